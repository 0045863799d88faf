// Kernel instantiation of the RHF gradient adjoint, class (dd|dp).
// Split across translation units only so that nvcc compiles them in parallel.
#include "grad_kernels.cuh"

namespace m2 {
void launch_grad2e_bra_dd_hi(int B, const Grad2eParams& P, dim3 grid, cudaStream_t s) {
  if (B == 4) k_grad2e<2, 2, 2, 1><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
