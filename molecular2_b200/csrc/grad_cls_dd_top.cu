// Kernel instantiation of the RHF gradient adjoint, class (dd|dd).
// Split across translation units only so that nvcc compiles them in parallel.
#include "grad_kernels.cuh"

namespace m2 {
void launch_grad2e_bra_dd_top(const Grad2eParams& P, dim3 grid, cudaStream_t s) {
  k_grad2e<2, 2, 2, 2><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
