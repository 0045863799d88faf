// Kernel instantiations of the RHF gradient adjoint, bra class ds.
// Split across translation units only so that nvcc compiles them in parallel.
#include "grad_kernels.cuh"

namespace m2 {
void launch_grad2e_bra_ds(int B, const Grad2eParams& P, dim3 grid, cudaStream_t s) {
  if (B == 0) k_grad2e<2, 0, 0, 0><<<grid, 64, 0, s>>>(P);
  if (B == 1) k_grad2e<2, 0, 1, 0><<<grid, 64, 0, s>>>(P);
  if (B == 2) k_grad2e<2, 0, 1, 1><<<grid, 64, 0, s>>>(P);
  if (B == 3) k_grad2e<2, 0, 2, 0><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
