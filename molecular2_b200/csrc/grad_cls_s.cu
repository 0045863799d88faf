// Kernel instantiations of the RHF gradient adjoint, bra classes ss, ps, pp.
// Split across translation units only so that nvcc compiles them in parallel.
#include "grad_kernels.cuh"

namespace m2 {
void launch_grad2e_bra_s(int A, int B, const Grad2eParams& P, dim3 grid, cudaStream_t s) {
  if (A == 0 && B == 0) k_grad2e<0, 0, 0, 0><<<grid, 64, 0, s>>>(P);
  if (A == 1 && B == 0) k_grad2e<1, 0, 0, 0><<<grid, 64, 0, s>>>(P);
  if (A == 1 && B == 1) k_grad2e<1, 0, 1, 0><<<grid, 64, 0, s>>>(P);
  if (A == 2 && B == 0) k_grad2e<1, 1, 0, 0><<<grid, 64, 0, s>>>(P);
  if (A == 2 && B == 1) k_grad2e<1, 1, 1, 0><<<grid, 64, 0, s>>>(P);
  if (A == 2 && B == 2) k_grad2e<1, 1, 1, 1><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
