// Kernel instantiations of the density-fitted gradient, three-index
// derivatives with fitting functions of angular momentum 3.  Split across
// translation units only so that nvcc compiles them in parallel.
#include "df_grad_kernels.cuh"

namespace m2 {
void launch_grad3_l3(int pc, const Grad3Params& P, cudaStream_t s) {
  dim3 grid((P.pairs.npair + 63) / 64, P.naux_shells, 4);  // z: the four shifted classes
  if (pc == 0) k_grad3<3, 0, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 1) k_grad3<3, 1, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 2) k_grad3<3, 1, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 3) k_grad3<3, 2, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 4) k_grad3<3, 2, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 5) k_grad3<3, 2, 2><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
