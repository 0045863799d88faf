// Kernel instantiations of the direct J/K build, bra class dp.
// Split across translation units only so that nvcc compiles them in parallel.
#include "jk_kernels.cuh"

namespace m2 {
void launch_jk_bra_dp(int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s) {
  if (B == 0) { if (nden == 2) k_jk_direct<2, 1, 0, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<2, 1, 0, 0><<<grid, 128, 0, s>>>(P); }
  if (B == 1) { if (nden == 2) k_jk_direct<2, 1, 1, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<2, 1, 1, 0><<<grid, 128, 0, s>>>(P); }
  if (B == 2) { if (nden == 2) k_jk_direct<2, 1, 1, 1, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<2, 1, 1, 1><<<grid, 128, 0, s>>>(P); }
  if (B == 3) { if (nden == 2) k_jk_direct<2, 1, 2, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<2, 1, 2, 0><<<grid, 128, 0, s>>>(P); }
  if (B == 4) { if (nden == 2) k_jk_direct<2, 1, 2, 1, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<2, 1, 2, 1><<<grid, 128, 0, s>>>(P); }
}

}  // namespace m2
