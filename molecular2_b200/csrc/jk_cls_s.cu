// Kernel instantiations of the direct J/K build, bra classes ss, ps, pp.
// Split across translation units only so that nvcc compiles them in parallel.
#include "jk_kernels.cuh"

namespace m2 {
void launch_jk_bra_s(int A, int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s) {
  if (A == 0 && B == 0) { if (nden == 2) k_jk_direct<0, 0, 0, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<0, 0, 0, 0><<<grid, 128, 0, s>>>(P); }
  if (A == 1 && B == 0) { if (nden == 2) k_jk_direct<1, 0, 0, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<1, 0, 0, 0><<<grid, 128, 0, s>>>(P); }
  if (A == 1 && B == 1) { if (nden == 2) k_jk_direct<1, 0, 1, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<1, 0, 1, 0><<<grid, 128, 0, s>>>(P); }
  if (A == 2 && B == 0) { if (nden == 2) k_jk_direct<1, 1, 0, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<1, 1, 0, 0><<<grid, 128, 0, s>>>(P); }
  if (A == 2 && B == 1) { if (nden == 2) k_jk_direct<1, 1, 1, 0, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<1, 1, 1, 0><<<grid, 128, 0, s>>>(P); }
  if (A == 2 && B == 2) { if (nden == 2) k_jk_direct<1, 1, 1, 1, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<1, 1, 1, 1><<<grid, 128, 0, s>>>(P); }
}

}  // namespace m2
