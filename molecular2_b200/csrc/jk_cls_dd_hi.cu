// Kernel instantiations of the direct J/K build, bra class dd with ket dp, dd.
// Split across translation units only so that nvcc compiles them in parallel.
#include "jk_kernels.cuh"

namespace m2 {
void launch_jk_bra_dd_hi(int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s) {
  if (B == 4) { if (nden == 2) k_jk_direct<2, 2, 2, 1, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<2, 2, 2, 1><<<grid, 128, 0, s>>>(P); }
  if (B == 5) { if (nden == 2) k_jk_direct<2, 2, 2, 2, 2><<<grid, 128, 0, s>>>(P); else k_jk_direct<2, 2, 2, 2><<<grid, 128, 0, s>>>(P); }
}

void launch_schwarz_dd(const SchwarzParams& P, dim3 grid, cudaStream_t s) {
  k_schwarz<2, 2><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
