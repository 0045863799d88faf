// Three-index (P|mn) kernel instantiations for fitting shells with l = 3.
// Split across translation units only so that nvcc compiles them in parallel.
#include "df_kernels.cuh"

namespace m2 {

void launch_eri3_l3(int pc, const Eri3Params& P, cudaStream_t s) {
  dim3 grid((P.pairs.npair + 63) / 64, P.naux_shells);
  if (pc == 0) k_eri3<3, 0, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 1) k_eri3<3, 1, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 2) k_eri3<3, 1, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 3) k_eri3<3, 2, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 4) k_eri3<3, 2, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 5) k_eri3<3, 2, 2><<<grid, 64, 0, s>>>(P);
}


void launch_eri3_tile_l3(int pc, const Eri3Params& P, const Eri3TileArgs& A, cudaStream_t s) {
  dim3 grid((A.nlist + 63) / 64, P.naux_shells);
  if (pc == 0) k_eri3_tile<3, 0, 0><<<grid, 64, 0, s>>>(P, A);
  if (pc == 1) k_eri3_tile<3, 1, 0><<<grid, 64, 0, s>>>(P, A);
  if (pc == 2) k_eri3_tile<3, 1, 1><<<grid, 64, 0, s>>>(P, A);
  if (pc == 3) k_eri3_tile<3, 2, 0><<<grid, 64, 0, s>>>(P, A);
  if (pc == 4) k_eri3_tile<3, 2, 1><<<grid, 64, 0, s>>>(P, A);
  if (pc == 5) k_eri3_tile<3, 2, 2><<<grid, 64, 0, s>>>(P, A);
}

}  // namespace m2
