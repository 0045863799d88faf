// Three-index (P|mn) kernel instantiations for fitting shells with l = 0.
// Split across translation units only so that nvcc compiles them in parallel.
#include "df_kernels.cuh"

namespace m2 {

void launch_eri3_l0(int pc, const Eri3Params& P, cudaStream_t s) {
  dim3 grid((P.pairs.npair + 63) / 64, P.naux_shells);
  if (pc == 0) k_eri3<0, 0, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 1) k_eri3<0, 1, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 2) k_eri3<0, 1, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 3) k_eri3<0, 2, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 4) k_eri3<0, 2, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 5) k_eri3<0, 2, 2><<<grid, 64, 0, s>>>(P);
}

void launch_eri2(int LP, int LQ, const Eri2Params& P, cudaStream_t s) {
  dim3 grid((P.nq + 63) / 64, P.np);
  if (LP == 0 && LQ == 0) k_eri2<0, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 1 && LQ == 0) k_eri2<1, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 1 && LQ == 1) k_eri2<1, 1><<<grid, 64, 0, s>>>(P);
  if (LP == 2 && LQ == 0) k_eri2<2, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 2 && LQ == 1) k_eri2<2, 1><<<grid, 64, 0, s>>>(P);
  if (LP == 2 && LQ == 2) k_eri2<2, 2><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 0) k_eri2<3, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 1) k_eri2<3, 1><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 2) k_eri2<3, 2><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 3) k_eri2<3, 3><<<grid, 64, 0, s>>>(P);
}

void launch_onebody(int pc, const OneBodyParams& P, cudaStream_t s) {
  dim3 grid((P.pairs.npair + 63) / 64);
  if (pc == 0) k_onebody<0, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 1) k_onebody<1, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 2) k_onebody<1, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 3) k_onebody<2, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 4) k_onebody<2, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 5) k_onebody<2, 2><<<grid, 64, 0, s>>>(P);
}


void launch_eri3_tile_l0(int pc, const Eri3Params& P, const Eri3TileArgs& A, cudaStream_t s) {
  dim3 grid((A.nlist + 63) / 64, P.naux_shells);
  if (pc == 0) k_eri3_tile<0, 0, 0><<<grid, 64, 0, s>>>(P, A);
  if (pc == 1) k_eri3_tile<0, 1, 0><<<grid, 64, 0, s>>>(P, A);
  if (pc == 2) k_eri3_tile<0, 1, 1><<<grid, 64, 0, s>>>(P, A);
  if (pc == 3) k_eri3_tile<0, 2, 0><<<grid, 64, 0, s>>>(P, A);
  if (pc == 4) k_eri3_tile<0, 2, 1><<<grid, 64, 0, s>>>(P, A);
  if (pc == 5) k_eri3_tile<0, 2, 2><<<grid, 64, 0, s>>>(P, A);
}

}  // namespace m2
