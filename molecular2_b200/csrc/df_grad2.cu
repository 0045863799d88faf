// Kernel instantiations of the density-fitted gradient, two-index (metric)
// derivatives for every ordered pair of fitting angular momenta.
#include "df_grad_kernels.cuh"

namespace m2 {
void launch_grad2(int LP, int LQ, const Grad2Params& P, cudaStream_t s) {
  dim3 grid((P.nq + 63) / 64, P.np);
  if (LP == 0 && LQ == 0) k_grad2<0, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 0 && LQ == 1) k_grad2<0, 1><<<grid, 64, 0, s>>>(P);
  if (LP == 0 && LQ == 2) k_grad2<0, 2><<<grid, 64, 0, s>>>(P);
  if (LP == 0 && LQ == 3) k_grad2<0, 3><<<grid, 64, 0, s>>>(P);
  if (LP == 1 && LQ == 0) k_grad2<1, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 1 && LQ == 1) k_grad2<1, 1><<<grid, 64, 0, s>>>(P);
  if (LP == 1 && LQ == 2) k_grad2<1, 2><<<grid, 64, 0, s>>>(P);
  if (LP == 1 && LQ == 3) k_grad2<1, 3><<<grid, 64, 0, s>>>(P);
  if (LP == 2 && LQ == 0) k_grad2<2, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 2 && LQ == 1) k_grad2<2, 1><<<grid, 64, 0, s>>>(P);
  if (LP == 2 && LQ == 2) k_grad2<2, 2><<<grid, 64, 0, s>>>(P);
  if (LP == 2 && LQ == 3) k_grad2<2, 3><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 0) k_grad2<3, 0><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 1) k_grad2<3, 1><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 2) k_grad2<3, 2><<<grid, 64, 0, s>>>(P);
  if (LP == 3 && LQ == 3) k_grad2<3, 3><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
