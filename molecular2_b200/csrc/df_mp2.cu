// Density-fitted MP2 correlation energy (MP2::dfmp2, molecular2
// src/mp2.cpp:477-583) over the fitted tensor of the DF J/K build.
//
// molecular2 inverts the metric explicitly and forms
//   (ia|jb) = sum_PQ B'_ia,P (P|Q)^-1 B'_jb,Q,  B'_ia,P = sum_mn C_mi C_na (P|mn);
// here the factorised inverse is used instead: with B = (mn|P) L^-T (the
// tensor jk_df_setup keeps, V = L L^T) the same integrals are
//   (ia|jb) = sum_K Z_ia,K Z_jb,K,  Z_ia,K = sum_xy C_xi C_ya B_xy,K,
// and the energy E = sum_ijab (ia|jb) [2 (ia|jb) - (ib|ja)] / (e_i + e_j - e_a
// - e_b) runs over the active occupied orbitals (the lowest nfrozen are kept
// out, molecular2's withcore = false).  All FP64 on the DMMA GEMM:
//   X[x][K][i] = sum_y B[x][K][y] C[y][i]            (one GEMM),
//   Z[i][a][K] = sum_x Cv[x][a] X[x][K][i]           (batched over i),
//   V_i[jb][a] = sum_K Z[i][a][K] Z[j][b][K]         (batched over blocks of i),
// and a reduction kernel that reads (ia|jb) and (ib|ja) from the same V_i.
#include <algorithm>
#include <string>
#include <vector>

#include "dense.cuh"
#include "engine.h"

namespace m2 {

// E += sum over the ib orbitals i0.. of the block, all j, a, b
__global__ void __launch_bounds__(256) k_mp2_energy(int ib, int i0, int act, int nv, const double* __restrict__ V,
                                                    const double* __restrict__ eo, const double* __restrict__ ev,
                                                    double* __restrict__ E) {
  const size_t per_i = (size_t)act * nv * nv;
  const size_t tot = per_i * ib;
  double acc = 0.0;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < tot; idx += (size_t)gridDim.x * blockDim.x) {
    const int bi = (int)(idx / per_i);
    const size_t r = idx % per_i;
    const int a = (int)(r % nv);
    const size_t jb = r / nv;
    const int b = (int)(jb % nv), j = (int)(jb / nv);
    const double* Vi = V + (size_t)bi * per_i;
    const double v = Vi[jb * nv + a];                        // (ia|jb)
    const double w = Vi[((size_t)j * nv + a) * nv + b];      // (ib|ja)
    acc += v * (2.0 * v - w) / (eo[i0 + bi] + eo[j] - ev[a] - ev[b]);
  }
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) atomicAdd(E, acc);
  }
}

static int df_mp2(jk_engine* e, const double* hC, const double* heps, int nmo, int nocc, int nfrozen, double* emp2) {
  DFState& d = e->df;
  if (e->tiled.metric_ready) return set_error(e, JK_ERR_STATE, "jk_df_mp2 needs the unpacked DF storage");
  if (!d.ready) {
    const int rc = df_setup(e);
    if (rc) return rc;
    if (e->tiled.metric_ready) return set_error(e, JK_ERR_STATE, "jk_df_mp2 needs the unpacked DF storage");
  }
  if (d.k0 != 0 || d.naux != e->aux.n_final)
    return set_error(e, JK_ERR_STATE, "jk_df_mp2 needs the whole fitting range (jk_df_set_range)");
  const int n = e->obs.n_final, naux = d.naux, act = nocc - nfrozen, nv = nmo - nocc;
  cudaStream_t s = e->stream;
  DevBuf<double> C, eps, X, Z, V, E;
  cudaError_t st = C.alloc((size_t)n * nmo);
  if (st == cudaSuccess) st = eps.alloc(nmo);
  if (st == cudaSuccess) st = X.alloc((size_t)n * naux * act);
  if (st == cudaSuccess) st = Z.alloc((size_t)act * nv * naux);
  if (st == cudaSuccess) st = E.alloc(1);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_df_mp2 allocation");
  if ((st = cudaMemcpyAsync(C.p, hC, sizeof(double) * n * nmo, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (st = cudaMemcpyAsync(eps.p, heps, sizeof(double) * nmo, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return check_cuda(e, st, "jk_df_mp2 upload");
  auto gemm = [&](const DGemm& g, const char* what) {
    const cudaError_t r = dgemm(g, s);
    return r == cudaSuccess ? JK_OK : check_cuda(e, r, what);
  };
  int rc;
  {
    DGemm g;  // X[x][K][i] = sum_y B[x][K][y] C[y][nfrozen + i]
    g.M = n * naux; g.N = act; g.K = n;
    g.A = d.B64.p; g.sam = n; g.sak = 1;
    g.B = C.p + (size_t)nfrozen * n; g.sbk = 1; g.sbn = n;
    g.C = X.p; g.scm = act; g.scn = 1;
    if ((rc = gemm(g, "jk_df_mp2: X = B C"))) return rc;
  }
  {
    DGemm g;  // Z[i][a][K] = sum_x Cv[x][a] X[x][K][i], one problem per i
    g.M = nv; g.N = naux; g.K = n; g.batch = act;
    g.A = C.p + (size_t)nocc * n; g.sam = n; g.sak = 1;
    g.B = X.p; g.sbk = (long long)naux * act; g.sbn = act; g.bsb = 1;
    g.C = Z.p; g.scm = naux; g.scn = 1; g.bsc = (long long)nv * naux;
    if ((rc = gemm(g, "jk_df_mp2: Z = Cv^T X"))) return rc;
  }
  X.reset();
  // blocks of i with V_i (nv x act*nv) resident, within a quarter of the free memory
  size_t fr = 0, tt = 0;
  cudaMemGetInfo(&fr, &tt);
  const double per_i = 8.0 * (double)nv * act * nv;
  const int ib = (int)std::max(1.0, std::min<double>(std::min(act, 64), 0.25 * (double)fr / per_i));
  if ((st = V.alloc((size_t)ib * act * nv * nv)) != cudaSuccess) return check_cuda(e, st, "jk_df_mp2 V block");
  cudaMemsetAsync(E.p, 0, sizeof(double), s);
  for (int i0 = 0; i0 < act; i0 += ib) {
    const int bcur = std::min(ib, act - i0);
    DGemm g;  // V_i[jb][a] = sum_K Z[i][a][K] Z[jb][K]
    g.M = nv; g.N = act * nv; g.K = naux; g.batch = bcur;
    g.A = Z.p + (size_t)i0 * nv * naux; g.sam = naux; g.sak = 1; g.bsa = (long long)nv * naux;
    g.B = Z.p; g.sbk = 1; g.sbn = naux;
    g.C = V.p; g.scm = 1; g.scn = nv; g.bsc = (long long)act * nv * nv;
    if ((rc = gemm(g, "jk_df_mp2: (ia|jb)"))) return rc;
    k_mp2_energy<<<4 * 148, 256, 0, s>>>(bcur, i0, act, nv, V.p, eps.p + nfrozen, eps.p + nocc, E.p);
  }
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaMemcpyAsync(emp2, E.p, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);
  return check_cuda(e, st, "jk_df_mp2");
}

}  // namespace m2

using namespace m2;

extern "C" int jk_df_mp2(jk_engine* e, const double* C, const double* eps, int nmo, int nocc, int nfrozen,
                         double* emp2) {
  if (!e || !C || !eps || !emp2) return JK_ERR_ARG;
  if (nmo < 1 || nmo > e->obs.n_final || nocc < 1 || nocc >= nmo || nfrozen < 0 || nfrozen >= nocc)
    return set_error(e, JK_ERR_ARG, "jk_df_mp2: need 0 <= nfrozen < nocc < nmo <= n");
  return df_mp2(e, C, eps, nmo, nocc, nfrozen, emp2);
}
