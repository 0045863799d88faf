// Density-fitted J/K (Fock::formJKdf / compute_2body_fock_df, molecular2
// src/fockbuild.cpp:171-174, 585-660), the three- and two-index integrals
// (IntegralEngine::compute_eris_3index/2index, src/eris.cpp:89-156, 304-356)
// and the one-body S, T, V matrices (IntegralEngine constructor,
// src/integrals.cpp:70-72).
//
// HBM layout.  The fitted three-index tensor is stored unpacked as
// B[x][K][y] (n x naux x n, x slowest): for every orbital x the slab B[x] is
// naux x n with y contiguous.  With that layout
//   X[x][K][i] = sum_y B[x][K][y] C[y][i]    is one GEMM (n*naux x n) . (n x o),
//   K          = X X^T                        is one SYRK over the n x (naux*o) matrix X,
//   gamma_K    = sum_{x,i} X[x][K][i] C[x][i] and
//   J[x][y]    = sum_K gamma_K B[x][K][y]     stream X and B once each.
// B = T L^-T with V = L L^T is formed once per geometry by a batched GEMM
// with L^-1 (the reference's O(n^2 naux^2) transform at :610-618); the
// Cholesky factor, L^-1 and every GEMM are this library's own FP64 kernels
// (dense.cu).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "dense.cuh"
#include "df_kernels.cuh"
#include "engine.h"

namespace m2 {

PrimView prim_view(const jk_engine* e);
ShellView shell_view(const jk_engine* e);

int prepare_aux(jk_engine* e) {
  if (!e->has_aux) return set_error(e, JK_ERR_STATE, "no fitting basis was given to jk_create");
  if (e->ap_p.p) return JK_OK;
  const HostBasis& a = e->aux;
  std::vector<double> p, x, y, z, K;
  std::vector<int> off;
  for (int s = 0; s < a.nshell; ++s) {
    off.push_back((int)p.size());
    for (int k = 0; k < a.nprim[s]; ++k) {
      p.push_back(a.exps[a.prim_off[s] + k]);
      x.push_back(a.xyz[3 * s]);
      y.push_back(a.xyz[3 * s + 1]);
      z.push_back(a.xyz[3 * s + 2]);
      K.push_back(a.coefs[a.prim_off[s] + k]);
    }
  }
  cudaStream_t st = e->stream;
  cudaError_t r = e->ap_p.upload(p, st);
  if (r == cudaSuccess) r = e->ap_x.upload(x, st);
  if (r == cudaSuccess) r = e->ap_y.upload(y, st);
  if (r == cudaSuccess) r = e->ap_z.upload(z, st);
  if (r == cudaSuccess) r = e->ap_K.upload(K, st);
  if (r == cudaSuccess) r = e->aux_prim_off.upload(off, st);
  for (int l = 0; l <= MAX_L_AUX && r == cudaSuccess; ++l) {
    std::vector<int> sh;
    for (int s = 0; s < a.nshell; ++s)
      if (a.l[s] == l) sh.push_back(s);
    e->aux_by_l_count[l] = (int)sh.size();
    r = e->aux_by_l[l].upload(sh, st);
  }
  if (r == cudaSuccess) r = cudaStreamSynchronize(st);
  return check_cuda(e, r, "prepare fitting basis");
}

static PrimView aux_view(const jk_engine* e) {
  return PrimView{e->ap_p.p, e->ap_x.p, e->ap_y.p, e->ap_z.p, e->ap_K.p};
}

// Launch parameters of the three-index kernels for fitting shells of angular
// momentum l and orbital pair class pc.
Eri3Params eri3_params(const jk_engine* e, int l, int pc) {
  Eri3Params P{};
  P.ap = aux_view(e);
  P.aux_shells = e->aux_by_l[l].p;
  P.naux_shells = e->aux_by_l_count[l];
  P.aux_prim_off = e->aux_prim_off.p;
  P.aux_nprim = e->daux.nprim.p;
  P.ax = e->daux.x.p;
  P.ay = e->daux.y.p;
  P.az = e->daux.z.p;
  P.aux_foff = e->daux.final_off.p;
  P.aux_pure = e->daux.pure.p;
  P.pairs = view(e->pcls[pc]);
  P.pp = prim_view(e);
  P.ox = e->dobs.x.p;
  P.oy = e->dobs.y.p;
  P.oz = e->dobs.z.p;
  P.obs_foff = e->dobs.final_off.p;
  P.obs_pure = e->dobs.pure.p;
  P.sph = e->dobs.sph.p;
  P.boys = e->boys.p;
  P.n = e->obs.n_final;
  P.naux = e->aux.n_final;
  return P;
}

// T3[x][P][y] = (P|xy), full n x naux x n.
static int compute_T3(jk_engine* e, double* T3, cudaStream_t s) {
  const int n = e->obs.n_final, naux = e->aux.n_final;
  cudaMemsetAsync(T3, 0, sizeof(double) * (size_t)n * naux * n, s);
  for (int l = 0; l <= MAX_L_AUX; ++l) {
    if (!e->aux_by_l_count[l]) continue;
    for (int pc = 0; pc < NPAIRCLASS; ++pc) {
      if (!e->pcls[pc].npair) continue;
      Eri3Params P = eri3_params(e, l, pc);
      P.T3 = T3;
      if (l == 0) launch_eri3_l0(pc, P, s);
      if (l == 1) launch_eri3_l1(pc, P, s);
      if (l == 2) launch_eri3_l2(pc, P, s);
      if (l == 3) launch_eri3_l3(pc, P, s);
    }
  }
  return check_cuda(e, cudaGetLastError(), "eri3 launch");
}

int compute_V(jk_engine* e, double* V, cudaStream_t s) {
  const int naux = e->aux.n_final;
  for (int lp = 0; lp <= MAX_L_AUX; ++lp)
    for (int lq = 0; lq <= lp; ++lq) {
      if (!e->aux_by_l_count[lp] || !e->aux_by_l_count[lq]) continue;
      Eri2Params P{};
      P.ap = aux_view(e);
      P.shells_p = e->aux_by_l[lp].p;
      P.np = e->aux_by_l_count[lp];
      P.shells_q = e->aux_by_l[lq].p;
      P.nq = e->aux_by_l_count[lq];
      P.aux_prim_off = e->aux_prim_off.p;
      P.aux_nprim = e->daux.nprim.p;
      P.ax = e->daux.x.p;
      P.ay = e->daux.y.p;
      P.az = e->daux.z.p;
      P.aux_foff = e->daux.final_off.p;
      P.aux_pure = e->daux.pure.p;
      P.sph = e->dobs.sph.p;
      P.boys = e->boys.p;
      P.naux = naux;
      P.V = V;
      launch_eri2(lp, lq, P, s);
    }
  return check_cuda(e, cudaGetLastError(), "eri2 launch");
}

// packed reference layout: Tp[(x(x+1)/2 + y) + P*npair], x >= y
__global__ void k_pack_T3(int n, int naux, const double* __restrict__ T3, double* __restrict__ Tp) {
  const size_t npair = (size_t)n * (n + 1) / 2;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= npair * naux) return;
  const int P = (int)(idx / npair);
  const size_t xy = idx % npair;
  int x = (int)floor((sqrt(8.0 * (double)xy + 1.0) - 1.0) * 0.5);
  while ((size_t)x * (x + 1) / 2 > xy) --x;
  while ((size_t)(x + 1) * (x + 2) / 2 <= xy) ++x;
  const int y = (int)(xy - (size_t)x * (x + 1) / 2);
  Tp[idx] = T3[((size_t)x * naux + P) * n + y];
}

// gamma_K = sum_{x,i} X[x][K][i] C[x][i]   (C column-major n x o)
__global__ void k_gamma(int n, int naux, int o, const double* __restrict__ X, const double* __restrict__ C,
                        double* __restrict__ g) {
  const int K = blockIdx.x;
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < n * o; idx += blockDim.x) {
    const int x = idx / o, i = idx % o;
    acc += X[((size_t)x * naux + K) * o + i] * C[(size_t)i * n + x];
  }
  __shared__ double red[32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (threadIdx.x == 0) g[K] = acc;
  }
}

// J[x][y] += sum_{K in [K0, K1)} gamma_K B[x][K][y] for y <= x (FP64 B).
// One block per (x, K range): ny = ceil((x+1)/2) threads of a K group read
// two consecutive y each (16-byte loads of one row of B), the block's other
// threads form further K groups, partial sums meet in shared memory and one
// atomic per (x, y) and block goes to J.  Only the lower triangle of J is
// written; k_mirror_lower fills the upper one.
constexpr int DFJ_THREADS = 256;
__global__ void __launch_bounds__(DFJ_THREADS) k_df_J_lower(int n, int naux, int kchunk,
                                                            const double* __restrict__ B,
                                                            const double* __restrict__ g, double* __restrict__ J) {
  __shared__ double part[DFJ_THREADS * 2];
  const int x = blockIdx.x;
  const int ny_all = (x + 2) / 2;
  const int K0 = blockIdx.y * kchunk, K1 = min(naux, K0 + kchunk);
  const int t = threadIdx.x;
  for (int yb = 0; yb < ny_all; yb += DFJ_THREADS) {
    const int ny = min(ny_all - yb, DFJ_THREADS);
    const int ngroups = DFJ_THREADS / ny;
    const int yi = t % ny, kg = t / ny;
    const int y = (yb + yi) * 2;
    double a0 = 0.0, a1 = 0.0;
    if (kg < ngroups) {
      const double* b = B + (size_t)x * naux * n + y;
      const bool pair = (y + 1 < n) && ((n & 1) == 0);   // 16-byte aligned pair
#pragma unroll 4
      for (int K = K0 + kg; K < K1; K += ngroups) {
        const double gk = __ldg(g + K);
        if (pair) {
          const double2 v = __ldg(reinterpret_cast<const double2*>(b + (size_t)K * n));
          a0 += gk * v.x;
          a1 += gk * v.y;
        } else {
          a0 += gk * __ldg(b + (size_t)K * n);
          if (y + 1 < n) a1 += gk * __ldg(b + (size_t)K * n + 1);
        }
      }
    }
    __syncthreads();
    part[t * 2] = a0;
    part[t * 2 + 1] = a1;
    __syncthreads();
    for (int idx = t; idx < ny * 2; idx += DFJ_THREADS) {
      const int yy = idx / 2, e = idx % 2, yo = (yb + yy) * 2 + e;
      if (yo > x || yo >= n) continue;
      double sum = 0.0;
      for (int k = 0; k < ngroups; ++k) sum += part[(k * ny + yy) * 2 + e];
      atomicAdd(J + (size_t)yo * n + x, sum);
    }
  }
}

__global__ void k_scale_mat(size_t n, double a, double* x) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= a;
}

// upper triangle of a column-major symmetric matrix from its lower triangle
__global__ void k_mirror_lower(int n, double* J) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n * n) return;
  const int i = (int)(idx % n), j = (int)(idx / n);
  if (i < j) J[idx] = J[(size_t)i * n + j];
}

// K (n x n, column-major) = X X^T for X given as n rows of length len
// (row x at X + x*len): lower tiles split over the SMs, then mirrored.
cudaError_t df_syrk_X(jk_engine* e, const double* X, int n, long long len, double* K, cudaStream_t s) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device);
  const int tiles = ((n + 127) / 128) * ((n + 127) / 128 + 1) / 2;
  const long long kt = (len + 15) / 16;
  DGemm g;
  g.M = n;
  g.N = n;
  g.K = (int)len;
  g.A = X;
  g.sam = len;
  g.sak = 1;
  g.B = X;
  g.sbk = 1;
  g.sbn = len;
  g.C = K;
  g.scm = 1;
  g.scn = n;
  g.c_lower = true;
  g.ksplit = (int)std::max(1LL, std::min<long long>((2LL * nsm + tiles - 1) / tiles, kt / 8));
  cudaError_t st = dgemm(g, s);
  if (st == cudaSuccess) mirror_lower(K, n, s);
  return st == cudaSuccess ? cudaGetLastError() : st;
}

int df_setup(jk_engine* e) {
  int rc = prepare_aux(e);
  if (rc) return rc;
  if (df_use_tiled(e)) return df_tiled_setup(e);
  cudaStream_t s = e->stream;
  const int n = e->obs.n_final, naux = e->aux.n_final;
  DFState& d = e->df;
  const int k0 = d.k0, k1 = d.k1 < 0 ? naux : d.k1, nloc = k1 - k0;
  if (k0 < 0 || k1 > naux || nloc <= 0) return set_error(e, JK_ERR_ARG, "DF range outside the fitting basis");
  DevBuf<double> T3, Linv;
  cudaError_t st = T3.alloc((size_t)n * naux * n);
  if (st == cudaSuccess) st = d.L.alloc((size_t)naux * naux);
  if (st == cudaSuccess) st = Linv.alloc((size_t)naux * naux);
  if (st == cudaSuccess) st = d.B64.alloc((size_t)n * nloc * n);
  if (st != cudaSuccess) return check_cuda(e, st, "df_setup allocation");
  if ((rc = compute_T3(e, T3.p, s))) return rc;
  if ((rc = compute_V(e, d.L.p, s))) return rc;
  // V = L L^T (own blocked Cholesky), then L^-1
  DevBuf<double> work;
  DevBuf<int> info;
  st = work.alloc((size_t)naux * naux);
  if (st == cudaSuccess) st = info.alloc(1);
  if (st != cudaSuccess) return check_cuda(e, st, "Cholesky workspace");
  if ((rc = cholesky(e, d.L.p, naux, work.p, info.p, s))) return rc;
  int hinfo = 0;
  st = cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);
  if (st != cudaSuccess) return check_cuda(e, st, "Cholesky");
  if (hinfo != 0)
    return set_error(e, JK_ERR_NOT_PD,
                     "fitting metric (P|Q) is not positive definite (leading minor " + std::to_string(hinfo) + ")");
  if ((rc = tri_inverse(e, d.L.p, Linv.p, naux, work.p, s))) return rc;
  // B[x] (nloc x n, y contiguous) = (rows k0..k1 of L^-1) . T[x]  for every x
  DGemm g;
  g.M = nloc;
  g.N = n;
  g.K = naux;
  g.batch = n;
  g.A = Linv.p + k0;
  g.sam = 1;
  g.sak = naux;
  g.a_lower = (k0 == 0);
  g.B = T3.p;
  g.sbk = n;
  g.sbn = 1;
  g.bsb = (long long)naux * n;
  g.C = d.B64.p;
  g.scm = n;
  g.scn = 1;
  g.bsc = (long long)nloc * n;
  st = dgemm(g, s);
  if (st != cudaSuccess) return check_cuda(e, st, "B = L^-1 T");
  st = d.Linv.alloc((size_t)naux * naux);
  if (st == cudaSuccess)
    st = cudaMemcpyAsync(d.Linv.p, Linv.p, sizeof(double) * naux * naux, cudaMemcpyDeviceToDevice, s);
  if (st != cudaSuccess) return check_cuda(e, st, "keep L^-1");
  st = cudaStreamSynchronize(s);
  if (st != cudaSuccess) return check_cuda(e, st, "df_setup");
  d.naux = nloc;
  d.ready = true;
  return JK_OK;
}

// Record stage boundary k of the DF build when profiling is on.
void stage_mark(jk_engine* e, int k, cudaStream_t s) {
  if (!e->profiling || k >= jk_engine::NSTAGE_EV) return;
  if (!e->ev[k]) cudaEventCreate(&e->ev[k]);
  cudaEventRecord(e->ev[k], s);
  e->nev_used = std::max(e->nev_used, k + 1);
}

int df_jk_device(jk_engine* e, const double* dC, int nocc, int mode, double* dJ, double* dK, cudaStream_t s) {
  DFState& d = e->df;
  e->kev_blocks = 0;
  if (e->tiled.metric_ready) return df_tiled_device(e, dC, nocc, mode, dJ, dK, s);
  if (!d.ready) return set_error(e, JK_ERR_STATE, "jk_df before jk_df_setup");
  if (mode == 1) return df_mixed_device(e, dC, nocc, dJ, dK, s);
  if (mode != 0) return set_error(e, JK_ERR_ARG, "jk_df: unsupported precision mode");
  const int n = e->obs.n_final, naux = d.naux;
  cudaError_t st = d.X64.alloc((size_t)n * naux * nocc);
  if (st == cudaSuccess) st = d.gamma.alloc(naux);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_df scratch");
  stage_mark(e, 0, s);
  // X[x][K][i] = sum_y B[x][K][y] C[y][i]: one GEMM over the n*naux rows (x, K)
  DGemm gx;
  gx.M = n * naux;
  gx.N = nocc;
  gx.K = n;
  gx.A = d.B64.p;
  gx.sam = n;
  gx.sak = 1;
  gx.B = dC;
  gx.sbk = 1;
  gx.sbn = n;
  gx.C = d.X64.p;
  gx.scm = nocc;
  gx.scn = 1;
  cudaError_t st2 = dgemm(gx, s);
  if (st2 != cudaSuccess) return check_cuda(e, st2, "X = B C");
  stage_mark(e, 1, s);
  // K = X X^T over the (K, i) index: lower tiles, split over the SMs, mirrored
  st2 = df_syrk_X(e, d.X64.p, n, (long long)naux * nocc, dK, s);
  if (st2 != cudaSuccess) return check_cuda(e, st2, "K = X X^T");
  stage_mark(e, 2, s);
  k_gamma<<<naux, 256, 0, s>>>(n, naux, nocc, d.X64.p, dC, d.gamma.p);
  stage_mark(e, 3, s);
  cudaMemsetAsync(dJ, 0, sizeof(double) * n * n, s);
  const int kchunk = (naux + 15) / 16;   // 16 K ranges per row x
  k_df_J_lower<<<dim3(n, (naux + kchunk - 1) / kchunk), DFJ_THREADS, 0, s>>>(n, naux, kchunk, d.B64.p, d.gamma.p,
                                                                              dJ);
  k_mirror_lower<<<(unsigned)(((size_t)n * n + 255) / 256), 256, 0, s>>>(n, dJ);
  stage_mark(e, 4, s);
  return check_cuda(e, cudaGetLastError(), "jk_df launch");
}

int one_body_device(jk_engine* e, double* S, double* T, double* V, cudaStream_t s) {
  const int n = e->obs.n_final;
  DevBuf<double> Z, C;
  cudaError_t st = Z.upload(e->Z, s);
  if (st == cudaSuccess) st = C.upload(e->atom_xyz, s);
  if (st != cudaSuccess) return check_cuda(e, st, "one_body upload");
  // shell pairs whose primitive products all vanish are not in the pair
  // lists; their blocks are zero, not whatever the buffers held before
  for (double* M : {S, T, V}) cudaMemsetAsync(M, 0, sizeof(double) * (size_t)n * n, s);
  for (int pc = 0; pc < NPAIRCLASS; ++pc) {
    if (!e->pcls[pc].npair) continue;
    OneBodyParams P{};
    P.pairs = view(e->pcls[pc]);
    P.pp = prim_view(e);
    P.pa = e->pp_a.p;
    P.ox = e->dobs.x.p;
    P.oy = e->dobs.y.p;
    P.oz = e->dobs.z.p;
    P.foff = e->dobs.final_off.p;
    P.pure = e->dobs.pure.p;
    P.sph = e->dobs.sph.p;
    P.boys = e->boys.p;
    P.natom = e->natom;
    P.Z = Z.p;
    P.cxyz = C.p;
    P.n = n;
    P.S = S;
    P.T = T;
    P.V = V;
    launch_onebody(pc, P, s);
  }
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);  // Z, C die on return
  return check_cuda(e, st, "one_body");
}

}  // namespace m2

using namespace m2;

extern "C" {

int jk_eri3(jk_engine* e, double* Tpacked) {
  if (!e || !Tpacked) return JK_ERR_ARG;
  int rc = prepare_aux(e);
  if (rc) return rc;
  const int n = e->obs.n_final, naux = e->aux.n_final;
  const size_t npair = (size_t)n * (n + 1) / 2;
  DevBuf<double> T3, Tp;
  cudaError_t st = T3.alloc((size_t)n * naux * n);
  if (st == cudaSuccess) st = Tp.alloc(npair * naux);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_eri3 allocation");
  if ((rc = compute_T3(e, T3.p, e->stream))) return rc;
  const size_t tot = npair * naux;
  k_pack_T3<<<(unsigned)((tot + 255) / 256), 256, 0, e->stream>>>(n, naux, T3.p, Tp.p);
  st = cudaMemcpyAsync(Tpacked, Tp.p, tot * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  return check_cuda(e, st, "jk_eri3");
}

int jk_eri2(jk_engine* e, double* V) {
  if (!e || !V) return JK_ERR_ARG;
  int rc = prepare_aux(e);
  if (rc) return rc;
  const int naux = e->aux.n_final;
  DevBuf<double> Vd;
  cudaError_t st = Vd.alloc((size_t)naux * naux);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_eri2 allocation");
  if ((rc = compute_V(e, Vd.p, e->stream))) return rc;
  st = cudaMemcpyAsync(V, Vd.p, sizeof(double) * naux * naux, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  return check_cuda(e, st, "jk_eri2");
}

int jk_df_setup(jk_engine* e) {
  if (!e) return JK_ERR_ARG;
  return df_setup(e);
}

int jk_df_set_range(jk_engine* e, int k0, int k1) {
  if (!e) return JK_ERR_ARG;
  if (e->df.ready) return set_error(e, JK_ERR_STATE, "jk_df_set_range after jk_df_setup");
  const int naux = e->has_aux ? e->aux.n_final : 0;
  if (k0 < 0 || k1 <= k0 || k1 > naux) return set_error(e, JK_ERR_ARG, "jk_df_set_range: need 0 <= k0 < k1 <= naux");
  e->df.k0 = k0;
  e->df.k1 = k1;
  return JK_OK;
}

int jk_df_device(jk_engine* e, const double* dC, int nocc, int prec_mode, double* dJ, double* dK, void* stream) {
  if (!e || !dC || !dJ || !dK || nocc <= 0) return JK_ERR_ARG;
  return df_jk_device(e, dC, nocc, prec_mode, dJ, dK, stream ? (cudaStream_t)stream : e->stream);
}

int jk_df(jk_engine* e, const double* C, int nocc, int prec_mode, double* J, double* K) {
  if (!e || !C || !J || !K || nocc <= 0) return JK_ERR_ARG;
  const int n = e->obs.n_final;
  DevBuf<double> dC;
  cudaError_t st = dC.alloc((size_t)n * nocc);
  if (st == cudaSuccess) st = e->Jfinal.alloc((size_t)n * n);
  if (st == cudaSuccess) st = e->Kfinal.alloc((size_t)n * n);
  if (st == cudaSuccess) st = cudaMemcpyAsync(dC.p, C, sizeof(double) * n * nocc, cudaMemcpyHostToDevice, e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_df upload");
  int rc = df_jk_device(e, dC.p, nocc, prec_mode, e->Jfinal.p, e->Kfinal.p, e->stream);
  if (rc) return rc;
  st = cudaMemcpyAsync(J, e->Jfinal.p, sizeof(double) * n * n, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaMemcpyAsync(K, e->Kfinal.p, sizeof(double) * n * n, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_df download");
  return prec_mode == 1 ? df_mixed_error(e) : JK_OK;
}

int jk_df_uhf_device(jk_engine* e, const double* dCa, int na, const double* dCb, int nb, int prec_mode,
                     double multiplier, double* dJa, double* dJb, double* dKa, double* dKb, void* stream) {
  if (!e || !dJa || !dJb || !dKa || !dKb || na < 0 || nb < 0 || (na > 0 && !dCa) || (nb > 0 && !dCb))
    return JK_ERR_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  const int n = e->obs.n_final;
  const size_t nn = (size_t)n * n;
  // UnrestrictedFock::formJKdf (src/fockbuild.cpp:365-372): compute_2body_fock_df
  // for each spin over the same fitted tensor, then both scaled by multiplier
  const double* Cs[2] = {dCa, dCb};
  const int no[2] = {na, nb};
  double* Js[2] = {dJa, dJb};
  double* Ks[2] = {dKa, dKb};
  for (int k = 0; k < 2; ++k) {
    if (no[k] == 0) {
      cudaMemsetAsync(Js[k], 0, sizeof(double) * nn, s);
      cudaMemsetAsync(Ks[k], 0, sizeof(double) * nn, s);
      continue;
    }
    int rc = df_jk_device(e, Cs[k], no[k], prec_mode, Js[k], Ks[k], s);
    if (rc) return rc;
    if (multiplier != 1.0) {
      k_scale_mat<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(nn, multiplier, Js[k]);
      k_scale_mat<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(nn, multiplier, Ks[k]);
    }
  }
  return check_cuda(e, cudaGetLastError(), "jk_df_uhf");
}

int jk_df_uhf(jk_engine* e, const double* Ca, int na, const double* Cb, int nb, int prec_mode, double multiplier,
              double* Ja, double* Jb, double* Ka, double* Kb) {
  if (!e || !Ja || !Jb || !Ka || !Kb || na < 0 || nb < 0 || (na > 0 && !Ca) || (nb > 0 && !Cb)) return JK_ERR_ARG;
  const int n = e->obs.n_final;
  const size_t nn = (size_t)n * n;
  DevBuf<double> d;
  cudaError_t st = d.alloc(4 * nn + (size_t)n * (na + nb));
  double* dCa = d.p + 4 * nn;
  double* dCb = dCa + (size_t)n * na;
  if (st == cudaSuccess && na)
    st = cudaMemcpyAsync(dCa, Ca, sizeof(double) * n * na, cudaMemcpyHostToDevice, e->stream);
  if (st == cudaSuccess && nb)
    st = cudaMemcpyAsync(dCb, Cb, sizeof(double) * n * nb, cudaMemcpyHostToDevice, e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_df_uhf upload");
  int rc = jk_df_uhf_device(e, dCa, na, dCb, nb, prec_mode, multiplier, d.p, d.p + nn, d.p + 2 * nn, d.p + 3 * nn,
                            nullptr);
  if (rc) return rc;
  double* outs[4] = {Ja, Jb, Ka, Kb};
  for (int k = 0; k < 4 && st == cudaSuccess; ++k)
    st = cudaMemcpyAsync(outs[k], d.p + k * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_df_uhf download");
  return prec_mode == 1 ? df_mixed_error(e) : JK_OK;
}

int jk_set_profiling(jk_engine* e, int on) {
  if (!e) return JK_ERR_ARG;
  e->profiling = on != 0;
  return JK_OK;
}

int jk_stage_ms(jk_engine* e, float* ms, int nmax, int* nwritten) {
  if (!e || !ms || !nwritten) return JK_ERR_ARG;
  *nwritten = 0;
  if (e->profiling && e->kev_blocks > 0) {
    // tiled mixed build: [GEMM1 total, GEMM2 total, J, finalize, fitted-function blocks]
    const int B = e->kev_blocks;
    cudaError_t st = cudaEventSynchronize(e->kev[3 * B + 1]);
    if (st != cudaSuccess) return check_cuda(e, st, "kernel events");
    float g1 = 0.f, g2 = 0.f, t = 0.f;
    for (int b = 0; b < B; ++b) {
      cudaEventElapsedTime(&t, e->kev[3 * b], e->kev[3 * b + 1]);
      g1 += t;
      cudaEventElapsedTime(&t, e->kev[3 * b + 1], e->kev[3 * b + 2]);
      g2 += t;
    }
    float jt = 0.f, ft = 0.f;
    cudaEventElapsedTime(&jt, e->kev[3 * B - 1], e->kev[3 * B]);
    cudaEventElapsedTime(&ft, e->kev[3 * B], e->kev[3 * B + 1]);
    const float vals[5] = {g1, g2, jt, ft, (float)B};
    int k = 0;
    for (; k < 5 && k < nmax; ++k) ms[k] = vals[k];
    *nwritten = k;
    return JK_OK;
  }
  if (!e->profiling || e->nev_used < 2) return set_error(e, JK_ERR_STATE, "profiling off or no build recorded");
  cudaError_t st = cudaEventSynchronize(e->ev[e->nev_used - 1]);
  if (st != cudaSuccess) return check_cuda(e, st, "stage events");
  int k = 0;
  for (; k + 1 < e->nev_used && k < nmax; ++k) {
    st = cudaEventElapsedTime(&ms[k], e->ev[k], e->ev[k + 1]);
    if (st != cudaSuccess) return check_cuda(e, st, "stage events");
  }
  *nwritten = k;
  return JK_OK;
}

int jk_one_body(jk_engine* e, double* S, double* T, double* V) {
  if (!e || !S || !T || !V) return JK_ERR_ARG;
  const int n = e->obs.n_final;
  DevBuf<double> dS, dT, dV;
  cudaError_t st = dS.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dT.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dV.alloc((size_t)n * n);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_one_body allocation");
  int rc = one_body_device(e, dS.p, dT.p, dV.p, e->stream);
  if (rc) return rc;
  const size_t b = sizeof(double) * n * n;
  st = cudaMemcpyAsync(S, dS.p, b, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaMemcpyAsync(T, dT.p, b, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaMemcpyAsync(V, dV.p, b, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  return check_cuda(e, st, "jk_one_body");
}

}  // extern "C"
