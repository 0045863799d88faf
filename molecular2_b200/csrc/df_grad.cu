// Density-fitted RHF nuclear gradient: the gradient of the energy that the
// DF Fock build of compute_2body_fock_df (molecular2 src/fockbuild.cpp:585-660)
// defines, plus the one-body and nuclear terms of Fock::compute_forces
// (src/rhfgrad.cpp:15-89).  molecular2 only differentiates the 4-index
// energy (compute_2body_fock_deriv<1>); with density fitting the consistent
// gradient differentiates the fitted integrals (mn|P) V^-1 (Q|ls):
//   dE2 = sum_{P,mn} (mn|P)^x W3_{mn,P} + sum_{PQ} (P|Q)^x W2_{PQ}
// (weights in df_grad_kernels.cuh).  Everything before the derivative
// kernels is dense linear algebra on the B tensor kept by jk_df_setup:
//   X[x][K][i]  = sum_y B[x][K][y] C[y][i]                     (DGEMM)
//   bt[K](i,j)  = sum_x X[x][K][i] C[x][j]                     (batched DGEMM)
//   gt_K        = 2 sum_i bt[K](i,i),  c = L^-T gt              (TRSV)
//   d           = bt L^-1  over K (d^P_ij = sum_Q V^-1_PQ (Q|ij))   (TRSM)
//   W2          = d^T d - 1/2 c c^T                            (DGEMM + DGER)
//   Z^P         = C d^P C^T,  W3^P = c_P D - 2 Z^P              (batched DGEMM)
#include <cmath>
#include <vector>

#include "df_grad_kernels.cuh"
#include "engine.h"

namespace m2 {

int grad_rhf_device(jk_engine* e, const double* dD, const double* dW, double precision, double* g2e, double* g1e,
                    cudaStream_t s, bool with_2e);
void launch_scale_K(int n, const double* K, const double* p, const double* alpha, double* K2a, double* K2b,
                    cudaStream_t s);
void nuclear_repulsion_grad(const jk_engine* e, std::vector<double>& gn);
PrimView prim_view(const jk_engine* e);

// gt_K = 2 sum_i bt[K](i,i)
__global__ void k_trace_bt(int naux, int o, const double* __restrict__ bt, double* __restrict__ g) {
  const int K = blockIdx.x * blockDim.x + threadIdx.x;
  if (K >= naux) return;
  double acc = 0.0;
  const double* b = bt + (size_t)K * o * o;
  for (int i = 0; i < o; ++i) acc += b[(size_t)i * o + i];
  g[K] = 2.0 * acc;
}

// W3[P] = c_P D - 2 Z[P], in place over n*n*naux elements
__global__ void k_w3(size_t nn, int naux, const double* __restrict__ c, const double* __restrict__ D,
                     double* __restrict__ Z) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn * naux) return;
  const int P = (int)(i / nn);
  Z[i] = c[P] * D[i % nn] - 2.0 * Z[i];
}

// 2 alpha K for the (P, unit) fitting primitives (alpha = p)
__global__ void k_scale_aux(int n, const double* __restrict__ K, const double* __restrict__ p,
                            double* __restrict__ K2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) K2[i] = 2.0 * p[i] * K[i];
}

static int cublas_fail(jk_engine* e, const char* what) { return set_error(e, JK_ERR_CUDA, what); }

// dC: n x nocc column-major occupied orbitals; dD = 2 C C^T; g2e receives
// the two-electron DF gradient (zeroed here).  Synchronises the stream.
int grad_df_2e_device(jk_engine* e, const double* dC, int nocc, const double* dD, double* g2e, cudaStream_t s) {
  DFState& d = e->df;
  const int n = e->obs.n_final, naux = d.naux, o = nocc, na = e->natom;
  const size_t nn = (size_t)n * n;
  for (int k = 0; k < e->aux.nshell; ++k)
    if (e->aux.atom[k] < 0 || e->aux.atom[k] >= na)
      return set_error(e, JK_ERR_ARG, "DF gradient: every fitting shell needs an owning atom (jk_basis.atom)");
  DevBuf<double> X, bt, c, W2, Z, K2a, K2b, ap2;
  cudaError_t st = X.alloc((size_t)n * naux * o);
  if (st == cudaSuccess) st = bt.alloc((size_t)o * o * naux);
  if (st == cudaSuccess) st = c.alloc(naux);
  if (st == cudaSuccess) st = W2.alloc((size_t)naux * naux);
  if (st == cudaSuccess) st = Z.alloc(nn * naux);
  if (st == cudaSuccess) st = K2a.alloc(e->pp_p.n);
  if (st == cudaSuccess) st = K2b.alloc(e->pp_p.n);
  if (st == cudaSuccess) st = ap2.alloc(e->ap_p.n);
  if (st != cudaSuccess) return check_cuda(e, st, "DF gradient allocation");
  const double one = 1.0, zero = 0.0, mhalf = -0.5;
  cublasSetStream(e->cublas, s);
  cublasHandle_t h = e->cublas;
  // X[x][K][i]: (o x n*naux) = C^T . B
  if (cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, o, n * naux, n, &one, dC, n, d.B64.p, n, &zero, X.p, o) !=
      CUBLAS_STATUS_SUCCESS)
    return cublas_fail(e, "DF gradient: X = B C");
  // bt[K] (o x o) = X_K (o x n, ld naux*o) . C (n x o)
  if (cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, o, o, n, &one, X.p, naux * o, (long long)o, dC, n, 0,
                                &zero, bt.p, o, (long long)o * o, naux) != CUBLAS_STATUS_SUCCESS)
    return cublas_fail(e, "DF gradient: C^T X");
  k_trace_bt<<<(naux + 127) / 128, 128, 0, s>>>(naux, o, bt.p, c.p);
  // c = L^-T gt;  d = bt L^-1 (bt as o^2 x naux)
  if (cublasDtrsv(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, naux, d.L.p, naux, c.p, 1) !=
      CUBLAS_STATUS_SUCCESS)
    return cublas_fail(e, "DF gradient: c = V^-1 gamma");
  if (cublasDtrsm(h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, o * o, naux, &one,
                  d.L.p, naux, bt.p, o * o) != CUBLAS_STATUS_SUCCESS)
    return cublas_fail(e, "DF gradient: d = V^-1 b");
  // W2 = d^T d - 1/2 c c^T
  if (cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, naux, naux, o * o, &one, bt.p, o * o, bt.p, o * o, &zero, W2.p,
                  naux) != CUBLAS_STATUS_SUCCESS ||
      cublasDger(h, naux, naux, &mhalf, c.p, 1, c.p, 1, W2.p, naux) != CUBLAS_STATUS_SUCCESS)
    return cublas_fail(e, "DF gradient: W2");
  // Y[P] = C d^P (n x o, reusing X), Z[P] = Y[P] C^T (n x n)
  if (cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, n, o, o, &one, dC, n, 0, bt.p, o, (long long)o * o,
                                &zero, X.p, n, (long long)n * o, naux) != CUBLAS_STATUS_SUCCESS ||
      cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_T, n, n, o, &one, X.p, n, (long long)n * o, dC, n, 0,
                                &zero, Z.p, n, (long long)nn, naux) != CUBLAS_STATUS_SUCCESS)
    return cublas_fail(e, "DF gradient: Z = C d C^T");
  k_w3<<<(unsigned)((nn * naux + 255) / 256), 256, 0, s>>>(nn, naux, c.p, dD, Z.p);
  // primitive weights of the shifted classes
  launch_scale_K((int)e->pp_p.n, e->pp_K.p, e->pp_p.p, e->pp_a.p, K2a.p, K2b.p, s);
  k_scale_aux<<<(unsigned)((e->ap_p.n + 255) / 256), 256, 0, s>>>((int)e->ap_p.n, e->ap_K.p, e->ap_p.p, ap2.p);
  cudaMemsetAsync(g2e, 0, sizeof(double) * 3 * na, s);
  const PrimView ap{e->ap_p.p, e->ap_x.p, e->ap_y.p, e->ap_z.p, e->ap_K.p};
  PrimView aps = ap;
  aps.K = ap2.p;
  // three-index derivatives
  for (int l = 0; l <= MAX_L_AUX; ++l) {
    if (!e->aux_by_l_count[l]) continue;
    for (int pc = 0; pc < NPAIRCLASS; ++pc) {
      if (!e->pcls[pc].npair) continue;
      Grad3Params P{};
      P.ap = ap;
      P.aux_shells = e->aux_by_l[l].p;
      P.naux_shells = e->aux_by_l_count[l];
      P.aux_prim_off = e->aux_prim_off.p;
      P.aux_nprim = e->daux.nprim.p;
      P.ax = e->daux.x.p;
      P.ay = e->daux.y.p;
      P.az = e->daux.z.p;
      P.aux_foff = e->daux.final_off.p;
      P.aux_pure = e->daux.pure.p;
      P.aux_atom = e->daux.atom.p;
      P.pairs = view(e->pcls[pc]);
      P.pp = prim_view(e);
      P.pp2a = P.pp;
      P.pp2a.K = K2a.p;
      P.pp2b = P.pp;
      P.pp2b.K = K2b.p;
      P.ox = e->dobs.x.p;
      P.oy = e->dobs.y.p;
      P.oz = e->dobs.z.p;
      P.obs_foff = e->dobs.final_off.p;
      P.obs_pure = e->dobs.pure.p;
      P.obs_atom = e->dobs.atom.p;
      P.sph_obs = e->dobs.sph.p;
      P.sph_aux = e->dobs.sph.p;
      P.boys = e->boys.p;
      P.n = n;
      P.W3 = Z.p;
      P.grad = g2e;
      if (l == 0) launch_grad3_l0(pc, P, s);
      if (l == 1) launch_grad3_l1(pc, P, s);
      if (l == 2) launch_grad3_l2(pc, P, s);
      if (l == 3) launch_grad3_l3(pc, P, s);
    }
  }
  // metric derivatives
  for (int lp = 0; lp <= MAX_L_AUX; ++lp)
    for (int lq = 0; lq <= MAX_L_AUX; ++lq) {
      if (!e->aux_by_l_count[lp] || !e->aux_by_l_count[lq]) continue;
      Grad2Params P{};
      P.ap = ap;
      P.ap2 = aps;
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
      P.aux_atom = e->daux.atom.p;
      P.sph = e->dobs.sph.p;
      P.boys = e->boys.p;
      P.naux = naux;
      P.W2 = W2.p;
      P.grad = g2e;
      launch_grad2(lp, lq, P, s);
    }
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);  // scratch dies on return
  return check_cuda(e, st, "DF gradient kernels");
}

}  // namespace m2

using namespace m2;

extern "C" int jk_grad_df(jk_engine* e, const double* Cocc, int nocc, const double* eps_occ, double* grad,
                          double* grad2e) {
  if (!e || !Cocc || !eps_occ || !grad) return JK_ERR_ARG;
  const int n = e->obs.n_final, na = e->natom;
  if (nocc <= 0 || nocc > n) return set_error(e, JK_ERR_ARG, "jk_grad_df: nocc out of range");
  if (e->df.k0 != 0 || (e->df.k1 >= 0 && e->df.k1 != e->aux.n_final))
    return set_error(e, JK_ERR_STATE, "jk_grad_df needs the whole fitting range (jk_df_set_range)");
  if (!e->df.ready) {
    int rc = df_setup(e);
    if (rc) return rc;
  }
  cudaStream_t s = e->stream;
  DevBuf<double> dC, dCe, dD, dW, g2, g1, dEps;
  cudaError_t st = dC.alloc((size_t)n * nocc);
  if (st == cudaSuccess) st = dCe.alloc((size_t)n * nocc);
  if (st == cudaSuccess) st = dD.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dW.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dEps.alloc(nocc);
  if (st == cudaSuccess) st = g2.alloc(3 * na);
  if (st == cudaSuccess) st = g1.alloc(3 * na);
  if (st == cudaSuccess) st = cudaMemcpyAsync(dC.p, Cocc, sizeof(double) * n * nocc, cudaMemcpyHostToDevice, s);
  if (st == cudaSuccess) st = cudaMemcpyAsync(dEps.p, eps_occ, sizeof(double) * nocc, cudaMemcpyHostToDevice, s);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_grad_df upload");
  // D = 2 C C^T, W = C diag(eps) C^T (src/rhfgrad.cpp:35-38)
  const double two = 2.0, one = 1.0, zero = 0.0;
  cublasSetStream(e->cublas, s);
  if (cublasDgemm(e->cublas, CUBLAS_OP_N, CUBLAS_OP_T, n, n, nocc, &two, dC.p, n, dC.p, n, &zero, dD.p, n) !=
          CUBLAS_STATUS_SUCCESS ||
      cublasDdgmm(e->cublas, CUBLAS_SIDE_RIGHT, n, nocc, dC.p, n, dEps.p, 1, dCe.p, n) != CUBLAS_STATUS_SUCCESS ||
      cublasDgemm(e->cublas, CUBLAS_OP_N, CUBLAS_OP_T, n, n, nocc, &one, dCe.p, n, dC.p, n, &zero, dW.p, n) !=
          CUBLAS_STATUS_SUCCESS)
    return set_error(e, JK_ERR_CUDA, "jk_grad_df: densities");
  int rc = grad_rhf_device(e, dD.p, dW.p, 0.0, nullptr, g1.p, s, false);
  if (rc) return rc;
  rc = grad_df_2e_device(e, dC.p, nocc, dD.p, g2.p, s);
  if (rc) return rc;
  std::vector<double> h2(3 * na), h1(3 * na), gn;
  st = cudaMemcpy(h2.data(), g2.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost);
  if (st == cudaSuccess) st = cudaMemcpy(h1.data(), g1.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_grad_df download");
  nuclear_repulsion_grad(e, gn);
  for (int i = 0; i < 3 * na; ++i) grad[i] = h1[i] + h2[i] + gn[i];
  if (grad2e)
    for (int i = 0; i < 3 * na; ++i) grad2e[i] = h2[i];
  return JK_OK;
}
