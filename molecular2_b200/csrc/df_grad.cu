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
#include "dense.cuh"
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

// Ce = C diag(eps), C column-major n x o
__global__ void k_scale_cols(int n, int o, const double* __restrict__ C, const double* __restrict__ eps,
                             double* __restrict__ Ce) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < (size_t)n * o) Ce[idx] = C[idx] * eps[idx / n];
}

int grad_df_2e_tiled(jk_engine* e, const double* dC, int nocc, const double* dD, double* g2e, cudaStream_t s);

// k_grad3 over every orbital pair class for the fitting shells `shells` (all
// of angular momentum l) with W3 holding fitting functions from w3_f0 on.
static void launch_grad3_all(jk_engine* e, int l, const int* shells, int nshells, const double* W3, int w3_f0,
                             const double* K2a, const double* K2b, double* g2e, cudaStream_t s) {
  const PrimView ap{e->ap_p.p, e->ap_x.p, e->ap_y.p, e->ap_z.p, e->ap_K.p};
  for (int pc = 0; pc < NPAIRCLASS; ++pc) {
    if (!e->pcls[pc].npair) continue;
    Grad3Params P{};
    P.ap = ap;
    P.aux_shells = shells;
    P.naux_shells = nshells;
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
    P.pp2a.K = K2a;
    P.pp2b = P.pp;
    P.pp2b.K = K2b;
    P.ox = e->dobs.x.p;
    P.oy = e->dobs.y.p;
    P.oz = e->dobs.z.p;
    P.obs_foff = e->dobs.final_off.p;
    P.obs_pure = e->dobs.pure.p;
    P.obs_atom = e->dobs.atom.p;
    P.sph_obs = e->dobs.sph.p;
    P.sph_aux = e->dobs.sph.p;
    P.boys = e->boys.p;
    P.n = e->obs.n_final;
    P.W3 = W3;
    P.w3_f0 = w3_f0;
    P.grad = g2e;
    if (l == 0) launch_grad3_l0(pc, P, s);
    if (l == 1) launch_grad3_l1(pc, P, s);
    if (l == 2) launch_grad3_l2(pc, P, s);
    if (l == 3) launch_grad3_l3(pc, P, s);
  }
}

// k_grad2 over every pair of fitting angular momenta with the weights W2.
static void launch_grad2_all(jk_engine* e, const double* ap2K, const double* W2, double* g2e, cudaStream_t s) {
  const PrimView ap{e->ap_p.p, e->ap_x.p, e->ap_y.p, e->ap_z.p, e->ap_K.p};
  PrimView aps = ap;
  aps.K = ap2K;
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
      P.naux = e->aux.n_final;
      P.W2 = W2;
      P.grad = g2e;
      launch_grad2(lp, lq, P, s);
    }
}


// dC: n x nocc column-major occupied orbitals; dD = 2 C C^T; g2e receives
// the two-electron DF gradient (zeroed here).  Synchronises the stream.
int grad_df_2e_device(jk_engine* e, const double* dC, int nocc, const double* dD, double* g2e, cudaStream_t s) {
  DFState& d = e->df;
  if (e->tiled.metric_ready || (!d.ready && df_use_tiled(e))) return grad_df_2e_tiled(e, dC, nocc, dD, g2e, s);
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
  if (!d.Linv.p) return set_error(e, JK_ERR_STATE, "DF gradient: L^-1 missing (run jk_df_setup)");
  DevBuf<double> dd, gt;
  st = dd.alloc((size_t)o * o * naux);
  if (st == cudaSuccess) st = gt.alloc(naux);
  if (st != cudaSuccess) return check_cuda(e, st, "DF gradient allocation");
  auto gemm = [&](const DGemm& g, const char* what) {
    const cudaError_t r = dgemm(g, s);
    return r == cudaSuccess ? JK_OK : check_cuda(e, r, what);
  };
  int rc;
  // X[x][K][i] = sum_y B[x][K][y] C[y][i]
  {
    DGemm g;
    g.M = n * naux; g.N = o; g.K = n;
    g.A = d.B64.p; g.sam = n; g.sak = 1;
    g.B = dC; g.sbk = 1; g.sbn = n;
    g.C = X.p; g.scm = o; g.scn = 1;
    if ((rc = gemm(g, "DF gradient: X = B C"))) return rc;
  }
  // bt[K](i, j) = sum_x X[x][K][i] C[x][j]   (o x o, column-major, per K)
  {
    DGemm g;
    g.M = o; g.N = o; g.K = n; g.batch = naux;
    g.A = X.p; g.sam = 1; g.sak = (long long)naux * o; g.bsa = o;
    g.B = dC; g.sbk = 1; g.sbn = n;
    g.C = bt.p; g.scm = 1; g.scn = o; g.bsc = (long long)o * o;
    if ((rc = gemm(g, "DF gradient: C^T X"))) return rc;
  }
  k_trace_bt<<<(naux + 127) / 128, 128, 0, s>>>(naux, o, bt.p, gt.p);
  // c = L^-T gamma
  {
    DGemm g;
    g.M = naux; g.N = 1; g.K = naux;
    g.A = d.Linv.p; g.sam = naux; g.sak = 1;
    g.B = gt.p; g.sbk = 1; g.sbn = 0;
    g.C = c.p; g.scm = 1; g.scn = 0;
    if ((rc = gemm(g, "DF gradient: c = V^-1 gamma"))) return rc;
  }
  // d (o^2 x naux) = bt L^-1
  {
    DGemm g;
    g.M = o * o; g.N = naux; g.K = naux;
    g.A = bt.p; g.sam = 1; g.sak = (long long)o * o;
    g.B = d.Linv.p; g.sbk = 1; g.sbn = naux; g.b_lower = true;
    g.C = dd.p; g.scm = 1; g.scn = (long long)o * o;
    if ((rc = gemm(g, "DF gradient: d = V^-1 b"))) return rc;
  }
  // W2 = d^T d - 1/2 c c^T
  {
    DGemm g;
    g.M = naux; g.N = naux; g.K = o * o;
    g.A = dd.p; g.sam = (long long)o * o; g.sak = 1;
    g.B = dd.p; g.sbk = 1; g.sbn = (long long)o * o;
    g.C = W2.p; g.scm = 1; g.scn = naux;
    if ((rc = gemm(g, "DF gradient: W2"))) return rc;
    DGemm r;
    r.M = naux; r.N = naux; r.K = 1;
    r.A = c.p; r.sam = 1; r.sak = 0;
    r.B = c.p; r.sbk = 0; r.sbn = 1;
    r.C = W2.p; r.scm = 1; r.scn = naux;
    r.alpha = -0.5; r.beta = 1.0;
    if ((rc = gemm(r, "DF gradient: W2"))) return rc;
  }
  // Y[P] = C d^P (n x o, reusing X), Z[P] = Y[P] C^T (n x n)
  {
    DGemm g;
    g.M = n; g.N = o; g.K = o; g.batch = naux;
    g.A = dC; g.sam = 1; g.sak = n;
    g.B = dd.p; g.sbk = 1; g.sbn = o; g.bsb = (long long)o * o;
    g.C = X.p; g.scm = 1; g.scn = n; g.bsc = (long long)n * o;
    if ((rc = gemm(g, "DF gradient: Y = C d"))) return rc;
    DGemm z;
    z.M = n; z.N = n; z.K = o; z.batch = naux;
    z.A = X.p; z.sam = 1; z.sak = n; z.bsa = (long long)n * o;
    z.B = dC; z.sbk = n; z.sbn = 1;
    z.C = Z.p; z.scm = 1; z.scn = n; z.bsc = (long long)nn;
    if ((rc = gemm(z, "DF gradient: Z = Y C^T"))) return rc;
  }
  k_w3<<<(unsigned)((nn * naux + 255) / 256), 256, 0, s>>>(nn, naux, c.p, dD, Z.p);
  // primitive weights of the shifted classes
  launch_scale_K((int)e->pp_p.n, e->pp_K.p, e->pp_p.p, e->pp_a.p, K2a.p, K2b.p, s);
  k_scale_aux<<<(unsigned)((e->ap_p.n + 255) / 256), 256, 0, s>>>((int)e->ap_p.n, e->ap_K.p, e->ap_p.p, ap2.p);
  cudaMemsetAsync(g2e, 0, sizeof(double) * 3 * na, s);
  // three-index derivatives
  for (int l = 0; l <= MAX_L_AUX; ++l)
    if (e->aux_by_l_count[l]) launch_grad3_all(e, l, e->aux_by_l[l].p, e->aux_by_l_count[l], Z.p, 0, K2a.p, K2b.p, g2e, s);
  // metric derivatives
  launch_grad2_all(e, ap2.p, W2.p, g2e, s);
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
  // tiled storage needs only the metric (df_tiled_metric, from the gradient itself)
  if (!e->df.ready && !e->tiled.metric_ready && !df_use_tiled(e)) {
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
  {
    DGemm g;
    g.M = n; g.N = n; g.K = nocc; g.alpha = 2.0;
    g.A = dC.p; g.sam = 1; g.sak = n;
    g.B = dC.p; g.sbk = n; g.sbn = 1;
    g.C = dD.p; g.scm = 1; g.scn = n;
    st = dgemm(g, s);
    if (st == cudaSuccess) {
      k_scale_cols<<<(unsigned)(((size_t)n * nocc + 255) / 256), 256, 0, s>>>(n, nocc, dC.p, dEps.p, dCe.p);
      g.alpha = 1.0;
      g.A = dCe.p;
      g.C = dW.p;
      st = dgemm(g, s);
    }
    if (st != cudaSuccess) return check_cuda(e, st, "jk_grad_df: densities");
  }
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

namespace m2 {

// The same gradient for tiled DF storage, where neither B nor (P|mn) is kept:
// one streamed pass gives X'[x][P][i] = sum_y (P|xy) C[y][i] in occupied
// slices, hence b'[P] = C^T (P|..) C and b[K] = sum_P L^-1[K][P] b'[P]; the
// rest follows the unpacked path, with W3 formed and contracted one block of
// fitting shells at a time (W3 for all of them would be n^2 naux doubles).
int grad_df_2e_tiled(jk_engine* e, const double* dC, int nocc, const double* dD, double* g2e, cudaStream_t s) {
  int rc = df_tiled_metric(e);
  if (rc) return rc;
  DFState& d = e->df;
  TiledDF& T = e->tiled;
  const int n = e->obs.n_final, naux = e->aux.n_final, o = nocc, na = e->natom, npad = T.npad;
  const size_t nn = (size_t)n * n, oo = (size_t)o * o;
  for (int k = 0; k < e->aux.nshell; ++k)
    if (e->aux.atom[k] < 0 || e->aux.atom[k] >= na)
      return set_error(e, JK_ERR_ARG, "DF gradient: every fitting shell needs an owning atom (jk_basis.atom)");
  DevBuf<double> btp, bt, dd, gt, c, W2, Cp, Tt, K2a, K2b, ap2;
  cudaError_t st = btp.alloc(oo * naux);
  if (st == cudaSuccess) st = dd.alloc(oo * naux);
  if (st == cudaSuccess) st = gt.alloc(naux);
  if (st == cudaSuccess) st = c.alloc(naux);
  if (st == cudaSuccess) st = W2.alloc((size_t)naux * naux);
  if (st == cudaSuccess) st = Cp.alloc((size_t)npad * o);
  if (st == cudaSuccess) st = Tt.alloc((size_t)DF_TILE * naux * DF_TILE);
  if (st == cudaSuccess) st = K2a.alloc(e->pp_p.n);
  if (st == cudaSuccess) st = K2b.alloc(e->pp_p.n);
  if (st == cudaSuccess) st = ap2.alloc(e->ap_p.n);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled DF gradient allocation");
  auto gemm = [&](const DGemm& g, const char* what) {
    const cudaError_t r = dgemm(g, s);
    return r == cudaSuccess ? JK_OK : check_cuda(e, r, what);
  };
  launch_pad_rows(n, npad, o, dC, Cp.p, s);
  {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    int oc = (int)std::min<double>(o, std::floor(0.8 * (double)fr / (8.0 * npad * naux)));
    if (oc < 1) return set_error(e, JK_ERR_NOMEM, "tiled DF gradient: no room for X'");
    const int nch = (o + oc - 1) / oc;
    oc = (o + nch - 1) / nch;
    DevBuf<double> X;
    if ((st = X.alloc((size_t)npad * naux * oc)) != cudaSuccess) return check_cuda(e, st, "tiled DF gradient X'");
    for (int ch = 0; ch < nch; ++ch) {
      const int i0 = ch * oc, ocur = std::min(oc, o - i0);
      if ((rc = tiled_xprime_pass(e, Cp.p, i0, ocur, X.p, Tt.p, s, nullptr))) return rc;
      DGemm g;  // b'[P](i, j) = sum_x C[x][i] X'[x][P][j]
      g.M = o; g.N = ocur; g.K = n; g.batch = naux;
      g.A = dC; g.sam = n; g.sak = 1;
      g.B = X.p; g.sbk = (long long)naux * ocur; g.sbn = 1; g.bsb = ocur;
      g.C = btp.p + (size_t)i0 * o; g.scm = 1; g.scn = o; g.bsc = (long long)oo;
      if ((rc = gemm(g, "tiled DF gradient: C^T X'"))) return rc;
    }
  }
  Tt.reset();
  if ((st = bt.alloc(oo * naux)) != cudaSuccess) return check_cuda(e, st, "tiled DF gradient b");
  {
    DGemm g;  // b (o^2 x naux) = b' L^-T
    g.M = (int)oo; g.N = naux; g.K = naux;
    g.A = btp.p; g.sam = 1; g.sak = (long long)oo;
    g.B = d.Linv.p; g.sbk = naux; g.sbn = 1;
    g.C = bt.p; g.scm = 1; g.scn = (long long)oo;
    if ((rc = gemm(g, "tiled DF gradient: b = b' L^-T"))) return rc;
  }
  btp.reset();
  k_trace_bt<<<(naux + 127) / 128, 128, 0, s>>>(naux, o, bt.p, gt.p);
  {
    DGemm g;  // c = L^-T gamma
    g.M = naux; g.N = 1; g.K = naux;
    g.A = d.Linv.p; g.sam = naux; g.sak = 1;
    g.B = gt.p; g.sbk = 1; g.sbn = 0;
    g.C = c.p; g.scm = 1; g.scn = 0;
    if ((rc = gemm(g, "tiled DF gradient: c"))) return rc;
    DGemm h;  // d = b L^-1
    h.M = (int)oo; h.N = naux; h.K = naux;
    h.A = bt.p; h.sam = 1; h.sak = (long long)oo;
    h.B = d.Linv.p; h.sbk = 1; h.sbn = naux; h.b_lower = true;
    h.C = dd.p; h.scm = 1; h.scn = (long long)oo;
    if ((rc = gemm(h, "tiled DF gradient: d"))) return rc;
  }
  bt.reset();
  {
    DGemm g;  // W2 = d^T d - 1/2 c c^T
    g.M = naux; g.N = naux; g.K = (int)oo;
    g.A = dd.p; g.sam = (long long)oo; g.sak = 1;
    g.B = dd.p; g.sbk = 1; g.sbn = (long long)oo;
    g.C = W2.p; g.scm = 1; g.scn = naux;
    if ((rc = gemm(g, "tiled DF gradient: W2"))) return rc;
    DGemm r;
    r.M = naux; r.N = naux; r.K = 1;
    r.A = c.p; r.sam = 1; r.sak = 0;
    r.B = c.p; r.sbk = 0; r.sbn = 1;
    r.C = W2.p; r.scm = 1; r.scn = naux;
    r.alpha = -0.5; r.beta = 1.0;
    if ((rc = gemm(r, "tiled DF gradient: W2"))) return rc;
  }
  launch_scale_K((int)e->pp_p.n, e->pp_K.p, e->pp_p.p, e->pp_a.p, K2a.p, K2b.p, s);
  k_scale_aux<<<(unsigned)((e->ap_p.n + 255) / 256), 256, 0, s>>>((int)e->ap_p.n, e->ap_K.p, e->ap_p.p, ap2.p);
  cudaMemsetAsync(g2e, 0, sizeof(double) * 3 * na, s);
  // W3 = c_P D - 2 C d^P C^T and its contraction, one block of fitting shells at a time
  {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    const double per_f = 8.0 * ((double)nn + (double)n * o);
    const int wmax = (int)std::max(16.0, std::min<double>(naux, 0.6 * (double)fr / per_f));
    DevBuf<double> Y, Z;
    if ((st = Y.alloc((size_t)n * o * wmax)) == cudaSuccess) st = Z.alloc(nn * wmax);
    if (st != cudaSuccess) return check_cuda(e, st, "tiled DF gradient W3 block");
    const HostBasis& ab = e->aux;
    DevBuf<int> lists[MAX_L_AUX + 1];
    for (int s0 = 0; s0 < ab.nshell;) {
      int s1 = s0;
      while (s1 < ab.nshell && ab.off_final[s1 + 1] - ab.off_final[s0] <= wmax) ++s1;
      if (s1 == s0) return set_error(e, JK_ERR_ARG, "tiled DF gradient: fitting shell wider than the block");
      const int f0 = ab.off_final[s0], w = ab.off_final[s1] - f0;
      DGemm y;  // Y[P] = C d^P (n x o)
      y.M = n; y.N = o; y.K = o; y.batch = w;
      y.A = dC; y.sam = 1; y.sak = n;
      y.B = dd.p + (size_t)f0 * oo; y.sbk = 1; y.sbn = o; y.bsb = (long long)oo;
      y.C = Y.p; y.scm = 1; y.scn = n; y.bsc = (long long)n * o;
      if ((rc = gemm(y, "tiled DF gradient: Y = C d"))) return rc;
      DGemm z;  // Z[P] = Y[P] C^T (n x n)
      z.M = n; z.N = n; z.K = o; z.batch = w;
      z.A = Y.p; z.sam = 1; z.sak = n; z.bsa = (long long)n * o;
      z.B = dC; z.sbk = n; z.sbn = 1;
      z.C = Z.p; z.scm = 1; z.scn = n; z.bsc = (long long)nn;
      if ((rc = gemm(z, "tiled DF gradient: Z = Y C^T"))) return rc;
      k_w3<<<(unsigned)((nn * w + 255) / 256), 256, 0, s>>>(nn, w, c.p + f0, dD, Z.p);
      for (int l = 0; l <= MAX_L_AUX; ++l) {
        std::vector<int> sh;
        for (int k = s0; k < s1; ++k)
          if (ab.l[k] == l) sh.push_back(k);
        if (sh.empty()) continue;
        if ((st = lists[l].upload(sh, s)) != cudaSuccess) return check_cuda(e, st, "tiled DF gradient shells");
        launch_grad3_all(e, l, lists[l].p, (int)sh.size(), Z.p, f0, K2a.p, K2b.p, g2e, s);
      }
      st = cudaStreamSynchronize(s);  // Y, Z and the shell lists are reused by the next block
      if (st != cudaSuccess) return check_cuda(e, st, "tiled DF gradient block");
      s0 = s1;
    }
  }
  launch_grad2_all(e, ap2.p, W2.p, g2e, s);
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);
  return check_cuda(e, st, "tiled DF gradient kernels");
}

}  // namespace m2
