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

// dC: n x nocc column-major occupied orbitals; dD = 2 C C^T; g2e receives
// the two-electron DF gradient (zeroed here).  Synchronises the stream.
int grad_df_2e_device(jk_engine* e, const double* dC, int nocc, const double* dD, double* g2e, cudaStream_t s) {
  DFState& d = e->df;
  if (e->tiled.ready) return grad_df_2e_tiled(e, dC, nocc, dD, g2e, s);
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
int grad_df_2e_tiled(jk_engine* e, const double*, int, const double*, double*, cudaStream_t) {
  return set_error(e, JK_ERR_STATE, "DF gradient with tiled storage: not available yet");
}
}  // namespace m2
