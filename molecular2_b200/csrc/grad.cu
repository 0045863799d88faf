// RHF nuclear gradient on the device: the B200 replacement for
// Fock::compute_forces (molecular2 src/rhfgrad.cpp:15-89) with
// compute_2body_fock_deriv<1> (:419-598) and the one-body derivative
// integrals (inc/integrals.hpp:169-349).
//   grad = (T' + V') . D - 2 S' . W + 1/4 G'(D) . D + nuclear repulsion
// with D the full density, W = Cocc diag(eps_occ) Cocc^T.  The two-electron
// term runs over the same unique shell quartets as the reference: both shell
// pairs in the overlap-screened pair list (|S block| >= 1e-12 or same centre,
// src/integrals.cpp:515-566) and max6(|D| blocks) Q_ab Q_cd >= precision.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "engine.h"
#include "grad_kernels.cuh"

namespace m2 {

PrimView prim_view(const jk_engine* e);
ShellView shell_view(const jk_engine* e);

// significance of each pair of one class from the final-basis overlap matrix
__global__ void k_pair_sig(PairView pairs, const int* __restrict__ foff, const double* __restrict__ x,
                           const double* __restrict__ y, const double* __restrict__ z, const double* __restrict__ S,
                           int n, unsigned char* __restrict__ sig) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pairs.npair) return;
  const int a = pairs.sa[i], b = pairs.sb[i];
  const bool same = x[a] == x[b] && y[a] == y[b] && z[a] == z[b];
  double s2 = 0.0;
  for (int p = foff[a]; p < foff[a + 1]; ++p)
    for (int q = foff[b]; q < foff[b + 1]; ++q) s2 += S[(size_t)q * n + p] * S[(size_t)q * n + p];
  sig[i] = (same || sqrt(s2) >= 1e-12) ? 1 : 0;
}

__global__ void k_scale_K(int n, const double* __restrict__ K, const double* __restrict__ p,
                          const double* __restrict__ alpha, double* __restrict__ K2a, double* __restrict__ K2b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  K2a[i] = 2.0 * alpha[i] * K[i];
  K2b[i] = 2.0 * (p[i] - alpha[i]) * K[i];
}

// kets per 64-thread block: one per thread, halved for classes with few bra
// pairs so that their blocks still spread over the SMs
static void launch_grad2e(const jk_engine* e, int A, int B, const Grad2eParams& Pin, int nbra, int nket,
                          cudaStream_t s) {
  Grad2eParams P = Pin;
  int nb = 0;
  bra_share(e, nbra, P.bra0, P.bra_step, nb);
  if (nb == 0) return;
  P.kchunk = 64;
  if ((long long)nb * ((nket + 63) / 64) < 4 * 148) P.kchunk = 32;
  dim3 grid(nb, (nket + P.kchunk - 1) / P.kchunk, 6);  // z: the six shifted classes
  if (A <= 2)
    launch_grad2e_bra_s(A, B, P, grid, s);
  else if (A == 3)
    launch_grad2e_bra_ds(B, P, grid, s);
  else if (A == 4)
    launch_grad2e_bra_dp(B, P, grid, s);
  else
    launch_grad2e_bra_dd(B, P, grid, s);
}

void launch_scale_K(int n, const double* K, const double* p, const double* alpha, double* K2a, double* K2b,
                    cudaStream_t s) {
  k_scale_K<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, K, p, alpha, K2a, K2b);
}

// dE_nuc/dx, natom x 3 (src/rhfgrad.cpp:59-86)
void nuclear_repulsion_grad(const jk_engine* e, std::vector<double>& gn) {
  const int na = e->natom;
  gn.assign(3 * (size_t)na, 0.0);
  for (int a1 = 1; a1 < na; ++a1)
    for (int a2 = 0; a2 < a1; ++a2) {
      double r[3], r2 = 0.0;
      for (int k = 0; k < 3; ++k) {
        r[k] = e->atom_xyz[3 * a1 + k] - e->atom_xyz[3 * a2 + k];
        r2 += r[k] * r[k];
      }
      const double f = e->Z[a1] * e->Z[a2] / (r2 * std::sqrt(r2));
      for (int k = 0; k < 3; ++k) {
        gn[3 * a1 + k] -= r[k] * f;
        gn[3 * a2 + k] += r[k] * f;
      }
    }
}

// dD, dW final-basis n x n on the device; g2e/g1e (3*natom) device
// accumulators, zeroed here (g2e only when with_2e).  Synchronises the stream
// before returning.
int grad_rhf_device(jk_engine* e, const double* dD, const double* dW, double precision, double* g2e, double* g1e,
                    cudaStream_t s, bool with_2e) {
  const int n = e->obs.n_final, nc = e->obs.n_cart, ns = e->obs.nshell, na = e->natom;
  for (int k = 0; k < ns; ++k)
    if (e->obs.atom[k] < 0 || e->obs.atom[k] >= na)
      return set_error(e, JK_ERR_ARG, "gradient: every shell needs an owning atom (jk_basis.atom)");
  const size_t npp = e->pp_p.n;
  DevBuf<double> S, T, V, Dc, Wc, Dn, Dmax, K2a, K2b, Z, C;
  DevBuf<int> atom;
  DevBuf<unsigned char> sig[NPAIRCLASS];
  cudaError_t st = cudaSuccess;
  for (auto* b : {&S, &T, &V})
    if (st == cudaSuccess) st = b->alloc((size_t)n * n);
  if (st == cudaSuccess) st = Dc.alloc((size_t)nc * nc);
  if (st == cudaSuccess) st = Wc.alloc((size_t)nc * nc);
  if (st == cudaSuccess) st = Dn.alloc((size_t)ns * ns);
  if (st == cudaSuccess) st = Dmax.alloc(2);
  if (st == cudaSuccess) st = K2a.alloc(npp);
  if (st == cudaSuccess) st = K2b.alloc(npp);
  if (st == cudaSuccess) st = atom.upload(e->obs.atom, s);
  if (st == cudaSuccess) st = Z.upload(e->Z, s);
  if (st == cudaSuccess) st = C.upload(e->atom_xyz, s);
  for (int k = 0; k < NPAIRCLASS && st == cudaSuccess; ++k)
    if (e->pcls[k].npair) st = sig[k].alloc(e->pcls[k].npair);
  if (st != cudaSuccess) return check_cuda(e, st, "gradient allocation");
  int rc = one_body_device(e, S.p, T.p, V.p, s);
  if (rc) return rc;
  for (int k = 0; k < NPAIRCLASS; ++k)
    if (e->pcls[k].npair)
      k_pair_sig<<<(e->pcls[k].npair + 127) / 128, 128, 0, s>>>(view(e->pcls[k]), e->dobs.final_off.p, e->dobs.x.p,
                                                               e->dobs.y.p, e->dobs.z.p, S.p, n, sig[k].p);
  k_scale_K<<<(unsigned)((npp + 255) / 256), 256, 0, s>>>((int)npp, e->pp_K.p, e->pp_p.p, e->pp_a.p, K2a.p, K2b.p);
  launch_shell_norms(e, dD, Dn.p, Dmax.p, s);
  launch_final_to_cart(e, dD, Dc.p, s);
  launch_final_to_cart(e, dW, Wc.p, s);
  if (with_2e) cudaMemsetAsync(g2e, 0, sizeof(double) * 3 * na, s);
  cudaMemsetAsync(g1e, 0, sizeof(double) * 3 * na, s);
  Grad2eParams P{};
  P.pp = prim_view(e);
  P.pp2a = P.pp;
  P.pp2a.K = K2a.p;
  P.pp2b = P.pp;
  P.pp2b.K = K2b.p;
  P.sh = shell_view(e);
  P.atom = atom.p;
  P.Dnorm = Dn.p;
  P.nshell = ns;
  P.Dmax = Dmax.p;
  P.Dc = Dc.p;
  P.nc = nc;
  P.precision = precision;
  P.boys = e->boys.p;
  P.grad = g2e;
  P.kchunk = 64;  // one ket per thread (64-thread blocks)
  // the class launches run on the engine's side streams, longest first (the
  // gradient is accumulated with atomics, so they commute)
  static const double ncp[6] = {1, 3, 9, 6, 18, 36};
  struct Item {
    int A, B;
    double cost;
  };
  std::vector<Item> items;
  for (int A = 0; A < NPAIRCLASS && with_2e; ++A)
    for (int B = 0; B <= A; ++B)
      if (e->pcls[A].npair && e->pcls[B].npair)
        items.push_back({A, B, (double)e->pcls[A].npair * e->pcls[B].npair * ncp[A] * ncp[B] * (A == B ? 0.5 : 1.0)});
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.cost > b.cost; });
  ClassStreams cs(e, s);
  for (const Item& it : items) {
    Grad2eParams Q = P;
    Q.bra = view(e->pcls[it.A]);
    Q.ket = view(e->pcls[it.B]);
    Q.bra_sig = sig[it.A].p;
    Q.ket_sig = sig[it.B].p;
    Q.same_class = (it.A == it.B);
    launch_grad2e(e, it.A, it.B, Q, e->pcls[it.A].npair, e->pcls[it.B].npair, cs.next(it.cost));
  }
  cs.join();
  // one-body terms: whole on the first rank of a partition, none on the others
  const bool with_1e = !(e->part_active && e->part_rank != 0);
  for (int k = 0; k < NPAIRCLASS && with_1e; ++k) {
    if (!e->pcls[k].npair) continue;
    Grad1eParams Q{};
    Q.pairs = view(e->pcls[k]);
    Q.pp = prim_view(e);
    Q.pa = e->pp_a.p;
    Q.ox = e->dobs.x.p;
    Q.oy = e->dobs.y.p;
    Q.oz = e->dobs.z.p;
    Q.coff = e->dobs.cart_off.p;
    Q.atom = atom.p;
    Q.sig = sig[k].p;
    Q.Dc = Dc.p;
    Q.Wc = Wc.p;
    Q.nc = nc;
    Q.boys = e->boys.p;
    Q.natom = na;
    Q.Z = Z.p;
    Q.cxyz = C.p;
    Q.grad = g1e;
    launch_grad1e(k, Q, s);
  }
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);  // scratch dies on return
  return check_cuda(e, st, "gradient kernels");
}

}  // namespace m2

using namespace m2;

extern "C" int jk_grad_rhf(jk_engine* e, const double* D, const double* W, double precision, double* grad,
                           double* grad2e) {
  if (!e || !D || !W || !grad) return JK_ERR_ARG;
  const int n = e->obs.n_final, na = e->natom;
  DevBuf<double> dD, dW, g2, g1;
  cudaError_t st = dD.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dW.alloc((size_t)n * n);
  if (st == cudaSuccess) st = g2.alloc(3 * na);
  if (st == cudaSuccess) st = g1.alloc(3 * na);
  if (st == cudaSuccess) st = cudaMemcpyAsync(dD.p, D, sizeof(double) * n * n, cudaMemcpyHostToDevice, e->stream);
  if (st == cudaSuccess) st = cudaMemcpyAsync(dW.p, W, sizeof(double) * n * n, cudaMemcpyHostToDevice, e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_grad_rhf upload");
  const bool first = e->part_rank == 0;
  int rc;
  {
    PartitionScope part(e);
    rc = grad_rhf_device(e, dD.p, dW.p, precision, g2.p, g1.p, e->stream, true);
  }
  if (rc) return rc;
  std::vector<double> h2(3 * na), h1(3 * na);
  st = cudaMemcpy(h2.data(), g2.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost);
  if (st == cudaSuccess) st = cudaMemcpy(h1.data(), g1.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_grad_rhf download");
  std::vector<double> gn;
  nuclear_repulsion_grad(e, gn);
  if (!first) std::fill(gn.begin(), gn.end(), 0.0);  // the first rank adds it
  for (int i = 0; i < 3 * na; ++i) grad[i] = h1[i] + h2[i] + gn[i];
  if (grad2e)
    for (int i = 0; i < 3 * na; ++i) grad2e[i] = h2[i];
  return JK_OK;
}
