// Two-electron part of the superposition-of-atomic-densities (SOAD) guess:
// Fock::compute_2body_fock_general (molecular2 src/fockbuild.cpp:477-583),
//   G(1,2) = sum_{3,4 in dbs} 2 D(3,4) (12|34) - D(3,4) (13|24),
// for a density D given in a second basis (the minimal STO-3G basis of
// Fock::compute_soad_guess, src/fock.cpp:174-225).
//
// The integral-direct J/K build already evaluates every needed quartet if
// both bases are one basis: with the orbital shells first and the density
// shells after them, and D placed in the density-density block (zero
// elsewhere), J[D] and K[D] restricted to the orbital block are
// sum D(3,4)(12|34) and sum D(3,4)(13|24), so G = 2 J - K there.  Quartets
// whose six density blocks are all zero are dropped by the density screen.
// With shelldiag != 0 only the shell-diagonal blocks of D are kept, as the
// reference's D_is_shelldiagonal loop does (:516-517).
#include <vector>

#include "engine.h"

namespace m2 {
int direct_jk_device(jk_engine* e, const double* dD, double precision, double mult, double* dJ, double* dK,
                     cudaStream_t s);
}
using namespace m2;

extern "C" int jk_fock_general(const jk_basis* obs, const jk_basis* dbs, const double* D, int shelldiag,
                               double precision, int device, double* G) {
  if (!obs || !dbs || !D || !G || obs->nshell <= 0 || dbs->nshell <= 0) return JK_ERR_ARG;
  if (!(precision >= 0.0)) return JK_ERR_ARG;
  // one basis: orbital shells, then density shells
  const int ns1 = obs->nshell, ns2 = dbs->nshell, ns = ns1 + ns2;
  std::vector<int> l(ns), nprim(ns), poff(ns), pure(ns, 0);
  std::vector<double> exps, coefs, xyz(3 * (size_t)ns);
  auto add = [&](const jk_basis* b, int base) {
    for (int s = 0; s < b->nshell; ++s) {
      l[base + s] = b->l[s];
      nprim[base + s] = b->nprim[s];
      poff[base + s] = (int)exps.size();
      pure[base + s] = b->pure ? b->pure[s] : 0;
      for (int k = 0; k < 3; ++k) xyz[3 * (size_t)(base + s) + k] = b->xyz[3 * s + k];
      for (int p = 0; p < b->nprim[s]; ++p) {
        exps.push_back(b->exps[b->prim_off[s] + p]);
        coefs.push_back(b->coefs[b->prim_off[s] + p]);
      }
    }
  };
  if (!obs->l || !obs->nprim || !obs->prim_off || !obs->exps || !obs->coefs || !obs->xyz || !dbs->l ||
      !dbs->nprim || !dbs->prim_off || !dbs->exps || !dbs->coefs || !dbs->xyz)
    return JK_ERR_ARG;
  add(obs, 0);
  add(dbs, ns1);
  jk_basis comb{ns, l.data(), nprim.data(), poff.data(), exps.data(), coefs.data(), xyz.data(), pure.data(), nullptr};
  jk_engine* e = nullptr;
  int rc = jk_create(&comb, nullptr, 0, nullptr, nullptr, device, &e);
  if (rc) {
    jk_destroy(e);
    return rc;
  }
  const int n = e->obs.n_final, n1 = e->obs.off_final[ns1], n2 = n - n1;
  // function offsets of the density shells inside the density basis
  std::vector<int> shell_of(n2);
  for (int s = ns1; s < ns; ++s)
    for (int f = e->obs.off_final[s]; f < e->obs.off_final[s + 1]; ++f) shell_of[f - n1] = s;
  std::vector<double> Dc((size_t)n * n, 0.0);
  for (int j = 0; j < n2; ++j)
    for (int i = 0; i < n2; ++i)
      if (!shelldiag || shell_of[i] == shell_of[j]) Dc[(size_t)(n1 + j) * n + n1 + i] = D[(size_t)j * n2 + i];
  DevBuf<double> dD, dJ, dK;
  cudaError_t st = dD.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dJ.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dK.alloc((size_t)n * n);
  if (st == cudaSuccess)
    st = cudaMemcpyAsync(dD.p, Dc.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice, e->stream);
  if (st != cudaSuccess) {
    jk_destroy(e);
    return JK_ERR_CUDA;
  }
  rc = direct_jk_device(e, dD.p, precision, 1.0, dJ.p, dK.p, e->stream);
  std::vector<double> J((size_t)n * n), K((size_t)n * n);
  if (!rc) {
    st = cudaMemcpyAsync(J.data(), dJ.p, sizeof(double) * n * n, cudaMemcpyDeviceToHost, e->stream);
    if (st == cudaSuccess)
      st = cudaMemcpyAsync(K.data(), dK.p, sizeof(double) * n * n, cudaMemcpyDeviceToHost, e->stream);
    if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
    if (st != cudaSuccess) rc = JK_ERR_CUDA;
  }
  dD.reset();
  dJ.reset();
  dK.reset();
  jk_destroy(e);
  if (rc) return rc;
  for (int j = 0; j < n1; ++j)
    for (int i = 0; i < n1; ++i) G[(size_t)j * n1 + i] = 2.0 * J[(size_t)j * n + i] - K[(size_t)j * n + i];
  return JK_OK;
}
