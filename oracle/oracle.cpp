// FP64 CPU oracle for the J/K Fock build — TEST INFRASTRUCTURE ONLY.
//
// This file is the parity checker for the CUDA engine in molecular2_b200.
// Only tests/, the smoke check in __graft_entry__.py and bench.py's
// cpu_baseline / --impl reference leg may load it; the product never does.
//
// It restates, in scalar C++ with no third-party code, the molecular2 hot path:
//   * Fock::formJKdirect            src/fockbuild.cpp:64-164
//   * Fock::compute_2body_fock_df   src/fockbuild.cpp:585-660
//   * Fock::compute_2body_fock_general (SOAD G)  src/fockbuild.cpp:477-583
//   * IntegralEngine::compute_eris_3index / _2index  src/eris.cpp:89-156, 304-356
//   * compute_schwarz_ints / compute_shellblock_norm / compute_shellpair_list
//                                    src/integrals.cpp:451-566
//   * Fock::compute_2body_fock_deriv<1>  src/rhfgrad.cpp:419-598
//   * compute_1body_ints(_deriv)     src/integrals.cpp:394-449, inc/integrals.hpp:169-349
// The integral arithmetic molecular2 takes from libint2 2.3.0-beta.3 (not
// vendored) is restated from the published methods instead of libint source:
//   * Obara & Saika, J. Chem. Phys. 84, 3963 (1986): vertical recursion;
//   * Head-Gordon & Pople, J. Chem. Phys. 89, 5777 (1988): horizontal recursion;
//   * Boys function by its convergent series (small T) and the erf closed form
//     with upward recursion (large T);
//   * real solid harmonics from the Cartesian recursion of Helgaker, Jorgensen
//     & Olsen, "Molecular Electronic-Structure Theory" eqs. 6.4.70-6.4.73,
//     normalised numerically.
// Conventions (shared with the CUDA engine; libint2's documented defaults):
//   Cartesian order  for a=l..0, b=l-a..0: x^a y^b z^(l-a-b)
//   pure order       m = -l..l, pure only for l >= 2 when a shell is flagged pure
//   normalisation    contracted x^l component has unit norm, every Cartesian
//                    component shares the same coefficients (libint2 Shell).
// Matrices are column-major n x n like Eigen::MatrixXd (all J/K/D symmetric).

#include <cmath>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <array>
#include <algorithm>
#include <thread>
#include <mutex>

namespace {

constexpr int LMAXC = 9;  // max Cartesian angular momentum handled by tables

double dfact(int n) {  // n!!, with (-1)!! = 1
  double r = 1.0;
  for (int k = n; k > 1; k -= 2) r *= k;
  return r;
}

int ncart(int l) { return (l + 1) * (l + 2) / 2; }
int ncum(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }  // #cart fns with total <= l

struct CartTables {
  std::vector<std::array<int, 3>> comp[LMAXC + 1];
  int gid[LMAXC + 1][LMAXC + 1][LMAXC + 1];  // global index over all totals
  int lid[LMAXC + 1][LMAXC + 1][LMAXC + 1];  // index within its total l
  std::vector<std::array<int, 3>> gcomp;     // global index -> exponents
  CartTables() {
    for (int l = 0; l <= LMAXC; ++l)
      for (int a = l; a >= 0; --a)
        for (int b = l - a; b >= 0; --b) {
          int c = l - a - b;
          lid[a][b][c] = (int)comp[l].size();
          comp[l].push_back({a, b, c});
          gid[a][b][c] = (int)gcomp.size();
          gcomp.push_back({a, b, c});
        }
  }
};
const CartTables& CT() {
  static CartTables t;
  return t;
}

// ---------------------------------------------------------------- Boys
void boys(int mmax, double T, double* F) {
  if (T < 40.0) {
    // F_m(T) = exp(-T) * sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)); evaluate
    // the highest order by the series, then recur downward (stable).
    double term = 1.0 / (2 * mmax + 1), sum = term;
    for (int k = 1; k < 400; ++k) {
      term *= 2.0 * T / (2 * mmax + 2 * k + 1);
      sum += term;
      if (term < 1e-17 * sum) break;
    }
    double e = std::exp(-T);
    F[mmax] = e * sum;
    for (int m = mmax - 1; m >= 0; --m) F[m] = (2.0 * T * F[m + 1] + e) / (2 * m + 1);
  } else {
    double e = std::exp(-T);
    F[0] = 0.5 * std::sqrt(M_PI / T) * std::erf(std::sqrt(T));
    for (int m = 0; m < mmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
  }
}

// ---------------------------------------------------------------- shells
struct Shell {
  int l = 0;
  bool pure = false;
  double A[3] = {0, 0, 0};
  std::vector<double> a, c;  // exponents, coefficients incl. primitive norms
  int atom = -1;
  int nbf() const { return pure ? 2 * l + 1 : ncart(l); }
};

// libint2::Shell semantics: multiply by primitive norms, then rescale so the
// contracted x^l function is normalised.
void normalise(Shell& s) {
  const int l = s.l;
  for (size_t p = 0; p < s.a.size(); ++p) {
    double al = s.a[p];
    double n2 = std::pow(4.0 * al, l) * std::pow(2.0 * al / M_PI, 1.5) / dfact(2 * l - 1);
    s.c[p] *= std::sqrt(n2);
  }
  double norm = 0.0;
  for (size_t p = 0; p < s.a.size(); ++p)
    for (size_t q = 0; q < s.a.size(); ++q) {
      double g = s.a[p] + s.a[q];
      norm += s.c[p] * s.c[q] * dfact(2 * l - 1) / std::pow(2.0 * g, l) * std::pow(M_PI / g, 1.5);
    }
  double f = 1.0 / std::sqrt(norm);
  for (auto& x : s.c) x *= f;
}

Shell unit_shell(const double* A) {
  Shell s;
  s.l = 0;
  s.A[0] = A[0];
  s.A[1] = A[1];
  s.A[2] = A[2];
  s.a = {0.0};
  s.c = {1.0};
  return s;
}

// real solid harmonics, rows m=-l..l, columns Cartesian components of l,
// in terms of x^l-normalised Cartesian functions.
struct Poly {  // polynomial as map over (a,b,c) with a+b+c = degree (dense over gid)
  std::vector<double> c;
  Poly() : c(CT().gcomp.size(), 0.0) {}
};

std::vector<std::vector<double>> solid_harmonics(int l) {
  const auto& T = CT();
  // S[l][m+l]
  std::vector<std::vector<Poly>> S(l + 1);
  S[0].resize(1);
  S[0][0].c[T.gid[0][0][0]] = 1.0;
  auto mul = [&](const Poly& p, int dx, int dy, int dz, double f, Poly& out) {
    for (size_t g = 0; g < p.c.size(); ++g)
      if (p.c[g] != 0.0) {
        auto e = T.gcomp[g];
        out.c[T.gid[e[0] + dx][e[1] + dy][e[2] + dz]] += f * p.c[g];
      }
  };
  for (int k = 0; k < l; ++k) {  // build k+1 from k (and k-1)
    S[k + 1].resize(2 * k + 3);
    double f = std::sqrt((k == 0 ? 2.0 : 1.0) * (2 * k + 1) / (2.0 * k + 2));
    // m = k+1
    {
      Poly out;
      mul(S[k][2 * k], 1, 0, 0, f, out);                       // x S_kk
      if (k > 0) mul(S[k][0], 0, 1, 0, -f, out);               // - y S_k,-k
      S[k + 1][2 * k + 2] = out;
    }
    // m = -(k+1)
    {
      Poly out;
      mul(S[k][2 * k], 0, 1, 0, f, out);                       // y S_kk
      if (k > 0) mul(S[k][0], 1, 0, 0, f, out);                // + x S_k,-k
      S[k + 1][0] = out;
    }
    for (int m = -k; m <= k; ++m) {
      Poly out;
      double den = std::sqrt((double)(k + m + 1) * (k - m + 1));
      mul(S[k][m + k], 0, 0, 1, (2 * k + 1) / den, out);
      if (k > 0 && std::abs(m) <= k - 1) {
        double g = -std::sqrt((double)(k + m) * (k - m)) / den;
        const Poly& q = S[k - 1][m + k - 1];
        mul(q, 2, 0, 0, g, out);
        mul(q, 0, 2, 0, g, out);
        mul(q, 0, 0, 2, g, out);
      }
      S[k + 1][m + k + 1] = out;
    }
  }
  const auto& comps = T.comp[l];
  std::vector<std::vector<double>> R(2 * l + 1, std::vector<double>(comps.size(), 0.0));
  for (int m = 0; m < 2 * l + 1; ++m) {
    for (size_t i = 0; i < comps.size(); ++i)
      R[m][i] = S[l][m].c[T.gid[comps[i][0]][comps[i][1]][comps[i][2]]];
    double nrm = 0.0;  // <S|S> in units of the x^l norm
    for (size_t i = 0; i < comps.size(); ++i)
      for (size_t j = 0; j < comps.size(); ++j) {
        int sx = comps[i][0] + comps[j][0], sy = comps[i][1] + comps[j][1], sz = comps[i][2] + comps[j][2];
        if (sx % 2 || sy % 2 || sz % 2) continue;
        nrm += R[m][i] * R[m][j] * dfact(sx - 1) * dfact(sy - 1) * dfact(sz - 1) / dfact(2 * l - 1);
      }
    for (auto& v : R[m]) v /= std::sqrt(nrm);
  }
  return R;
}

const std::vector<std::vector<double>>& SH(int l) {
  static std::vector<std::vector<std::vector<double>>> cache(LMAXC + 1);
  static std::mutex mu;
  std::lock_guard<std::mutex> g(mu);
  if (cache[l].empty()) cache[l] = solid_harmonics(l);
  return cache[l];
}

// ---------------------------------------------------------------- ERIs
// Contracted Cartesian block (ab|cd) for arbitrary exps/coefs, by OS VRR on
// [e0|f0]^(m), contraction, then HGP HRR on both sides.
// out layout: ((ia*nb + ib)*nc + ic)*nd + id over Cartesian components.
void cart_eri(int la, const double* A, const std::vector<double>& aa, const std::vector<double>& ca,
              int lb, const double* B, const std::vector<double>& ab, const std::vector<double>& cb,
              int lc, const double* C, const std::vector<double>& ac, const std::vector<double>& cc,
              int ld, const double* D, const std::vector<double>& ad, const std::vector<double>& cd,
              std::vector<double>& out) {
  const auto& T = CT();
  const int Ea = la + lb, Ef = lc + ld, L = Ea + Ef, M = L + 1;
  const int NE = ncum(Ea), NF = ncum(Ef);
  std::vector<double> V((size_t)NE * NF * M);
  std::vector<double> X((size_t)NE * NF, 0.0);  // contracted [e0|f0]
  double AB[3], CD[3], AB2 = 0, CD2 = 0;
  for (int i = 0; i < 3; ++i) {
    AB[i] = A[i] - B[i];
    CD[i] = C[i] - D[i];
    AB2 += AB[i] * AB[i];
    CD2 += CD[i] * CD[i];
  }
  std::vector<double> F(M);
  auto at = [&](int e, int f, int m) -> double& { return V[((size_t)e * NF + f) * M + m]; };
  for (size_t pa = 0; pa < aa.size(); ++pa)
    for (size_t pb = 0; pb < ab.size(); ++pb) {
      const double al = aa[pa], be = ab[pb], zeta = al + be;
      const double Kab = std::exp(-al * be / zeta * AB2);
      double P[3], PA[3];
      for (int i = 0; i < 3; ++i) {
        P[i] = (al * A[i] + be * B[i]) / zeta;
        PA[i] = P[i] - A[i];
      }
      for (size_t pc = 0; pc < ac.size(); ++pc)
        for (size_t pd = 0; pd < ad.size(); ++pd) {
          const double ga = ac[pc], de = ad[pd], eta = ga + de;
          const double Kcd = std::exp(-ga * de / eta * CD2);
          const double coef = ca[pa] * cb[pb] * cc[pc] * cd[pd];
          double Q[3], QC[3], W[3], WP[3], WQ[3], PQ2 = 0;
          for (int i = 0; i < 3; ++i) {
            Q[i] = (ga * C[i] + de * D[i]) / eta;
            QC[i] = Q[i] - C[i];
            W[i] = (zeta * P[i] + eta * Q[i]) / (zeta + eta);
            WP[i] = W[i] - P[i];
            WQ[i] = W[i] - Q[i];
            PQ2 += (P[i] - Q[i]) * (P[i] - Q[i]);
          }
          const double rho = zeta * eta / (zeta + eta);
          const double pref = 2.0 * std::pow(M_PI, 2.5) / (zeta * eta * std::sqrt(zeta + eta)) * Kab * Kcd;
          boys(L, rho * PQ2, F.data());
          for (int m = 0; m <= L; ++m) at(0, 0, m) = pref * F[m];
          // bra build, f = 0
          for (int et = 1; et <= Ea; ++et)
            for (auto t : T.comp[et]) {
              int i = t[0] ? 0 : (t[1] ? 1 : 2);
              auto e = t;
              e[i] -= 1;
              int g_t = T.gid[t[0]][t[1]][t[2]], g_e = T.gid[e[0]][e[1]][e[2]];
              int g_e2 = -1;
              if (e[i] > 0) {
                auto e2 = e;
                e2[i] -= 1;
                g_e2 = T.gid[e2[0]][e2[1]][e2[2]];
              }
              for (int m = 0; m <= L - et; ++m) {
                double v = PA[i] * at(g_e, 0, m) + WP[i] * at(g_e, 0, m + 1);
                if (g_e2 >= 0) v += e[i] / (2 * zeta) * (at(g_e2, 0, m) - rho / zeta * at(g_e2, 0, m + 1));
                at(g_t, 0, m) = v;
              }
            }
          // ket build
          for (int ft = 1; ft <= Ef; ++ft)
            for (auto t : T.comp[ft]) {
              int i = t[0] ? 0 : (t[1] ? 1 : 2);
              auto f = t;
              f[i] -= 1;
              int g_t = T.gid[t[0]][t[1]][t[2]], g_f = T.gid[f[0]][f[1]][f[2]];
              int g_f2 = -1;
              if (f[i] > 0) {
                auto f2 = f;
                f2[i] -= 1;
                g_f2 = T.gid[f2[0]][f2[1]][f2[2]];
              }
              for (int et = 0; et <= Ea; ++et)
                for (auto e : T.comp[et]) {
                  int g_e = T.gid[e[0]][e[1]][e[2]];
                  int g_em = -1;
                  if (e[i] > 0) {
                    auto em = e;
                    em[i] -= 1;
                    g_em = T.gid[em[0]][em[1]][em[2]];
                  }
                  for (int m = 0; m <= L - et - ft; ++m) {
                    double v = QC[i] * at(g_e, g_f, m) + WQ[i] * at(g_e, g_f, m + 1);
                    if (g_f2 >= 0) v += f[i] / (2 * eta) * (at(g_e, g_f2, m) - rho / eta * at(g_e, g_f2, m + 1));
                    if (g_em >= 0) v += e[i] / (2 * (zeta + eta)) * at(g_em, g_f, m + 1);
                    at(g_e, g_t, m) = v;
                  }
                }
            }
          for (int e = 0; e < NE; ++e)
            for (int f = 0; f < NF; ++f) X[(size_t)e * NF + f] += coef * at(e, f, 0);
        }
    }
  // ket HRR: (e|c d) from (e|f0), f total in [lc, lc+ld]
  const int NC = ncum(Ef), ND = ncum(ld);
  std::vector<double> Y((size_t)NE * NC * ND, 0.0);
  auto y = [&](std::vector<double>& arr, int e, int c, int d) -> double& {
    return arr[((size_t)e * NC + c) * ND + d];
  };
  for (int e = 0; e < NE; ++e)
    for (int f = 0; f < NF; ++f) y(Y, e, f, 0) = X[(size_t)e * NF + f];
  for (int k = 0; k < ld; ++k) {  // from dtot=k to k+1
    for (auto dn : T.comp[k + 1]) {
      int i = dn[0] ? 0 : (dn[1] ? 1 : 2);
      auto dd = dn;
      dd[i] -= 1;
      int g_dn = T.gid[dn[0]][dn[1]][dn[2]], g_d = T.gid[dd[0]][dd[1]][dd[2]];
      for (int ct = lc; ct <= Ef - k - 1; ++ct)
        for (auto c : T.comp[ct]) {
          auto cp = c;
          cp[i] += 1;
          int g_c = T.gid[c[0]][c[1]][c[2]], g_cp = T.gid[cp[0]][cp[1]][cp[2]];
          for (int e = 0; e < NE; ++e) y(Y, e, g_c, g_dn) = y(Y, e, g_cp, g_d) + CD[i] * y(Y, e, g_c, g_d);
        }
    }
  }
  // bra HRR on each (c,d) of the final ket shells
  const int nc = ncart(lc), nd = ncart(ld), na = ncart(la), nb = ncart(lb);
  out.assign((size_t)na * nb * nc * nd, 0.0);
  const int NA = ncum(Ea), NB = ncum(lb);
  std::vector<double> Z((size_t)NA * NB);
  for (int ic = 0; ic < nc; ++ic)
    for (int id = 0; id < nd; ++id) {
      auto c = T.comp[lc][ic];
      auto d = T.comp[ld][id];
      int g_c = T.gid[c[0]][c[1]][c[2]], g_d = T.gid[d[0]][d[1]][d[2]];
      std::fill(Z.begin(), Z.end(), 0.0);
      for (int e = 0; e < NE; ++e) Z[(size_t)e * NB + 0] = y(Y, e, g_c, g_d);
      for (int k = 0; k < lb; ++k)
        for (auto bn : T.comp[k + 1]) {
          int i = bn[0] ? 0 : (bn[1] ? 1 : 2);
          auto bb = bn;
          bb[i] -= 1;
          int g_bn = T.gid[bn[0]][bn[1]][bn[2]], g_b = T.gid[bb[0]][bb[1]][bb[2]];
          for (int at_ = la; at_ <= Ea - k - 1; ++at_)
            for (auto a : T.comp[at_]) {
              auto ap = a;
              ap[i] += 1;
              int g_a = T.gid[a[0]][a[1]][a[2]], g_ap = T.gid[ap[0]][ap[1]][ap[2]];
              Z[(size_t)g_a * NB + g_bn] = Z[(size_t)g_ap * NB + g_b] + AB[i] * Z[(size_t)g_a * NB + g_b];
            }
        }
      for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib) {
          auto a = T.comp[la][ia];
          auto b = T.comp[lb][ib];
          out[(((size_t)ia * nb + ib) * nc + ic) * nd + id] =
              Z[(size_t)T.gid[a[0]][a[1]][a[2]] * NB + T.gid[b[0]][b[1]][b[2]]];
        }
    }
}

// Transform a Cartesian 4-index block to the shells' final (pure/Cartesian) basis.
void to_final(const int l[4], const bool pure[4], std::vector<double>& blk) {
  int n[4];
  for (int k = 0; k < 4; ++k) n[k] = ncart(l[k]);
  for (int k = 0; k < 4; ++k) {
    if (!pure[k] || l[k] < 2) continue;
    const auto& R = SH(l[k]);
    int nk = 2 * l[k] + 1;
    int pre = 1, post = 1;
    for (int j = 0; j < k; ++j) pre *= n[j];
    for (int j = k + 1; j < 4; ++j) post *= n[j];
    std::vector<double> o((size_t)pre * nk * post, 0.0);
    for (int p = 0; p < pre; ++p)
      for (int m = 0; m < nk; ++m)
        for (int i = 0; i < n[k]; ++i) {
          double r = R[m][i];
          if (r == 0.0) continue;
          for (int q = 0; q < post; ++q)
            o[((size_t)p * nk + m) * post + q] += r * blk[((size_t)p * n[k] + i) * post + q];
        }
    blk.swap(o);
    n[k] = nk;
  }
}

void shell_eri(const Shell& s1, const Shell& s2, const Shell& s3, const Shell& s4, std::vector<double>& out) {
  cart_eri(s1.l, s1.A, s1.a, s1.c, s2.l, s2.A, s2.a, s2.c, s3.l, s3.A, s3.a, s3.c, s4.l, s4.A, s4.a, s4.c, out);
  int l[4] = {s1.l, s2.l, s3.l, s4.l};
  bool p[4] = {s1.pure, s2.pure, s3.pure, s4.pure};
  to_final(l, p, out);
}

// Derivative of the (s1 s2|s3 s4) block with respect to the centre of shell
// `which` (0..3), direction xyz: d/dA_i g_a = 2 alpha g_{a+1_i} - a_i g_{a-1_i}.
void shell_eri_deriv(const Shell* s[4], int which, int xyz, std::vector<double>& out) {
  const auto& T = CT();
  const Shell& w = *s[which];
  std::vector<double> c2(w.c.size());
  for (size_t p = 0; p < w.c.size(); ++p) c2[p] = 2.0 * w.a[p] * w.c[p];
  int l[4] = {s[0]->l, s[1]->l, s[2]->l, s[3]->l};
  int n[4];
  for (int k = 0; k < 4; ++k) n[k] = ncart(l[k]);
  auto call = [&](int lw, const std::vector<double>& cw, std::vector<double>& o) {
    const Shell* t[4] = {s[0], s[1], s[2], s[3]};
    int ll[4] = {l[0], l[1], l[2], l[3]};
    ll[which] = lw;
    const std::vector<double>* cc[4] = {&t[0]->c, &t[1]->c, &t[2]->c, &t[3]->c};
    cc[which] = &cw;
    cart_eri(ll[0], t[0]->A, t[0]->a, *cc[0], ll[1], t[1]->A, t[1]->a, *cc[1], ll[2], t[2]->A, t[2]->a, *cc[2],
             ll[3], t[3]->A, t[3]->a, *cc[3], o);
  };
  std::vector<double> up, dn;
  call(l[which] + 1, c2, up);
  if (l[which] > 0) call(l[which] - 1, w.c, dn);
  int nup[4] = {n[0], n[1], n[2], n[3]}, ndn[4] = {n[0], n[1], n[2], n[3]};
  nup[which] = ncart(l[which] + 1);
  ndn[which] = l[which] > 0 ? ncart(l[which] - 1) : 0;
  out.assign((size_t)n[0] * n[1] * n[2] * n[3], 0.0);
  for (int i0 = 0; i0 < n[0]; ++i0)
    for (int i1 = 0; i1 < n[1]; ++i1)
      for (int i2 = 0; i2 < n[2]; ++i2)
        for (int i3 = 0; i3 < n[3]; ++i3) {
          int idx[4] = {i0, i1, i2, i3};
          auto e = T.comp[l[which]][idx[which]];
          auto ep = e;
          ep[xyz] += 1;
          int iu[4] = {i0, i1, i2, i3};
          iu[which] = T.lid[ep[0]][ep[1]][ep[2]];
          double v = up[(((size_t)iu[0] * nup[1] + iu[1]) * nup[2] + iu[2]) * nup[3] + iu[3]];
          if (e[xyz] > 0) {
            auto em = e;
            em[xyz] -= 1;
            int id_[4] = {i0, i1, i2, i3};
            id_[which] = T.lid[em[0]][em[1]][em[2]];
            v -= e[xyz] * dn[(((size_t)id_[0] * ndn[1] + id_[1]) * ndn[2] + id_[2]) * ndn[3] + id_[3]];
          }
          out[(((size_t)i0 * n[1] + i1) * n[2] + i2) * n[3] + i3] = v;
        }
  bool p[4] = {s[0]->pure, s[1]->pure, s[2]->pure, s[3]->pure};
  to_final(l, p, out);
}

// ---------------------------------------------------------------- 1e ints
// 1D overlap table S[i][j] for Gaussians on A, B (OS).
void overlap1d(int imax, int jmax, double PA, double PB, double p, std::vector<double>& S, int ld) {
  S.assign((size_t)(imax + 1) * ld, 0.0);
  S[0] = 1.0;  // prefactor applied outside
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      double v;
      if (i > 0) {
        v = PA * S[(i - 1) * ld + j];
        if (i > 1) v += (i - 1) / (2 * p) * S[(i - 2) * ld + j];
        if (j > 0) v += j / (2 * p) * S[(i - 1) * ld + j - 1];
      } else {
        v = PB * S[i * ld + j - 1];
        if (j > 1) v += (j - 1) / (2 * p) * S[i * ld + j - 2];
      }
      S[i * ld + j] = v;
    }
}

// Cartesian overlap and kinetic blocks for shells a, b (contracted).
void cart_ST(int la, const double* A, const std::vector<double>& aa, const std::vector<double>& ca, int lb,
             const double* B, const std::vector<double>& ab, const std::vector<double>& cb, std::vector<double>* S,
             std::vector<double>* Tk) {
  const auto& T = CT();
  int na = ncart(la), nb = ncart(lb);
  if (S) S->assign((size_t)na * nb, 0.0);
  if (Tk) Tk->assign((size_t)na * nb, 0.0);
  double AB2 = 0;
  for (int i = 0; i < 3; ++i) AB2 += (A[i] - B[i]) * (A[i] - B[i]);
  std::vector<double> s1d[3];
  const int ld = lb + 3;
  for (size_t pa = 0; pa < aa.size(); ++pa)
    for (size_t pb = 0; pb < ab.size(); ++pb) {
      double al = aa[pa], be = ab[pb], p = al + be;
      double pref = ca[pa] * cb[pb] * std::exp(-al * be / p * AB2) * std::pow(M_PI / p, 1.5);
      for (int i = 0; i < 3; ++i) {
        double P = (al * A[i] + be * B[i]) / p;
        overlap1d(la + 1, lb + 2, P - A[i], P - B[i], p, s1d[i], ld);
      }
      for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib) {
          auto a = T.comp[la][ia];
          auto b = T.comp[lb][ib];
          double sx = s1d[0][a[0] * ld + b[0]], sy = s1d[1][a[1] * ld + b[1]], sz = s1d[2][a[2] * ld + b[2]];
          if (S) (*S)[ia * nb + ib] += pref * sx * sy * sz;
          if (Tk) {
            double t[3];
            for (int d = 0; d < 3; ++d) {
              int i = a[d], j = b[d];
              const auto& s = s1d[d];
              double v = -2.0 * be * be * s[i * ld + j + 2] + be * (2 * j + 1) * s[i * ld + j];
              if (j > 1) v -= 0.5 * j * (j - 1) * s[i * ld + j - 2];
              t[d] = v;
            }
            (*Tk)[ia * nb + ib] += pref * (t[0] * sy * sz + sx * t[1] * sz + sx * sy * t[2]);
          }
        }
    }
}

// Cartesian nuclear attraction block of a single unit charge at C (no -Z),
// i.e. (a| 1/|r-C| |b), by OS VRR on the bra plus HRR.
void cart_V1(int la, const double* A, const std::vector<double>& aa, const std::vector<double>& ca, int lb,
             const double* B, const std::vector<double>& ab, const std::vector<double>& cb, const double* C,
             std::vector<double>& out) {
  const auto& T = CT();
  const int Ea = la + lb, M = Ea + 1, NE = ncum(Ea);
  std::vector<double> V((size_t)NE * M), X(NE, 0.0), F(M);
  double AB[3], AB2 = 0;
  for (int i = 0; i < 3; ++i) {
    AB[i] = A[i] - B[i];
    AB2 += AB[i] * AB[i];
  }
  for (size_t pa = 0; pa < aa.size(); ++pa)
    for (size_t pb = 0; pb < ab.size(); ++pb) {
      double al = aa[pa], be = ab[pb], p = al + be;
      double P[3], PA[3], PC[3], PC2 = 0;
      for (int i = 0; i < 3; ++i) {
        P[i] = (al * A[i] + be * B[i]) / p;
        PA[i] = P[i] - A[i];
        PC[i] = P[i] - C[i];
        PC2 += PC[i] * PC[i];
      }
      double pref = 2.0 * M_PI / p * std::exp(-al * be / p * AB2) * ca[pa] * cb[pb];
      boys(Ea, p * PC2, F.data());
      for (int m = 0; m <= Ea; ++m) V[m] = pref * F[m];
      for (int et = 1; et <= Ea; ++et)
        for (auto t : T.comp[et]) {
          int i = t[0] ? 0 : (t[1] ? 1 : 2);
          auto e = t;
          e[i] -= 1;
          int g_t = T.gid[t[0]][t[1]][t[2]], g_e = T.gid[e[0]][e[1]][e[2]];
          int g_e2 = -1;
          if (e[i] > 0) {
            auto e2 = e;
            e2[i] -= 1;
            g_e2 = T.gid[e2[0]][e2[1]][e2[2]];
          }
          for (int m = 0; m <= Ea - et; ++m) {
            double v = PA[i] * V[g_e * M + m] - PC[i] * V[g_e * M + m + 1];
            if (g_e2 >= 0) v += e[i] / (2 * p) * (V[g_e2 * M + m] - V[g_e2 * M + m + 1]);
            V[g_t * M + m] = v;
          }
        }
      for (int e = 0; e < NE; ++e) X[e] += V[e * M];
    }
  const int NB = ncum(lb), na = ncart(la), nb = ncart(lb);
  std::vector<double> Z((size_t)NE * NB, 0.0);
  for (int e = 0; e < NE; ++e) Z[(size_t)e * NB] = X[e];
  for (int k = 0; k < lb; ++k)
    for (auto bn : T.comp[k + 1]) {
      int i = bn[0] ? 0 : (bn[1] ? 1 : 2);
      auto bb = bn;
      bb[i] -= 1;
      int g_bn = T.gid[bn[0]][bn[1]][bn[2]], g_b = T.gid[bb[0]][bb[1]][bb[2]];
      for (int at_ = la; at_ <= Ea - k - 1; ++at_)
        for (auto a : T.comp[at_]) {
          auto ap = a;
          ap[i] += 1;
          int g_a = T.gid[a[0]][a[1]][a[2]], g_ap = T.gid[ap[0]][ap[1]][ap[2]];
          Z[(size_t)g_a * NB + g_bn] = Z[(size_t)g_ap * NB + g_b] + AB[i] * Z[(size_t)g_a * NB + g_b];
        }
    }
  out.assign((size_t)na * nb, 0.0);
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib) {
      auto a = T.comp[la][ia];
      auto b = T.comp[lb][ib];
      out[ia * nb + ib] = Z[(size_t)T.gid[a[0]][a[1]][a[2]] * NB + T.gid[b[0]][b[1]][b[2]]];
    }
}

void to_final2(int la, bool pa, int lb, bool pb, std::vector<double>& blk) {
  int l[4] = {la, lb, 0, 0};
  bool p[4] = {pa, pb, false, false};
  to_final(l, p, blk);
}

// ---------------------------------------------------------------- basis plumbing
struct Basis {
  std::vector<Shell> sh;
  std::vector<int> off;
  int n = 0;
};

}  // namespace

extern "C" {

// Same shape as jk_basis in include/jk_engine.h.
typedef struct {
  int nshell;
  const int* l;
  const int* nprim;
  const int* prim_off;
  const double* exps;
  const double* coefs;  // as printed in the basis file (normalised primitives)
  const double* xyz;    // 3*nshell, bohr
  const int* pure;      // 1 = spherical (l >= 2 only)
  const int* atom;      // owning atom per shell (may be NULL)
} orc_basis;
}

namespace {
Basis make_basis(const orc_basis* b) {
  Basis B;
  B.sh.resize(b->nshell);
  for (int s = 0; s < b->nshell; ++s) {
    Shell& x = B.sh[s];
    x.l = b->l[s];
    x.pure = b->pure ? (b->pure[s] != 0 && x.l >= 2) : false;
    for (int i = 0; i < 3; ++i) x.A[i] = b->xyz[3 * s + i];
    x.a.assign(b->exps + b->prim_off[s], b->exps + b->prim_off[s] + b->nprim[s]);
    x.c.assign(b->coefs + b->prim_off[s], b->coefs + b->prim_off[s] + b->nprim[s]);
    x.atom = b->atom ? b->atom[s] : -1;
    normalise(x);
  }
  B.off.resize(b->nshell + 1);
  B.off[0] = 0;
  for (int s = 0; s < b->nshell; ++s) B.off[s + 1] = B.off[s] + B.sh[s].nbf();
  B.n = B.off[b->nshell];
  return B;
}

template <class F>
void parallel_for(int n, int nthreads, F f) {
  if (nthreads <= 1) {
    for (int i = 0; i < n; ++i) f(i, 0);
    return;
  }
  std::vector<std::thread> th;
  std::mutex mu;
  int next = 0;
  for (int t = 0; t < nthreads; ++t)
    th.emplace_back([&, t] {
      for (;;) {
        int i;
        {
          std::lock_guard<std::mutex> g(mu);
          i = next++;
        }
        if (i >= n) break;
        f(i, t);
      }
    });
  for (auto& x : th) x.join();
}

// max |A| over a shell block (Eigen lpNorm<Infinity>), src/integrals.cpp:451-469
std::vector<double> shellblock_norm(const Basis& B, const double* D) {
  int ns = (int)B.sh.size();
  std::vector<double> out((size_t)ns * ns, 0.0);
  for (int s1 = 0; s1 < ns; ++s1)
    for (int s2 = 0; s2 < ns; ++s2) {
      double m = 0.0;
      for (int i = B.off[s1]; i < B.off[s1 + 1]; ++i)
        for (int j = B.off[s2]; j < B.off[s2 + 1]; ++j) m = std::max(m, std::fabs(D[(size_t)j * B.n + i]));
      out[(size_t)s1 * ns + s2] = m;
    }
  return out;
}
}  // namespace

extern "C" {

void orc_boys(int mmax, double T, double* F) { boys(mmax, T, F); }

int orc_nbf(const orc_basis* b) { return make_basis(b).n; }

// Normalised coefficients (after libint2-style normalisation), per primitive.
void orc_normalised_coefs(const orc_basis* b, double* out) {
  Basis B = make_basis(b);
  for (int s = 0; s < b->nshell; ++s)
    for (int p = 0; p < b->nprim[s]; ++p) out[b->prim_off[s] + p] = B.sh[s].c[p];
}

// Solid-harmonic transform rows m=-l..l over Cartesian columns.
void orc_solid_harmonics(int l, double* out) {
  const auto& R = SH(l);
  int nc = ncart(l);
  for (int m = 0; m < 2 * l + 1; ++m)
    for (int i = 0; i < nc; ++i) out[m * nc + i] = R[m][i];
}

// One shell quartet in libint order f1234 = ((f1*n2+f2)*n3+f3)*n4+f4.
void orc_eri_quartet(const orc_basis* b, int s1, int s2, int s3, int s4, double* out) {
  Basis B = make_basis(b);
  std::vector<double> v;
  shell_eri(B.sh[s1], B.sh[s2], B.sh[s3], B.sh[s4], v);
  std::memcpy(out, v.data(), v.size() * sizeof(double));
}

// Full ERI tensor (n^4, index ((i*n+j)*n+k)*n+l) for small tests.
void orc_eri_full(const orc_basis* b, double* out) {
  Basis B = make_basis(b);
  int ns = (int)B.sh.size(), n = B.n;
  std::vector<double> v;
  for (int s1 = 0; s1 < ns; ++s1)
    for (int s2 = 0; s2 < ns; ++s2)
      for (int s3 = 0; s3 < ns; ++s3)
        for (int s4 = 0; s4 < ns; ++s4) {
          shell_eri(B.sh[s1], B.sh[s2], B.sh[s3], B.sh[s4], v);
          int n1 = B.sh[s1].nbf(), n2 = B.sh[s2].nbf(), n3 = B.sh[s3].nbf(), n4 = B.sh[s4].nbf();
          for (int f1 = 0, f = 0; f1 < n1; ++f1)
            for (int f2 = 0; f2 < n2; ++f2)
              for (int f3 = 0; f3 < n3; ++f3)
                for (int f4 = 0; f4 < n4; ++f4, ++f) {
                  size_t i = B.off[s1] + f1, j = B.off[s2] + f2, k = B.off[s3] + f3, l = B.off[s4] + f4;
                  out[((i * n + j) * n + k) * n + l] = v[f];
                }
        }
}

// Schwarz matrix Q(s1,s2) = sqrt(max_i |(ab|ab)_ii|), src/integrals.cpp:472-513
void orc_schwarz(const orc_basis* b, double* Q) {
  Basis B = make_basis(b);
  int ns = (int)B.sh.size();
  std::vector<double> v;
  for (int s1 = 0; s1 < ns; ++s1)
    for (int s2 = 0; s2 <= s1; ++s2) {
      shell_eri(B.sh[s1], B.sh[s2], B.sh[s1], B.sh[s2], v);
      int n12 = B.sh[s1].nbf() * B.sh[s2].nbf();
      double m = 0.0;
      for (int i = 0; i < n12; ++i) m = std::max(m, std::fabs(v[(size_t)i * n12 + i]));
      Q[(size_t)s1 * ns + s2] = Q[(size_t)s2 * ns + s1] = std::sqrt(m);
    }
}

void orc_shellblock_norm(const orc_basis* b, const double* D, double* out) {
  Basis B = make_basis(b);
  auto v = shellblock_norm(B, D);
  std::memcpy(out, v.data(), v.size() * sizeof(double));
}

// Fock::formJKdirect (src/fockbuild.cpp:64-164).  Outputs are w.r.t. the full
// D passed in (jints = J[D], kints = K[D]); multiplier as in the reference.
// Q may be NULL (no screening, as when the Schwarz matrix is empty).
// Returns the number of quartets computed.
long orc_jk_direct(const orc_basis* b, const double* Q, const double* D, double precision, double multiplier,
                   double* J, double* K, int nthreads) {
  Basis B = make_basis(b);
  const int ns = (int)B.sh.size(), n = B.n;
  const bool screen = Q != nullptr;
  auto Dn = shellblock_norm(B, D);
  if (nthreads < 1) nthreads = 1;
  std::vector<std::vector<double>> Jt(nthreads, std::vector<double>((size_t)n * n, 0.0));
  std::vector<std::vector<double>> Kt(nthreads, std::vector<double>((size_t)n * n, 0.0));
  std::vector<long> cnt(nthreads, 0);
  auto dn = [&](int a, int c) { return Dn[(size_t)a * ns + c]; };
  auto Dm = [&](int i, int j) { return D[(size_t)j * n + i]; };
  parallel_for(ns, nthreads, [&](int s1, int t) {
    std::vector<double> buf;
    double* Jm = Jt[t].data();
    double* Km = Kt[t].data();
    auto J_ = [&](int i, int j) -> double& { return Jm[(size_t)j * n + i]; };
    auto K_ = [&](int i, int j) -> double& { return Km[(size_t)j * n + i]; };
    for (int s2 = 0; s2 <= s1; ++s2) {
      const double Dnorm12 = screen ? dn(s1, s2) : 0.0;
      for (int s3 = 0; s3 <= s1; ++s3) {
        const double Dnorm123 = screen ? std::max(dn(s1, s3), std::max(dn(s2, s3), Dnorm12)) : 0.0;
        const int s4_max = (s1 == s3) ? s2 : s3;
        for (int s4 = 0; s4 <= s4_max; ++s4) {
          const double Dnorm1234 =
              screen ? std::max(dn(s1, s4), std::max(dn(s2, s4), std::max(dn(s3, s4), Dnorm123))) : 0.0;
          if (screen && Dnorm1234 * Q[(size_t)s1 * ns + s2] * Q[(size_t)s3 * ns + s4] < precision) continue;
          double s12_deg = (s1 == s2) ? 1.0 : 2.0;
          double s34_deg = (s3 == s4) ? 1.0 : 2.0;
          double s12_34_deg = (s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0;
          double deg = s12_deg * s34_deg * s12_34_deg;
          shell_eri(B.sh[s1], B.sh[s2], B.sh[s3], B.sh[s4], buf);
          ++cnt[t];
          int n1 = B.sh[s1].nbf(), n2 = B.sh[s2].nbf(), n3 = B.sh[s3].nbf(), n4 = B.sh[s4].nbf();
          for (int f1 = 0, f = 0; f1 < n1; ++f1) {
            int b1 = B.off[s1] + f1;
            for (int f2 = 0; f2 < n2; ++f2) {
              int b2 = B.off[s2] + f2;
              for (int f3 = 0; f3 < n3; ++f3) {
                int b3 = B.off[s3] + f3;
                for (int f4 = 0; f4 < n4; ++f4, ++f) {
                  int b4 = B.off[s4] + f4;
                  double v = buf[f] * deg;
                  J_(b1, b2) += multiplier * Dm(b3, b4) * v;
                  J_(b3, b4) += multiplier * Dm(b1, b2) * v;
                  K_(b1, b3) += 0.5 * multiplier * Dm(b2, b4) * v;
                  K_(b2, b4) += 0.5 * multiplier * Dm(b1, b3) * v;
                  K_(b1, b4) += 0.5 * multiplier * Dm(b2, b3) * v;
                  K_(b2, b3) += 0.5 * multiplier * Dm(b1, b4) * v;
                }
              }
            }
          }
        }
      }
    }
  });
  long total = 0;
  for (int t = 0; t < nthreads; ++t) total += cnt[t];
  for (size_t i = 0; i < (size_t)n * n; ++i) {
    double js = 0, ks = 0;
    for (int t = 0; t < nthreads; ++t) {
      js += Jt[t][i];
      ks += Kt[t][i];
    }
    Jt[0][i] = js;
    Kt[0][i] = ks;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      J[(size_t)j * n + i] = 0.25 * (Jt[0][(size_t)j * n + i] + Jt[0][(size_t)i * n + j]);
      K[(size_t)j * n + i] = 0.25 * (Kt[0][(size_t)j * n + i] + Kt[0][(size_t)i * n + j]);
    }
  return total;
}

// UnrestrictedFock::formJKdirect (src/fockbuild.cpp:266-362): the loop of
// formJKdirect with the screen built from the shell-block norms of Da + Db and
// every integral batch digested into both spin densities.  Outputs are w.r.t.
// each full spin density, times multiplier.  Returns the quartet count.
long orc_jk_direct_uhf(const orc_basis* b, const double* Q, const double* Da, const double* Db, double precision,
                       double multiplier, double* Ja, double* Jb, double* Ka, double* Kb, int nthreads) {
  Basis B = make_basis(b);
  const int ns = (int)B.sh.size(), n = B.n;
  const size_t nn = (size_t)n * n;
  const bool screen = Q != nullptr;
  std::vector<double> Dt(nn);
  for (size_t i = 0; i < nn; ++i) Dt[i] = Da[i] + Db[i];
  auto Dn = shellblock_norm(B, Dt.data());
  if (nthreads < 1) nthreads = 1;
  // per thread: Ja, Jb, Ka, Kb accumulators
  std::vector<std::vector<double>> acc(nthreads, std::vector<double>(4 * nn, 0.0));
  std::vector<long> cnt(nthreads, 0);
  auto dn = [&](int a, int c) { return Dn[(size_t)a * ns + c]; };
  parallel_for(ns, nthreads, [&](int s1, int t) {
    std::vector<double> buf;
    double* A = acc[t].data();
    for (int s2 = 0; s2 <= s1; ++s2) {
      const double Dnorm12 = screen ? dn(s1, s2) : 0.0;
      for (int s3 = 0; s3 <= s1; ++s3) {
        const double Dnorm123 = screen ? std::max(dn(s1, s3), std::max(dn(s2, s3), Dnorm12)) : 0.0;
        const int s4_max = (s1 == s3) ? s2 : s3;
        for (int s4 = 0; s4 <= s4_max; ++s4) {
          const double Dnorm1234 =
              screen ? std::max(dn(s1, s4), std::max(dn(s2, s4), std::max(dn(s3, s4), Dnorm123))) : 0.0;
          if (screen && Dnorm1234 * Q[(size_t)s1 * ns + s2] * Q[(size_t)s3 * ns + s4] < precision) continue;
          const double deg = ((s1 == s2) ? 1.0 : 2.0) * ((s3 == s4) ? 1.0 : 2.0) *
                             ((s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0);
          shell_eri(B.sh[s1], B.sh[s2], B.sh[s3], B.sh[s4], buf);
          ++cnt[t];
          const int n1 = B.sh[s1].nbf(), n2 = B.sh[s2].nbf(), n3 = B.sh[s3].nbf(), n4 = B.sh[s4].nbf();
          for (int spin = 0; spin < 2; ++spin) {
            const double* D = spin ? Db : Da;
            double* Jm = A + spin * nn;
            double* Km = A + (2 + spin) * nn;
            auto Dm = [&](int i, int j) { return D[(size_t)j * n + i]; };
            for (int f1 = 0, f = 0; f1 < n1; ++f1) {
              const int b1 = B.off[s1] + f1;
              for (int f2 = 0; f2 < n2; ++f2) {
                const int b2 = B.off[s2] + f2;
                for (int f3 = 0; f3 < n3; ++f3) {
                  const int b3 = B.off[s3] + f3;
                  for (int f4 = 0; f4 < n4; ++f4, ++f) {
                    const int b4 = B.off[s4] + f4;
                    const double v = multiplier * buf[f] * deg;
                    Jm[(size_t)b2 * n + b1] += Dm(b3, b4) * v;
                    Jm[(size_t)b4 * n + b3] += Dm(b1, b2) * v;
                    Km[(size_t)b3 * n + b1] += 0.5 * Dm(b2, b4) * v;
                    Km[(size_t)b4 * n + b2] += 0.5 * Dm(b1, b3) * v;
                    Km[(size_t)b4 * n + b1] += 0.5 * Dm(b2, b3) * v;
                    Km[(size_t)b3 * n + b2] += 0.5 * Dm(b1, b4) * v;
                  }
                }
              }
            }
          }
        }
      }
    }
  });
  long total = 0;
  for (int t = 0; t < nthreads; ++t) total += cnt[t];
  for (int t = 1; t < nthreads; ++t)
    for (size_t i = 0; i < 4 * nn; ++i) acc[0][i] += acc[t][i];
  double* outs[4] = {Ja, Jb, Ka, Kb};
  for (int k = 0; k < 4; ++k) {
    const double* X = acc[0].data() + k * nn;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) outs[k][(size_t)j * n + i] = 0.25 * (X[(size_t)j * n + i] + X[(size_t)i * n + j]);
  }
  return total;
}

// Time-bounded variant for the CPU baseline: runs the same loop for s1 in
// [s1_begin, s1_end) only and returns the number of quartets computed.
long orc_jk_direct_rows(const orc_basis* b, const double* Q, const double* D, double precision, int s1_begin,
                        int s1_end, double* J, double* K) {
  Basis B = make_basis(b);
  const int ns = (int)B.sh.size(), n = B.n;
  auto Dn = shellblock_norm(B, D);
  long cnt = 0;
  std::vector<double> buf;
  auto dn = [&](int a, int c) { return Dn[(size_t)a * ns + c]; };
  for (int s1 = s1_begin; s1 < std::min(s1_end, ns); ++s1)
    for (int s2 = 0; s2 <= s1; ++s2) {
      const double Dnorm12 = dn(s1, s2);
      for (int s3 = 0; s3 <= s1; ++s3) {
        const double Dnorm123 = std::max(dn(s1, s3), std::max(dn(s2, s3), Dnorm12));
        const int s4_max = (s1 == s3) ? s2 : s3;
        for (int s4 = 0; s4 <= s4_max; ++s4) {
          const double Dnorm1234 = std::max(dn(s1, s4), std::max(dn(s2, s4), std::max(dn(s3, s4), Dnorm123)));
          if (Dnorm1234 * Q[(size_t)s1 * ns + s2] * Q[(size_t)s3 * ns + s4] < precision) continue;
          double deg = ((s1 == s2) ? 1.0 : 2.0) * ((s3 == s4) ? 1.0 : 2.0) * ((s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0);
          shell_eri(B.sh[s1], B.sh[s2], B.sh[s3], B.sh[s4], buf);
          ++cnt;
          int n1 = B.sh[s1].nbf(), n2 = B.sh[s2].nbf(), n3 = B.sh[s3].nbf(), n4 = B.sh[s4].nbf();
          for (int f1 = 0, f = 0; f1 < n1; ++f1)
            for (int f2 = 0; f2 < n2; ++f2)
              for (int f3 = 0; f3 < n3; ++f3)
                for (int f4 = 0; f4 < n4; ++f4, ++f) {
                  size_t b1 = B.off[s1] + f1, b2 = B.off[s2] + f2, b3 = B.off[s3] + f3, b4 = B.off[s4] + f4;
                  double v = buf[f] * deg;
                  J[b2 * n + b1] += D[b4 * n + b3] * v;
                  J[b4 * n + b3] += D[b2 * n + b1] * v;
                  K[b3 * n + b1] += 0.5 * D[b4 * n + b2] * v;
                  K[b4 * n + b2] += 0.5 * D[b3 * n + b1] * v;
                  K[b4 * n + b1] += 0.5 * D[b3 * n + b2] * v;
                  K[b3 * n + b2] += 0.5 * D[b4 * n + b1] * v;
                }
        }
      }
    }
  return cnt;
}

// Fock::compute_2body_fock_general (src/fockbuild.cpp:477-583): G over obs
// from a density D in basis dbs (shell-diagonal when shelldiag != 0).
void orc_fock_general(const orc_basis* obs, const orc_basis* dbs, const double* D, int shelldiag, double* G) {
  Basis B = make_basis(obs), Bd = make_basis(dbs);
  const int ns = (int)B.sh.size(), nsd = (int)Bd.sh.size(), n = B.n, nd = Bd.n;
  const int nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::vector<double>> Gt(nthreads, std::vector<double>((size_t)n * n, 0.0));
  auto Dm = [&](int i, int j) { return D[(size_t)j * nd + i]; };
  parallel_for(ns, nthreads, [&](int s1, int t) {
    std::vector<double> buf;
    double* Gm = Gt[t].data();
    for (int s2 = 0; s2 <= s1; ++s2)
      for (int s3 = 0; s3 < nsd; ++s3) {
        int s4b = shelldiag ? s3 : 0, s4e = shelldiag ? s3 + 1 : nsd;
        for (int s4 = s4b; s4 < s4e; ++s4) {
          int n1 = B.sh[s1].nbf(), n2 = B.sh[s2].nbf(), n3 = Bd.sh[s3].nbf(), n4 = Bd.sh[s4].nbf();
          double s12_deg = (s1 == s2) ? 1.0 : 2.0;
          if (s3 >= s4) {
            double deg = s12_deg * ((s3 == s4) ? 1.0 : 2.0);
            shell_eri(B.sh[s1], B.sh[s2], Bd.sh[s3], Bd.sh[s4], buf);
            for (int f1 = 0, f = 0; f1 < n1; ++f1)
              for (int f2 = 0; f2 < n2; ++f2)
                for (int f3 = 0; f3 < n3; ++f3)
                  for (int f4 = 0; f4 < n4; ++f4, ++f) {
                    int b1 = B.off[s1] + f1, b2 = B.off[s2] + f2, b3 = Bd.off[s3] + f3, b4 = Bd.off[s4] + f4;
                    Gm[(size_t)b2 * n + b1] += 2.0 * Dm(b3, b4) * buf[f] * deg;
                  }
          }
          shell_eri(B.sh[s1], Bd.sh[s3], B.sh[s2], Bd.sh[s4], buf);
          for (int f1 = 0, f = 0; f1 < n1; ++f1)
            for (int f3 = 0; f3 < n3; ++f3)
              for (int f2 = 0; f2 < n2; ++f2)
                for (int f4 = 0; f4 < n4; ++f4, ++f) {
                  int b1 = B.off[s1] + f1, b2 = B.off[s2] + f2, b3 = Bd.off[s3] + f3, b4 = Bd.off[s4] + f4;
                  Gm[(size_t)b2 * n + b1] -= Dm(b3, b4) * buf[f] * s12_deg;
                }
        }
      }
  });
  for (int t = 1; t < nthreads; ++t)
    for (size_t i = 0; i < (size_t)n * n; ++i) Gt[0][i] += Gt[t][i];
  const double* Gm = Gt[0].data();
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) G[(size_t)j * n + i] = 0.5 * (Gm[(size_t)j * n + i] + Gm[(size_t)i * n + j]);
}

// IntegralEngine::compute_eris_3index (src/eris.cpp:89-156): column-major
// (n(n+1)/2) x naux, row index x(x+1)/2 + y for x >= y.
void orc_eri3(const orc_basis* obs, const orc_basis* aux, double* T) {
  Basis B = make_basis(obs), Ba = make_basis(aux);
  const int n = B.n, npair = n * (n + 1) / 2;
  std::vector<double> buf;
  parallel_for((int)Ba.sh.size(), (int)std::max(1u, std::thread::hardware_concurrency()), [&](int s1, int) {
    std::vector<double> v;
    Shell u = unit_shell(Ba.sh[s1].A);
    for (size_t s2 = 0; s2 < B.sh.size(); ++s2)
      for (size_t s3 = 0; s3 <= s2; ++s3) {
        shell_eri(Ba.sh[s1], u, B.sh[s2], B.sh[s3], v);
        int n1 = Ba.sh[s1].nbf(), n2 = B.sh[s2].nbf(), n3 = B.sh[s3].nbf();
        for (int f1 = 0, f = 0; f1 < n1; ++f1)
          for (int f2 = 0; f2 < n2; ++f2)
            for (int f3 = 0; f3 < n3; ++f3, ++f) {
              int b1 = Ba.off[s1] + f1, b2 = B.off[s2] + f2, b3 = B.off[s3] + f3;
              if (b2 >= b3) T[(size_t)b1 * npair + (size_t)b2 * (b2 + 1) / 2 + b3] = v[f];
            }
      }
  });
}

// IntegralEngine::compute_eris_2index (src/eris.cpp:304-356)
void orc_eri2(const orc_basis* aux, double* V) {
  Basis Ba = make_basis(aux);
  const int na = Ba.n;
  std::vector<double> v;
  for (size_t s1 = 0; s1 < Ba.sh.size(); ++s1)
    for (size_t s2 = 0; s2 <= s1; ++s2) {
      Shell u1 = unit_shell(Ba.sh[s1].A), u2 = unit_shell(Ba.sh[s2].A);
      shell_eri(Ba.sh[s1], u1, Ba.sh[s2], u2, v);
      int n1 = Ba.sh[s1].nbf(), n2 = Ba.sh[s2].nbf();
      for (int f1 = 0, f = 0; f1 < n1; ++f1)
        for (int f2 = 0; f2 < n2; ++f2, ++f) {
          int b1 = Ba.off[s1] + f1, b2 = Ba.off[s2] + f2;
          V[(size_t)b2 * na + b1] = v[f];
          V[(size_t)b1 * na + b2] = v[f];
        }
    }
}

// Cholesky V = L L^T (lower, column-major).  Returns 0, or k+1 when the
// leading minor k is not positive definite (Eigen::LLT's failure mode).
int orc_cholesky(int N, const double* V, double* L) {
  std::memset(L, 0, sizeof(double) * (size_t)N * N);
  for (int j = 0; j < N; ++j) {
    double d = V[(size_t)j * N + j];
    for (int k = 0; k < j; ++k) d -= L[(size_t)k * N + j] * L[(size_t)k * N + j];
    if (!(d > 0.0)) return j + 1;
    double ljj = std::sqrt(d);
    L[(size_t)j * N + j] = ljj;
    for (int i = j + 1; i < N; ++i) {
      double s = V[(size_t)j * N + i];
      for (int k = 0; k < j; ++k) s -= L[(size_t)k * N + i] * L[(size_t)k * N + j];
      L[(size_t)j * N + i] = s / ljj;
    }
  }
  return 0;
}

// First-call setup of compute_2body_fock_df (src/fockbuild.cpp:598-619):
// B(xy,K) = sum_P T(xy,P) Linv(K,P), Linv = L^-1, V = L L^T.
int orc_df_B(int npair, int naux, const double* T, const double* V, double* B, int nthreads) {
  std::vector<double> L((size_t)naux * naux), Li((size_t)naux * naux, 0.0);
  int st = orc_cholesky(naux, V, L.data());
  if (st) return st;
  // Li = L^-1 by forward substitution on the identity (column-major)
  for (int c = 0; c < naux; ++c) {
    for (int i = 0; i < naux; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) s -= L[(size_t)k * naux + i] * Li[(size_t)c * naux + k];
      Li[(size_t)c * naux + i] = (i < c) ? 0.0 : s / L[(size_t)i * naux + i];
    }
  }
  if (nthreads < 1) nthreads = 1;
  parallel_for(npair, nthreads, [&](int xy, int) {
    std::vector<double> row(naux);
    for (int P = 0; P < naux; ++P) row[P] = T[(size_t)P * npair + xy];
    for (int K = 0; K < naux; ++K) {
      double s = 0;
      for (int P = 0; P <= K; ++P) s += row[P] * Li[(size_t)P * naux + K];
      B[(size_t)K * npair + xy] = s;
    }
  });
  return 0;
}

// Per-iteration part of compute_2body_fock_df (src/fockbuild.cpp:621-659),
// the same naive loops: J, K w.r.t. C C^T; Cocc column-major n x o.
// Restricted to K in [k_begin, k_end) when those bound a sub-range (used to
// time a bounded sample); the full build passes 0, naux.
void orc_df_jk(int n, int naux, int nocc, const double* B, const double* C, double* J, double* K, int k_begin,
               int k_end, int nthreads) {
  const size_t npair = (size_t)n * (n + 1) / 2;
  auto Bx = [&](int x, int y, int Kq) {
    int X = std::max(x, y), Y = std::min(x, y);
    return B[(size_t)Kq * npair + (size_t)X * (X + 1) / 2 + Y];
  };
  const int nK = k_end - k_begin;
  // xiK(x*nocc+i, K)
  std::vector<double> xiK((size_t)n * nocc * nK, 0.0);
  if (nthreads < 1) nthreads = 1;
  parallel_for(n, nthreads, [&](int x, int) {
    for (int i = 0; i < nocc; ++i)
      for (int Kq = k_begin; Kq < k_end; ++Kq) {
        double s = 0;
        for (int y = 0; y < n; ++y) s += Bx(x, y, Kq) * C[(size_t)i * n + y];
        xiK[(size_t)(Kq - k_begin) * n * nocc + (size_t)x * nocc + i] = s;
      }
  });
  parallel_for(n, nthreads, [&](int x, int) {
    for (int y = 0; y <= x; ++y) {
      double s = 0;
      for (int i = 0; i < nocc; ++i)
        for (int Kq = 0; Kq < nK; ++Kq)
          s += xiK[(size_t)Kq * n * nocc + (size_t)x * nocc + i] * xiK[(size_t)Kq * n * nocc + (size_t)y * nocc + i];
      K[(size_t)y * n + x] = s;
      K[(size_t)x * n + y] = s;
    }
  });
  std::vector<double> g(nK, 0.0);
  for (int Kq = 0; Kq < nK; ++Kq)
    for (int x = 0; x < n; ++x)
      for (int i = 0; i < nocc; ++i)
        g[Kq] += xiK[(size_t)Kq * n * nocc + (size_t)x * nocc + i] * C[(size_t)i * n + x];
  parallel_for(n, nthreads, [&](int x, int) {
    for (int y = 0; y <= x; ++y) {
      double s = 0;
      for (int Kq = 0; Kq < nK; ++Kq) s += Bx(x, y, Kq + k_begin) * g[Kq];
      J[(size_t)y * n + x] = s;
      J[(size_t)x * n + y] = s;
    }
  });
}


// compute_1body_ints for S, T, V (src/integrals.cpp:394-449); V sums -Z_C over
// the point charges (natom, Z, xyz). Outputs column-major n x n (symmetric).
void orc_one_body(const orc_basis* obs, int natom, const double* Z, const double* xyz, double* S, double* T,
                  double* V) {
  Basis B = make_basis(obs);
  const int ns = (int)B.sh.size(), n = B.n;
  std::vector<double> s, t, v, vt;
  for (int s1 = 0; s1 < ns; ++s1)
    for (int s2 = 0; s2 < ns; ++s2) {
      const Shell &a = B.sh[s1], &b = B.sh[s2];
      cart_ST(a.l, a.A, a.a, a.c, b.l, b.A, b.a, b.c, &s, &t);
      v.assign(s.size(), 0.0);
      for (int C = 0; C < natom; ++C) {
        cart_V1(a.l, a.A, a.a, a.c, b.l, b.A, b.a, b.c, xyz + 3 * C, vt);
        for (size_t i = 0; i < v.size(); ++i) v[i] -= Z[C] * vt[i];
      }
      to_final2(a.l, a.pure, b.l, b.pure, s);
      to_final2(a.l, a.pure, b.l, b.pure, t);
      to_final2(a.l, a.pure, b.l, b.pure, v);
      int n1 = a.nbf(), n2 = b.nbf();
      for (int f1 = 0; f1 < n1; ++f1)
        for (int f2 = 0; f2 < n2; ++f2) {
          size_t i = B.off[s1] + f1, j = B.off[s2] + f2;
          if (S) S[j * n + i] = s[f1 * n2 + f2];
          if (T) T[j * n + i] = t[f1 * n2 + f2];
          if (V) V[j * n + i] = v[f1 * n2 + f2];
        }
    }
}

}  // extern "C"

namespace {
// d/dA_i of a 2-index Cartesian block where only shell a moves.
template <class F>
void deriv_bra(int la, const std::vector<double>& aa, const std::vector<double>& ca, int lb, int xyz, F blockfn,
               std::vector<double>& out) {
  const auto& T = CT();
  std::vector<double> c2(ca.size()), up, dn;
  for (size_t p = 0; p < ca.size(); ++p) c2[p] = 2.0 * aa[p] * ca[p];
  blockfn(la + 1, c2, up);
  if (la > 0) blockfn(la - 1, ca, dn);
  int na = ncart(la), nb = ncart(lb), nu = ncart(la + 1);
  out.assign((size_t)na * nb, 0.0);
  for (int ia = 0; ia < na; ++ia) {
    auto e = T.comp[la][ia];
    auto ep = e;
    ep[xyz] += 1;
    int iu = T.lid[ep[0]][ep[1]][ep[2]];
    int idn = -1;
    if (e[xyz] > 0) {
      auto em = e;
      em[xyz] -= 1;
      idn = T.lid[em[0]][em[1]][em[2]];
    }
    for (int ib = 0; ib < nb; ++ib) {
      double v = up[(size_t)iu * nb + ib];
      if (idn >= 0) v -= e[xyz] * dn[(size_t)idn * nb + ib];
      out[(size_t)ia * nb + ib] = v;
    }
  }
  (void)nu;
}
}  // namespace

extern "C" {

// compute_1body_ints_deriv<kinetic/nuclear/overlap>(1) (inc/integrals.hpp:169-349):
// 3*natom matrices each (coord = 3*atom + xyz), column-major n x n.
// shell_atom maps shells to atoms (src/integrals.cpp:384-392).
void orc_one_body_deriv(const orc_basis* obs, const int* shell_atom, int natom, const double* Z,
                        const double* xyz, double* S1, double* T1, double* V1) {
  Basis B = make_basis(obs);
  const int ns = (int)B.sh.size(), n = B.n;
  const size_t nn = (size_t)n * n;
  if (S1) std::memset(S1, 0, sizeof(double) * nn * 3 * natom);
  if (T1) std::memset(T1, 0, sizeof(double) * nn * 3 * natom);
  if (V1) std::memset(V1, 0, sizeof(double) * nn * 3 * natom);
  for (int s1 = 0; s1 < ns; ++s1)
    for (int s2 = 0; s2 < ns; ++s2) {
      const Shell &a = B.sh[s1], &b = B.sh[s2];
      const int n1 = a.nbf(), n2 = b.nbf();
      auto put = [&](double* M, int coord, std::vector<double> blk, double scale) {
        to_final2(a.l, a.pure, b.l, b.pure, blk);
        for (int f1 = 0; f1 < n1; ++f1)
          for (int f2 = 0; f2 < n2; ++f2) {
            size_t i = B.off[s1] + f1, j = B.off[s2] + f2;
            M[(size_t)coord * nn + j * n + i] += scale * blk[f1 * n2 + f2];
          }
      };
      for (int x = 0; x < 3; ++x) {
        std::vector<double> dA_s, dA_t, dB_s, dB_t, tmp;
        // d/dA: move a; d/dB: move b (via the transposed problem)
        deriv_bra(a.l, a.a, a.c, b.l, x,
                  [&](int l, const std::vector<double>& c, std::vector<double>& o) {
                    cart_ST(l, a.A, a.a, c, b.l, b.A, b.a, b.c, &o, nullptr);
                  }, dA_s);
        deriv_bra(a.l, a.a, a.c, b.l, x,
                  [&](int l, const std::vector<double>& c, std::vector<double>& o) {
                    cart_ST(l, a.A, a.a, c, b.l, b.A, b.a, b.c, nullptr, &o);
                  }, dA_t);
        // translational invariance for S and T: d/dB = -d/dA
        if (S1) {
          put(S1, 3 * shell_atom[s1] + x, dA_s, 1.0);
          put(S1, 3 * shell_atom[s2] + x, dA_s, -1.0);
        }
        if (T1) {
          put(T1, 3 * shell_atom[s1] + x, dA_t, 1.0);
          put(T1, 3 * shell_atom[s2] + x, dA_t, -1.0);
        }
        if (V1) {
          // per nucleus C: d/dA, d/dB explicit; d/dC = -(d/dA + d/dB)
          for (int C = 0; C < natom; ++C) {
            std::vector<double> dA_v, dB_vT, dB_v((size_t)ncart(a.l) * ncart(b.l));
            deriv_bra(a.l, a.a, a.c, b.l, x,
                      [&](int l, const std::vector<double>& c, std::vector<double>& o) {
                        cart_V1(l, a.A, a.a, c, b.l, b.A, b.a, b.c, xyz + 3 * C, o);
                      }, dA_v);
            deriv_bra(b.l, b.a, b.c, a.l, x,
                      [&](int l, const std::vector<double>& c, std::vector<double>& o) {
                        cart_V1(l, b.A, b.a, c, a.l, a.A, a.a, a.c, xyz + 3 * C, o);
                      }, dB_vT);
            int na = ncart(a.l), nb = ncart(b.l);
            for (int i = 0; i < na; ++i)
              for (int j = 0; j < nb; ++j) dB_v[(size_t)i * nb + j] = dB_vT[(size_t)j * na + i];
            std::vector<double> dC(dA_v.size());
            for (size_t k = 0; k < dC.size(); ++k) dC[k] = -(dA_v[k] + dB_v[k]);
            put(V1, 3 * shell_atom[s1] + x, dA_v, -Z[C]);
            put(V1, 3 * shell_atom[s2] + x, dB_v, -Z[C]);
            put(V1, 3 * C + x, dC, -Z[C]);
          }
        }
      }
    }
}

// compute_shellpair_list (src/integrals.cpp:515-566): flags[s1*ns+s2] = 1 for
// s2 <= s1 with the same centre or overlap-block Frobenius norm >= threshold.
void orc_shellpair_list(const orc_basis* obs, double threshold, int* flags) {
  Basis B = make_basis(obs);
  const int ns = (int)B.sh.size();
  std::vector<double> s;
  for (int s1 = 0; s1 < ns; ++s1)
    for (int s2 = 0; s2 < ns; ++s2) {
      int f = 0;
      if (s2 <= s1) {
        const Shell &a = B.sh[s1], &b = B.sh[s2];
        bool same = a.A[0] == b.A[0] && a.A[1] == b.A[1] && a.A[2] == b.A[2];
        if (same) {
          f = 1;
        } else {
          cart_ST(a.l, a.A, a.a, a.c, b.l, b.A, b.a, b.c, &s, nullptr);
          to_final2(a.l, a.pure, b.l, b.pure, s);
          double nrm = 0;
          for (double x : s) nrm += x * x;
          f = std::sqrt(nrm) >= threshold;
        }
      }
      flags[(size_t)s1 * ns + s2] = f;
    }
}

// Fock::compute_2body_fock_deriv<1> (src/rhfgrad.cpp:419-598) followed by
// the contraction of compute_forces (:48-57): returns grad[3*natom] =
// 0.25 * sum_ab G1[coord](a,b) D(a,b), and, when G1 != NULL, the 3*natom
// symmetrised derivative Fock matrices (column-major).  Q is the Schwarz
// matrix; screening uses D as the reference does with its member density.
static void grad2e_rows(const orc_basis* obs, const int* shell_atom, int natom, const double* D, const double* Q,
                        double precision, double* G1, double* grad, int nthreads, int s1_begin, int s1_step);

void orc_grad2e(const orc_basis* obs, const int* shell_atom, int natom, const double* D, const double* Q,
                double precision, double* G1, double* grad, int nthreads) {
  grad2e_rows(obs, shell_atom, natom, D, Q, precision, G1, grad, nthreads, 0, 1);
}

// Time-bounded variant for the CPU baseline: the same loop over the shell rows
// s1 = s1_begin, s1_begin + s1_step, ... only (one thread).
void orc_grad2e_rows(const orc_basis* obs, const int* shell_atom, int natom, const double* D, const double* Q,
                     double precision, int s1_begin, int s1_step, double* grad) {
  grad2e_rows(obs, shell_atom, natom, D, Q, precision, nullptr, grad, 1, s1_begin, s1_step);
}

static void grad2e_rows(const orc_basis* obs, const int* shell_atom, int natom, const double* D, const double* Q,
                        double precision, double* G1, double* grad, int nthreads, int s1_begin, int s1_step) {
  Basis B = make_basis(obs);
  const int ns = (int)B.sh.size(), n = B.n;
  std::vector<int> rows;
  for (int s = s1_begin; s < ns; s += s1_step) rows.push_back(s);
  const size_t nn = (size_t)n * n;
  auto Dn = shellblock_norm(B, D);
  std::vector<int> flags((size_t)ns * ns);
  orc_shellpair_list(obs, 1e-12, flags.data());
  std::vector<std::vector<int>> plist(ns);
  for (int s1 = 0; s1 < ns; ++s1)
    for (int s2 = 0; s2 <= s1; ++s2)
      if (flags[(size_t)s1 * ns + s2]) plist[s1].push_back(s2);
  if (nthreads < 1) nthreads = 1;
  std::vector<std::vector<double>> Gt(nthreads, std::vector<double>(nn * 3 * natom, 0.0));
  auto dn = [&](int a, int c) { return Dn[(size_t)a * ns + c]; };
  auto Dm = [&](size_t i, size_t j) { return D[j * n + i]; };
  parallel_for((int)rows.size(), nthreads, [&](int r, int t) {
    const int s1 = rows[r];
    double* G = Gt[t].data();
    std::vector<double> buf;
    for (int s2 : plist[s1]) {
      const double Dnorm12 = dn(s1, s2);
      for (int s3 = 0; s3 <= s1; ++s3) {
        const double Dnorm123 = std::max(dn(s1, s3), std::max(dn(s2, s3), Dnorm12));
        const int s4_max = (s1 == s3) ? s2 : s3;
        for (int s4 : plist[s3]) {
          if (s4 > s4_max) break;
          const double Dnorm1234 = std::max(dn(s1, s4), std::max(dn(s2, s4), std::max(dn(s3, s4), Dnorm123)));
          if (Dnorm1234 * Q[(size_t)s1 * ns + s2] * Q[(size_t)s3 * ns + s4] < precision) continue;
          double deg = ((s1 == s2) ? 1.0 : 2.0) * ((s3 == s4) ? 1.0 : 2.0) * ((s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0);
          const Shell* sh[4] = {&B.sh[s1], &B.sh[s2], &B.sh[s3], &B.sh[s4]};
          const int ss[4] = {s1, s2, s3, s4};
          int n1 = sh[0]->nbf(), n2 = sh[1]->nbf(), n3 = sh[2]->nbf(), n4 = sh[3]->nbf();
          for (int d = 0; d < 12; ++d) {
            const int c = d / 3, x = d % 3;
            shell_eri_deriv(sh, c, x, buf);
            double* g = G + (size_t)(3 * shell_atom[ss[c]] + x) * nn;
            for (int f1 = 0, f = 0; f1 < n1; ++f1) {
              size_t b1 = B.off[s1] + f1;
              for (int f2 = 0; f2 < n2; ++f2) {
                size_t b2 = B.off[s2] + f2;
                for (int f3 = 0; f3 < n3; ++f3) {
                  size_t b3 = B.off[s3] + f3;
                  for (int f4 = 0; f4 < n4; ++f4, ++f) {
                    size_t b4 = B.off[s4] + f4;
                    double w = buf[f] * deg;
                    g[b2 * n + b1] += Dm(b3, b4) * w;
                    g[b4 * n + b3] += Dm(b1, b2) * w;
                    g[b3 * n + b1] -= 0.25 * Dm(b2, b4) * w;
                    g[b4 * n + b2] -= 0.25 * Dm(b1, b3) * w;
                    g[b4 * n + b1] -= 0.25 * Dm(b2, b3) * w;
                    g[b3 * n + b2] -= 0.25 * Dm(b1, b4) * w;
                  }
                }
              }
            }
          }
        }
      }
    }
  });
  for (int t = 1; t < nthreads; ++t)
    for (size_t i = 0; i < Gt[0].size(); ++i) Gt[0][i] += Gt[t][i];
  for (int cidx = 0; cidx < 3 * natom; ++cidx) {
    const double* g = Gt[0].data() + (size_t)cidx * nn;
    double acc = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double sym = 0.5 * (g[(size_t)j * n + i] + g[(size_t)i * n + j]);
        if (G1) G1[(size_t)cidx * nn + (size_t)j * n + i] = sym;
        acc += sym * D[(size_t)j * n + i];
      }
    grad[cidx] = 0.25 * acc;
  }
}

// Three-index derivative block (P|mn)' for the DF gradient: d/d(center c) of
// shell set (aux s1 | obs s2 s3), c in {0: aux, 2: obs s2, 3: obs s3}.
void orc_eri3_deriv_block(const orc_basis* obs, const orc_basis* aux, int sa, int s2, int s3, int center, int xyz,
                          double* out) {
  Basis B = make_basis(obs), Ba = make_basis(aux);
  Shell u = unit_shell(Ba.sh[sa].A);
  const Shell* sh[4] = {&Ba.sh[sa], &u, &B.sh[s2], &B.sh[s3]};
  std::vector<double> v;
  shell_eri_deriv(sh, center, xyz, v);
  std::memcpy(out, v.data(), v.size() * sizeof(double));
}

// Two-electron part of the density-fitted RHF gradient, the contraction step
// (test restatement of the derivative of the DF energy of
// src/fockbuild.cpp:585-660): with the three-index weights M3[P][m][n]
// (naux x n x n, n fastest) and the metric weights M2[P][Q] (naux x naux),
//   grad[3 A + x] = sum_{P,m,n} d(P|mn)/dA_x M3[P][m][n]
//                 + sum_{P,Q}   d(P|Q)/dA_x  M2[P][Q],
// every derivative integral from shell_eri_deriv (all shell combinations, no
// screening).  The weights come from oracle.df_grad2e.
void orc_df_grad_contract(const orc_basis* obs, const orc_basis* aux, const int* obs_atom, const int* aux_atom,
                          int natom, const double* M3, const double* M2, double* grad, int nthreads) {
  Basis B = make_basis(obs), Ba = make_basis(aux);
  const int ns = (int)B.sh.size(), na = (int)Ba.sh.size(), n = B.n, naux = Ba.n;
  if (nthreads < 1) nthreads = 1;
  std::vector<std::vector<double>> gt(nthreads, std::vector<double>(3 * (size_t)natom, 0.0));
  parallel_for(na, nthreads, [&](int sa, int t) {
    double* g = gt[t].data();
    std::vector<double> buf;
    const Shell u = unit_shell(Ba.sh[sa].A);
    const int np = Ba.sh[sa].nbf();
    for (int s2 = 0; s2 < ns; ++s2)
      for (int s3 = 0; s3 < ns; ++s3) {
        const Shell* sh[4] = {&Ba.sh[sa], &u, &B.sh[s2], &B.sh[s3]};
        const int n2 = B.sh[s2].nbf(), n3 = B.sh[s3].nbf();
        const int centre_atom[4] = {aux_atom[sa], -1, obs_atom[s2], obs_atom[s3]};
        for (int c : {0, 2, 3})
          for (int x = 0; x < 3; ++x) {
            shell_eri_deriv(sh, c, x, buf);
            double acc = 0.0;
            for (int fp = 0, f = 0; fp < np; ++fp)
              for (int f2 = 0; f2 < n2; ++f2)
                for (int f3 = 0; f3 < n3; ++f3, ++f)
                  acc += buf[f] * M3[((size_t)(Ba.off[sa] + fp) * n + B.off[s2] + f2) * n + B.off[s3] + f3];
            g[3 * centre_atom[c] + x] += acc;
          }
      }
    for (int sb = 0; sb < na; ++sb) {
      const Shell u2 = unit_shell(Ba.sh[sb].A);
      const Shell* sh[4] = {&Ba.sh[sa], &u, &Ba.sh[sb], &u2};
      const int nq = Ba.sh[sb].nbf();
      const int centre_atom[4] = {aux_atom[sa], -1, aux_atom[sb], -1};
      for (int c : {0, 2})
        for (int x = 0; x < 3; ++x) {
          shell_eri_deriv(sh, c, x, buf);
          double acc = 0.0;
          for (int fp = 0, f = 0; fp < np; ++fp)
            for (int fq = 0; fq < nq; ++fq, ++f) acc += buf[f] * M2[(size_t)(Ba.off[sa] + fp) * naux + Ba.off[sb] + fq];
          g[3 * centre_atom[c] + x] += acc;
        }
    }
  });
  for (int k = 0; k < 3 * natom; ++k) {
    double a = 0.0;
    for (int t = 0; t < nthreads; ++t) a += gt[t][k];
    grad[k] = a;
  }
}

void orc_eri4_deriv_block(const orc_basis* obs, int s1, int s2, int s3, int s4, int center, int xyz, double* out) {
  Basis B = make_basis(obs);
  const Shell* sh[4] = {&B.sh[s1], &B.sh[s2], &B.sh[s3], &B.sh[s4]};
  std::vector<double> v;
  shell_eri_deriv(sh, center, xyz, v);
  std::memcpy(out, v.data(), v.size() * sizeof(double));
}

}  // extern "C"
