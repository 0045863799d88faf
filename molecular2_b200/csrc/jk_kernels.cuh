// Device side of the integral-direct J/K build and the Schwarz bounds (FP64).
// Included by the per-class translation units jk_cls_*.cu and jk_direct.cu.
#pragma once
#include "md.cuh"

namespace m2 {

struct PairView {
  const int* sa;
  const int* sb;
  const int* prim_off;
  const int* nprim;
  const double* Q;
  int npair;
};
struct PrimView {
  const double *p, *x, *y, *z, *K;
};
struct ShellView {
  const double *x, *y, *z;
  const int* coff;  // Cartesian function offset
};

__host__ __device__ constexpr double PI25X2() { return 34.986836655249725; }  // 2 pi^(5/2)

// Hermite triples and Cartesian exponents by index, for the classes whose
// loops stay rolled (tables cover totals up to 9).
struct HermTab {
  unsigned char t[nherm(9)], u[nherm(9)], v[nherm(9)];
};
__host__ __device__ constexpr HermTab make_herm_tab() {
  HermTab h{};
  int i = 0;
  for (int k = 0; k <= 9; ++k)
    for (int j = 0; j < ncart(k); ++j, ++i) {
      h.t[i] = (unsigned char)cart_a(k, j);
      h.u[i] = (unsigned char)cart_b(k, j);
      h.v[i] = (unsigned char)cart_c(k, j);
    }
  return h;
}
__constant__ constexpr HermTab c_herm = make_herm_tab();

// Classes with more than this many Cartesian integrals keep their component
// loops rolled (small code, arrays in local memory); the rest unroll fully.
constexpr int UNROLL_LIMIT = 100;

// Contracted Cartesian (ab|cd) for one quartet of shell pairs, accumulated
// over primitive pairs.  out[((ia*NB+ib)*NC+ic)*ND+id].
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void quartet_cart(const PrimView& pp, int b0, int nb, double Ax, double Ay, double Az,
                                             double Bx, double By, double Bz, const PrimView& kp, int k0, int nk,
                                             double Cx, double Cy, double Cz, double Dx, double Dy, double Dz,
                                             const double* __restrict__ boys_tab, double* out) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int LAB = LA + LB, LCD = LC + LD, L = LAB + LCD;
  constexpr int NAB = NA * NB, NCD = NC * ND;
  constexpr bool BIG = NAB * NCD > UNROLL_LIMIT;
#pragma unroll
  for (int i = 0; i < NAB * NCD; ++i) out[i] = 0.0;
  for (int ib = b0; ib < b0 + nb; ++ib) {
    const double p = __ldg(pp.p + ib), Px = __ldg(pp.x + ib), Py = __ldg(pp.y + ib), Pz = __ldg(pp.z + ib);
    const double Kab = __ldg(pp.K + ib);
    E1<LA, LB> ex, ey, ez;
    const double oo2p = 0.5 / p;
    md_E1<LA, LB>(Px - Ax, Px - Bx, oo2p, ex);
    md_E1<LA, LB>(Py - Ay, Py - By, oo2p, ey);
    md_E1<LA, LB>(Pz - Az, Pz - Bz, oo2p, ez);
    for (int ik = k0; ik < k0 + nk; ++ik) {
      const double q = __ldg(kp.p + ik), Qx = __ldg(kp.x + ik), Qy = __ldg(kp.y + ik), Qz = __ldg(kp.z + ik);
      const double Kcd = __ldg(kp.K + ik);
      E1<LC, LD> fx, fy, fz;
      const double oo2q = 0.5 / q;
      md_E1<LC, LD>(Qx - Cx, Qx - Dx, oo2q, fx);
      md_E1<LC, LD>(Qy - Cy, Qy - Dy, oo2q, fy);
      md_E1<LC, LD>(Qz - Cz, Qz - Dz, oo2q, fz);
      const double pq = p + q;
      const double alpha = p * q / pq;
      const double pref = PI25X2() / (p * q * sqrt(pq)) * Kab * Kcd;
      const double X = Px - Qx, Y = Py - Qy, Z = Pz - Qz;
      double F[L + 1];
      boys<L>(alpha * (X * X + Y * Y + Z * Z), boys_tab, F);
      double R[nherm(L)];
      md_R<L>(alpha, X, Y, Z, F, R);
      if constexpr (!BIG) {
#pragma unroll
        for (int icd = 0; icd < NCD; ++icd) {
          const int ic = icd / ND, id = icd % ND;
          const int cx = cart_a(LC, ic), cy = cart_b(LC, ic), cz = cart_c(LC, ic);
          const int dx = cart_a(LD, id), dy = cart_b(LD, id), dz = cart_c(LD, id);
          double W[nherm(LAB)];
#pragma unroll
          for (int h = 0; h < nherm(LAB); ++h) {
            int k = 0;
            while (nherm(k) <= h) ++k;
            const int i = h - (k > 0 ? nherm(k - 1) : 0);
            const int t = cart_a(k, i), u = cart_b(k, i), v = cart_c(k, i);
            double s = 0.0;
#pragma unroll
            for (int tau = 0; tau <= cx + dx; ++tau)
#pragma unroll
              for (int nu = 0; nu <= cy + dy; ++nu)
#pragma unroll
                for (int phi = 0; phi <= cz + dz; ++phi) {
                  const double e = fx.e[cx][dx][tau] * fy.e[cy][dy][nu] * fz.e[cz][dz][phi];
                  const double r = R[hidx(t + tau, u + nu, v + phi)];
                  s += ((tau + nu + phi) & 1) ? -e * r : e * r;
                }
            W[h] = s;
          }
#pragma unroll
          for (int iab = 0; iab < NAB; ++iab) {
            const int ia = iab / NB, ibb = iab % NB;
            const int ax = cart_a(LA, ia), ay = cart_b(LA, ia), az = cart_c(LA, ia);
            const int bx = cart_a(LB, ibb), by = cart_b(LB, ibb), bz = cart_c(LB, ibb);
            double acc = 0.0;
#pragma unroll
            for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
              for (int u = 0; u <= ay + by; ++u)
#pragma unroll
                for (int v = 0; v <= az + bz; ++v)
                  acc += ex.e[ax][bx][t] * ey.e[ay][by][u] * ez.e[az][bz][v] * W[hidx(t, u, v)];
            out[iab * NCD + icd] += pref * acc;
          }
        }
      } else {
        const int cbase = nherm(LC - 1 < 0 ? -1 : LC - 1) * (LC > 0);
        const int dbase = nherm(LD - 1 < 0 ? -1 : LD - 1) * (LD > 0);
        const int abase = nherm(LA - 1 < 0 ? -1 : LA - 1) * (LA > 0);
        const int bbase = nherm(LB - 1 < 0 ? -1 : LB - 1) * (LB > 0);
#pragma unroll 1
        for (int icd = 0; icd < NCD; ++icd) {
          const int ic = icd / ND, id = icd % ND;
          const int cx = c_herm.t[cbase + ic], cy = c_herm.u[cbase + ic], cz = c_herm.v[cbase + ic];
          const int dx = c_herm.t[dbase + id], dy = c_herm.u[dbase + id], dz = c_herm.v[dbase + id];
          double W[nherm(LAB)];
#pragma unroll 1
          for (int h = 0; h < nherm(LAB); ++h) {
            const int t = c_herm.t[h], u = c_herm.u[h], v = c_herm.v[h];
            double s = 0.0;
            for (int tau = 0; tau <= cx + dx; ++tau)
              for (int nu = 0; nu <= cy + dy; ++nu) {
                const double exy = fx.e[cx][dx][tau] * fy.e[cy][dy][nu];
                for (int phi = 0; phi <= cz + dz; ++phi) {
                  const double e = exy * fz.e[cz][dz][phi];
                  const double r = R[hidx(t + tau, u + nu, v + phi)];
                  s += ((tau + nu + phi) & 1) ? -e * r : e * r;
                }
              }
            W[h] = s;
          }
#pragma unroll 1
          for (int iab = 0; iab < NAB; ++iab) {
            const int ia = iab / NB, ibb = iab % NB;
            const int ax = c_herm.t[abase + ia], ay = c_herm.u[abase + ia], az = c_herm.v[abase + ia];
            const int bx = c_herm.t[bbase + ibb], by = c_herm.u[bbase + ibb], bz = c_herm.v[bbase + ibb];
            double acc = 0.0;
            for (int t = 0; t <= ax + bx; ++t)
              for (int u = 0; u <= ay + by; ++u) {
                const double exy = ex.e[ax][bx][t] * ey.e[ay][by][u];
                for (int v = 0; v <= az + bz; ++v) acc += exy * ez.e[az][bz][v] * W[hidx(t, u, v)];
              }
            out[iab * NCD + icd] += pref * acc;
          }
        }
      }
    }
  }
}

struct JKParams {
  PairView bra, ket;
  int same_class;
  PrimView pp;
  ShellView sh;
  const double* Dnorm;  // nshell x nshell (final-basis shell-block max norms)
  int nshell;
  const double* Dmax;   // device scalar
  const double* Dc;     // Cartesian density, nc x nc (NDEN of them, dstride apart)
  int nc;
  double* Jc;           // raw accumulators (NDEN of each, dstride apart)
  double* Kc;
  size_t dstride;       // elements between consecutive densities / accumulators
  double precision;
  const double* boys;
  unsigned long long* counter;
  unsigned long long* work;  // NULL or this class pair's [quartets, sum bra primitive pairs, sum primitive quartets]
  int kchunk;
  int bra0, bra_step;        // block x handles bra pair bra0 + x * bra_step (a rank's share of the class)
};

// Pairs of a class are sorted by Schwarz bound Q descending and then, inside
// consecutive windows of PAIR_WINDOW pairs, by contraction length, so that
// the 32 kets of a warp have similar primitive counts.  The Q prefix of a
// threshold is therefore rounded up to a whole window; the per-ket screen
// drops the extra kets.  Every Q of a window is >= every Q of the next one,
// so a binary search lands inside the window holding the cut; window_up
// returns the end of the window containing index k (k itself included).
constexpr int PAIR_WINDOW = 256;
__device__ __forceinline__ int window_up(int k, int n) {
  return min(n, (k / PAIR_WINDOW + 1) * PAIR_WINDOW);
}

// number of kets in [0, n) whose Q >= thr (Q sorted descending)
__device__ __forceinline__ int q_prefix(const double* Q, int n, double thr) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(Q + mid) >= thr)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void atomic_add_f64(double* a, double v) {
  if (v != 0.0) atomicAdd(a, v);
}

// NDEN densities (1: RHF; 2: the alpha and beta densities of UHF,
// UnrestrictedFock::formJKdirect, src/fockbuild.cpp:266-362) are digested from
// the same integrals; the screen uses the norms of their sum.
template <int LA, int LB, int LC, int LD, int NDEN = 1>
__global__ void __launch_bounds__(128) k_jk_direct(const JKParams P) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr bool BIG = NA * NB * NC * ND > UNROLL_LIMIT;
  const int bra = P.bra0 + blockIdx.x * P.bra_step;
  const int a = P.bra.sa[bra], b = P.bra.sb[bra];
  const double Qab = P.bra.Q[bra];
  const double Dmax = *P.Dmax;
  if (!(Qab * Dmax > 0.0)) return;
  int nket = window_up(q_prefix(P.ket.Q, P.ket.npair, P.precision / (Qab * Dmax)), P.ket.npair);
  if (P.same_class) nket = min(nket, bra + 1);
  const int start = blockIdx.y * P.kchunk;
  if (start >= nket) return;
  const int end = min(start + P.kchunk, nket);

  const double Ax = P.sh.x[a], Ay = P.sh.y[a], Az = P.sh.z[a];
  const double Bx = P.sh.x[b], By = P.sh.y[b], Bz = P.sh.z[b];
  const int a0 = P.sh.coff[a], b0 = P.sh.coff[b];
  const int bp0 = P.bra.prim_off[bra], bnp = P.bra.nprim[bra];
  const int nc = P.nc;

  double jab[NDEN][NA * NB];
#pragma unroll
  for (int dd = 0; dd < NDEN; ++dd)
#pragma unroll
    for (int i = 0; i < NA * NB; ++i) jab[dd][i] = 0.0;
  unsigned long long cnt = 0, wb = 0, wq = 0;

  for (int kl = start + threadIdx.x; kl < end; kl += blockDim.x) {
    const int c = P.ket.sa[kl], d = P.ket.sb[kl];
    const double Qcd = P.ket.Q[kl];
    const double* Dn = P.Dnorm;
    const int ns = P.nshell;
    double dn = fmax(fmax(Dn[a * ns + b], Dn[c * ns + d]), fmax(Dn[a * ns + c], Dn[a * ns + d]));
    dn = fmax(dn, fmax(Dn[b * ns + c], Dn[b * ns + d]));
    if (dn * Qab * Qcd < P.precision) continue;
    ++cnt;
    wb += bnp;
    wq += (unsigned long long)bnp * P.ket.nprim[kl];
    double eri[NA * NB * NC * ND];
    quartet_cart<LA, LB, LC, LD>(P.pp, bp0, bnp, Ax, Ay, Az, Bx, By, Bz, P.pp, P.ket.prim_off[kl], P.ket.nprim[kl],
                                 P.sh.x[c], P.sh.y[c], P.sh.z[c], P.sh.x[d], P.sh.y[d], P.sh.z[d], P.boys, eri);
    const double deg = ((a == b) ? 1.0 : 2.0) * ((c == d) ? 1.0 : 2.0) * ((P.same_class && kl == bra) ? 1.0 : 2.0);
    const int c0 = P.sh.coff[c], d0 = P.sh.coff[d];
#pragma unroll
    for (int dd = 0; dd < NDEN; ++dd) {
    const double* __restrict__ Dc = P.Dc + dd * P.dstride;
    double* __restrict__ Jd = P.Jc + dd * P.dstride;
    double* __restrict__ Kd = P.Kc + dd * P.dstride;
    double jcd[NC * ND], kac[NA * NC], kbd[NB * ND], kad[NA * ND], kbc[NB * NC];
#pragma unroll
    for (int i = 0; i < NC * ND; ++i) jcd[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NA * NC; ++i) kac[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NB * ND; ++i) kbd[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NA * ND; ++i) kad[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NB * NC; ++i) kbc[i] = 0.0;
    if constexpr (!BIG) {
#pragma unroll
      for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
          const double dab = Dc[(size_t)(a0 + ia) * nc + b0 + ib];
#pragma unroll
          for (int ic = 0; ic < NC; ++ic) {
            const double dac = Dc[(size_t)(a0 + ia) * nc + c0 + ic];
            const double dbc = Dc[(size_t)(b0 + ib) * nc + c0 + ic];
#pragma unroll
            for (int id = 0; id < ND; ++id) {
              const double v = eri[((ia * NB + ib) * NC + ic) * ND + id] * deg;
              jab[dd][ia * NB + ib] += Dc[(size_t)(c0 + ic) * nc + d0 + id] * v;
              jcd[ic * ND + id] += dab * v;
              kac[ia * NC + ic] += Dc[(size_t)(b0 + ib) * nc + d0 + id] * v;
              kbd[ib * ND + id] += dac * v;
              kad[ia * ND + id] += dbc * v;
              kbc[ib * NC + ic] += Dc[(size_t)(a0 + ia) * nc + d0 + id] * v;
            }
          }
        }
    } else {
#pragma unroll 1
      for (int ia = 0; ia < NA; ++ia)
#pragma unroll 1
        for (int ib = 0; ib < NB; ++ib) {
          const double dab = Dc[(size_t)(a0 + ia) * nc + b0 + ib];
          double jsum = 0.0;
#pragma unroll 1
          for (int ic = 0; ic < NC; ++ic) {
            const double dac = Dc[(size_t)(a0 + ia) * nc + c0 + ic];
            const double dbc = Dc[(size_t)(b0 + ib) * nc + c0 + ic];
            double kacs = 0.0, kbcs = 0.0;
#pragma unroll
            for (int id = 0; id < ND; ++id) {
              const double v = eri[((ia * NB + ib) * NC + ic) * ND + id] * deg;
              jsum += Dc[(size_t)(c0 + ic) * nc + d0 + id] * v;
              jcd[ic * ND + id] += dab * v;
              kacs += Dc[(size_t)(b0 + ib) * nc + d0 + id] * v;
              kbd[ib * ND + id] += dac * v;
              kad[ia * ND + id] += dbc * v;
              kbcs += Dc[(size_t)(a0 + ia) * nc + d0 + id] * v;
            }
            kac[ia * NC + ic] += kacs;
            kbc[ib * NC + ic] += kbcs;
          }
          jab[dd][ia * NB + ib] += jsum;
        }
    }
#pragma unroll
    for (int i = 0; i < NC * ND; ++i) atomic_add_f64(Jd + (size_t)(c0 + i / ND) * nc + d0 + i % ND, jcd[i]);
#pragma unroll
    for (int i = 0; i < NA * NC; ++i) atomic_add_f64(Kd + (size_t)(a0 + i / NC) * nc + c0 + i % NC, kac[i]);
#pragma unroll
    for (int i = 0; i < NB * ND; ++i) atomic_add_f64(Kd + (size_t)(b0 + i / ND) * nc + d0 + i % ND, kbd[i]);
#pragma unroll
    for (int i = 0; i < NA * ND; ++i) atomic_add_f64(Kd + (size_t)(a0 + i / ND) * nc + d0 + i % ND, kad[i]);
#pragma unroll
    for (int i = 0; i < NB * NC; ++i) atomic_add_f64(Kd + (size_t)(b0 + i / NC) * nc + c0 + i % NC, kbc[i]);
    }  // densities
  }
  // J_ab: the whole block shares the bra pair
  const unsigned lane = threadIdx.x & 31;
#pragma unroll
  for (int dd = 0; dd < NDEN; ++dd)
#pragma unroll
    for (int i = 0; i < NA * NB; ++i) {
      double v = jab[dd][i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) atomic_add_f64(P.Jc + dd * P.dstride + (size_t)(a0 + i / NB) * nc + b0 + i % NB, v);
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    wb += __shfl_down_sync(0xffffffffu, wb, o);
    wq += __shfl_down_sync(0xffffffffu, wq, o);
  }
  if (lane == 0 && cnt) {
    atomicAdd(P.counter, cnt);
    if (P.work) {
      atomicAdd(P.work, cnt);
      atomicAdd(P.work + 1, wb);
      atomicAdd(P.work + 2, wq);
    }
  }
}

// Schwarz bound of each pair of one class: sqrt(max diag (ab|ab)) over the
// final (pure or Cartesian) functions (compute_schwarz_ints, src/integrals.cpp:472-513).
struct SchwarzParams {
  PairView pairs;
  PrimView pp;
  ShellView sh;
  const int* l;
  const int* pure;
  const double* sph;
  const double* boys;
  double* Qout;
};

template <int LA, int LB>
__global__ void __launch_bounds__(64) k_schwarz(const SchwarzParams P) {
  constexpr int NA = ncart(LA), NB = ncart(LB);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.pairs.npair) return;
  const int a = P.pairs.sa[i], b = P.pairs.sb[i];
  double eri[NA * NB * NA * NB];
  const int p0 = P.pairs.prim_off[i], np = P.pairs.nprim[i];
  const double Ax = P.sh.x[a], Ay = P.sh.y[a], Az = P.sh.z[a], Bx = P.sh.x[b], By = P.sh.y[b], Bz = P.sh.z[b];
  quartet_cart<LA, LB, LA, LB>(P.pp, p0, np, Ax, Ay, Az, Bx, By, Bz, P.pp, p0, np, Ax, Ay, Az, Bx, By, Bz, P.boys,
                               eri);
  const int pa = P.pure[a], pb = P.pure[b];
  const int ma = pa ? 2 * LA + 1 : NA, mb = pb ? 2 * LB + 1 : NB;
  double m = 0.0;
#pragma unroll 1
  for (int mu = 0; mu < ma; ++mu)
#pragma unroll 1
    for (int nu = 0; nu < mb; ++nu) {
      double v = 0.0;
#pragma unroll 1
      for (int a1 = 0; a1 < NA; ++a1) {
        const double t1 = pa ? P.sph[sph_off(LA) + mu * NA + a1] : (a1 == mu ? 1.0 : 0.0);
        if (t1 == 0.0) continue;
#pragma unroll 1
        for (int b1 = 0; b1 < NB; ++b1) {
          const double t2 = pb ? P.sph[sph_off(LB) + nu * NB + b1] : (b1 == nu ? 1.0 : 0.0);
          if (t2 == 0.0) continue;
#pragma unroll 1
          for (int a2 = 0; a2 < NA; ++a2) {
            const double t3 = pa ? P.sph[sph_off(LA) + mu * NA + a2] : (a2 == mu ? 1.0 : 0.0);
            if (t3 == 0.0) continue;
#pragma unroll 1
            for (int b2 = 0; b2 < NB; ++b2) {
              const double t4 = pb ? P.sph[sph_off(LB) + nu * NB + b2] : (b2 == nu ? 1.0 : 0.0);
              if (t4 == 0.0) continue;
              v += t1 * t2 * t3 * t4 * eri[((a1 * NB + b1) * NA + a2) * NB + b2];
            }
          }
        }
      }
      m = fmax(m, fabs(v));
    }
  P.Qout[i] = sqrt(m);
}

struct PairClassDev;
PairView view(const PairClassDev& c);

// per-translation-unit launchers (jk_cls_*.cu); A, B are pair-class ids
// nden: densities digested per quartet (1 or 2)
void launch_jk_bra_s(int A, int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s);   // A in {0,1,2}
void launch_jk_bra_ds(int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s);         // A = 3
void launch_jk_bra_dp(int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s);         // A = 4
void launch_jk_bra_dd_lo(int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s);      // A = 5, B < 4
void launch_jk_bra_dd_hi(int B, int nden, const JKParams& P, dim3 grid, cudaStream_t s);      // A = 5, B >= 4
void launch_schwarz_dd(const SchwarzParams& P, dim3 grid, cudaStream_t s);

}  // namespace m2
