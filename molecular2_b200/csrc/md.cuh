// McMurchie-Davidson integral machinery for sm_100a (FP64).
//
// Gaussian products are expanded in Hermite Gaussians with the E coefficients
//   E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}
//   E^{i,j+1}_t = E^{ij}_{t-1}/(2p) + X_PB E^{ij}_t + (t+1) E^{ij}_{t+1}
// and Coulomb integrals over Hermite functions use the R recursion
//   R^{(n)}_{000} = (-2a)^n F_n(a R_PQ^2),
//   R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} + X_PQ R^{(n+1)}_{t,u,v}
// (McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978); Helgaker,
// Jorgensen & Olsen, "Molecular Electronic-Structure Theory" ch. 9).
// The Boys function is a 7-term Taylor expansion about the nearest point of
// a table with spacing 1/20 at the highest order needed, then downward
// recursion F_m = (2T F_{m+1} + e^{-T})/(2m+1); for T >= 36 the asymptotic
// F_0 = sqrt(pi/T)/2 and upward recursion.
//
// Index conventions: a Cartesian component (a,b,c) of total l sits at
// cidx = (l-a)(l-a+1)/2 + c (libint2 order x^l, x^{l-1}y, ...); Hermite
// triples (t,u,v) with t+u+v <= L are stored by total, each total in the
// same order: hidx = k(k+1)(k+2)/6 + cidx.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace m2 {

constexpr int BOYS_MMAX = 14;      // highest order the engine evaluates
constexpr int BOYS_TAYLOR = 7;     // Taylor terms
constexpr int BOYS_NGRID = 721;    // grid points 0 .. 36 step 1/20
constexpr double BOYS_STEP = 0.05;
constexpr double BOYS_TMAX = 36.0;
constexpr int BOYS_NCOL = BOYS_MMAX + BOYS_TAYLOR;  // orders stored per grid point

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nherm(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
__host__ __device__ constexpr int cidx(int a, int b, int c) { return (b + c) * (b + c + 1) / 2 + c; }
__host__ __device__ constexpr int hidx(int t, int u, int v) {
  return (t + u + v) * (t + u + v + 1) * (t + u + v + 2) / 6 + cidx(t, u, v);
}
// exponents of Cartesian component i of total l
__host__ __device__ constexpr int cart_a(int l, int i) {
  int a = l, pos = 0;
  while (pos + (l - a + 1) <= i) {
    pos += l - a + 1;
    --a;
  }
  return a;
}
__host__ __device__ constexpr int cart_c(int l, int i) {
  int a = cart_a(l, i);
  return i - (l - a) * (l - a + 1) / 2;
}
__host__ __device__ constexpr int cart_b(int l, int i) { return l - cart_a(l, i) - cart_c(l, i); }
// offset of the (2l+1) x ncart(l) solid-harmonic block of l in the packed table
__host__ __device__ constexpr int sph_off(int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += (2 * k + 1) * ncart(k);
  return o;
}
constexpr int SPH_LMAX = 4;

// ---------------------------------------------------------------- Boys
// F_0..F_M at T; table is BOYS_NGRID x BOYS_NCOL doubles (row = grid point).
template <int M>
__device__ __forceinline__ void boys(double T, const double* __restrict__ table, double* F) {
  static_assert(M <= BOYS_MMAX, "Boys order too high");
  if (T < BOYS_TMAX) {
    const int k = __double2int_rn(T * (1.0 / BOYS_STEP));
    const double d = k * BOYS_STEP - T;  // expand at grid point: F(T) = sum F_{m+j}(Tk) (Tk-T)^j / j!
    const double* row = table + k * BOYS_NCOL + M;
    double acc = __ldg(row + BOYS_TAYLOR - 1);
#pragma unroll
    for (int j = BOYS_TAYLOR - 1; j >= 1; --j) acc = __ldg(row + j - 1) + acc * d * (1.0 / j);
    F[M] = acc;
    const double e = exp(-T);
#pragma unroll
    for (int m = M - 1; m >= 0; --m) F[m] = (2.0 * T * F[m + 1] + e) * (1.0 / (2 * m + 1));
  } else {
    const double e = exp(-T);
    const double it = 1.0 / T;
    F[0] = 0.886226925452758014 * sqrt(it);  // sqrt(pi)/2 / sqrt(T)
#pragma unroll
    for (int m = 0; m < M; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * 0.5 * it;
  }
}

// ---------------------------------------------------------------- R table
// In place: after the call R[hidx(t,u,v)] = R^{(0)}_{tuv}, t+u+v <= L.
// `a` is the reduced exponent; F holds F_0..F_L(a |PQ|^2).
template <int L>
__device__ __forceinline__ void md_R(double a, double X, double Y, double Z, const double* F, double* R) {
  const double m2a = -2.0 * a;
  double pw[L + 1];
  pw[0] = 1.0;
#pragma unroll
  for (int n = 1; n <= L; ++n) pw[n] = pw[n - 1] * m2a;
  R[0] = F[L] * pw[L];
#pragma unroll
  for (int n = L - 1; n >= 0; --n) {
#pragma unroll
    for (int k = L - n; k >= 1; --k) {
#pragma unroll
      for (int i = 0; i < ncart(k); ++i) {
        const int t = cart_a(k, i), v = cart_c(k, i), u = k - t - v;
        double val;
        if (t > 0) {
          val = X * R[hidx(t - 1, u, v)];
          if (t > 1) val += (t - 1) * R[hidx(t - 2, u, v)];
        } else if (u > 0) {
          val = Y * R[hidx(t, u - 1, v)];
          if (u > 1) val += (u - 1) * R[hidx(t, u - 2, v)];
        } else {
          val = Z * R[hidx(t, u, v - 1)];
          if (v > 1) val += (v - 1) * R[hidx(t, u, v - 2)];
        }
        R[hidx(t, u, v)] = val;
      }
    }
    R[0] = F[n] * pw[n];
  }
}

// ---------------------------------------------------------------- E coefficients
// One Cartesian direction: E[i][j][t] for i <= LA, j <= LB, t <= i + j, with
// E^{00}_0 = 1 (the Gaussian prefactor exp(-mu X_AB^2) is applied elsewhere).
template <int LA, int LB>
struct E1 {
  double e[LA + 1][LB + 1][LA + LB + 1];
};

template <int LA, int LB>
__device__ __forceinline__ void md_E1(double PA, double PB, double oo2p, E1<LA, LB>& E) {
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j)
#pragma unroll
      for (int t = 0; t <= LA + LB; ++t) E.e[i][j][t] = 0.0;
  E.e[0][0][0] = 1.0;
#pragma unroll
  for (int i = 0; i <= LA; ++i) {
#pragma unroll
    for (int j = 0; j <= LB; ++j) {
      if (i == 0 && j == 0) continue;
#pragma unroll
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (j == 0) {  // from (i-1, 0)
          v = PA * E.e[i - 1][0][t];
          if (t > 0) v += oo2p * E.e[i - 1][0][t - 1];
          if (t + 1 <= i - 1) v += (t + 1) * E.e[i - 1][0][t + 1];
        } else {  // from (i, j-1)
          v = PB * E.e[i][j - 1][t];
          if (t > 0) v += oo2p * E.e[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += (t + 1) * E.e[i][j - 1][t + 1];
        }
        E.e[i][j][t] = v;
      }
    }
  }
}

}  // namespace m2
