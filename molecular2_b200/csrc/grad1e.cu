// One-body part of the RHF nuclear gradient: overlap, kinetic and
// nuclear-attraction derivative integrals contracted at once with D and W,
//   (T' + V') . D  and  -2 S' . W   (Fock::compute_forces, molecular2
// src/rhfgrad.cpp:23-45; derivative integrals inc/integrals.hpp:169-349),
// one thread per canonical shell pair (times 2 for a != b).
#include "grad_kernels.cuh"

namespace m2 {

// sum_tuv E^{ab}_t E_u E_v R[t+st, u+su, v+sv] for one Cartesian pair (a, b).
// Bound: every caller passes components with |a| + |b| + st + su + sv <=
// LA + LB + 1 = L (the Hellmann-Feynman term: |a| = LA, |b| = LB and one unit
// shift; the centre terms: a or b raised or lowered by one, no shift), so
// hidx(...) < nherm(L) = NR for every term; the static_assert ties NR to the
// class.  Kept out of line: inlined into k_grad1e, the CUDA 12.9 build at
// ptxas -O1 and above gave wrong nuclear-attraction sums for the p-shell
// classes, while -O0 and this out-of-line form agree with a host build of the
// same source.  Reading the kernel found no out-of-bounds index or other
// source defect behind it, so the out-of-line form is a workaround kept for a
// compiler behaviour whose cause is not known.
template <int LA1, int LB2, int NR>
__device__ __noinline__ double herm_sum(const E1<LA1, LB2>& ex, const E1<LA1, LB2>& ey, const E1<LA1, LB2>& ez,
                                        int ax, int ay, int az, int bx, int by, int bz, const double* R, int st,
                                        int su, int sv) {
  static_assert(NR == nherm(LA1 + LB2 - 2), "R table length must be nherm(LA + LB + 1)");
  double acc = 0.0;
  for (int t = 0; t <= ax + bx; ++t)
    for (int u = 0; u <= ay + by; ++u) {
      const double exy = ex.e[ax][bx][t] * ey.e[ay][by][u];
      for (int v = 0; v <= az + bz; ++v) acc += exy * ez.e[az][bz][v] * R[hidx(t + st, u + su, v + sv)];
    }
  return acc;
}

template <int LA, int LB>
__global__ void __launch_bounds__(64) k_grad1e(const Grad1eParams P) {
  constexpr int NA = ncart(LA), NB = ncart(LB), L = LA + LB + 1;
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.pairs.npair || !P.sig[ip]) return;
  const int a = P.pairs.sa[ip], b = P.pairs.sb[ip];
  const double sym = (a == b) ? 1.0 : 2.0;
  const double Ax = P.ox[a], Ay = P.oy[a], Az = P.oz[a], Bx = P.ox[b], By = P.oy[b], Bz = P.oz[b];
  const int a0 = P.coff[a], b0 = P.coff[b];
  double gA[3] = {0, 0, 0};  // d/dA of T.D - 2 S.W (d/dB = -d/dA for S and T)
  double gVA[3] = {0, 0, 0}, gVB[3] = {0, 0, 0};
  const int p0 = P.pairs.prim_off[ip], np = P.pairs.nprim[ip];
  for (int k = p0; k < p0 + np; ++k) {
    const double p = P.pp.p[k], Px = P.pp.x[k], Py = P.pp.y[k], Pz = P.pp.z[k], K = P.pp.K[k];
    const double al = P.pa[k], be = p - al;
    E1<LA + 1, LB + 2> ex, ey, ez;
    const double oo2p = 0.5 / p;
    md_E1<LA + 1, LB + 2>(Px - Ax, Px - Bx, oo2p, ex);
    md_E1<LA + 1, LB + 2>(Py - Ay, Py - By, oo2p, ey);
    md_E1<LA + 1, LB + 2>(Pz - Az, Pz - Bz, oo2p, ez);
    const double pip = M_PI / p;
    const double ov = K * pip * sqrt(pip);  // K (pi/p)^{3/2}
    // Nuclear attraction.  Centre terms use the nucleus-summed Hermite
    // integrals Rsum = sum_C -Z_C R^C; the Hellmann-Feynman term of nucleus C
    // follows from d/dC_x R_tuv(P - C) = -R_{t+1,u,v}.
    const double v2p = 2.0 * M_PI / p * K;
    double Rsum[nherm(L)];
    for (int h = 0; h < nherm(L); ++h) Rsum[h] = 0.0;
    for (int cn = 0; cn < P.natom; ++cn) {
      const double X = Px - P.cxyz[3 * cn], Y = Py - P.cxyz[3 * cn + 1], Zc = Pz - P.cxyz[3 * cn + 2];
      double F[L + 1], R[nherm(L)];
      boys<L>(p * (X * X + Y * Y + Zc * Zc), P.boys, F);
      md_R<L>(p, X, Y, Zc, F, R);
      const double zc = P.Z[cn];
      for (int h = 0; h < nherm(L); ++h) Rsum[h] -= zc * R[h];
      double hf[3] = {0, 0, 0};
      for (int ia = 0; ia < NA; ++ia) {
        const int ax = c_herm.t[nherm(LA - 1) + ia], ay = c_herm.u[nherm(LA - 1) + ia],
                  az = c_herm.v[nherm(LA - 1) + ia];
        for (int ib = 0; ib < NB; ++ib) {
          const int bx = c_herm.t[nherm(LB - 1) + ib], by = c_herm.u[nherm(LB - 1) + ib],
                    bz = c_herm.v[nherm(LB - 1) + ib];
          const double dab = sym * P.Dc[(size_t)(a0 + ia) * P.nc + b0 + ib];
          hf[0] += dab * herm_sum<LA + 1, LB + 2, nherm(L)>(ex, ey, ez, ax, ay, az, bx, by, bz, R, 1, 0, 0);
          hf[1] += dab * herm_sum<LA + 1, LB + 2, nherm(L)>(ex, ey, ez, ax, ay, az, bx, by, bz, R, 0, 1, 0);
          hf[2] += dab * herm_sum<LA + 1, LB + 2, nherm(L)>(ex, ey, ez, ax, ay, az, bx, by, bz, R, 0, 0, 1);
        }
      }
      // V_C = -Z_C v2p sum E R  =>  dV_C/dC_x = +Z_C v2p sum E R_{t+1}
      for (int x = 0; x < 3; ++x) atomicAdd(P.grad + 3 * cn + x, zc * v2p * hf[x]);
    }
    for (int ia = 0; ia < NA; ++ia) {
      const int ax = c_herm.t[nherm(LA - 1) + ia], ay = c_herm.u[nherm(LA - 1) + ia], az = c_herm.v[nherm(LA - 1) + ia];
      for (int ib = 0; ib < NB; ++ib) {
        const int bx = c_herm.t[nherm(LB - 1) + ib], by = c_herm.u[nherm(LB - 1) + ib],
                  bz = c_herm.v[nherm(LB - 1) + ib];
        const double dab = sym * P.Dc[(size_t)(a0 + ia) * P.nc + b0 + ib];
        const int ea[3] = {ax, ay, az}, eb[3] = {bx, by, bz};
        for (int x = 0; x < 3; ++x) {
          int up[3] = {ax, ay, az}, dn[3] = {ax, ay, az}, bu[3] = {bx, by, bz}, bd[3] = {bx, by, bz};
          up[x] += 1;
          dn[x] -= 1;
          bu[x] += 1;
          bd[x] -= 1;
          double dA = 2.0 * al * herm_sum<LA + 1, LB + 2, nherm(L)>(ex, ey, ez, up[0], up[1], up[2], bx, by, bz, Rsum, 0, 0, 0);
          if (ea[x] > 0) dA -= ea[x] * herm_sum<LA + 1, LB + 2, nherm(L)>(ex, ey, ez, dn[0], dn[1], dn[2], bx, by, bz, Rsum, 0, 0, 0);
          double dB = 2.0 * be * herm_sum<LA + 1, LB + 2, nherm(L)>(ex, ey, ez, ax, ay, az, bu[0], bu[1], bu[2], Rsum, 0, 0, 0);
          if (eb[x] > 0) dB -= eb[x] * herm_sum<LA + 1, LB + 2, nherm(L)>(ex, ey, ez, ax, ay, az, bd[0], bd[1], bd[2], Rsum, 0, 0, 0);
          gVA[x] += dab * v2p * dA;
          gVB[x] += dab * v2p * dB;
        }
      }
    }
    // overlap and kinetic
    for (int ia = 0; ia < NA; ++ia) {
      const int ax = c_herm.t[nherm(LA - 1) + ia], ay = c_herm.u[nherm(LA - 1) + ia], az = c_herm.v[nherm(LA - 1) + ia];
      for (int ib = 0; ib < NB; ++ib) {
        const int bx = c_herm.t[nherm(LB - 1) + ib], by = c_herm.u[nherm(LB - 1) + ib],
                  bz = c_herm.v[nherm(LB - 1) + ib];
        const double dab = sym * P.Dc[(size_t)(a0 + ia) * P.nc + b0 + ib];
        const double wab = sym * P.Wc[(size_t)(a0 + ia) * P.nc + b0 + ib];
        auto kin = [&](const E1<LA + 1, LB + 2>& e, int i, int j) {
          double r = -2.0 * be * be * e.e[i][j + 2][0] + be * (2 * j + 1) * e.e[i][j][0];
          if (j > 1) r -= 0.5 * j * (j - 1) * e.e[i][j - 2][0];
          return r;
        };
        auto ST = [&](int i, int j, int k2, double& S, double& T) {
          const double sx = ex.e[i][bx][0], sy = ey.e[j][by][0], sz = ez.e[k2][bz][0];
          S = ov * sx * sy * sz;
          T = ov * (kin(ex, i, bx) * sy * sz + sx * kin(ey, j, by) * sz + sx * sy * kin(ez, k2, bz));
        };
        const int ea[3] = {ax, ay, az};
        for (int x = 0; x < 3; ++x) {
          int up[3] = {ax, ay, az}, dn[3] = {ax, ay, az};
          up[x] += 1;
          dn[x] -= 1;
          double Su, Tu, Sd = 0.0, Td = 0.0;
          ST(up[0], up[1], up[2], Su, Tu);
          if (ea[x] > 0) ST(dn[0], dn[1], dn[2], Sd, Td);
          const double dS = 2.0 * al * Su - ea[x] * Sd;
          const double dT = 2.0 * al * Tu - ea[x] * Td;
          gA[x] += dab * dT - 2.0 * wab * dS;
        }
      }
    }
  }
  for (int x = 0; x < 3; ++x) {
    atomicAdd(P.grad + 3 * P.atom[a] + x, gA[x] + gVA[x]);
    atomicAdd(P.grad + 3 * P.atom[b] + x, -gA[x] + gVB[x]);
  }
}

void launch_grad1e(int pc, const Grad1eParams& P, cudaStream_t s) {
  dim3 grid((P.pairs.npair + 63) / 64);
  if (pc == 0) k_grad1e<0, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 1) k_grad1e<1, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 2) k_grad1e<1, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 3) k_grad1e<2, 0><<<grid, 64, 0, s>>>(P);
  if (pc == 4) k_grad1e<2, 1><<<grid, 64, 0, s>>>(P);
  if (pc == 5) k_grad1e<2, 2><<<grid, 64, 0, s>>>(P);
}

}  // namespace m2
