// Device side of the density-fitting integrals: three-index (P|mn) and
// two-index (P|Q) Coulomb integrals over the fitting basis, and the one-body
// S, T, V integrals.  McMurchie-Davidson through quartet_cart with a unit
// s function as the partner of each fitting function (libint2 BraKet::xs_xx
// and xs_xs in molecular2, src/eris.cpp:89-156, 304-356).
#pragma once
#include "jk_kernels.cuh"

namespace m2 {

// Transform index k (0..2) of a 3-index Cartesian block (dims n[0..2]) to the
// final basis of its shell (pure block of sph when p != 0).  Rolled loops:
// these kernels run once per geometry.
__device__ __forceinline__ void sph_index(const double* in, double* out, int k, const int* n, int l,
                                          const double* sph) {
  const int nf = 2 * l + 1, ncl = ncart(l);
  int pre = 1, post = 1;
  for (int j = 0; j < k; ++j) pre *= n[j];
  for (int j = k + 1; j < 3; ++j) post *= n[j];
  const double* T = sph + sph_off(l);
  for (int a = 0; a < pre; ++a)
    for (int m = 0; m < nf; ++m)
      for (int c = 0; c < post; ++c) {
        double v = 0.0;
        for (int i = 0; i < ncl; ++i) v += T[m * ncl + i] * in[(a * ncl + i) * post + c];
        out[(a * nf + m) * post + c] = v;
      }
}

struct Eri3Params {
  PrimView ap;            // fitting primitives as (P, unit) pairs
  const int* aux_shells;  // fitting shells of this class (angular momentum LP)
  int naux_shells;
  const int* aux_prim_off;
  const int* aux_nprim;
  const double *ax, *ay, *az;
  const int* aux_foff;    // final function offsets
  const int* aux_pure;
  PairView pairs;         // orbital pairs of one class
  PrimView pp;
  const double *ox, *oy, *oz;
  const int* obs_foff;
  const int* obs_pure;
  const double* sph;
  const double* boys;
  int n, naux;
  double* T3;             // [x][P][y]
};

// Final-basis block (P|mn) of fitting shell sP and orbital shell pair ip of
// the class: out[(a * dims[1] + x) * dims[2] + y]; c and t are scratch of
// NP*NM*NN doubles each, the result is one of them.
template <int LP, int LM, int LN>
__device__ __forceinline__ const double* eri3_block(const Eri3Params& P, int sP, int ip, double* c, double* t,
                                                    int* dims) {
  const int m = P.pairs.sa[ip], n = P.pairs.sb[ip];
  const double Ax = P.ax[sP], Ay = P.ay[sP], Az = P.az[sP];
  quartet_cart<LP, 0, LM, LN>(P.ap, P.aux_prim_off[sP], P.aux_nprim[sP], Ax, Ay, Az, Ax, Ay, Az, P.pp,
                              P.pairs.prim_off[ip], P.pairs.nprim[ip], P.ox[m], P.oy[m], P.oz[m], P.ox[n], P.oy[n],
                              P.oz[n], P.boys, c);
  dims[0] = ncart(LP);
  dims[1] = ncart(LM);
  dims[2] = ncart(LN);
  double* cur = c;
  double* nxt = t;
  const int pure[3] = {P.aux_pure[sP], P.obs_pure[m], P.obs_pure[n]};
  const int ls[3] = {LP, LM, LN};
  for (int k = 0; k < 3; ++k)
    if (pure[k]) {
      sph_index(cur, nxt, k, dims, ls[k], P.sph);
      dims[k] = 2 * ls[k] + 1;
      double* sw = cur;
      cur = nxt;
      nxt = sw;
    }
  return cur;
}

template <int LP, int LM, int LN>
__global__ void __launch_bounds__(64) k_eri3(const Eri3Params P) {
  constexpr int N3 = ncart(LP) * ncart(LM) * ncart(LN);
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  const int is = blockIdx.y;
  if (ip >= P.pairs.npair || is >= P.naux_shells) return;
  const int sP = P.aux_shells[is];
  const int m = P.pairs.sa[ip], n = P.pairs.sb[ip];
  double c[N3], t[N3];
  int dims[3];
  const double* cur = eri3_block<LP, LM, LN>(P, sP, ip, c, t, dims);
  const int f0 = P.aux_foff[sP], m0 = P.obs_foff[m], n0 = P.obs_foff[n];
  const size_t nQ = (size_t)P.naux * P.n;
  for (int a = 0; a < dims[0]; ++a)
    for (int x = 0; x < dims[1]; ++x)
      for (int y = 0; y < dims[2]; ++y) {
        const double v = cur[(a * dims[1] + x) * dims[2] + y];
        P.T3[(size_t)(m0 + x) * nQ + (size_t)(f0 + a) * P.n + n0 + y] = v;
        P.T3[(size_t)(n0 + y) * nQ + (size_t)(f0 + a) * P.n + m0 + x] = v;
      }
}

// One tile pair of the tiled three-index tensor: T[r][P][c] = (P | x y) for
// x = x0 + r and y = y0 + c inside the TB x TB tile (TB = 128), over the
// shell pairs `plist` of the class that touch the tile pair (either
// orientation).  Entries of the block outside the tile are not written.
struct Eri3TileArgs {
  const int* plist;  // indices into the class's pair list
  int nlist;
  int x0, y0;        // first function of the row tile and of the column tile
  int naux;
  double* T;         // [r][P][c], TB * naux * TB doubles
};
constexpr int DF_TILE = 128;

template <int LP, int LM, int LN>
__global__ void __launch_bounds__(64) k_eri3_tile(const Eri3Params P, const Eri3TileArgs A) {
  constexpr int N3 = ncart(LP) * ncart(LM) * ncart(LN);
  const int il = blockIdx.x * blockDim.x + threadIdx.x;
  const int is = blockIdx.y;
  if (il >= A.nlist || is >= P.naux_shells) return;
  const int ip = A.plist[il];
  const int sP = P.aux_shells[is];
  const int m = P.pairs.sa[ip], n = P.pairs.sb[ip];
  double c[N3], t[N3];
  int dims[3];
  const double* cur = eri3_block<LP, LM, LN>(P, sP, ip, c, t, dims);
  const int f0 = P.aux_foff[sP], m0 = P.obs_foff[m], n0 = P.obs_foff[n];
  const size_t rs = (size_t)A.naux * DF_TILE;  // stride of r
  for (int a = 0; a < dims[0]; ++a)
    for (int x = 0; x < dims[1]; ++x)
      for (int y = 0; y < dims[2]; ++y) {
        const double v = cur[(a * dims[1] + x) * dims[2] + y];
        const int X = m0 + x, Y = n0 + y;
        const unsigned r1 = (unsigned)(X - A.x0), c1 = (unsigned)(Y - A.y0);
        if (r1 < DF_TILE && c1 < DF_TILE) A.T[r1 * rs + (size_t)(f0 + a) * DF_TILE + c1] = v;
        const unsigned r2 = (unsigned)(Y - A.x0), c2 = (unsigned)(X - A.y0);
        if (r2 < DF_TILE && c2 < DF_TILE) A.T[r2 * rs + (size_t)(f0 + a) * DF_TILE + c2] = v;
      }
}

struct Eri2Params {
  PrimView ap;
  const int* shells_p;
  int np;
  const int* shells_q;
  int nq;
  const int* aux_prim_off;
  const int* aux_nprim;
  const double *ax, *ay, *az;
  const int* aux_foff;
  const int* aux_pure;
  const double* sph;
  const double* boys;
  int naux;
  double* V;  // naux x naux
};

template <int LP, int LQ>
__global__ void __launch_bounds__(64) k_eri2(const Eri2Params P) {
  constexpr int NP = ncart(LP), NQ = ncart(LQ);
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  const int ip = blockIdx.y;
  if (iq >= P.nq || ip >= P.np) return;
  const int sP = P.shells_p[ip], sQ = P.shells_q[iq];
  const double Ax = P.ax[sP], Ay = P.ay[sP], Az = P.az[sP];
  const double Cx = P.ax[sQ], Cy = P.ay[sQ], Cz = P.az[sQ];
  double c[NP * NQ], t[NP * NQ];
  quartet_cart<LP, 0, LQ, 0>(P.ap, P.aux_prim_off[sP], P.aux_nprim[sP], Ax, Ay, Az, Ax, Ay, Az, P.ap,
                             P.aux_prim_off[sQ], P.aux_nprim[sQ], Cx, Cy, Cz, Cx, Cy, Cz, P.boys, c);
  int dims[3] = {NP, NQ, 1};
  double* cur = c;
  double* nxt = t;
  if (P.aux_pure[sP]) {
    sph_index(cur, nxt, 0, dims, LP, P.sph);
    dims[0] = 2 * LP + 1;
    double* sw = cur;
    cur = nxt;
    nxt = sw;
  }
  if (P.aux_pure[sQ]) {
    sph_index(cur, nxt, 1, dims, LQ, P.sph);
    dims[1] = 2 * LQ + 1;
    double* sw = cur;
    cur = nxt;
    nxt = sw;
  }
  const int p0 = P.aux_foff[sP], q0 = P.aux_foff[sQ];
  for (int a = 0; a < dims[0]; ++a)
    for (int b = 0; b < dims[1]; ++b) {
      const double v = cur[a * dims[1] + b];
      P.V[(size_t)(q0 + b) * P.naux + p0 + a] = v;
      P.V[(size_t)(p0 + a) * P.naux + q0 + b] = v;
    }
}

// ---------------------------------------------------------------- one-body
struct OneBodyParams {
  PairView pairs;
  PrimView pp;
  const double* pa;  // exponent of shell a per primitive pair
  const double *ox, *oy, *oz;
  const int* foff;
  const int* pure;
  const double* sph;
  const double* boys;
  int natom;
  const double* Z;
  const double* cxyz;  // 3*natom
  int n;
  double *S, *T, *V;   // n x n final basis
};

template <int LA, int LB>
__global__ void __launch_bounds__(64) k_onebody(const OneBodyParams P) {
  constexpr int NA = ncart(LA), NB = ncart(LB), L = LA + LB;
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.pairs.npair) return;
  const int a = P.pairs.sa[ip], b = P.pairs.sb[ip];
  const double Ax = P.ox[a], Ay = P.oy[a], Az = P.oz[a], Bx = P.ox[b], By = P.oy[b], Bz = P.oz[b];
  double s[NA * NB], t[NA * NB], v[NA * NB];
  for (int i = 0; i < NA * NB; ++i) s[i] = t[i] = v[i] = 0.0;
  const int p0 = P.pairs.prim_off[ip], np = P.pairs.nprim[ip];
  for (int k = p0; k < p0 + np; ++k) {
    const double p = P.pp.p[k], Px = P.pp.x[k], Py = P.pp.y[k], Pz = P.pp.z[k], K = P.pp.K[k];
    const double al = P.pa[k], be = p - al;
    E1<LA, LB + 2> ex, ey, ez;
    const double oo2p = 0.5 / p;
    md_E1<LA, LB + 2>(Px - Ax, Px - Bx, oo2p, ex);
    md_E1<LA, LB + 2>(Py - Ay, Py - By, oo2p, ey);
    md_E1<LA, LB + 2>(Pz - Az, Pz - Bz, oo2p, ez);
    const double ov = K * pow(M_PI / p, 1.5);
    // nuclear attraction: sum_C -Z_C 2 pi/p K sum_tuv E_t E_u E_v R_tuv(p, P-C)
    double Rsum[nherm(L)];
    for (int h = 0; h < nherm(L); ++h) Rsum[h] = 0.0;
    for (int c = 0; c < P.natom; ++c) {
      const double X = Px - P.cxyz[3 * c], Y = Py - P.cxyz[3 * c + 1], Zc = Pz - P.cxyz[3 * c + 2];
      double F[L + 1], R[nherm(L)];
      boys<L>(p * (X * X + Y * Y + Zc * Zc), P.boys, F);
      md_R<L>(p, X, Y, Zc, F, R);
      const double z = P.Z[c];
      for (int h = 0; h < nherm(L); ++h) Rsum[h] -= z * R[h];
    }
    const double vp = 2.0 * M_PI / p * K;
#pragma unroll
    for (int ia = 0; ia < NA; ++ia) {
      const int ax = cart_a(LA, ia), ay = cart_b(LA, ia), az = cart_c(LA, ia);
#pragma unroll
      for (int ib = 0; ib < NB; ++ib) {
        const int bx = cart_a(LB, ib), by = cart_b(LB, ib), bz = cart_c(LB, ib);
        const double sx = ex.e[ax][bx][0], sy = ey.e[ay][by][0], sz = ez.e[az][bz][0];
        s[ia * NB + ib] += ov * sx * sy * sz;
        auto kin = [&](const E1<LA, LB + 2>& e, int i, int j) {
          double r = -2.0 * be * be * e.e[i][j + 2][0] + be * (2 * j + 1) * e.e[i][j][0];
          if (j > 1) r -= 0.5 * j * (j - 1) * e.e[i][j - 2][0];
          return r;
        };
        t[ia * NB + ib] += ov * (kin(ex, ax, bx) * sy * sz + sx * kin(ey, ay, by) * sz + sx * sy * kin(ez, az, bz));
        double acc = 0.0;
        for (int tt = 0; tt <= ax + bx; ++tt)
          for (int u = 0; u <= ay + by; ++u)
            for (int w = 0; w <= az + bz; ++w)
              acc += ex.e[ax][bx][tt] * ey.e[ay][by][u] * ez.e[az][bz][w] * Rsum[hidx(tt, u, w)];
        v[ia * NB + ib] += vp * acc;
      }
    }
  }
  // final basis and store both orientations
  double* blocks[3] = {s, t, v};
  double* outs[3] = {P.S, P.T, P.V};
  const int pa = P.pure[a], pb = P.pure[b];
  const int fa = pa ? 2 * LA + 1 : NA, fb = pb ? 2 * LB + 1 : NB;
  const int a0 = P.foff[a], b0 = P.foff[b];
  for (int k = 0; k < 3; ++k) {
    const double* c = blocks[k];
    for (int m = 0; m < fa; ++m)
      for (int q = 0; q < fb; ++q) {
        double val = 0.0;
        for (int i = 0; i < NA; ++i) {
          const double ta = pa ? P.sph[sph_off(LA) + m * NA + i] : (i == m ? 1.0 : 0.0);
          if (ta == 0.0) continue;
          for (int j = 0; j < NB; ++j) {
            const double tb = pb ? P.sph[sph_off(LB) + q * NB + j] : (j == q ? 1.0 : 0.0);
            val += ta * tb * c[i * NB + j];
          }
        }
        outs[k][(size_t)(b0 + q) * P.n + a0 + m] = val;
        outs[k][(size_t)(a0 + m) * P.n + b0 + q] = val;
      }
  }
}

// launchers in df_cls_*.cu
void launch_eri3_l0(int pair_class_id, const Eri3Params& P, cudaStream_t s);
void launch_eri3_l1(int pair_class_id, const Eri3Params& P, cudaStream_t s);
void launch_eri3_l2(int pair_class_id, const Eri3Params& P, cudaStream_t s);
void launch_eri3_l3(int pair_class_id, const Eri3Params& P, cudaStream_t s);
void launch_eri3_tile_l0(int pair_class_id, const Eri3Params& P, const Eri3TileArgs& A, cudaStream_t s);
void launch_eri3_tile_l1(int pair_class_id, const Eri3Params& P, const Eri3TileArgs& A, cudaStream_t s);
void launch_eri3_tile_l2(int pair_class_id, const Eri3Params& P, const Eri3TileArgs& A, cudaStream_t s);
void launch_eri3_tile_l3(int pair_class_id, const Eri3Params& P, const Eri3TileArgs& A, cudaStream_t s);
void launch_eri2(int LP, int LQ, const Eri2Params& P, cudaStream_t s);
void launch_onebody(int pair_class_id, const OneBodyParams& P, cudaStream_t s);

}  // namespace m2
