// Device side of the density-fitted RHF gradient: derivative three-index
// (mn|P)^x and two-index (P|Q)^x integrals contracted at once with their
// weights, recomputed per shell pair / aux shell (nothing derivative is
// stored).  With c = V^-1 gamma, gamma_P = sum_mn (P|mn) D_mn, and
// d^P_ij = sum_Q (V^-1)_PQ (Q|ij) over the occupied orbitals, the two-electron
// energy of compute_2body_fock_df (molecular2 src/fockbuild.cpp:585-660),
//   E2 = 1/2 gamma^T V^-1 gamma - sum_ij sum_PQ (P|ij) (V^-1)_PQ (Q|ij),
// has the nuclear derivative
//   dE2 = sum_{P,mn} (mn|P)^x W3_{mn,P} + sum_{PQ} (P|Q)^x W2_{PQ},
//   W3_{mn,P} = c_P D_mn - 2 sum_ij C_mi C_nj d^P_ij,
//   W2_{PQ}   = -1/2 c_P c_Q + sum_ij d^P_ij d^Q_ij.
// Derivatives of the orbital centres are taken as in grad_kernels.cuh (shifted
// classes weighted by 2 alpha); the fitting centre of (mn|P) follows from
// translational invariance, and for (P|Q) d/dQ = -d/dP.
#pragma once
#include "df_kernels.cuh"
#include "grad_kernels.cuh"

namespace m2 {

// Adjoint of sph_index: index k of a 3-index block goes from the final (pure)
// functions of shell l back to its Cartesian components.
__device__ __forceinline__ void sph_index_adj(const double* in, double* out, int k, const int* n, int l,
                                              const double* sph) {
  const int nf = 2 * l + 1, ncl = ncart(l);
  int pre = 1, post = 1;
  for (int j = 0; j < k; ++j) pre *= n[j];
  for (int j = k + 1; j < 3; ++j) post *= n[j];
  const double* T = sph + sph_off(l);
  for (int a = 0; a < pre; ++a)
    for (int i = 0; i < ncl; ++i)
      for (int c = 0; c < post; ++c) {
        double v = 0.0;
        for (int m = 0; m < nf; ++m) v += T[m * ncl + i] * in[(a * nf + m) * post + c];
        out[(a * ncl + i) * post + c] = v;
      }
}

// quartet_cart kept out of line for the derivative classes: inlined into
// k_grad3, the CUDA 12.9 build (with ptxas -O3 and with -O0 alike) gave wrong
// contributions for the fitting classes d and f with p-p orbital pairs, while
// a host build of the same source and this out-of-line form both agree with
// finite differences of the integrals.
template <int LA, int LB, int LC, int LD>
__device__ __noinline__ void quartet_cart_ool(const PrimView& pp, int b0, int nb, double Ax, double Ay, double Az,
                                              double Bx, double By, double Bz, const PrimView& kp, int k0, int nk,
                                              double Cx, double Cy, double Cz, double Dx, double Dy, double Dz,
                                              const double* __restrict__ boys_tab, double* out) {
  quartet_cart<LA, LB, LC, LD>(pp, b0, nb, Ax, Ay, Az, Bx, By, Bz, kp, k0, nk, Cx, Cy, Cz, Dx, Dy, Dz, boys_tab, out);
}

struct Grad3Params {
  PrimView ap;            // fitting primitives as (P, unit) pairs
  const int* aux_shells;  // fitting shells of this angular momentum
  int naux_shells;
  const int* aux_prim_off;
  const int* aux_nprim;
  const double *ax, *ay, *az;
  const int* aux_foff;
  const int* aux_pure;
  const int* aux_atom;
  PairView pairs;         // orbital pairs of one class
  PrimView pp, pp2a, pp2b;
  const double *ox, *oy, *oz;
  const int* obs_foff;
  const int* obs_pure;
  const int* obs_atom;
  const double* sph_obs;
  const double* sph_aux;
  const double* boys;
  int n;
  const double* W3;       // [P - w3_f0][n][m] final basis: W3[((P - w3_f0) * n + y) * n + x]
  int w3_f0;              // first fitting function held in W3
  double* grad;           // 3 * natom
};

// One shifted class per block layer: blockIdx.z = 0, 1 (orbital centre m
// raised, lowered), 2, 3 (n); the fitting centre's derivative is minus their
// sum (translational invariance).  All threads of a block share the fitting
// shell, so its atom's term is reduced over the warp first.
template <int LP, int LM, int LN>
__global__ void __launch_bounds__(64) k_grad3(const Grad3Params P) {
  constexpr int NP = ncart(LP), NM = ncart(LM), NN = ncart(LN);
  constexpr int N3 = NP * NM * NN;
  const int sh = blockIdx.z;
  if ((sh == 1 && LM == 0) || (sh == 3 && LN == 0)) return;
  const int is = blockIdx.y;
  if (is >= P.naux_shells) return;
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  const int sP = P.aux_shells[is];
  double g[3] = {0, 0, 0};
  if (ip < P.pairs.npair) {
    const int m = P.pairs.sa[ip], n = P.pairs.sb[ip];
    // weights of this block, final basis -> Cartesian
    const int pure[3] = {P.aux_pure[sP], P.obs_pure[m], P.obs_pure[n]};
    const int ls[3] = {LP, LM, LN};
    int dims[3] = {pure[0] ? 2 * LP + 1 : NP, pure[1] ? 2 * LM + 1 : NM, pure[2] ? 2 * LN + 1 : NN};
    double w0[N3], w1[N3];
    const int f0 = P.aux_foff[sP], m0 = P.obs_foff[m], n0 = P.obs_foff[n];
    for (int a = 0; a < dims[0]; ++a)
      for (int x = 0; x < dims[1]; ++x)
        for (int y = 0; y < dims[2]; ++y)
          w0[(a * dims[1] + x) * dims[2] + y] = P.W3[((size_t)(f0 - P.w3_f0 + a) * P.n + n0 + y) * P.n + m0 + x];
    double* cur = w0;
    double* nxt = w1;
    for (int k = 0; k < 3; ++k)
      if (pure[k]) {
        sph_index_adj(cur, nxt, k, dims, ls[k], k == 0 ? P.sph_aux : P.sph_obs);
        dims[k] = ncart(ls[k]);
        double* sw = cur;
        cur = nxt;
        nxt = sw;
      }
    const double* Wt = cur;  // [a][x][y] Cartesian, as a (LP, 0 | LM, LN) block
    const double Px = P.ax[sP], Py = P.ay[sP], Pz = P.az[sP];
    const double Ax = P.ox[m], Ay = P.oy[m], Az = P.oz[m], Bx = P.ox[n], By = P.oy[n], Bz = P.oz[n];
    const int ap0 = P.aux_prim_off[sP], anp = P.aux_nprim[sP];
    const int kp0 = P.pairs.prim_off[ip], knp = P.pairs.nprim[ip];
    if (sh == 0) {
      double I[NP * ncart(LM + 1) * NN];
      quartet_cart_ool<LP, 0, LM + 1, LN>(P.ap, ap0, anp, Px, Py, Pz, Px, Py, Pz, P.pp2a, kp0, knp, Ax, Ay, Az, Bx,
                                          By, Bz, P.boys, I);
      contract_shift<LP, 0, LM, LN, 2, 1>(I, Wt, g);
    } else if (sh == 1) {
      if constexpr (LM > 0) {
        double I[NP * ncart(LM - 1) * NN];
        quartet_cart_ool<LP, 0, LM - 1, LN>(P.ap, ap0, anp, Px, Py, Pz, Px, Py, Pz, P.pp, kp0, knp, Ax, Ay, Az, Bx,
                                            By, Bz, P.boys, I);
        contract_shift<LP, 0, LM, LN, 2, -1>(I, Wt, g);
      }
    } else if (sh == 2) {
      double I[NP * NM * ncart(LN + 1)];
      quartet_cart_ool<LP, 0, LM, LN + 1>(P.ap, ap0, anp, Px, Py, Pz, Px, Py, Pz, P.pp2b, kp0, knp, Ax, Ay, Az, Bx,
                                          By, Bz, P.boys, I);
      contract_shift<LP, 0, LM, LN, 3, 1>(I, Wt, g);
    } else {
      if constexpr (LN > 0) {
        double I[NP * NM * ncart(LN - 1)];
        quartet_cart_ool<LP, 0, LM, LN - 1>(P.ap, ap0, anp, Px, Py, Pz, Px, Py, Pz, P.pp, kp0, knp, Ax, Ay, Az, Bx,
                                            By, Bz, P.boys, I);
        contract_shift<LP, 0, LM, LN, 3, -1>(I, Wt, g);
      }
    }
    // the sum over ordered (m, n) counts an off-diagonal canonical pair twice
    const double deg = (m == n) ? 1.0 : 2.0;
    const int at = P.obs_atom[sh < 2 ? m : n];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      g[x] *= deg;
      if (g[x] != 0.0) atomicAdd(P.grad + 3 * at + x, g[x]);
    }
  }
  // the fitting centre: minus the orbital centres' terms, one atomic per warp
  const int aP = P.aux_atom[sP];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    double v = g[x];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(P.grad + 3 * aP + x, -v);
  }
}

struct Grad2Params {
  PrimView ap, ap2;       // fitting primitives; ap2 has K * 2 alpha
  const int* shells_p;
  int np;
  const int* shells_q;
  int nq;
  const int* aux_prim_off;
  const int* aux_nprim;
  const double *ax, *ay, *az;
  const int* aux_foff;
  const int* aux_pure;
  const int* aux_atom;
  const double* sph;
  const double* boys;
  int naux;
  const double* W2;       // naux x naux, symmetric
  double* grad;
};

// one thread per ordered pair (P, Q) of fitting shells: W2 . d/dP (P|Q)
// goes to P's atom and its negative to Q's atom
template <int LP, int LQ>
__global__ void __launch_bounds__(64) k_grad2(const Grad2Params P) {
  constexpr int NP = ncart(LP), NQ = ncart(LQ);
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  const int ip = blockIdx.y;
  if (iq >= P.nq || ip >= P.np) return;
  const int sP = P.shells_p[ip], sQ = P.shells_q[iq];
  const int aP = P.aux_atom[sP], aQ = P.aux_atom[sQ];
  if (aP == aQ) return;  // one-centre: d/dP + d/dQ = 0 on the same atom
  const int pure[3] = {P.aux_pure[sP], P.aux_pure[sQ], 0};
  const int ls[3] = {LP, LQ, 0};
  int dims[3] = {pure[0] ? 2 * LP + 1 : NP, pure[1] ? 2 * LQ + 1 : NQ, 1};
  double w0[NP * NQ], w1[NP * NQ];
  const int p0 = P.aux_foff[sP], q0 = P.aux_foff[sQ];
  for (int a = 0; a < dims[0]; ++a)
    for (int b = 0; b < dims[1]; ++b) w0[a * dims[1] + b] = P.W2[(size_t)(q0 + b) * P.naux + p0 + a];
  double* cur = w0;
  double* nxt = w1;
  for (int k = 0; k < 2; ++k)
    if (pure[k]) {
      sph_index_adj(cur, nxt, k, dims, ls[k], P.sph);
      dims[k] = ncart(ls[k]);
      double* sw = cur;
      cur = nxt;
      nxt = sw;
    }
  const double Ax = P.ax[sP], Ay = P.ay[sP], Az = P.az[sP];
  const double Cx = P.ax[sQ], Cy = P.ay[sQ], Cz = P.az[sQ];
  double g[3] = {0, 0, 0};
  {
    double I[ncart(LP + 1) * NQ];
    quartet_cart<LP + 1, 0, LQ, 0>(P.ap2, P.aux_prim_off[sP], P.aux_nprim[sP], Ax, Ay, Az, Ax, Ay, Az, P.ap,
                                   P.aux_prim_off[sQ], P.aux_nprim[sQ], Cx, Cy, Cz, Cx, Cy, Cz, P.boys, I);
    contract_shift<LP, 0, LQ, 0, 0, 1>(I, cur, g);
  }
  if constexpr (LP > 0) {
    double I[ncart(LP - 1) * NQ];
    quartet_cart<LP - 1, 0, LQ, 0>(P.ap, P.aux_prim_off[sP], P.aux_nprim[sP], Ax, Ay, Az, Ax, Ay, Az, P.ap,
                                   P.aux_prim_off[sQ], P.aux_nprim[sQ], Cx, Cy, Cz, Cx, Cy, Cz, P.boys, I);
    contract_shift<LP, 0, LQ, 0, 0, -1>(I, cur, g);
  }
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    atomicAdd(P.grad + 3 * aP + x, g[x]);
    atomicAdd(P.grad + 3 * aQ + x, -g[x]);
  }
}

// launchers (df_grad_l*.cu, df_grad2.cu)
void launch_grad3_l0(int pair_class_id, const Grad3Params& P, cudaStream_t s);
void launch_grad3_l1(int pair_class_id, const Grad3Params& P, cudaStream_t s);
void launch_grad3_l2(int pair_class_id, const Grad3Params& P, cudaStream_t s);
void launch_grad3_l3(int pair_class_id, const Grad3Params& P, cudaStream_t s);
void launch_grad2(int LP, int LQ, const Grad2Params& P, cudaStream_t s);

}  // namespace m2
