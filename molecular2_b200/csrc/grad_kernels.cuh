// Device side of the RHF nuclear gradient (FP64): the adjoint of the direct
// J/K build and of the one-body matrices.  Derivative integrals are recomputed
// per shell quartet / pair and contracted at once with the density weights, so
// no derivative integral or derivative Fock matrix is ever stored
// (molecular2 builds 3N derivative Fock matrices, src/rhfgrad.cpp:419-598).
//
// Derivative of a primitive Cartesian Gaussian with respect to its centre:
//   d/dA_x  x_A^a e^{-alpha r_A^2} = 2 alpha x_A^{a+1} e^{..} - a x_A^{a-1} e^{..},
// so d/dA_x (ab|cd) = (a+1_x b|cd)~ - a_x (a-1_x b|cd) where ~ marks primitive
// pairs weighted by 2 alpha.  Centres A, B, C are differentiated this way and
// D by translational invariance, d/dD = -(d/dA + d/dB + d/dC).
#pragma once
#include "jk_kernels.cuh"

namespace m2 {

// Contract a Cartesian block of class (.., L+SHIFT on centre WHICH, ..) with
// the weights Wt(a,b,c,d) of class (LA,LB,LC,LD), for the three directions:
// g[x] += sum Wt * I(component shifted by +-1 along x), times a_x for SHIFT < 0.
template <int LA, int LB, int LC, int LD, int WHICH, int SHIFT>
__device__ __forceinline__ void contract_shift(const double* I, const double* Wt, double* g) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int LW = WHICH == 0 ? LA : (WHICH == 1 ? LB : (WHICH == 2 ? LC : LD));
  constexpr int NSH = ncart(LW + SHIFT);
  constexpr int NS1 = WHICH == 1 ? NSH : NB, NS2 = WHICH == 2 ? NSH : NC, NS3 = WHICH == 3 ? NSH : ND;
#pragma unroll 1
  for (int ia = 0; ia < NA; ++ia)
#pragma unroll 1
    for (int ib = 0; ib < NB; ++ib)
#pragma unroll 1
      for (int ic = 0; ic < NC; ++ic)
#pragma unroll 1
        for (int id = 0; id < ND; ++id) {
          const double w = Wt[((ia * NB + ib) * NC + ic) * ND + id];
          if (w == 0.0) continue;
          int idx[4] = {ia, ib, ic, id};
          const int i0 = idx[WHICH];
          const int base = nherm(LW - 1);
          const int ex[3] = {c_herm.t[base + i0], c_herm.u[base + i0], c_herm.v[base + i0]};
#pragma unroll
          for (int x = 0; x < 3; ++x) {
            int e2[3] = {ex[0], ex[1], ex[2]};
            e2[x] += SHIFT;
            if (e2[x] < 0) continue;
            const double f = SHIFT > 0 ? 1.0 : -(double)ex[x];
            idx[WHICH] = cidx(e2[0], e2[1], e2[2]);
            g[x] += f * w * I[((idx[0] * NS1 + idx[1]) * NS2 + idx[2]) * NS3 + idx[3]];
            idx[WHICH] = i0;
          }
        }
}

struct Grad2eParams {
  PairView bra, ket;
  int same_class;
  PrimView pp;         // K
  PrimView pp2a;       // K * 2 alpha (exponent of the pair's first shell)
  PrimView pp2b;       // K * 2 beta  (exponent of the pair's second shell)
  ShellView sh;
  const int* atom;     // shell -> atom
  const unsigned char* bra_sig;  // overlap significance of each pair (shell-pair list)
  const unsigned char* ket_sig;
  const double* Dnorm;
  int nshell;
  const double* Dmax;
  const double* Dc;    // Cartesian density, nc x nc
  int nc;
  double precision;
  const double* boys;
  double* grad;        // 3 * natom
  int kchunk;
  int bra0, bra_step;        // block x handles bra pair bra0 + x * bra_step (a rank's share of the class)
};

// One shifted class per block layer: blockIdx.z = 0, 1 (centre a raised,
// lowered), 2, 3 (b), 4, 5 (c); the derivative with respect to centre d follows
// from translational invariance (minus the sum of the other three).  Splitting
// the six shifted quartets over blocks shortens each thread's serial work six
// times, which is what bounds the d classes of small molecules.
template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(64) k_grad2e(const Grad2eParams P) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int N4 = NA * NB * NC * ND;
  const int sh = blockIdx.z, centre = sh >> 1;
  if ((sh == 1 && LA == 0) || (sh == 3 && LB == 0) || (sh == 5 && LC == 0)) return;
  const int bra = P.bra0 + blockIdx.x * P.bra_step;
  if (!P.bra_sig[bra]) return;
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
  const double* __restrict__ Dc = P.Dc;
  double gbra[3] = {0, 0, 0};  // this thread's share for the bra centre (centre 0 or 1: one atom per block)

  for (int kl = start + threadIdx.x; kl < end; kl += blockDim.x) {
    if (!P.ket_sig[kl]) continue;
    const int c = P.ket.sa[kl], d = P.ket.sb[kl];
    const double* Dn = P.Dnorm;
    const int ns = P.nshell;
    double dn = fmax(fmax(Dn[a * ns + b], Dn[c * ns + d]), fmax(Dn[a * ns + c], Dn[a * ns + d]));
    dn = fmax(dn, fmax(Dn[b * ns + c], Dn[b * ns + d]));
    if (dn * Qab * P.ket.Q[kl] < P.precision) continue;
    const double deg = ((a == b) ? 1.0 : 2.0) * ((c == d) ? 1.0 : 2.0) * ((P.same_class && kl == bra) ? 1.0 : 2.0);
    const int c0 = P.sh.coff[c], d0 = P.sh.coff[d];
    const double Cx = P.sh.x[c], Cy = P.sh.y[c], Cz = P.sh.z[c];
    const double Ex = P.sh.x[d], Ey = P.sh.y[d], Ez = P.sh.z[d];
    const int kp0 = P.ket.prim_off[kl], knp = P.ket.nprim[kl];
    // density weights of the 2e energy: 1/2 D_ab D_cd - 1/8 (D_ac D_bd + D_ad D_bc)
    double Wt[N4];
#pragma unroll 1
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll 1
      for (int ib = 0; ib < NB; ++ib) {
        const double dab = Dc[(size_t)(a0 + ia) * nc + b0 + ib];
#pragma unroll 1
        for (int ic = 0; ic < NC; ++ic) {
          const double dac = Dc[(size_t)(a0 + ia) * nc + c0 + ic], dbc = Dc[(size_t)(b0 + ib) * nc + c0 + ic];
#pragma unroll 1
          for (int id = 0; id < ND; ++id) {
            const double dcd = Dc[(size_t)(c0 + ic) * nc + d0 + id];
            const double dbd = Dc[(size_t)(b0 + ib) * nc + d0 + id], dad = Dc[(size_t)(a0 + ia) * nc + d0 + id];
            Wt[((ia * NB + ib) * NC + ic) * ND + id] = 0.5 * dab * dcd - 0.125 * (dac * dbd + dad * dbc);
          }
        }
      }
    double g[3] = {0, 0, 0};
    if (sh == 0) {
      double I[ncart(LA + 1) * NB * NC * ND];
      quartet_cart<LA + 1, LB, LC, LD>(P.pp2a, bp0, bnp, Ax, Ay, Az, Bx, By, Bz, P.pp, kp0, knp, Cx, Cy, Cz, Ex, Ey,
                                       Ez, P.boys, I);
      contract_shift<LA, LB, LC, LD, 0, 1>(I, Wt, g);
    } else if (sh == 1) {
      if constexpr (LA > 0) {
        double I[ncart(LA - 1) * NB * NC * ND];
        quartet_cart<LA - 1, LB, LC, LD>(P.pp, bp0, bnp, Ax, Ay, Az, Bx, By, Bz, P.pp, kp0, knp, Cx, Cy, Cz, Ex, Ey,
                                         Ez, P.boys, I);
        contract_shift<LA, LB, LC, LD, 0, -1>(I, Wt, g);
      }
    } else if (sh == 2) {
      double I[NA * ncart(LB + 1) * NC * ND];
      quartet_cart<LA, LB + 1, LC, LD>(P.pp2b, bp0, bnp, Ax, Ay, Az, Bx, By, Bz, P.pp, kp0, knp, Cx, Cy, Cz, Ex, Ey,
                                       Ez, P.boys, I);
      contract_shift<LA, LB, LC, LD, 1, 1>(I, Wt, g);
    } else if (sh == 3) {
      if constexpr (LB > 0) {
        double I[NA * ncart(LB - 1) * NC * ND];
        quartet_cart<LA, LB - 1, LC, LD>(P.pp, bp0, bnp, Ax, Ay, Az, Bx, By, Bz, P.pp, kp0, knp, Cx, Cy, Cz, Ex, Ey,
                                         Ez, P.boys, I);
        contract_shift<LA, LB, LC, LD, 1, -1>(I, Wt, g);
      }
    } else if (sh == 4) {
      double I[NA * NB * ncart(LC + 1) * ND];
      quartet_cart<LA, LB, LC + 1, LD>(P.pp, bp0, bnp, Ax, Ay, Az, Bx, By, Bz, P.pp2a, kp0, knp, Cx, Cy, Cz, Ex, Ey,
                                       Ez, P.boys, I);
      contract_shift<LA, LB, LC, LD, 2, 1>(I, Wt, g);
    } else {
      if constexpr (LC > 0) {
        double I[NA * NB * ncart(LC - 1) * ND];
        quartet_cart<LA, LB, LC - 1, LD>(P.pp, bp0, bnp, Ax, Ay, Az, Bx, By, Bz, P.pp, kp0, knp, Cx, Cy, Cz, Ex, Ey,
                                         Ez, P.boys, I);
        contract_shift<LA, LB, LC, LD, 2, -1>(I, Wt, g);
      }
    }
    const int atd = P.atom[d];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      const double v = deg * g[x];
      if (centre < 2)
        gbra[x] += v;
      else
        atomicAdd(P.grad + 3 * P.atom[c] + x, v);
      atomicAdd(P.grad + 3 * atd + x, -v);  // d: minus the derivative of the shifted centre
    }
  }
  if (centre < 2) {  // the bra centre's atom is the same for the whole block: one atomic per warp
    const int at = P.atom[centre == 0 ? a : b];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      double v = gbra[x];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(P.grad + 3 * at + x, v);
    }
  }
}

// ---------------------------------------------------------------- one-body
// Arguments of k_grad1e (grad1e.cu).
struct Grad1eParams {
  PairView pairs;
  PrimView pp;
  const double* pa;
  const double *ox, *oy, *oz;
  const int* coff;
  const int* atom;
  const unsigned char* sig;
  const double* Dc;  // Cartesian D, nc x nc
  const double* Wc;  // Cartesian W
  int nc;
  const double* boys;
  int natom;
  const double* Z;
  const double* cxyz;
  double* grad;
};

// launchers (grad_cls_*.cu, grad1e.cu)
void launch_grad2e_bra_s(int A, int B, const Grad2eParams& P, dim3 grid, cudaStream_t s);
void launch_grad2e_bra_ds(int B, const Grad2eParams& P, dim3 grid, cudaStream_t s);
void launch_grad2e_bra_dp(int B, const Grad2eParams& P, dim3 grid, cudaStream_t s);
void launch_grad2e_bra_dd(int B, const Grad2eParams& P, dim3 grid, cudaStream_t s);
void launch_grad1e(int pc, const Grad1eParams& P, cudaStream_t s);

}  // namespace m2
