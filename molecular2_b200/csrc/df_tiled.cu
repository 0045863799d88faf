// Density-fitted J/K for systems whose unpacked fitted tensor does not fit in
// HBM ((H2O)64 / aug-cc-pVDZ + AVDZ-JKFIT: n = 2624, naux = 9600, the
// unpacked FP64 B is 529 GB, molecular2's packed FP64 B 264 GB).  Same
// contraction as compute_2body_fock_df (molecular2 src/fockbuild.cpp:585-660).
//
// Storage.  B_K[x][y] is symmetric in (x, y), so only the tiles on and below
// the diagonal of a 128 x 128 tiling of the function pairs are kept: tile pair
// t = I(I+1)/2 + J (I >= J) holds B_K[128I + r][128J + c] for r, c < 128, as
// split BF16 (hi + lo) in [K][t][r][c] order (145 GB at the size above).
// Set-up builds it one tile pair at a time: the three-index integrals
// T[r][P][c] = (P | x y) of the tile pair (k_eri3_tile), B = L^-1 T on the
// FP64 DMMA GEMM, then the BF16 split; the FP64 B is never stored whole.
//
// Mixed build (prec_mode 1), per block of fitted functions:
//   GEMM1  X_K[x][i] = sum_y B_K[x][y] C[y][i]: one work item = (K, row tile
//          I, half of the occupied orbitals); its k loop runs over the row
//          of tiles, reading tile (I, J) as stored (K-major A) for J <= I and
//          tile (J, I) transposed (MN-major A descriptor, same bytes) for
//          J > I.  TMA -> 3-stage ring -> tcgen05.mma (M = 128, N = 160) ->
//          double-buffered TMEM; the epilogue writes X as BF16 hi/lo and adds
//          gamma_K = sum_{x,i} X C.
//   GEMM2  K += X X^T over the block (the tcgen05 kernel of df_mixed.cu).
// then J = sum_K gamma_K B_K over the stored tiles (HBM stream) and K, J are
// assembled from their lower triangles.
//
// FP64 build (prec_mode 0) keeps nothing per fitted function: per slice of
// the occupied orbitals it recomputes every tile pair's T, forms
// X'[x][P][i] = sum_y (P|xy) C[y][i] (two DMMA GEMMs per tile pair, one per
// orientation), Y = L^-1 X' and K += Y Y^T; d_P = sum_xy (P|xy) D_xy comes
// with the first pass and J = sum_P (xy|P) (V^-1 d)_P with the second.
#include <algorithm>
#include <cmath>
#include <functional>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "dense.cuh"
#include "df_kernels.cuh"
#include "engine.h"
#include "tc_gemm.cuh"

namespace m2 {
using namespace tc;

PrimView prim_view(const jk_engine* e);
Eri3Params eri3_params(const jk_engine* e, int l, int pc);
void stage_mark(jk_engine* e, int k, cudaStream_t s);

namespace {

constexpr int TB = DF_TILE;        // tile edge (functions)
constexpr long long TT = (long long)TB * TB;
constexpr int SN = 160;            // occupied orbitals per GEMM1 work item (MMA N)
constexpr int SBK = 64;            // BF16 per 128-byte swizzle row
constexpr int S1_A = TB * SBK * 2;         // 16 KB: one 128 x 64 operand tile
constexpr int S1_C = SN * SBK * 2;         // 20 KB
constexpr int S1_STAGE = 2 * S1_A + 2 * S1_C;
constexpr int S1_STAGES = 3;
constexpr int S1_SMEM = S1_STAGES * S1_STAGE + 1024 + 1024;
constexpr int S1_ACC = 256;        // TMEM columns per accumulator buffer (160 used)
constexpr int S1_EPI = 3;          // epilogue warps per TMEM lane quadrant
constexpr int S1_THREADS = 64 + 4 * 32 * S1_EPI;
static_assert(S1_SMEM <= 227 * 1024, "GEMM1 ring exceeds shared memory");

enum : int { ERR_WAIT_PRODUCER = 1, ERR_WAIT_MMA = 2, ERR_WAIT_EPILOGUE = 3 };
__device__ __forceinline__ void report(int* err, int code) { atomicCAS(err, 0, code); }

__host__ __device__ __forceinline__ void tile_of(int t, int& I, int& J) {
  int a = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (a * (a + 1) / 2 > t) --a;
  while ((a + 1) * (a + 2) / 2 <= t) ++a;
  I = a;
  J = t - a * (a + 1) / 2;
}

// ---------------------------------------------------------------- GEMM1 (symmetric tiles)
struct S1Params {
  int nt, npt;       // tile rows, stored tile pairs
  int k0, wstride;   // first fitted function of the block; X row stride in K
  int nhalf, nitems;
  int nocc, n, NPX;
  const float* Cx;   // [x][i] npad x NPX, C in FP32 (zero padded)
  __nv_bfloat16* Xh;  // [x][K_local][NPX]
  __nv_bfloat16* Xl;
  double* gamma;     // global fitted index
  double* Kt;        // K accumulator: receives the diagonal lo*lo term
  int* err;
};

__device__ __forceinline__ void s1_item(const S1Params& P, int item, int& Kl, int& I, int& h) {
  h = item % P.nhalf;
  const int r = item / P.nhalf;
  I = r % P.nt;
  Kl = r / P.nt;
}

// Accumulation groups of S1_GROUP 64-wide k chunks: the MMA warp restarts the
// TMEM accumulator for each group and the epilogue sums the FP32 group
// partials with round-to-nearest additions, so the downward drift of the
// tensor-core accumulation stays that of one group.  With two accumulator
// buffers the MMA warp runs at most two groups ahead of the epilogue, so a
// group must outlast the epilogue's per-item work (gamma, split, stores).
constexpr int S1_GROUP = 8;

// One epilogue warp's share of a work item: TMEM columns [16*C0, 16*C1) of its
// 32 rows summed over the item's accumulation groups (global group counter gt,
// buffer gt & 1, each released as soon as it is in registers), then added to
// gamma and written as BF16 hi/lo.  Returns false when a wait timed out.
template <int C0, int C1>
__device__ __forceinline__ bool s1_epilogue_item(uint32_t tbase, int& gt, int ngroups, int x, int Kl, int h,
                                                 const S1Params& P, uint64_t* tfull, uint64_t* tempty, int lane) {
  constexpr int NV = (C1 - C0) * 16;
  float v[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = 0.0f;
  for (int g = 0; g < ngroups; ++g, ++gt) {
    const int b = gt & 1;
    if (!mbar_wait(&tfull[b], (gt >> 1) & 1)) return false;
    tc_fence_after();
    const uint32_t taddr = tbase + b * S1_ACC;
#pragma unroll
    for (int c = C0; c < C1; ++c) {
      float w[16];
      tmem_ld16(taddr + c * 16, w);
      tmem_ld_wait();
#pragma unroll
      for (int e = 0; e < 16; ++e) v[(c - C0) * 16 + e] += w[e];
    }
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(&tempty[b]);
  }
  const int i0 = h * SN + C0 * 16;
  if (x < P.n) {  // gamma_K += sum_i X[x][K][i] C[x][i], the row of C as 16-byte vectors
    const float4* c4 = reinterpret_cast<const float4*>(P.Cx + (size_t)x * P.NPX + i0);
    double g4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < NV / 4; ++i) {
      const float4 c = __ldg(c4 + i);
      g4[0] += (double)v[4 * i] * c.x;
      g4[1] += (double)v[4 * i + 1] * c.y;
      g4[2] += (double)v[4 * i + 2] * c.z;
      g4[3] += (double)v[4 * i + 3] * c.w;
    }
    atomicAdd(P.gamma + P.k0 + Kl, (g4[0] + g4[1]) + (g4[2] + g4[3]));
  }
  const size_t row = ((size_t)x * P.wstride + Kl) * P.NPX + i0;
  uint4* oh = reinterpret_cast<uint4*>(P.Xh + row);
  uint4* ol = reinterpret_cast<uint4*>(P.Xl + row);
  float lsq = 0.0f;
#pragma unroll
  for (int c = 0; c < NV / 8; ++c) {
    __align__(16) __nv_bfloat16 hh[8], ll[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const float f = v[c * 8 + e];
      hh[e] = __float2bfloat16_rn(f);
      ll[e] = __float2bfloat16_rn(f - __bfloat162float(hh[e]));
      const float lf = __bfloat162float(ll[e]);
      lsq = fmaf(lf, lf, lsq);
    }
    oh[c] = *reinterpret_cast<const uint4*>(hh);
    ol[c] = *reinterpret_cast<const uint4*>(ll);
  }
  // the lo*lo term GEMM2 drops is sum_k lo_k^2 > 0 on the diagonal of K
  if (x < P.n) atomicAdd(P.Kt + (size_t)x * P.n + x, (double)lsq);
  return true;
}

__global__ void __launch_bounds__(S1_THREADS, 1)
    k_gemm1_sym(const __grid_constant__ CUtensorMap tBhK, const __grid_constant__ CUtensorMap tBlK,
                const __grid_constant__ CUtensorMap tBhM, const __grid_constant__ CUtensorMap tBlM,
                const __grid_constant__ CUtensorMap tCh, const __grid_constant__ CUtensorMap tCl, const S1Params P) {
  constexpr int S = S1_STAGES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + S * S1_STAGE);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kchunks = 2 * P.nt;  // 64-wide k chunks per work item

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4 * S1_EPI);
    }
    mbar_init(drain, 1);
    fence_barrier_init();
    prefetch_tmap(&tBhK);
    prefetch_tmap(&tBlK);
    prefetch_tmap(&tBhM);
    prefetch_tmap(&tBlM);
    prefetch_tmap(&tCh);
    prefetch_tmap(&tCl);
  }
  if (warp == 0) tmem_alloc(tmem_slot, 2 * S1_ACC);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int it = 0, last_s = -1;
      uint32_t last_par = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < P.nitems && ok; item += gridDim.x) {
        int Kl, I, h;
        s1_item(P, item, Kl, I, h);
        const long long K = P.k0 + Kl;
        for (int q = 0; q < kchunks; ++q, ++it) {
          const int J = q >> 1, cc = q & 1;
          const int s = it % S;
          const uint32_t j = it / S;
          if (!mbar_wait(&empty[s], (j & 1) ^ 1)) {
            report(P.err, ERR_WAIT_PRODUCER);
            ok = false;
            break;
          }
          uint8_t* st = smem + s * S1_STAGE;
          mbar_arrive_expect_tx(&full[s], S1_STAGE);
          if (J <= I) {  // stored tile (I, J): rows x of I, columns y of J
            const int row = (int)((K * P.npt + I * (I + 1) / 2 + J) * TB);
            tma_load_2d(st, &tBhK, SBK * cc, row, &full[s]);
            tma_load_2d(st + S1_A, &tBlK, SBK * cc, row, &full[s]);
          } else {       // stored tile (J, I): rows y of J (k), columns x of I (m)
            const int row = (int)((K * P.npt + J * (J + 1) / 2 + I) * TB) + SBK * cc;
            tma_load_2d(st, &tBhM, 0, row, &full[s]);
            tma_load_2d(st + S1_A / 2, &tBhM, SBK, row, &full[s]);
            tma_load_2d(st + S1_A, &tBlM, 0, row, &full[s]);
            tma_load_2d(st + S1_A + S1_A / 2, &tBlM, SBK, row, &full[s]);
          }
          const int ycol = TB * J + SBK * cc;
          tma_load_2d(st + 2 * S1_A, &tCh, ycol, h * SN, &full[s]);
          tma_load_2d(st + 2 * S1_A + S1_C, &tCl, ycol, h * SN, &full[s]);
          last_s = s;
          last_par = j & 1;
        }
      }
      if (last_s >= 0) mbar_wait(&full[last_s], last_par);  // no copy still in flight at exit
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idk = idesc_bf16_f32(TB, SN);
      constexpr uint32_t idm = idesc_bf16_f32_amn(TB, SN);
      int it = 0, gt = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < P.nitems && ok; item += gridDim.x) {
        int Kl, I, h;
        s1_item(P, item, Kl, I, h);
        for (int qg = 0; qg < kchunks && ok; qg += S1_GROUP, ++gt) {
          const int b = gt & 1;
          if (!mbar_wait(&tempty[b], ((gt >> 1) & 1) ^ 1)) {
            report(P.err, ERR_WAIT_MMA);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + b * S1_ACC;
          const int qend = min(qg + S1_GROUP, kchunks);
          for (int q = qg; q < qend; ++q, ++it) {
            const int J = q >> 1;
            const int s = it % S;
            const uint32_t j = it / S;
            if (!mbar_wait(&full[s], j & 1)) {
              report(P.err, ERR_WAIT_MMA);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint8_t* st = smem + s * S1_STAGE;
            const bool mn = J > I;
#pragma unroll
            for (int k = 0; k < SBK / 16; ++k) {
              uint64_t ah, al;
              if (!mn) {
                ah = sdesc_kmajor_sw128(st + k * 32);
                al = sdesc_kmajor_sw128(st + S1_A + k * 32);
              } else {
                ah = sdesc_mnmajor_sw128(st + k * 2048, S1_A / 2, 1024);
                al = sdesc_mnmajor_sw128(st + S1_A + k * 2048, S1_A / 2, 1024);
              }
              const uint64_t bh = sdesc_kmajor_sw128(st + 2 * S1_A + k * 32);
              const uint64_t bl = sdesc_kmajor_sw128(st + 2 * S1_A + S1_C + k * 32);
              const uint32_t id = mn ? idm : idk;
              umma_bf16(d, ah, bh, id, (q > qg || k > 0) ? 1u : 0u);
              umma_bf16(d, ah, bl, id, 1u);
              umma_bf16(d, al, bh, id, 1u);
            }
            umma_commit(&empty[s]);
          }
          if (ok) umma_commit(&tfull[b]);
        }
      }
      umma_commit(drain);  // every issued MMA has finished before TMEM is freed
      mbar_wait(drain, 0);
    }
  } else {  // epilogue: warp w drains TMEM lanes 32*(w%4).. and part (w-2)/4 of the 10 column chunks
    const int qd = warp & 3, part = (warp - 2) >> 2;
    const int ngroups = (kchunks + S1_GROUP - 1) / S1_GROUP;
    const uint32_t tbase = tmem + ((uint32_t)(32 * qd) << 16);
    int gt = 0;
    for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
      int Kl, I, h;
      s1_item(P, item, Kl, I, h);
      const int x = TB * I + 32 * qd + lane;
      bool ok;
      if (part == 0)
        ok = s1_epilogue_item<0, 4>(tbase, gt, ngroups, x, Kl, h, P, tfull, tempty, lane);
      else if (part == 1)
        ok = s1_epilogue_item<4, 7>(tbase, gt, ngroups, x, Kl, h, P, tfull, tempty, lane);
      else
        ok = s1_epilogue_item<7, 10>(tbase, gt, ngroups, x, Kl, h, P, tfull, tempty, lane);
      if (!ok) {
        report(P.err, ERR_WAIT_EPILOGUE);
        break;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * S1_ACC);
  }
}

// ---------------------------------------------------------------- J over the stored tiles
// J[x][y] (lower triangle) += sum_{K in range} gamma_K (Bh + Bl)[K][t][r][c]:
// block = (tile pair, 2048 elements, K range), 8 consecutive elements per thread.
constexpr int JT_THREADS = 256;
__global__ void __launch_bounds__(JT_THREADS) k_J_tiles(int npt, int naux, int kchunk, int n,
                                                        const __nv_bfloat16* __restrict__ Bh,
                                                        const __nv_bfloat16* __restrict__ Bl,
                                                        const double* __restrict__ gamma, double* __restrict__ J) {
  const int t = blockIdx.x;
  const int e0 = blockIdx.y * (JT_THREADS * 8) + threadIdx.x * 8;
  const int K0 = blockIdx.z * kchunk, K1 = min(naux, K0 + kchunk);
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
  for (int K = K0; K < K1; ++K) {
    const float g = (float)__ldg(gamma + K);
    const size_t off = ((size_t)K * npt + t) * TT + e0;
    const uint4 hv = __ldg(reinterpret_cast<const uint4*>(Bh + off));
    const uint4 lv = __ldg(reinterpret_cast<const uint4*>(Bl + off));
    const __nv_bfloat16* hh = reinterpret_cast<const __nv_bfloat16*>(&hv);
    const __nv_bfloat16* ll = reinterpret_cast<const __nv_bfloat16*>(&lv);
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[e] += g * (__bfloat162float(hh[e]) + __bfloat162float(ll[e]));
  }
  int I, Jt;
  tile_of(t, I, Jt);
  const int r = e0 / TB, c0 = e0 % TB;
  const int x = TB * I + r;
  if (x >= n) return;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int y = TB * Jt + c0 + e;
    if (y < n && y <= x) atomicAdd(J + (size_t)y * n + x, (double)acc[e]);
  }
}

// ---------------------------------------------------------------- set-up helpers
// Bt64[r][K][c] (FP64) -> Bh/Bl[K][t][r][c]
__global__ void k_store_tile(int t, int npt, int naux, const double* __restrict__ Bt, __nv_bfloat16* __restrict__ Bh,
                             __nv_bfloat16* __restrict__ Bl) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)TB * naux * TB;
  if (idx >= tot) return;
  const int c = (int)(idx % TB);
  const size_t rk = idx / TB;
  const int K = (int)(rk % naux), r = (int)(rk / naux);
  const double v = Bt[idx];
  const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
  const size_t dst = (((size_t)K * npt + t) * TB + r) * TB + c;
  Bh[dst] = h;
  Bl[dst] = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
}

// ---------------------------------------------------------------- FP64-build helpers
// d_P += w * sum_{r,c} T[r][P][c] D[x][y], x = x0 + r, y = y0 + c (D column-major n x n)
__global__ void __launch_bounds__(256) k_tile_d(int naux, int n, int x0, int y0, double w, const double* __restrict__ T,
                                                const double* __restrict__ D, double* __restrict__ d) {
  const int r = blockIdx.y, x = x0 + r;
  const int P = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (P >= naux || x >= n) return;
  const double* tr = T + ((size_t)r * naux + P) * TB;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < TB / 32; ++k) {
    const int c = lane + 32 * k, y = y0 + c;
    if (y < n) acc += tr[c] * D[(size_t)y * n + x];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) atomicAdd(d + P, w * acc);
}

// J[x][y] (lower triangle) += sum_P T[r][P][c] cv_P over a range of P
__global__ void __launch_bounds__(TB) k_tile_J(int naux, int n, int x0, int y0, int pchunk, const double* __restrict__ T,
                                              const double* __restrict__ cv, double* __restrict__ J) {
  const int r = blockIdx.y, c = threadIdx.x, x = x0 + r, y = y0 + c;
  const int P0 = blockIdx.x * pchunk, P1 = min(naux, P0 + pchunk);
  if (x >= n || y >= n || y > x) return;
  const double* tr = T + (size_t)r * naux * TB + c;
  double acc = 0.0;
  for (int P = P0; P < P1; ++P) acc += tr[(size_t)P * TB] * __ldg(cv + P);
  atomicAdd(J + (size_t)y * n + x, acc);
}

// Cpad (npad x nocc column-major, zero rows beyond n) from C (n x nocc)
__global__ void k_pad_rows(int n, int npad, int nocc, const double* __restrict__ C, double* __restrict__ Cp) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)npad * nocc) return;
  const int x = (int)(idx % npad), i = (int)(idx / npad);
  Cp[idx] = x < n ? C[(size_t)i * n + x] : 0.0;
}

}  // namespace

// ---------------------------------------------------------------- host
bool df_use_tiled(jk_engine* e) {
  if (e->df_storage == 2) return true;
  if (e->df_storage == 1) return false;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return false;
  const double n = e->obs.n_final, q = e->aux.n_final;
  // the unpacked path holds T3 and B64 (FP64) at set-up, then B64 and its split copy
  return 16.0 * n * n * q > 0.8 * (double)fr;
}

// Per tile pair and pair class: the shell pairs whose function ranges touch
// the tile pair in either orientation (pairs with a negligible Schwarz bound
// are left out: their integrals are below 1e-15 times the fitting norm).
static int build_tile_lists(jk_engine* e) {
  TiledDF& T = e->tiled;
  const HostBasis& b = e->obs;
  const int ns = b.nshell;
  std::vector<std::vector<int>> lists((size_t)T.npt * NPAIRCLASS);
  for (int pc = 0; pc < NPAIRCLASS; ++pc) {
    const int np = e->pcls[pc].npair;
    if (!np) continue;
    std::vector<int> sa(np), sb(np);
    cudaError_t st = cudaMemcpy(sa.data(), e->pcls[pc].sa.p, sizeof(int) * np, cudaMemcpyDeviceToHost);
    if (st == cudaSuccess) st = cudaMemcpy(sb.data(), e->pcls[pc].sb.p, sizeof(int) * np, cudaMemcpyDeviceToHost);
    if (st != cudaSuccess) return check_cuda(e, st, "tiled DF: pair lists");
    for (int ip = 0; ip < np; ++ip) {
      const int a = sa[ip], c = sb[ip];
      if (e->schwarz_host[(size_t)a * ns + c] < 1e-15) continue;
      const int fa0 = b.off_final[a], fa1 = b.off_final[a + 1], fc0 = b.off_final[c], fc1 = b.off_final[c + 1];
      for (int I = fa0 / TB; I <= (fa1 - 1) / TB; ++I)
        for (int J = fc0 / TB; J <= (fc1 - 1) / TB; ++J) {
          const int hi = std::max(I, J), lo = std::min(I, J);
          std::vector<int>& L = lists[(size_t)(hi * (hi + 1) / 2 + lo) * NPAIRCLASS + pc];
          if (L.empty() || L.back() != ip) L.push_back(ip);
        }
    }
  }
  T.list_off.assign(lists.size() + 1, 0);
  std::vector<int> flat;
  for (size_t k = 0; k < lists.size(); ++k) {
    T.list_off[k] = (long long)flat.size();
    flat.insert(flat.end(), lists[k].begin(), lists[k].end());
  }
  T.list_off[lists.size()] = (long long)flat.size();
  if (flat.empty()) flat.push_back(0);
  cudaError_t st = T.plist.upload(flat, e->stream);
  return check_cuda(e, st, "tiled DF: tile lists");
}

// T[r][P][c] = (P | x y) for tile pair t (zeroed first)
static int tile_integrals(jk_engine* e, int t, double* T, cudaStream_t s) {
  TiledDF& D = e->tiled;
  const int naux = e->aux.n_final;
  int I, J;
  tile_of(t, I, J);
  cudaMemsetAsync(T, 0, sizeof(double) * TB * (size_t)naux * TB, s);
  // the (fitting l, pair class) launches write disjoint parts of T: they run
  // longest first on the side streams (cost: pairs x fitting functions x
  // Cartesian sizes), so that the small ones fill the tails of the large ones
  static const double ncp[NPAIRCLASS] = {1, 3, 9, 6, 18, 36};
  struct Item {
    int l, pc;
    double cost;
  };
  Item items[(MAX_L_AUX + 1) * NPAIRCLASS];
  int nitems = 0;
  for (int l = 0; l <= MAX_L_AUX; ++l) {
    if (!e->aux_by_l_count[l]) continue;
    for (int pc = 0; pc < NPAIRCLASS; ++pc) {
      const long long o0 = D.list_off[(size_t)t * NPAIRCLASS + pc], o1 = D.list_off[(size_t)t * NPAIRCLASS + pc + 1];
      if (o1 > o0) items[nitems++] = {l, pc, (double)(o1 - o0) * e->aux_by_l_count[l] * ncp[pc] * (l + 1) * (l + 2)};
    }
  }
  std::sort(items, items + nitems, [](const Item& a, const Item& b) { return a.cost > b.cost; });
  ClassStreams cs(e, s);
  for (int k = 0; k < nitems; ++k) {
    const int l = items[k].l, pc = items[k].pc;
    const long long o0 = D.list_off[(size_t)t * NPAIRCLASS + pc];
    const Eri3Params P = eri3_params(e, l, pc);
    Eri3TileArgs A{};
    A.plist = D.plist.p + o0;
    A.nlist = (int)(D.list_off[(size_t)t * NPAIRCLASS + pc + 1] - o0);
    A.x0 = TB * I;
    A.y0 = TB * J;
    A.naux = naux;
    A.T = T;
    cudaStream_t q = cs.next(items[k].cost);
    if (l == 0) launch_eri3_tile_l0(pc, P, A, q);
    if (l == 1) launch_eri3_tile_l1(pc, P, A, q);
    if (l == 2) launch_eri3_tile_l2(pc, P, A, q);
    if (l == 3) launch_eri3_tile_l3(pc, P, A, q);
  }
  cs.join();
  return check_cuda(e, cudaGetLastError(), "tile integrals");
}

// Metric, its Cholesky factor and inverse, and the tile-pair lists: all the
// tiled builds and the tiled gradient need, without the fitted tensor.
int df_tiled_metric(jk_engine* e) {
  TiledDF& T = e->tiled;
  if (T.metric_ready) return JK_OK;
  int rc = prepare_aux(e);
  if (rc) return rc;
  cudaStream_t s = e->stream;
  DFState& d = e->df;
  if (d.k0 != 0 || (d.k1 >= 0 && d.k1 != e->aux.n_final))
    return set_error(e, JK_ERR_STATE, "tiled DF storage keeps the whole fitting range (no jk_df_set_range)");
  const int n = e->obs.n_final, naux = e->aux.n_final;
  T.nt = (n + TB - 1) / TB;
  T.npt = T.nt * (T.nt + 1) / 2;
  T.npad = T.nt * TB;
  cudaError_t st = d.L.alloc((size_t)naux * naux);
  if (st == cudaSuccess) st = d.Linv.alloc((size_t)naux * naux);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled DF: metric allocation");
  if ((rc = compute_V(e, d.L.p, s))) return rc;
  {
    DevBuf<double> work;
    DevBuf<int> info;
    st = work.alloc((size_t)naux * naux);
    if (st == cudaSuccess) st = info.alloc(1);
    if (st != cudaSuccess) return check_cuda(e, st, "Cholesky workspace");
    if ((rc = cholesky(e, d.L.p, naux, work.p, info.p, s))) return rc;
    int hinfo = 0;
    st = cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (st == cudaSuccess) st = cudaStreamSynchronize(s);
    if (st != cudaSuccess) return check_cuda(e, st, "Cholesky");
    if (hinfo != 0)
      return set_error(e, JK_ERR_NOT_PD,
                       "fitting metric (P|Q) is not positive definite (leading minor " + std::to_string(hinfo) + ")");
    if ((rc = tri_inverse(e, d.L.p, d.Linv.p, naux, work.p, s))) return rc;
  }
  if ((rc = build_tile_lists(e))) return rc;
  st = cudaStreamSynchronize(s);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled DF metric");
  T.metric_ready = true;
  return JK_OK;
}

int df_tiled_setup(jk_engine* e) {
  int rc = df_tiled_metric(e);
  if (rc) return rc;
  cudaStream_t s = e->stream;
  DFState& d = e->df;
  TiledDF& T = e->tiled;
  const int naux = e->aux.n_final;
  cudaError_t st;
  const size_t nB = (size_t)naux * T.npt * TT;
  st = T.Bh.alloc(nB);
  if (st == cudaSuccess) st = T.Bl.alloc(nB);
  if (st != cudaSuccess) {
    T.Bh.reset();
    T.Bl.reset();
    return set_error(e, JK_ERR_NOMEM, "tiled DF: the split-BF16 fitted tensor (" +
                                          std::to_string(2.0 * nB * 2 / 1e9) + " GB) does not fit on the device");
  }
  DevBuf<double> Tt, Bt;
  st = Tt.alloc((size_t)TB * naux * TB);
  if (st == cudaSuccess) st = Bt.alloc((size_t)TB * naux * TB);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled DF: tile buffers");
  const size_t tot = (size_t)TB * naux * TB;
  for (int t = 0; t < T.npt; ++t) {
    if ((rc = tile_integrals(e, t, Tt.p, s))) return rc;
    // Bt[r][K][c] = sum_P Linv[K][P] T[r][P][c]
    DGemm g;
    g.M = naux;
    g.N = TB;
    g.K = naux;
    g.batch = TB;
    g.A = d.Linv.p;
    g.sam = 1;
    g.sak = naux;
    g.a_lower = true;
    g.B = Tt.p;
    g.sbk = TB;
    g.sbn = 1;
    g.bsb = (long long)naux * TB;
    g.C = Bt.p;
    g.scm = TB;
    g.scn = 1;
    g.bsc = (long long)naux * TB;
    st = dgemm(g, s);
    if (st != cudaSuccess) return check_cuda(e, st, "tiled DF: B = L^-1 T");
    k_store_tile<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(t, T.npt, naux, Bt.p, T.Bh.p, T.Bl.p);
  }
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled DF set-up");
  d.naux = naux;
  d.ready = true;
  T.ready = true;
  return JK_OK;
}

// Scratch of the mixed build, sized for the largest occupied count seen so far
// (a smaller count reuses it with tensor maps for its own row length, so the
// varying column counts of incremental builds allocate nothing).
static int tiled_mixed_prepare(jk_engine* e, int nocc) {
  TiledDF& T = e->tiled;
  const int naux = e->aux.n_final, n = e->obs.n_final;
  const int nhalf = (nocc + SN - 1) / SN;
  const int NPX = nhalf * SN;
  cudaError_t st;
  if (!T.Xh.p || NPX > T.NPX_cap) {
    T.Ch.reset();
    T.Cl.reset();
    T.Xh.reset();
    T.Xl.reset();
    st = T.Ch.alloc((size_t)NPX * T.npad);
    if (st == cudaSuccess) st = T.Cx.alloc((size_t)NPX * T.npad);
    if (st == cudaSuccess) st = T.Cl.alloc((size_t)NPX * T.npad);
    if (st == cudaSuccess) st = T.Kt.alloc((size_t)n * n);
    if (st == cudaSuccess) st = T.err.alloc(1);
    if (st == cudaSuccess) st = e->df.gamma.alloc(naux);
    if (st != cudaSuccess) return check_cuda(e, st, "tiled mixed scratch");
    // X block: as many fitted functions as fit in a quarter of the free memory (at most all)
    size_t fr = 0, tt = 0;
    cudaMemGetInfo(&fr, &tt);
    const double per_k = 4.0 * T.npad * NPX;  // hi + lo BF16
    int w = (int)std::min<double>(naux, std::max(64.0, 0.25 * fr / per_k));
    if (T.waux_max > 0) w = std::min(w, T.waux_max);
    w = std::max(1, std::min(naux, w));
    // X rows are padded to an even number of fitted functions, so that a row
    // is a whole number of 64-wide k blocks (NPX is a multiple of 160)
    for (;; w = w / 2) {
      const int ws = w + (w & 1);
      st = T.Xh.alloc((size_t)T.npad * ws * NPX);
      if (st == cudaSuccess) st = T.Xl.alloc((size_t)T.npad * ws * NPX);
      if (st == cudaSuccess) break;
      T.Xh.reset();
      T.Xl.reset();
      cudaGetLastError();
      if (w <= 16) return check_cuda(e, st, "tiled mixed X block");
    }
    T.waux = w;
    T.wstride = w + (w & 1);
    T.NPX_cap = NPX;
    T.NPX = 0;
    cudaMemsetAsync(T.err.p, 0, sizeof(int), e->stream);
    const uint64_t brows = (uint64_t)naux * T.npt * TB;
    const bool ok = make_map(&T.maps[0], T.Bh.p, TB, brows, SBK, TB) && make_map(&T.maps[1], T.Bl.p, TB, brows, SBK, TB) &&
                    make_map(&T.maps[2], T.Bh.p, TB, brows, SBK, SBK) && make_map(&T.maps[3], T.Bl.p, TB, brows, SBK, SBK);
    if (!ok) return set_error(e, JK_ERR_CUDA, "cuTensorMapEncodeTiled failed (tiled DF)");
  }
  if (T.NPX != NPX) {
    const bool ok = make_map(&T.maps[4], T.Ch.p, T.npad, NPX, SBK, SN) && make_map(&T.maps[5], T.Cl.p, T.npad, NPX, SBK, SN) &&
                    make_map(&T.maps[6], T.Xh.p, (uint64_t)T.wstride * NPX, T.npad, SBK, TB) &&
                    make_map(&T.maps[7], T.Xl.p, (uint64_t)T.wstride * NPX, T.npad, SBK, TB);
    if (!ok) return set_error(e, JK_ERR_CUDA, "cuTensorMapEncodeTiled failed (tiled DF)");
    T.NPX = NPX;
  }
  T.nocc = nocc;
  return JK_OK;
}

static int tiled_mixed(jk_engine* e, const double* dC, int nocc, double* dJ, double* dK, cudaStream_t s) {
  int rc = tiled_mixed_prepare(e, nocc);
  if (rc) return rc;
  TiledDF& T = e->tiled;
  DFState& d = e->df;
  const int n = e->obs.n_final, naux = e->aux.n_final;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device);
  stage_mark(e, 0, s);
  cudaError_t st = launch_split_C(n, nocc, T.NPX, T.npad, dC, T.Ch.p, T.Cl.p, s);
  if (st == cudaSuccess) st = launch_rows_C(n, nocc, T.NPX, T.npad, dC, T.Cx.p, s);
  if (st != cudaSuccess) return check_cuda(e, st, "split C");
  cudaMemsetAsync(d.gamma.p, 0, sizeof(double) * naux, s);
  cudaMemsetAsync(T.Kt.p, 0, sizeof(double) * n * n, s);
  cudaMemsetAsync(dJ, 0, sizeof(double) * n * n, s);
  st = cudaFuncSetAttribute(k_gemm1_sym, cudaFuncAttributeMaxDynamicSharedMemorySize, S1_SMEM);
  if (st != cudaSuccess) return check_cuda(e, st, "gemm1 attribute");
  const int nblocks = (naux + T.waux - 1) / T.waux;
  e->kev_blocks = 0;
  auto kmark = [&](size_t k) {
    if (!e->profiling) return;
    while (e->kev.size() <= k) {
      cudaEvent_t ev;
      cudaEventCreate(&ev);
      e->kev.push_back(ev);
    }
    cudaEventRecord(e->kev[k], s);
  };
  int blk = 0;
  for (int k0 = 0; k0 < naux; k0 += T.waux, ++blk) {
    kmark(3 * blk);
    const int w = std::min(T.waux, naux - k0);
    S1Params P{};
    P.nt = T.nt;
    P.npt = T.npt;
    P.k0 = k0;
    P.wstride = T.wstride;
    P.nhalf = T.NPX / SN;
    P.nitems = w * T.nt * P.nhalf;
    P.nocc = nocc;
    P.n = n;
    P.NPX = T.NPX;
    P.Cx = T.Cx.p;
    P.Xh = T.Xh.p;
    P.Xl = T.Xl.p;
    P.gamma = d.gamma.p;
    P.Kt = T.Kt.p;
    P.err = T.err.p;
    k_gemm1_sym<<<std::min(nsm, P.nitems), S1_THREADS, S1_SMEM, s>>>(T.maps[0], T.maps[1], T.maps[2], T.maps[3],
                                                                       T.maps[4], T.maps[5], P);
    st = cudaGetLastError();
    if (st != cudaSuccess) return check_cuda(e, st, "gemm1 (tiled) launch");
    kmark(3 * blk + 1);
    // GEMM2 reads whole 64-wide k blocks: when w * NPX is not a multiple of
    // 64 (odd w with an odd number of 160-orbital halves) the tail of each X
    // row holds the previous block's values, so clear it
    const int kbl = (w * T.NPX + SBK - 1) / SBK;
    if (kbl * SBK != w * T.NPX) {
      const size_t pitch = (size_t)T.wstride * T.NPX * sizeof(__nv_bfloat16);
      const size_t off = (size_t)w * T.NPX, width = (size_t)kbl * SBK - off;
      cudaMemset2DAsync(T.Xh.p + off, pitch, 0, width * sizeof(__nv_bfloat16), T.npad, s);
      cudaMemset2DAsync(T.Xl.p + off, pitch, 0, width * sizeof(__nv_bfloat16), T.npad, s);
    }
    st = launch_gemm2(T.maps[6], T.maps[7], n, kbl, T.Kt.p, T.err.p, nsm, s);
    if (st != cudaSuccess) return check_cuda(e, st, "gemm2 (tiled) launch");
    kmark(3 * blk + 2);
  }
  stage_mark(e, 1, s);
  const int ksplit = 8, kchunk = (naux + ksplit - 1) / ksplit;
  k_J_tiles<<<dim3(T.npt, (unsigned)(TT / (JT_THREADS * 8)), ksplit), JT_THREADS, 0, s>>>(T.npt, naux, kchunk, n,
                                                                                        T.Bh.p, T.Bl.p, d.gamma.p, dJ);
  stage_mark(e, 2, s);
  kmark(3 * nblocks);
  st = launch_finalize_mixed(n, T.Kt.p, dJ, dK, s);
  stage_mark(e, 3, s);
  kmark(3 * nblocks + 1);
  if (e->profiling) e->kev_blocks = nblocks;
  return check_cuda(e, st, "tiled mixed DF");
}

static int tiled_mixed_error(jk_engine* e) {
  TiledDF& T = e->tiled;
  if (!T.err.p) return JK_OK;
  int h = 0;
  cudaError_t st = cudaMemcpyAsync(&h, T.err.p, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled DF error word");
  if (h) {
    cudaMemsetAsync(T.err.p, 0, sizeof(int), e->stream);
    return set_error(e, JK_ERR_CUDA, "tiled DF: tensor-core pipeline wait timed out (stage " + std::to_string(h) + ")");
  }
  return JK_OK;
}

// One pass over every tile pair: X'[x][P][i] = sum_y (P|xy) Cp[y][i0 + i] for
// i < ocur (X zeroed here; Cp is the npad x nocc zero-padded C).  hook(t, I, J)
// runs after tile pair t's integrals are in Tt.
int tiled_xprime_pass(jk_engine* e, const double* Cp, int i0, int ocur, double* X, double* Tt, cudaStream_t s,
                      const std::function<int(int, int, int)>& hook) {
  TiledDF& T = e->tiled;
  const int naux = e->aux.n_final, npad = T.npad;
  cudaMemsetAsync(X, 0, sizeof(double) * (size_t)npad * naux * ocur, s);
  int rc;
  cudaError_t st;
  for (int t = 0; t < T.npt; ++t) {
    int I, J;
    tile_of(t, I, J);
    if ((rc = tile_integrals(e, t, Tt, s))) return rc;
    if (hook && (rc = hook(t, I, J))) return rc;
    // X'[x in I][P][i] += sum_c T[r][P][c] C[128J + c][i]: rows (r, P) in one GEMM
    DGemm a;
    a.M = TB * naux;
    a.N = ocur;
    a.K = TB;
    a.A = Tt;
    a.sam = TB;
    a.sak = 1;
    a.B = Cp + (size_t)TB * J + (size_t)i0 * npad;
    a.sbk = 1;
    a.sbn = npad;
    a.C = X + (size_t)TB * I * naux * ocur;
    a.scm = ocur;
    a.scn = 1;
    a.beta = 1.0;
    if ((st = dgemm(a, s)) != cudaSuccess) return check_cuda(e, st, "X' (rows)");
    if (I != J) {  // X'[y in J][P][i] += sum_r T[r][P][c] C[128I + r][i], one GEMM per P
      DGemm b;
      b.M = TB;
      b.N = ocur;
      b.K = TB;
      b.batch = naux;
      b.A = Tt;
      b.sam = 1;
      b.sak = (long long)naux * TB;
      b.bsa = TB;
      b.B = Cp + (size_t)TB * I + (size_t)i0 * npad;
      b.sbk = 1;
      b.sbn = npad;
      b.C = X + (size_t)TB * J * naux * ocur;
      b.scm = (long long)naux * ocur;
      b.scn = 1;
      b.bsc = ocur;
      b.beta = 1.0;
      if ((st = dgemm(b, s)) != cudaSuccess) return check_cuda(e, st, "X' (columns)");
    }
  }
  return JK_OK;
}

void launch_pad_rows(int n, int npad, int nocc, const double* C, double* Cp, cudaStream_t s) {
  k_pad_rows<<<(unsigned)(((size_t)npad * nocc + 255) / 256), 256, 0, s>>>(n, npad, nocc, C, Cp);
}

// FP64 build with the three-index integrals recomputed per occupied slice.
static int tiled_fp64(jk_engine* e, const double* dC, int nocc, double* dJ, double* dK, cudaStream_t s) {
  TiledDF& T = e->tiled;
  DFState& d = e->df;
  const int n = e->obs.n_final, naux = e->aux.n_final, npad = T.npad;
  const size_t tbytes = sizeof(double) * (size_t)TB * naux * TB;
  // scratch that does not depend on the slice
  DevBuf<double> Tt, Cp, Dm, dv, cv, tv;
  cudaError_t st = Tt.alloc(tbytes / sizeof(double));
  if (st == cudaSuccess) st = Cp.alloc((size_t)npad * nocc);
  if (st == cudaSuccess) st = Dm.alloc((size_t)n * n);
  if (st == cudaSuccess) st = dv.alloc(naux);
  if (st == cudaSuccess) st = cv.alloc(naux);
  if (st == cudaSuccess) st = tv.alloc(naux);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled FP64 scratch");
  // the mixed build's X block is released (its next call allocates it again)
  // so that the occupied slices, each one more integral pass, are as wide as
  // the memory allows
  if (T.Xh.p) {
    T.Xh.reset();
    T.Xl.reset();
  }
  // occupied slice: X' (npad x naux x oc) and a Y batch of XB rows must fit
  constexpr int XB = 64;
  size_t fr = 0, tt = 0;
  cudaMemGetInfo(&fr, &tt);
  const double per_o = 8.0 * (double)(npad + XB) * naux;
  int oc = (int)std::min<double>(nocc, std::floor(0.94 * (double)fr / per_o));
  if (T.oc_max > 0) oc = std::min(oc, T.oc_max);
  if (oc < 1) return set_error(e, JK_ERR_NOMEM, "tiled FP64 DF: no room for one occupied orbital's X'");
  const int nch = (nocc + oc - 1) / oc;
  oc = (nocc + nch - 1) / nch;
  DevBuf<double> X, Yb;
  st = X.alloc((size_t)npad * naux * oc);
  if (st == cudaSuccess) st = Yb.alloc((size_t)XB * naux * oc);
  if (st != cudaSuccess) return check_cuda(e, st, "tiled FP64 X'");
  k_pad_rows<<<(unsigned)(((size_t)npad * nocc + 255) / 256), 256, 0, s>>>(n, npad, nocc, dC, Cp.p);
  {
    DGemm g;  // D = C C^T
    g.M = n;
    g.N = n;
    g.K = nocc;
    g.A = dC;
    g.sam = 1;
    g.sak = n;
    g.B = dC;
    g.sbk = n;
    g.sbn = 1;
    g.C = Dm.p;
    g.scm = 1;
    g.scn = n;
    if ((st = dgemm(g, s)) != cudaSuccess) return check_cuda(e, st, "D = C C^T");
  }
  cudaMemsetAsync(dv.p, 0, sizeof(double) * naux, s);
  cudaMemsetAsync(dJ, 0, sizeof(double) * n * n, s);
  cudaMemsetAsync(dK, 0, sizeof(double) * n * n, s);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device);
  int rc;
  auto j_pass_tile = [&](int t, int I, int J) {
    const int pchunk = (naux + 15) / 16;
    k_tile_J<<<dim3((naux + pchunk - 1) / pchunk, TB), TB, 0, s>>>(naux, n, TB * I, TB * J, pchunk, Tt.p, cv.p, dJ);
    (void)t;
  };
  stage_mark(e, 0, s);
  for (int ch = 0; ch < nch; ++ch) {
    const int i0 = ch * oc, ocur = std::min(oc, nocc - i0);
    rc = tiled_xprime_pass(e, Cp.p, i0, ocur, X.p, Tt.p, s, [&](int t, int I, int J) {
      (void)t;
      if (ch == 0)
        k_tile_d<<<dim3((naux + 7) / 8, TB), 256, 0, s>>>(naux, n, TB * I, TB * J, I == J ? 1.0 : 2.0, Tt.p, Dm.p, dv.p);
      if (ch == 1) j_pass_tile(t, I, J);
      return JK_OK;
    });
    if (rc) return rc;
    if (ch == 0) stage_mark(e, 1, s);  // profiling: first integral + X' pass
    if (ch == 0) {  // c = V^-1 d = L^-T (L^-1 d)
      DGemm g;
      g.M = naux;
      g.N = 1;
      g.K = naux;
      g.A = d.Linv.p;
      g.sam = 1;
      g.sak = naux;
      g.a_lower = true;
      g.B = dv.p;
      g.sbk = 1;
      g.C = tv.p;
      g.scm = 1;
      if ((st = dgemm(g, s)) != cudaSuccess) return check_cuda(e, st, "L^-1 d");
      g.A = d.Linv.p;
      g.sam = naux;
      g.sak = 1;
      g.a_lower = false;
      g.B = tv.p;
      g.C = cv.p;
      if ((st = dgemm(g, s)) != cudaSuccess) return check_cuda(e, st, "L^-T (L^-1 d)");
    }
    // Y = L^-1 X' for every row x, XB rows at a time
    for (int x0 = 0; x0 < n; x0 += XB) {
      const int xb = std::min(XB, n - x0);
      DGemm y;
      y.M = naux;
      y.N = ocur;
      y.K = naux;
      y.batch = xb;
      y.A = d.Linv.p;
      y.sam = 1;
      y.sak = naux;
      y.a_lower = true;
      y.B = X.p + (size_t)x0 * naux * ocur;
      y.sbk = ocur;
      y.sbn = 1;
      y.bsb = (long long)naux * ocur;
      y.C = Yb.p;
      y.scm = ocur;
      y.scn = 1;
      y.bsc = (long long)naux * ocur;
      if ((st = dgemm(y, s)) != cudaSuccess) return check_cuda(e, st, "Y = L^-1 X'");
      st = cudaMemcpyAsync(X.p + (size_t)x0 * naux * ocur, Yb.p, sizeof(double) * (size_t)xb * naux * ocur,
                           cudaMemcpyDeviceToDevice, s);
      if (st != cudaSuccess) return check_cuda(e, st, "Y copy");
    }
    if (ch == 0) stage_mark(e, 2, s);  // profiling: Y = L^-1 X' of the first slice
    // K += Y Y^T over (P, i)
    {
      const long long len = (long long)naux * ocur;
      const int tiles = ((n + 127) / 128) * ((n + 127) / 128 + 1) / 2;
      DGemm k;
      k.M = n;
      k.N = n;
      k.K = (int)len;
      k.A = X.p;
      k.sam = len;
      k.sak = 1;
      k.B = X.p;
      k.sbk = 1;
      k.sbn = len;
      k.C = dK;
      k.scm = 1;
      k.scn = n;
      k.beta = 1.0;
      k.c_lower = true;
      k.ksplit = (int)std::max(1LL, std::min<long long>((2LL * nsm + tiles - 1) / tiles, len / 128));
      if ((st = dgemm(k, s)) != cudaSuccess) return check_cuda(e, st, "K += Y Y^T");
    }
    if (ch == 0) stage_mark(e, 3, s);  // profiling: K of the first slice
  }
  if (nch == 1)  // J needs V^-1 d, known only after the first pass
    for (int t = 0; t < T.npt; ++t) {
      int I, J;
      tile_of(t, I, J);
      if ((rc = tile_integrals(e, t, Tt.p, s))) return rc;
      j_pass_tile(t, I, J);
    }
  mirror_lower(dJ, n, s);
  mirror_lower(dK, n, s);
  stage_mark(e, 4, s);
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);  // scratch dies on return
  return check_cuda(e, st, "tiled FP64 DF");
}

int df_tiled_device(jk_engine* e, const double* dC, int nocc, int mode, double* dJ, double* dK, cudaStream_t s) {
  if (!e->tiled.metric_ready) return set_error(e, JK_ERR_STATE, "jk_df before jk_df_setup");
  if (mode == 0) return tiled_fp64(e, dC, nocc, dJ, dK, s);  // needs only the metric
  if (mode != 1) return set_error(e, JK_ERR_ARG, "jk_df: unsupported precision mode");
  if (!e->tiled.ready) {  // first mixed build after an FP64-only set-up: build the fitted tensor now
    const int rc = df_tiled_setup(e);
    if (rc) return rc;
  }
  int rc = tiled_mixed(e, dC, nocc, dJ, dK, s);
  return rc ? rc : JK_OK;
}

int df_tiled_error(jk_engine* e) { return tiled_mixed_error(e); }

}  // namespace m2

using namespace m2;

extern "C" int jk_df_set_storage(jk_engine* e, int mode) {
  if (!e) return JK_ERR_ARG;
  if (mode < 0 || mode > 2) return set_error(e, JK_ERR_ARG, "jk_df_set_storage: mode must be 0, 1 or 2");
  if (e->df.ready || e->tiled.metric_ready)
    return set_error(e, JK_ERR_STATE, "jk_df_set_storage after jk_df_setup");
  e->df_storage = mode;
  return JK_OK;
}

extern "C" int jk_df_set_tiled_blocks(jk_engine* e, int waux_max, int oc_max) {
  if (!e) return JK_ERR_ARG;
  if (waux_max < 0 || oc_max < 0) return set_error(e, JK_ERR_ARG, "jk_df_set_tiled_blocks: negative cap");
  e->tiled.waux_max = waux_max;
  e->tiled.oc_max = oc_max;
  e->tiled.NPX_cap = 0;  // re-plan the mixed scratch on the next build
  e->tiled.NPX = 0;
  return JK_OK;
}

extern "C" long long jk_df_tensor_bytes(const jk_engine* e) {
  if (!e) return -1;
  if (e->tiled.ready) return (long long)(e->tiled.Bh.n + e->tiled.Bl.n) * (long long)sizeof(__nv_bfloat16);
  if (e->df.ready)
    return (long long)e->df.B64.n * (long long)sizeof(double) +
           (long long)(e->mixed.Bh.n + e->mixed.Bl.n) * (long long)sizeof(__nv_bfloat16);
  return 0;
}

extern "C" int jk_df_storage(const jk_engine* e) {
  if (!e) return -1;
  return (e->tiled.ready || e->tiled.metric_ready) ? 2 : (e->df.ready ? 1 : 0);
}
