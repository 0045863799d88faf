// Mixed-precision DF J/K on the tcgen05 tensor cores (prec_mode 1).
//
// Same contraction as the FP64 path (compute_2body_fock_df, molecular2
// src/fockbuild.cpp:621-659), with B = Bhi + Blo and C = Chi + Clo split into
// BF16 pairs and every product formed as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory (~16 significant bits per operand), restarted
// every ACC_GROUP k-blocks and summed in registers:
//   GEMM1  X[m][i] = sum_y B[m][y] C[y][i],  m = (x,K): persistent kernel over
//          128-row tiles, TMA -> 4-stage smem ring -> tcgen05.mma (M=128,
//          N=nocc padded to 16) -> double-buffered TMEM accumulators.  The
//          epilogue re-splits X into BF16 hi/lo for GEMM2 and accumulates
//          gamma_K = sum_{x,i} X[x][K][i] C[x][i] (FP64 atomics).
//   GEMM2  K = X X^T over the naux*nocc index: 128x256 blocks of the lower
//          triangle, split-K across the SMs, register totals, FP64 atomics.
//   J      J[x][y] = sum_K gamma_K B[x][K][y] over y <= x: HBM-bound stream of
//          the lower half of B (hi + lo).
// One warp issues TMA, one issues MMA, the rest drain TMEM; all waits are bounded
// and report through an error word instead of hanging.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "engine.h"
#include "tc_gemm.cuh"

namespace m2 {
using namespace tc;

constexpr int BM = 128;           // MMA / tile rows
constexpr int BK = 64;            // BF16 elements per 128-byte swizzle row
constexpr int TILE_A_BYTES = BM * BK * 2;
constexpr int SMEM_LIMIT = 227 * 1024;

enum : int { ERR_NONE = 0, ERR_WAIT_PRODUCER = 1, ERR_WAIT_MMA = 2, ERR_WAIT_EPILOGUE = 3 };

__device__ __forceinline__ void report(int* err, int code) { atomicCAS(err, 0, code); }

// ---------------------------------------------------------------- GEMM1
struct G1Params {
  int M;            // n * naux rows of B
  int kblocks;      // ldb / 64
  int nocc;
  int n, naux;
  int ntiles;
  const float* Cx;  // [x][i] n x NP, C in FP32 (zero padded)
  __nv_bfloat16* Xhi;  // [m][NP]
  __nv_bfloat16* Xlo;
  double* gamma;
  double* Kt;       // K accumulator: receives the diagonal lo*lo term
  int* err;
};

template <int NP>
struct G1Layout {
  static constexpr int B_BYTES = NP * BK * 2;
  static constexpr int STAGE = 2 * TILE_A_BYTES + 2 * B_BYTES;
  static constexpr int STAGES = std::min(4, (SMEM_LIMIT - 4096) / STAGE);
  static constexpr int SMEM = STAGES * STAGE + 1024 /*barriers*/ + 1024 /*alignment*/;
  static constexpr int ACC_STRIDE = NP <= 128 ? 128 : 256;  // TMEM columns per accumulator buffer
  static constexpr int TMEM_COLS = 2 * ACC_STRIDE;
};

// Accumulation groups.  tcgen05.mma accumulates in FP32 and its additions
// lose low-order bits in one direction, so a long accumulation drifts toward
// zero (about -1e-4 relative after ~2000 k-blocks).  The MMA warp therefore
// restarts the TMEM accumulator every G1_GROUP (GEMM1) or ACC_GROUP (GEMM2)
// k-blocks of 64 inner-index values and the epilogue adds the group partials
// in registers with round-to-nearest arithmetic; the drift is then that of
// one group.
constexpr int G1_GROUP = 4;
constexpr int ACC_GROUP = 4;

// One epilogue warp's share of a GEMM1 tile: TMEM columns [16*C0, 16*C1) of
// its 32 rows, summed over the tile's `ngroups` accumulation groups (global
// group counter gt, buffer gt & 1).  Each buffer is released as soon as its
// values are in registers; the sum is then added to gamma and written as
// BF16 hi/lo.  Returns false when a wait timed out.
template <int NP, int C0, int C1>
__device__ __forceinline__ bool g1_epilogue_tile(uint32_t tbase, int& gt, int ngroups, int m, const G1Params& P,
                                                 uint64_t* tfull, uint64_t* tempty, int lane) {
  using Lay = G1Layout<NP>;
  constexpr int NV = (C1 - C0) * 16;
  float v[NV > 0 ? NV : 1];
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = 0.0f;
  for (int g = 0; g < ngroups; ++g, ++gt) {
    const int b = gt & 1;
    if (!mbar_wait(&tfull[b], (gt >> 1) & 1)) return false;
    tc_fence_after();
    const uint32_t taddr = tbase + b * Lay::ACC_STRIDE;
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
  if (NV == 0 || m >= P.M) return true;
  const int x = m / P.naux, K = m - x * P.naux;
  // gamma_K += sum_i X[x][K][i] C[x][i]: the row of C as 16-byte vectors
  const float4* c4 = reinterpret_cast<const float4*>(P.Cx + (size_t)x * NP + C0 * 16);
  double g4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < NV / 4; ++i) {
    const float4 c = __ldg(c4 + i);
    g4[0] += (double)v[4 * i] * c.x;
    g4[1] += (double)v[4 * i + 1] * c.y;
    g4[2] += (double)v[4 * i + 2] * c.z;
    g4[3] += (double)v[4 * i + 3] * c.w;
  }
  atomicAdd(P.gamma + K, (g4[0] + g4[1]) + (g4[2] + g4[3]));
  uint4* oh = reinterpret_cast<uint4*>(P.Xhi + (size_t)m * NP + C0 * 16);
  uint4* ol = reinterpret_cast<uint4*>(P.Xlo + (size_t)m * NP + C0 * 16);
  float lsq = 0.0f;
#pragma unroll
  for (int c = 0; c < NV / 8; ++c) {
    __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const float f = v[c * 8 + e];
      h[e] = __float2bfloat16_rn(f);
      l[e] = __float2bfloat16_rn(f - __bfloat162float(h[e]));
      const float lf = __bfloat162float(l[e]);
      lsq = fmaf(lf, lf, lsq);
    }
    oh[c] = *reinterpret_cast<const uint4*>(h);
    ol[c] = *reinterpret_cast<const uint4*>(l);
  }
  // GEMM2 forms hi*hi + hi*lo + lo*hi; the dropped lo*lo term averages out off
  // the diagonal but is sum_k lo_k^2 > 0 on it, so it is added here (one
  // atomic per warp when the warp's rows share x, as all but boundary rows do)
  double lq = (double)lsq;
  const unsigned mask = __activemask();
  if (mask == 0xffffffffu && __all_sync(mask, x == __shfl_sync(mask, x, 0))) {
    for (int o = 16; o > 0; o >>= 1) lq += __shfl_xor_sync(mask, lq, o);
    if (lane == 0) atomicAdd(P.Kt + (size_t)x * P.n + x, lq);
  } else {
    atomicAdd(P.Kt + (size_t)x * P.n + x, lq);
  }
  return true;
}

constexpr int G1_EPI = 3;                            // epilogue warps per TMEM lane quadrant
constexpr int G1_THREADS = 64 + 4 * 32 * G1_EPI;     // TMA warp, MMA warp, epilogue warps

template <int NP>
__global__ void __launch_bounds__(G1_THREADS, 1)
    k_gemm1(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
            const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl, const G1Params P) {
  using Lay = G1Layout<NP>;
  constexpr int S = Lay::STAGES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + S * Lay::STAGE);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4 * G1_EPI);
    }
    mbar_init(drain, 1);
    fence_barrier_init();
    prefetch_tmap(&tAh);
    prefetch_tmap(&tAl);
    prefetch_tmap(&tBh);
    prefetch_tmap(&tBl);
  }
  if (warp == 0) tmem_alloc(tmem_slot, Lay::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int it = 0, last_s = -1;
      uint32_t last_par = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < P.ntiles && ok; t += gridDim.x)
        for (int kb = 0; kb < P.kblocks; ++kb, ++it) {
          const int s = it % S;
          const uint32_t j = it / S;
          if (!mbar_wait(&empty[s], (j & 1) ^ 1)) {
            report(P.err, ERR_WAIT_PRODUCER);
            ok = false;
            break;
          }
          uint8_t* st = smem + s * Lay::STAGE;
          mbar_arrive_expect_tx(&full[s], Lay::STAGE);
          tma_load_2d(st, &tAh, kb * BK, t * BM, &full[s]);
          tma_load_2d(st + TILE_A_BYTES, &tAl, kb * BK, t * BM, &full[s]);
          tma_load_2d(st + 2 * TILE_A_BYTES, &tBh, kb * BK, 0, &full[s]);
          tma_load_2d(st + 2 * TILE_A_BYTES + Lay::B_BYTES, &tBl, kb * BK, 0, &full[s]);
          last_s = s;
          last_par = j & 1;
        }
      if (last_s >= 0) mbar_wait(&full[last_s], last_par);  // no copy still in flight at exit
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = idesc_bf16_f32(BM, NP);
      int it = 0, gt = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < P.ntiles && ok; t += gridDim.x)
        for (int kg = 0; kg < P.kblocks && ok; kg += G1_GROUP, ++gt) {
          const int b = gt & 1;
          if (!mbar_wait(&tempty[b], ((gt >> 1) & 1) ^ 1)) {
            report(P.err, ERR_WAIT_MMA);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + b * Lay::ACC_STRIDE;
          const int kend = min(kg + G1_GROUP, P.kblocks);
          for (int kb = kg; kb < kend; ++kb, ++it) {
            const int s = it % S;
            const uint32_t j = it / S;
            if (!mbar_wait(&full[s], j & 1)) {
              report(P.err, ERR_WAIT_MMA);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint8_t* st = smem + s * Lay::STAGE;
#pragma unroll
            for (int k = 0; k < BK / 16; ++k) {
              const uint64_t ah = sdesc_kmajor_sw128(st + k * 32);
              const uint64_t al = sdesc_kmajor_sw128(st + TILE_A_BYTES + k * 32);
              const uint64_t bh = sdesc_kmajor_sw128(st + 2 * TILE_A_BYTES + k * 32);
              const uint64_t bl = sdesc_kmajor_sw128(st + 2 * TILE_A_BYTES + Lay::B_BYTES + k * 32);
              umma_bf16(d, ah, bh, idesc, (kb > kg || k > 0) ? 1u : 0u);
              umma_bf16(d, ah, bl, idesc, 1u);
              umma_bf16(d, al, bh, idesc, 1u);
            }
            umma_commit(&empty[s]);
          }
          if (ok) umma_commit(&tfull[b]);
        }
      umma_commit(drain);  // every issued MMA has finished before TMEM is freed
      mbar_wait(drain, 0);
    }
  } else {  // epilogue: warp w drains TMEM lanes 32*(w%4).. and part (w-2)/4 of the 16-column chunks
    const int q = warp & 3, part = (warp - 2) >> 2;
    constexpr int NCH = NP / 16;
    constexpr int CH1 = (NCH + G1_EPI - 1) / G1_EPI, CH2 = (2 * NCH + G1_EPI - 1) / G1_EPI;
    const int ngroups = (P.kblocks + G1_GROUP - 1) / G1_GROUP;
    const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16);
    int gt = 0;
    for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
      const int m = t * BM + 32 * q + lane;
      static_assert(G1_EPI == 3, "chunk split below is written for three parts");
      bool ok;
      if (part == 0)
        ok = g1_epilogue_tile<NP, 0, CH1>(tbase, gt, ngroups, m, P, tfull, tempty, lane);
      else if (part == 1)
        ok = g1_epilogue_tile<NP, CH1, CH2>(tbase, gt, ngroups, m, P, tfull, tempty, lane);
      else
        ok = g1_epilogue_tile<NP, CH2, NCH>(tbase, gt, ngroups, m, P, tfull, tempty, lane);
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
    tmem_dealloc(tmem, Lay::TMEM_COLS);
  }
}

// ---------------------------------------------------------------- GEMM2
// K = X X^T over blocks of 128 rows x 256 columns of the lower triangle (row
// tile tx, column tiles 2cp and 2cp+1 <= tx + 1): each k block loads 128 rows
// of A and 256 rows of B, 4/3 the flops per loaded byte of square 128 x 128
// tiles.  Blocks whose second column tile lies above the diagonal (or past the
// last row) run N = 128.
struct G2Params {
  int n;
  int kblocks;      // (naux*NP)/64
  int ntile_n;      // ceil(n/128)
  int nblocks;      // lower-triangle 128 x 256 blocks
  int splits;
  double* Kt;       // n x n, Kt[y*n + x] = K[x][y] for tile(x) >= tile(y); FP64 so
                    // the split-K sum does not depend on the atomics' order
  int* err;
};

constexpr int G2_BN = 256;
constexpr int G2_STAGE = 6 * TILE_A_BYTES;           // A hi, lo (128 rows) + B hi, lo (256 rows)
constexpr int G2_STAGES = 2;
constexpr int G2_SMEM = G2_STAGES * G2_STAGE + 1024 + 1024;
constexpr int G2_EPI = 2;                            // epilogue warps per TMEM lane quadrant
constexpr int G2_THREADS = 64 + 4 * 32 * G2_EPI;     // TMA warp, MMA warp, epilogue warps
constexpr int G2_COLS = G2_BN / G2_EPI;              // accumulator columns per epilogue warp
static_assert(G2_SMEM <= SMEM_LIMIT, "GEMM2 ring exceeds shared memory");

__host__ __device__ inline int g2_block_count(int nt) {
  int c = 0;
  for (int tx = 0; tx < nt; ++tx) c += tx / 2 + 1;
  return c;
}
__device__ inline void g2_block(int b, int nt, int& tx, int& cp) {
  tx = 0;
  for (; tx < nt; ++tx) {
    const int c = tx / 2 + 1;
    if (b < c) break;
    b -= c;
  }
  cp = b;
}

// Accumulation groups of ACC_GROUP k-blocks go to alternating TMEM buffers of
// 256 columns; the epilogue adds each group's FP32 partial to FP32 totals in
// registers (round-to-nearest) and adds the totals to Kt once at the end.
__global__ void __launch_bounds__(G2_THREADS, 1)
    k_gemm2(const __grid_constant__ CUtensorMap tXh, const __grid_constant__ CUtensorMap tXl, const G2Params P) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + G2_STAGES * G2_STAGE);
  uint64_t* empty = full + G2_STAGES;
  uint64_t* tfull = empty + G2_STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // which block of the lower triangle and which slice of the inner index
  const int blk = blockIdx.x % P.nblocks, split = blockIdx.x / P.nblocks;
  int tx, cp;
  g2_block(blk, P.ntile_n, tx, cp);
  // the second column tile is used when it lies on or below the diagonal
  const bool wide = 2 * cp + 1 <= tx;
  const int kb0 = (int)((long long)P.kblocks * split / P.splits);
  const int kb1 = (int)((long long)P.kblocks * (split + 1) / P.splits);

  if (threadIdx.x == 0) {
    for (int s = 0; s < G2_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4 * G2_EPI);
    }
    mbar_init(drain, 1);
    fence_barrier_init();
    prefetch_tmap(&tXh);
    prefetch_tmap(&tXl);
  }
  if (warp == 0) tmem_alloc(tmem_slot, 2 * G2_BN);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const bool have_work = kb1 > kb0;

  if (warp == 0) {
    if (lane == 0 && have_work) {
      int last_s = -1;
      uint32_t last_par = 0;
      const uint32_t bytes = wide ? G2_STAGE : 4 * TILE_A_BYTES;
      for (int kb = kb0, it = 0; kb < kb1; ++kb, ++it) {
        const int s = it % G2_STAGES;
        const uint32_t j = it / G2_STAGES;
        if (!mbar_wait(&empty[s], (j & 1) ^ 1)) {
          report(P.err, ERR_WAIT_PRODUCER);
          break;
        }
        uint8_t* st = smem + s * G2_STAGE;
        mbar_arrive_expect_tx(&full[s], bytes);
        tma_load_2d(st, &tXh, kb * BK, tx * BM, &full[s]);
        tma_load_2d(st + TILE_A_BYTES, &tXl, kb * BK, tx * BM, &full[s]);
        // B: 256 (or 128) rows from column tile 2cp, hi then lo
        tma_load_2d(st + 2 * TILE_A_BYTES, &tXh, kb * BK, 2 * cp * BM, &full[s]);
        tma_load_2d(st + 4 * TILE_A_BYTES, &tXl, kb * BK, 2 * cp * BM, &full[s]);
        if (wide) {
          tma_load_2d(st + 3 * TILE_A_BYTES, &tXh, kb * BK, (2 * cp + 1) * BM, &full[s]);
          tma_load_2d(st + 5 * TILE_A_BYTES, &tXl, kb * BK, (2 * cp + 1) * BM, &full[s]);
        }
        last_s = s;
        last_par = j & 1;
      }
      if (last_s >= 0) mbar_wait(&full[last_s], last_par);
    }
  } else if (warp == 1) {
    if (lane == 0 && have_work) {
      const uint32_t idesc = wide ? idesc_bf16_f32(BM, G2_BN) : idesc_bf16_f32(BM, BM);
      bool ok = true;
      int it = 0, gt = 0;
      for (int kg = kb0; kg < kb1 && ok; kg += ACC_GROUP, ++gt) {
        const int b = gt & 1;
        if (!mbar_wait(&tempty[b], ((gt >> 1) & 1) ^ 1)) {
          report(P.err, ERR_WAIT_MMA);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + b * G2_BN;
        const int kend = min(kg + ACC_GROUP, kb1);
        for (int kb = kg; kb < kend; ++kb, ++it) {
          const int s = it % G2_STAGES;
          const uint32_t j = it / G2_STAGES;
          if (!mbar_wait(&full[s], j & 1)) {
            report(P.err, ERR_WAIT_MMA);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint8_t* st = smem + s * G2_STAGE;
#pragma unroll
          for (int k = 0; k < BK / 16; ++k) {
            const uint64_t ah = sdesc_kmajor_sw128(st + k * 32);
            const uint64_t al = sdesc_kmajor_sw128(st + TILE_A_BYTES + k * 32);
            const uint64_t bh = sdesc_kmajor_sw128(st + 2 * TILE_A_BYTES + k * 32);
            const uint64_t bl = sdesc_kmajor_sw128(st + 4 * TILE_A_BYTES + k * 32);
            umma_bf16(d, ah, bh, idesc, (kb > kg || k > 0) ? 1u : 0u);
            umma_bf16(d, ah, bl, idesc, 1u);
            umma_bf16(d, al, bh, idesc, 1u);
          }
          umma_commit(&empty[s]);
        }
        if (ok) umma_commit(&tfull[b]);
      }
      umma_commit(drain);
      mbar_wait(drain, 0);
    }
  } else if (have_work) {  // warp w: TMEM lanes 32*(w%4).., columns [G2_COLS*part, +G2_COLS)
    const int q = warp & 3, part = (warp - 2) >> 2;
    const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + part * G2_COLS;
    float acc[G2_COLS];
#pragma unroll
    for (int e = 0; e < G2_COLS; ++e) acc[e] = 0.0f;
    bool ok = true;
    for (int kg = kb0, gt = 0; kg < kb1; kg += ACC_GROUP, ++gt) {
      const int b = gt & 1;
      if (!mbar_wait(&tfull[b], (gt >> 1) & 1)) {
        report(P.err, ERR_WAIT_EPILOGUE);
        ok = false;
        break;
      }
      tc_fence_after();
      if (part == 0 || wide) {
#pragma unroll
        for (int c = 0; c < G2_COLS / 16; ++c) {
          float v[16];
          tmem_ld16(tbase + b * G2_BN + c * 16, v);
          tmem_ld_wait();
#pragma unroll
          for (int e = 0; e < 16; ++e) acc[c * 16 + e] += v[e];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
    }
    const int x = tx * BM + 32 * q + lane;
    if (ok && x < P.n && (part == 0 || wide)) {
#pragma unroll
      for (int e = 0; e < G2_COLS; ++e) {
        const int y = 2 * cp * BM + part * G2_COLS + e;
        if (y < P.n) atomicAdd(P.Kt + (size_t)y * P.n + x, (double)acc[e]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * G2_BN);
  }
}

// ---------------------------------------------------------------- small kernels
// B64[x][K][y] (ld n) -> Bhi/Blo[x][K][y] (ld ldb, zero padded)
__global__ void k_split_B(size_t rows, int n, int ldb, const double* __restrict__ B, __nv_bfloat16* __restrict__ Bh,
                          __nv_bfloat16* __restrict__ Bl) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * ldb) return;
  const size_t r = i / ldb;
  const int y = (int)(i % ldb);
  const float f = y < n ? (float)B[r * n + y] : 0.0f;
  const double dv = y < n ? B[r * n + y] : 0.0;
  const __nv_bfloat16 h = __float2bfloat16_rn(f);
  Bh[i] = h;
  Bl[i] = __float2bfloat16_rn((float)(dv - (double)__bfloat162float(h)));
}

// C (n x nocc col-major FP64) -> ChiT/CloT[i][y] (NP x ldb, zero padded)
__global__ void k_split_C(int n, int nocc, int NP, int ldb, const double* __restrict__ C, __nv_bfloat16* Ch,
                          __nv_bfloat16* Cl) {
  const int i = blockIdx.y, y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= ldb) return;
  const double dv = (i < nocc && y < n) ? C[(size_t)i * n + y] : 0.0;
  const __nv_bfloat16 h = __float2bfloat16_rn((float)dv);
  Ch[(size_t)i * ldb + y] = h;
  Cl[(size_t)i * ldb + y] = __float2bfloat16_rn((float)(dv - (double)__bfloat162float(h)));
}

// J[x][y] += sum_{K in [K0, K1)} gamma_K (Bhi + Blo)[x][K][y] for y <= x.
// One block per (x, K range): the ny = ceil((x+1)/8) threads of a K group
// read 8 consecutive y each (16-byte loads of one row of B), and the block's
// remaining threads form further K groups, so short rows (small x) still keep
// the whole block busy.  Partial sums meet in shared memory; one atomic per
// (x, y) per block.
constexpr int JM_THREADS = 256;
__global__ void __launch_bounds__(JM_THREADS) k_J_mixed(int n, int naux, int ldb, int kchunk,
                                                        const __nv_bfloat16* __restrict__ Bh,
                                                        const __nv_bfloat16* __restrict__ Bl,
                                                        const double* __restrict__ gamma, double* __restrict__ J) {
  __shared__ float part[JM_THREADS * 8];
  const int x = blockIdx.x;
  const int ny_all = (x + 8) / 8;                  // y groups of 8 covering 0..x
  const int K0 = blockIdx.y * kchunk, K1 = min(naux, K0 + kchunk);
  const int t = threadIdx.x;
  for (int yb = 0; yb < ny_all; yb += JM_THREADS) {   // one pass unless x >= 8 * JM_THREADS
    const int ny = min(ny_all - yb, JM_THREADS);
    const int ngroups = JM_THREADS / ny;               // K groups
    const int yi = t % ny, kg = t / ny;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (kg < ngroups) {
      const size_t base = (size_t)x * naux * ldb + (size_t)(yb + yi) * 8;
#pragma unroll 4
      for (int K = K0 + kg; K < K1; K += ngroups) {
        const float g = (float)__ldg(gamma + K);
        const uint4 hv = __ldg(reinterpret_cast<const uint4*>(Bh + base + (size_t)K * ldb));
        const uint4 lv = __ldg(reinterpret_cast<const uint4*>(Bl + base + (size_t)K * ldb));
        const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&hv);
        const __nv_bfloat16* l = reinterpret_cast<const __nv_bfloat16*>(&lv);
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[e] += g * (__bfloat162float(h[e]) + __bfloat162float(l[e]));
      }
    }
    __syncthreads();  // the previous pass's readers are done with part[]
#pragma unroll
    for (int e = 0; e < 8; ++e) part[t * 8 + e] = acc[e];
    __syncthreads();
    // the first ny*8 threads each sum the K groups of one y = 8 (yb + yy) + e
    for (int idx = t; idx < ny * 8; idx += JM_THREADS) {
      const int yy = idx / 8, e = idx % 8, y = (yb + yy) * 8 + e;
      if (y > x || y >= n) continue;
      float sum = 0.0f;
      for (int k = 0; k < ngroups; ++k) sum += part[(k * ny + yy) * 8 + e];
      atomicAdd(J + (size_t)y * n + x, (double)sum);
    }
  }
}

// J: mirror the lower triangle; K: assemble from the lower-triangle tiles of Kt
__global__ void k_finalize_mixed(int n, const double* __restrict__ Kt, double* __restrict__ J, double* __restrict__ K) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n * n) return;
  const int i = (int)(idx % n), j = (int)(idx / n);  // element (i, j), column-major
  const int ti = i / BM, tj = j / BM;
  K[idx] = (ti >= tj) ? Kt[(size_t)j * n + i] : Kt[(size_t)i * n + j];
  if (i < j) J[idx] = J[(size_t)i * n + j];
}
__global__ void k_zero_upper(int n, double* J) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n * n) return;
  if ((int)(idx % n) < (int)(idx / n)) J[idx] = 0.0;
}

// ---------------------------------------------------------------- host
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 2-D BF16 tensor map: inner extent `cols` (contiguous), `rows`, box box_cols x box_rows, 128B swizzle.
bool make_map(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint32_t box_cols,
                     uint32_t box_rows) {
  auto enc = get_encode();
  if (!enc) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NP>
static cudaError_t launch_g1(const CUtensorMap* m, const G1Params& P, int grid, cudaStream_t s) {
  using Lay = G1Layout<NP>;
  cudaError_t st = cudaFuncSetAttribute(k_gemm1<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::SMEM);
  if (st != cudaSuccess) return st;
  k_gemm1<NP><<<grid, G1_THREADS, Lay::SMEM, s>>>(m[0], m[1], m[2], m[3], P);
  return cudaGetLastError();
}

static cudaError_t dispatch_g1(int NP, const CUtensorMap* m, const G1Params& P, int grid, cudaStream_t s) {
  switch (NP) {
#define CASE(v) \
  case v:       \
    return launch_g1<v>(m, P, grid, s);
    CASE(16) CASE(32) CASE(48) CASE(64) CASE(80) CASE(96) CASE(112) CASE(128)
    CASE(144) CASE(160) CASE(176) CASE(192) CASE(208) CASE(224) CASE(240) CASE(256)
#undef CASE
    default:
      return cudaErrorInvalidValue;
  }
}

int df_mixed_prepare(jk_engine* e, int nocc) {
  DFState& d = e->df;
  MixedState& m = e->mixed;
  const int n = e->obs.n_final, naux = d.naux;
  const int NP = ((nocc + 15) / 16) * 16;
  if (NP > 256) return set_error(e, JK_ERR_ARG, "mixed DF: nocc above 256 is not supported");
  const int ldb = ((n + BK - 1) / BK) * BK;
  cudaStream_t s = e->stream;
  cudaError_t st = cudaSuccess;
  if (!m.ready || m.ldb != ldb) {
    const size_t rows = (size_t)n * naux;
    st = m.Bh.alloc(rows * ldb);
    if (st == cudaSuccess) st = m.Bl.alloc(rows * ldb);
    if (st != cudaSuccess) return check_cuda(e, st, "mixed B allocation");
    const size_t tot = rows * ldb;
    k_split_B<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(rows, n, ldb, d.B64.p, m.Bh.p, m.Bl.p);
    st = cudaGetLastError();
    if (st != cudaSuccess) return check_cuda(e, st, "split B");
    m.ldb = ldb;
    m.NP = 0;
    m.NP_cap = 0;
    m.ready = true;
  }
  if (m.NP != NP) {
    // scratch sized for the largest occupied count so far; smaller counts
    // reuse it with tensor maps for their own row length
    if (NP > m.NP_cap) {
      st = m.Ch.alloc((size_t)NP * ldb);
      if (st == cudaSuccess) st = m.Cx.alloc((size_t)n * NP);
      if (st == cudaSuccess) st = m.Cl.alloc((size_t)NP * ldb);
      if (st == cudaSuccess) st = m.Xh.alloc((size_t)n * naux * NP);
      if (st == cudaSuccess) st = m.Xl.alloc((size_t)n * naux * NP);
      if (st == cudaSuccess) st = m.Kt.alloc((size_t)n * n);
      if (st == cudaSuccess) st = m.err.alloc(1);
      if (st == cudaSuccess) st = d.gamma.alloc(naux);
      if (st != cudaSuccess) return check_cuda(e, st, "mixed scratch allocation");
      cudaMemsetAsync(m.err.p, 0, sizeof(int), s);
      m.NP_cap = NP;
    }
    bool ok = make_map(&m.maps[0], m.Bh.p, ldb, (uint64_t)n * naux, BK, BM) &&
              make_map(&m.maps[1], m.Bl.p, ldb, (uint64_t)n * naux, BK, BM) &&
              make_map(&m.maps[2], m.Ch.p, ldb, NP, BK, NP) && make_map(&m.maps[3], m.Cl.p, ldb, NP, BK, NP) &&
              make_map(&m.maps[4], m.Xh.p, (uint64_t)naux * NP, n, BK, BM) &&
              make_map(&m.maps[5], m.Xl.p, (uint64_t)naux * NP, n, BK, BM);
    if (!ok) return set_error(e, JK_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    m.NP = NP;
  }
  return JK_OK;
}

int df_mixed_device(jk_engine* e, const double* dC, int nocc, double* dJ, double* dK, cudaStream_t s) {
  int rc = df_mixed_prepare(e, nocc);
  if (rc) return rc;
  DFState& d = e->df;
  MixedState& m = e->mixed;
  const int n = e->obs.n_final, naux = d.naux, NP = m.NP, ldb = m.ldb;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device);
  stage_mark(e, 0, s);
  k_split_C<<<dim3((ldb + 127) / 128, NP), 128, 0, s>>>(n, nocc, NP, ldb, dC, m.Ch.p, m.Cl.p);
  launch_rows_C(n, nocc, NP, n, dC, m.Cx.p, s);
  cudaMemsetAsync(d.gamma.p, 0, sizeof(double) * naux, s);
  cudaMemsetAsync(m.Kt.p, 0, sizeof(double) * n * n, s);
  cudaMemsetAsync(dJ, 0, sizeof(double) * n * n, s);
  G1Params P1{};
  P1.M = n * naux;
  P1.kblocks = ldb / BK;
  P1.nocc = nocc;
  P1.n = n;
  P1.naux = naux;
  P1.ntiles = (P1.M + BM - 1) / BM;
  P1.Cx = m.Cx.p;
  P1.Xhi = m.Xh.p;
  P1.Xlo = m.Xl.p;
  P1.gamma = d.gamma.p;
  P1.Kt = m.Kt.p;
  P1.err = m.err.p;
  cudaError_t st = dispatch_g1(NP, m.maps, P1, std::min(nsm, P1.ntiles), s);
  if (st != cudaSuccess) return check_cuda(e, st, "gemm1 launch");
  stage_mark(e, 1, s);
  st = launch_gemm2(m.maps[4], m.maps[5], n, (naux * NP) / BK, m.Kt.p, m.err.p, nsm, s);
  if (st != cudaSuccess) return check_cuda(e, st, "gemm2 launch");
  stage_mark(e, 2, s);
  const int kchunk = (naux + 15) / 16;   // 16 K ranges per row x
  k_J_mixed<<<dim3(n, (naux + kchunk - 1) / kchunk), JM_THREADS, 0, s>>>(n, naux, ldb, kchunk, m.Bh.p, m.Bl.p,
                                                                         d.gamma.p, dJ);
  stage_mark(e, 3, s);
  const size_t nn = (size_t)n * n;
  k_finalize_mixed<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(n, m.Kt.p, dJ, dK);
  stage_mark(e, 4, s);
  return check_cuda(e, cudaGetLastError(), "mixed DF launch");
}

// The bounded wait of the tensor-core kernels on a barrier that nothing
// completes (status[0]: 1 if it gave up) and on one that completes (status[1]:
// 1 if it gave up), with `limit` polls.
__global__ void k_wait_selftest(uint32_t limit, int* status) {
  __shared__ __align__(8) uint64_t bar[2];
  if (threadIdx.x != 0) return;
  mbar_init(&bar[0], 1);
  mbar_init(&bar[1], 1);
  fence_barrier_init();
  mbar_arrive(&bar[1]);
  status[0] = mbar_wait_n(&bar[0], 0, limit) ? 0 : 1;
  status[1] = mbar_wait_n(&bar[1], 0, limit) ? 0 : 1;
}

int df_mixed_error(jk_engine* e) {
  if (e->tiled.ready) return df_tiled_error(e);
  if (!e->mixed.err.p) return JK_OK;
  int h = 0;
  cudaError_t st = cudaMemcpyAsync(&h, e->mixed.err.p, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "mixed DF error word");
  if (h) {
    cudaMemsetAsync(e->mixed.err.p, 0, sizeof(int), e->stream);
    return set_error(e, JK_ERR_CUDA, "mixed DF: tensor-core pipeline wait timed out (stage " + std::to_string(h) + ")");
  }
  return JK_OK;
}

// ---------------------------------------------------------------- shared with the tiled path
__global__ void k_rows_C(int n, int nocc, int NP, int nrow, const double* __restrict__ C, float* __restrict__ Cx) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)nrow * NP) return;
  const int x = (int)(idx / NP), i = (int)(idx % NP);
  Cx[idx] = (x < n && i < nocc) ? (float)C[x + (size_t)i * n] : 0.0f;
}

cudaError_t launch_rows_C(int n, int nocc, int NP, int nrow, const double* C, float* Cx, cudaStream_t s) {
  const size_t tot = (size_t)nrow * NP;
  k_rows_C<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n, nocc, NP, nrow, C, Cx);
  return cudaGetLastError();
}

cudaError_t launch_split_C(int n, int nocc, int NP, int ld, const double* C, __nv_bfloat16* Ch, __nv_bfloat16* Cl,
                           cudaStream_t s) {
  k_split_C<<<dim3((ld + 127) / 128, NP), 128, 0, s>>>(n, nocc, NP, ld, C, Ch, Cl);
  return cudaGetLastError();
}

// Kt (+)= X X^T over the lower-triangle 128 x 256 blocks of the n rows of X
// (tensor maps tXh, tXl over rows of `kblocks` * 64 BF16, boxes of 64 x 128),
// split-K over the SMs.
cudaError_t launch_gemm2(const CUtensorMap& tXh, const CUtensorMap& tXl, int n, int kblocks, double* Kt, int* err,
                         int nsm, cudaStream_t s) {
  G2Params P2{};
  P2.n = n;
  P2.kblocks = kblocks;
  P2.ntile_n = (n + BM - 1) / BM;
  P2.nblocks = g2_block_count(P2.ntile_n);
  // splits so that the CTA count is close to a whole number of waves
  int best = 1;
  double best_eff = 0.0;
  for (int sp = 1; sp <= 64 && sp <= kblocks; ++sp) {
    const int ctas = P2.nblocks * sp;
    const double waves = std::ceil((double)ctas / nsm);
    const double eff = (double)ctas / (waves * nsm);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = sp;
    }
    if (eff > 0.97) break;
  }
  P2.splits = best;
  P2.Kt = Kt;
  P2.err = err;
  cudaError_t st = cudaFuncSetAttribute(k_gemm2, cudaFuncAttributeMaxDynamicSharedMemorySize, G2_SMEM);
  if (st != cudaSuccess) return st;
  k_gemm2<<<P2.nblocks * P2.splits, G2_THREADS, G2_SMEM, s>>>(tXh, tXl, P2);
  return cudaGetLastError();
}

cudaError_t launch_finalize_mixed(int n, const double* Kt, double* J, double* K, cudaStream_t s) {
  const size_t nn = (size_t)n * n;
  k_finalize_mixed<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(n, Kt, J, K);
  return cudaGetLastError();
}

}  // namespace m2

using namespace m2;

extern "C" int jk_wait_selftest(jk_engine* e, unsigned polls, int* timed_out, int* completed_timed_out) {
  if (!e || !timed_out || !completed_timed_out || polls == 0) return JK_ERR_ARG;
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != e->device)
    return set_error(e, JK_ERR_ARG, "jk_wait_selftest: the engine's device must be current");
  DevBuf<int> st;
  cudaError_t r = st.alloc(2);
  if (r == cudaSuccess) r = cudaMemsetAsync(st.p, 0xff, 2 * sizeof(int), e->stream);
  if (r != cudaSuccess) return check_cuda(e, r, "jk_wait_selftest");
  k_wait_selftest<<<1, 32, 0, e->stream>>>(polls, st.p);
  int h[2] = {-1, -1};
  r = cudaGetLastError();
  if (r == cudaSuccess) r = cudaMemcpyAsync(h, st.p, sizeof(h), cudaMemcpyDeviceToHost, e->stream);
  if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
  if (r != cudaSuccess) return check_cuda(e, r, "jk_wait_selftest");
  *timed_out = h[0];
  *completed_timed_out = h[1];
  return JK_OK;
}
