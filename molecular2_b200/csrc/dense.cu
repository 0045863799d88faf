// FP64 GEMM, blocked Cholesky and triangular inverse (dense.cuh).
//
// GEMM: 128 x 128 output tiles, 256 threads = 8 warps in a 2 x 4 grid, each
// warp a 64 x 32 block of 8 x 4 FP64 tensor-core tiles (mma.sync m8n8k4,
// the DMMA path), k tiles of 16 staged through a two-buffer shared-memory
// ring by cp.async (8-byte copies, so any stride works; the thread-to-element
// map follows whichever operand dimension is contiguous so the copies
// coalesce).  Out-of-range elements are copied as zeros (cp.async with
// source size 0).  The shared-memory pitches (136 doubles for [k][m], 20 for
// [m][k] tiles) put the 32 lanes of a fragment load (4 k x 8 consecutive m)
// and of a copy into the fewest bank wavefronts.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "dense.cuh"

namespace m2 {
namespace {

constexpr int GBM = 128, GBN = 128, GBK = 16, GT = 256;
constexpr int LDS = GBM + 8;   // [k][m] rows (doubles): 1088 B, 16-byte aligned, conflict-free fragments
constexpr int LDK = GBK + 4;   // [m][k] rows (doubles): 160 B, so 4 rows of 4 k fill the 32 banks once
constexpr int OPER = (GBK * LDS > GBM * LDK) ? GBK * LDS : GBM * LDK;  // doubles per operand buffer
constexpr int GSMEM = 4 * OPER * (int)sizeof(double);                  // A and B, two buffers each

__device__ __forceinline__ void cp8(double* dst, const double* src, bool ok) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
// D = A B + D for one 8 x 8 x 4 FP64 tile: a = A(lane/4, lane%4),
// b = B(lane%4, lane/4), d = D(lane/4, 2*(lane%4) + {0, 1}).
__device__ __forceinline__ void dmma(double* d, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ void tri_tile(int t, int& tm, int& tn) {
  int m = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (m * (m + 1) / 2 > t) --m;
  while ((m + 1) * (m + 2) / 2 <= t) ++m;
  tm = m;
  tn = t - m * (m + 1) / 2;
}

// Operand tiles in shared memory follow the operand's contiguous dimension in
// global memory: an operand whose k is contiguous (AK1 for A, !BN1 for B) is
// kept as [m][k] (pitch LDK), the other as [k][m] (pitch LDS), so that the
// 8-byte copies of a warp land in distinct banks.
template <bool AK1, bool BN1>
__global__ void __launch_bounds__(GT) k_dgemm(const DGemm g, int tiles_n) {
  extern __shared__ __align__(16) double gsm[];
  double* As = gsm;             // two buffers of OPER doubles
  double* Bs = gsm + 2 * OPER;
  auto aidx = [](int buf, int k, int m) { return buf * OPER + (AK1 ? m * LDK + k : k * LDS + m); };
  auto bidx = [](int buf, int k, int n) { return buf * OPER + (BN1 ? k * LDS + n : n * LDK + k); };
  int tm, tn;
  if (g.c_lower)
    tri_tile(blockIdx.x, tm, tn);
  else {
    tm = blockIdx.x / tiles_n;
    tn = blockIdx.x % tiles_n;
  }
  const int m0 = tm * GBM, n0 = tn * GBN;
  const long long bz = blockIdx.z;
  const double* A = g.A + bz * g.bsa;
  const double* B = g.B + bz * g.bsb;
  double* C = g.C + bz * g.bsc;
  int kb = 0, ke = g.K;
  if (g.a_lower) ke = min(ke, m0 + GBM);
  if (g.b_lower) kb = min(ke, n0);
  kb = (kb / GBK) * GBK;
  if (g.ksplit > 1) {
    const int len = max(0, ke - kb);
    const int chunk = ((len + g.ksplit - 1) / g.ksplit + GBK - 1) / GBK * GBK;
    const int s0 = kb + (int)blockIdx.y * chunk;
    const int s1 = min(ke, s0 + chunk);
    if (s0 >= s1) return;
    kb = s0;
    ke = s1;
  }
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, wm = warp >> 2, wn = warp & 3;

  auto load = [&](int buf, int k0) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      int m, k;
      if (AK1) {
        k = t & 15;
        m = (t >> 4) + 16 * r;
      } else {
        m = t & 127;
        k = (t >> 7) + 2 * r;
      }
      const int gm = m0 + m, gk = k0 + k;
      const bool ok = gm < g.M && gk < ke;
      cp8(As + aidx(buf, k, m), ok ? A + (long long)gm * g.sam + (long long)gk * g.sak : A, ok);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      int n, k;
      if (BN1) {
        n = t & 127;
        k = (t >> 7) + 2 * r;
      } else {
        k = t & 15;
        n = (t >> 4) + 16 * r;
      }
      const int gn = n0 + n, gk = k0 + k;
      const bool ok = gn < g.N && gk < ke;
      cp8(Bs + bidx(buf, k, n), ok ? B + (long long)gk * g.sbk + (long long)gn * g.sbn : B, ok);
    }
  };

  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int nk = ke > kb ? (ke - kb + GBK - 1) / GBK : 0;
  if (nk > 0) load(0, kb);
  cp_commit();
  const int fk = lane & 3, fr = lane >> 2;
  for (int it = 0; it < nk; ++it) {
    if (it + 1 < nk) load((it + 1) & 1, kb + (it + 1) * GBK);
    cp_commit();
    cp_wait1();
    __syncthreads();
    const int buf = it & 1;
#pragma unroll
    for (int k4 = 0; k4 < GBK; k4 += 4) {
      double a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = As[aidx(buf, k4 + fk, wm * 64 + i * 8 + fr)];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[bidx(buf, k4 + fk, wn * 32 + j * 8 + fr)];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gm = m0 + wm * 64 + i * 8 + fr;
    if (gm >= g.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gn = n0 + wn * 32 + j * 8 + 2 * fk + h;
        if (gn >= g.N) continue;
        double* c = C + (long long)gm * g.scm + (long long)gn * g.scn;
        if (g.ksplit > 1)
          atomicAdd(c, g.alpha * acc[i][j][h]);
        else
          *c = g.beta == 0.0 ? g.alpha * acc[i][j][h] : g.alpha * acc[i][j][h] + g.beta * *c;
      }
  }
}

__global__ void k_scale(double* C, int M, int N, long long scm, long long scn, long long bsc, double beta) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)M * N) return;
  const int m = (int)(idx % M), n = (int)(idx / M);
  double* c = C + (long long)blockIdx.y * bsc + (long long)m * scm + (long long)n * scn;
  *c = beta == 0.0 ? 0.0 : beta * *c;
}

// ---------------------------------------------------------------- Cholesky
constexpr int CNB = 64;  // panel width

// Factor the b x b diagonal block at (j, j) in place (lower triangle; the
// strict upper part of the block is zeroed) and write its inverse to Dinv
// (CNB x CNB, column-major, ld CNB).  A non-positive pivot sets *info to 1 +
// its index (first one wins) and the block continues with a unit pivot so
// that every later value stays finite.
__global__ void __launch_bounds__(256) k_potrf_diag(double* A, int n, int j, double* Dinv, int* info) {
  extern __shared__ double psm[];
  double(*S)[CNB + 1] = reinterpret_cast<double(*)[CNB + 1]>(psm);
  double(*I)[CNB + 1] = reinterpret_cast<double(*)[CNB + 1]>(psm + CNB * (CNB + 1));
  const int b = min(CNB, n - j);
  const int t = threadIdx.x;
  for (int idx = t; idx < b * b; idx += blockDim.x) {
    const int r = idx % b, c = idx / b;
    S[r][c] = A[(size_t)(j + c) * n + j + r];
  }
  __syncthreads();
  for (int c = 0; c < b; ++c) {
    if (t == 0) {
      double d = S[c][c];
      if (!(d > 0.0)) {
        atomicCAS(info, 0, 1 + j + c);
        d = 1.0;
      }
      S[c][c] = sqrt(d);
    }
    __syncthreads();
    const double inv = 1.0 / S[c][c];
    for (int r = c + 1 + t; r < b; r += blockDim.x) S[r][c] *= inv;
    __syncthreads();
    const int rem = b - c - 1;
    for (int idx = t; idx < rem * rem; idx += blockDim.x) {
      const int r = c + 1 + idx % rem, cc = c + 1 + idx / rem;
      if (cc <= r) S[r][cc] -= S[r][c] * S[cc][c];
    }
    __syncthreads();
  }
  // inverse of the lower-triangular block, one column per thread
  if (t < b) {
    const int col = t;
    for (int r = 0; r < col; ++r) I[r][col] = 0.0;
    I[col][col] = 1.0 / S[col][col];
    for (int r = col + 1; r < b; ++r) {
      double acc = 0.0;
      for (int k = col; k < r; ++k) acc += S[r][k] * I[k][col];
      I[r][col] = -acc / S[r][r];
    }
  }
  __syncthreads();
  for (int idx = t; idx < b * b; idx += blockDim.x) {
    const int r = idx % b, c = idx / b;
    A[(size_t)(j + c) * n + j + r] = r >= c ? S[r][c] : 0.0;
    Dinv[(size_t)c * CNB + r] = r >= c ? I[r][c] : 0.0;
  }
}

__global__ void k_zero_upper(double* A, int n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n * n) return;
  if ((int)(idx % n) < (int)(idx / n)) A[idx] = 0.0;
}

__global__ void k_mirror(double* C, int n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n * n) return;
  const int i = (int)(idx % n), j = (int)(idx / n);
  if (i < j) C[idx] = C[(size_t)i * n + j];
}

// Inverse of each CNB x CNB diagonal block of the lower-triangular L into
// Linv (same positions); one block of threads per diagonal block.
__global__ void __launch_bounds__(CNB) k_trinv_diag(const double* L, double* Linv, int n) {
  __shared__ double S[CNB][CNB + 1];
  const int j = blockIdx.x * CNB, b = min(CNB, n - j), t = threadIdx.x;
  for (int idx = t; idx < b * b; idx += blockDim.x) {
    const int r = idx % b, c = idx / b;
    S[r][c] = L[(size_t)(j + c) * n + j + r];
  }
  __syncthreads();
  if (t < b) {
    const int col = t;
    double x[CNB];
    for (int r = 0; r < b; ++r) x[r] = 0.0;
    x[col] = 1.0 / S[col][col];
    for (int r = col + 1; r < b; ++r) {
      double acc = 0.0;
      for (int k = col; k < r; ++k) acc += S[r][k] * x[k];
      x[r] = -acc / S[r][r];
    }
    for (int r = 0; r < b; ++r) Linv[(size_t)(j + col) * n + j + r] = x[r];
  }
}

}  // namespace

cudaError_t dgemm(const DGemm& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return cudaSuccess;
  if (g.c_lower && g.M != g.N) return cudaErrorInvalidValue;
  if (g.batch > 65535 || g.ksplit < 1 || g.ksplit > 65535) return cudaErrorInvalidValue;
  DGemm h = g;
  if (h.ksplit > 1 && h.beta != 1.0) {
    const long long tot = (long long)h.M * h.N;
    k_scale<<<dim3((unsigned)((tot + 255) / 256), h.batch), 256, 0, s>>>(h.C, h.M, h.N, h.scm, h.scn, h.bsc,
                                                                           h.beta);
    h.beta = 1.0;
  }
  const int tm = (h.M + GBM - 1) / GBM, tn = (h.N + GBN - 1) / GBN;
  const long long tiles = h.c_lower ? (long long)tm * (tm + 1) / 2 : (long long)tm * tn;
  dim3 grid((unsigned)tiles, h.ksplit, h.batch);
  const bool ak1 = h.sak == 1, bn1 = h.sbn == 1;
  auto launch = [&](auto kern) {
    cudaError_t st = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, GSMEM);
    if (st != cudaSuccess) return st;
    kern<<<grid, GT, GSMEM, s>>>(h, tn);
    return cudaGetLastError();
  };
  if (ak1 && bn1) return launch(k_dgemm<true, true>);
  if (ak1) return launch(k_dgemm<true, false>);
  if (bn1) return launch(k_dgemm<false, true>);
  return launch(k_dgemm<false, false>);
}

void mirror_lower(double* C, int n, cudaStream_t s) {
  const size_t nn = (size_t)n * n;
  k_mirror<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(C, n);
}

int cholesky(jk_engine* e, double* A, int n, double* work, int* info, cudaStream_t s) {
  cudaMemsetAsync(info, 0, sizeof(int), s);
  constexpr int PSMEM = 2 * CNB * (CNB + 1) * (int)sizeof(double);
  cudaError_t sa = cudaFuncSetAttribute(k_potrf_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, PSMEM);
  if (sa != cudaSuccess) return check_cuda(e, sa, "cholesky attribute");
  for (int j = 0; j < n; j += CNB) {
    const int b = std::min(CNB, n - j);
    k_potrf_diag<<<1, 256, PSMEM, s>>>(A, n, j, work, info);
    const int R = n - j - b;
    if (R <= 0) break;
    // L21 = A21 L11^-T, in place (each output tile reads only its own rows)
    DGemm p;
    p.M = R;
    p.N = b;
    p.K = b;
    p.A = A + (size_t)j * n + j + b;
    p.sam = 1;
    p.sak = n;
    p.B = work;      // B(k, c) = Dinv(c, k)
    p.sbk = CNB;
    p.sbn = 1;
    p.C = A + (size_t)j * n + j + b;
    p.scm = 1;
    p.scn = n;
    cudaError_t st = dgemm(p, s);
    if (st != cudaSuccess) return check_cuda(e, st, "cholesky panel");
    // A22 -= L21 L21^T on the tiles on or below the diagonal
    DGemm u;
    u.M = R;
    u.N = R;
    u.K = b;
    u.A = A + (size_t)j * n + j + b;
    u.sam = 1;
    u.sak = n;
    u.B = A + (size_t)j * n + j + b;  // B(k, r') = L21(r', k)
    u.sbk = n;
    u.sbn = 1;
    u.C = A + (size_t)(j + b) * n + j + b;
    u.scm = 1;
    u.scn = n;
    u.alpha = -1.0;
    u.beta = 1.0;
    u.c_lower = true;
    st = dgemm(u, s);
    if (st != cudaSuccess) return check_cuda(e, st, "cholesky update");
  }
  const size_t nn = (size_t)n * n;
  k_zero_upper<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(A, n);
  return check_cuda(e, cudaGetLastError(), "cholesky");
}

// Linv[lo:hi, lo:hi] from its diagonal blocks (already inverted):
// Linv21 = -Linv22 L21 Linv11 for a split at `mid`.
static int tri_inverse_rec(jk_engine* e, const double* L, double* Linv, int n, int lo, int hi, double* work,
                           cudaStream_t s) {
  if (hi - lo <= CNB) return JK_OK;
  const int nb = (hi - lo + CNB - 1) / CNB;
  const int mid = lo + ((nb + 1) / 2) * CNB;
  int rc = tri_inverse_rec(e, L, Linv, n, lo, mid, work, s);
  if (!rc) rc = tri_inverse_rec(e, L, Linv, n, mid, hi, work, s);
  if (rc) return rc;
  const int r = hi - mid, c = mid - lo;
  // T (r x c, column-major ld r) = L21 Linv11
  DGemm a;
  a.M = r;
  a.N = c;
  a.K = c;
  a.A = L + (size_t)lo * n + mid;
  a.sam = 1;
  a.sak = n;
  a.B = Linv + (size_t)lo * n + lo;
  a.sbk = 1;
  a.sbn = n;
  a.b_lower = true;
  a.C = work;
  a.scm = 1;
  a.scn = r;
  cudaError_t st = dgemm(a, s);
  if (st != cudaSuccess) return check_cuda(e, st, "triangular inverse");
  DGemm b;
  b.M = r;
  b.N = c;
  b.K = r;
  b.A = Linv + (size_t)mid * n + mid;
  b.sam = 1;
  b.sak = n;
  b.a_lower = true;
  b.B = work;
  b.sbk = 1;
  b.sbn = r;
  b.C = Linv + (size_t)lo * n + mid;
  b.scm = 1;
  b.scn = n;
  b.alpha = -1.0;
  st = dgemm(b, s);
  return check_cuda(e, st, "triangular inverse");
}

int tri_inverse(jk_engine* e, const double* L, double* Linv, int n, double* work, cudaStream_t s) {
  cudaMemsetAsync(Linv, 0, sizeof(double) * (size_t)n * n, s);
  k_trinv_diag<<<(n + CNB - 1) / CNB, CNB, 0, s>>>(L, Linv, n);
  cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) return check_cuda(e, st, "triangular inverse (diagonal blocks)");
  return tri_inverse_rec(e, L, Linv, n, 0, n, work, s);
}

}  // namespace m2
