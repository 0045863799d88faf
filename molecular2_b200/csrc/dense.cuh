// FP64 dense linear algebra on the FP64 pipe (sm_100a): a strided, batched
// GEMM with triangular-operand and lower-output variants and split-K, and the
// blocked Cholesky factorisation and triangular inverse built on it.  These
// are the contractions of the FP64 density-fitted build (molecular2
// src/fockbuild.cpp:602-659: the metric factorisation V = L L^T, B = T L^-T,
// X = B C, K = X X^T) and of the DF gradient algebra.
#pragma once
#include <cuda_runtime.h>

#include "engine.h"

namespace m2 {

// C(m, n) = alpha * sum_k A(m, k) B(k, n) + beta * C(m, n), for `batch`
// independent problems.  Element (m, k) of A sits at A[m*sam + k*sak +
// b*bsa], and likewise for B and C, so any transpose or row/column-major
// layout is a choice of strides.
struct DGemm {
  int M = 0, N = 0, K = 0, batch = 1;
  const double* A = nullptr;
  long long sam = 0, sak = 0, bsa = 0;
  const double* B = nullptr;
  long long sbk = 0, sbn = 0, bsb = 0;
  double* C = nullptr;
  long long scm = 0, scn = 0, bsc = 0;
  double alpha = 1.0, beta = 0.0;
  bool a_lower = false;  // A(m, k) = 0 for k > m: the k loop of a row tile stops at its last row
  bool b_lower = false;  // B(k, n) = 0 for k < n: the k loop of a column tile starts at its first column
  bool c_lower = false;  // only tiles on or below the diagonal (tile_n <= tile_m) are computed
  int ksplit = 1;        // > 1: the k range is split over blocks whose sums are added atomically
};

// Launch on stream s.  Returns the launch status.
cudaError_t dgemm(const DGemm& g, cudaStream_t s);

// Blocked Cholesky V = L L^T of the n x n column-major matrix A (ld = n), in
// place: the lower triangle becomes L, the strict upper triangle is zeroed.
// work: n * 64 doubles; info: one int on the device, set to 1 + the index of
// the first non-positive pivot (0 when positive definite).
int cholesky(jk_engine* e, double* A, int n, double* work, int* info, cudaStream_t s);

// Inverse of the lower-triangular n x n column-major L (ld = n) into Linv
// (ld = n, strict upper triangle zero).  work: n * n doubles.
int tri_inverse(jk_engine* e, const double* L, double* Linv, int n, double* work, cudaStream_t s);

// C (column-major, ld = n): copy the lower triangle into the upper one.
void mirror_lower(double* C, int n, cudaStream_t s);

}  // namespace m2
