// RHF SCF driver with every n x n quantity resident in HBM: the caller of the
// J/K engine, restated from molecular2
//   SCF::rhf                        src/scf.cpp:90-185
//   SCF::calcE / calcErr            src/scf.cpp:29-58
//   DIISEngine::compute / solve     src/diis.cpp:22-116
//   Fock::makeFock / addDiis / average / transform / diagonalise / makeDens
//                                   src/fockbuild.cpp:176-222, src/fock.cpp:124-244
// Linear algebra: cuSOLVER syevd (S^-1/2 once, the Fock eigenproblem every
// iteration), cuBLAS GEMM/dot/nrm2; only the <= (maxdiis+1)^2 DIIS system is
// solved on the host (full-pivot LU with its rank, as Eigen::FullPivLU).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"

namespace m2 {

__global__ void k_add_diag(double* A, const double* d, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[(size_t)i * n + i] += d[i];
}
__global__ void k_scale_columns(const double* __restrict__ U, int n, int r, const double* __restrict__ sc,
                                double* __restrict__ out) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < (size_t)n * r) out[idx] = U[idx] * sc[idx / n];
}
static void launch_scale_columns(const double* U, int n, int r, const double* sc, double* out, cudaStream_t s) {
  k_scale_columns<<<(unsigned)(((size_t)n * r + 255) / 256), 256, 0, s>>>(U, n, r, sc, out);
}
static void launch_add_diag(double* A, const double* d, int n, cudaStream_t s) {
  k_add_diag<<<(n + 255) / 256, 256, 0, s>>>(A, d, n);
}


namespace {

struct Gpu {
  jk_engine* e;
  cudaStream_t s;
  int n;
  const double one = 1.0, zero = 0.0, mone = -1.0;

  // C = alpha op(A) op(B) + beta C, all n x n unless k given
  bool gemm(bool ta, bool tb, int m, int nn, int k, double alpha, const double* A, int lda, const double* B, int ldb,
            double beta, double* C, int ldc) {
    return cublasDgemm(e->cublas, ta ? CUBLAS_OP_T : CUBLAS_OP_N, tb ? CUBLAS_OP_T : CUBLAS_OP_N, m, nn, k, &alpha,
                       A, lda, B, ldb, &beta, C, ldc) == CUBLAS_STATUS_SUCCESS;
  }
  bool mm(bool ta, bool tb, const double* A, const double* B, double* C, double alpha = 1.0, double beta = 0.0) {
    return gemm(ta, tb, n, n, n, alpha, A, n, B, n, beta, C, n);
  }
  bool axpy(double a, const double* x, double* y, size_t len) {
    return cublasDaxpy(e->cublas, (int)len, &a, x, 1, y, 1) == CUBLAS_STATUS_SUCCESS;
  }
  bool copy(const double* x, double* y, size_t len) {
    return cudaMemcpyAsync(y, x, len * sizeof(double), cudaMemcpyDeviceToDevice, s) == cudaSuccess;
  }
  bool scal(double a, double* x, size_t len) {
    return cublasDscal(e->cublas, (int)len, &a, x, 1) == CUBLAS_STATUS_SUCCESS;
  }
  double dot(const double* x, const double* y, size_t len) {
    double r = 0.0;
    cublasDdot(e->cublas, (int)len, x, 1, y, 1, &r);  // host pointer mode: synchronous
    return r;
  }
  double nrm2(const double* x, size_t len) {
    double r = 0.0;
    cublasDnrm2(e->cublas, (int)len, x, 1, &r);
    return r;
  }
};

// Eigen::FullPivLU-style solve with rank (threshold eps * size * max pivot).
void full_piv_solve(std::vector<double> A, int N, std::vector<double> b, std::vector<double>& x, int& rank) {
  std::vector<int> rp(N), cp(N);
  for (int i = 0; i < N; ++i) rp[i] = cp[i] = i;
  auto a = [&](int i, int j) -> double& { return A[(size_t)i * N + j]; };
  double maxpiv = 0.0;
  rank = 0;
  for (int k = 0; k < N; ++k) {
    int pi = k, pj = k;
    double best = -1.0;
    for (int i = k; i < N; ++i)
      for (int j = k; j < N; ++j)
        if (std::fabs(a(i, j)) > best) {
          best = std::fabs(a(i, j));
          pi = i;
          pj = j;
        }
    if (k == 0) maxpiv = best;
    if (best <= maxpiv * 2.220446049250313e-16 * N || best == 0.0) break;
    ++rank;
    if (pi != k) {
      for (int j = 0; j < N; ++j) std::swap(a(k, j), a(pi, j));
      std::swap(b[k], b[pi]);
      std::swap(rp[k], rp[pi]);
    }
    if (pj != k) {
      for (int i = 0; i < N; ++i) std::swap(a(i, k), a(i, pj));
      std::swap(cp[k], cp[pj]);
    }
    for (int i = k + 1; i < N; ++i) {
      double f = a(i, k) / a(k, k);
      if (f == 0.0) continue;
      for (int j = k; j < N; ++j) a(i, j) -= f * a(k, j);
      b[i] -= f * b[k];
    }
  }
  std::vector<double> y(N, 0.0);
  for (int i = rank - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < rank; ++j) s -= a(i, j) * y[j];
    y[i] = s / a(i, i);
  }
  x.assign(N, 0.0);
  for (int i = 0; i < N; ++i) x[cp[i]] = y[i];
}

// FIFO of at most `cap` device vectors backed by buffers allocated once, so
// the SCF loop never allocates (cudaFree would synchronise the device).
struct Ring {
  std::vector<std::unique_ptr<DevBuf<double>>> pool;
  std::vector<double*> order;  // oldest first
  std::vector<double*> spare;
  cudaError_t init(int cap, size_t len) {
    for (int i = 0; i < cap + 1; ++i) {
      pool.emplace_back(new DevBuf<double>());
      cudaError_t st = pool.back()->alloc(len);
      if (st != cudaSuccess) return st;
      spare.push_back(pool.back()->p);
    }
    return cudaSuccess;
  }
  void pop_front() {
    spare.push_back(order.front());
    order.erase(order.begin());
  }
  double* push() {
    if (spare.empty()) pop_front();
    double* p = spare.back();
    spare.pop_back();
    order.push_back(p);
    return p;
  }
  size_t size() const { return order.size(); }
  double* operator[](size_t i) const { return order[i]; }
  void clear() {
    for (double* p : order) spare.push_back(p);
    order.clear();
  }
};

struct Diis {  // DIISEngine (src/diis.cpp) with error vectors in HBM
  int max = 8;
  bool use = true;
  Ring errs;
  std::vector<double> lastB{0.0};
  int lastB_dim = 1;

  static std::vector<double> solve(const std::vector<double>& B, int dim, int start) {
    const int size = dim - start;
    double norm = 1.0;
    if (B[(size_t)start * dim + start] > 1e-10) norm = 1.0 / B[(size_t)start * dim + start];
    std::vector<double> nB((size_t)size * size, 0.0);
    for (int i = 0; i < size - 1; ++i) {
      for (int j = i; j < size - 1; ++j)
        nB[(size_t)i * size + j] = nB[(size_t)j * size + i] = norm * B[(size_t)(i + start) * dim + j + start];
      nB[(size_t)i * size + size - 1] = nB[(size_t)(size - 1) * size + i] = -1.0;
    }
    nB[(size_t)(size - 1) * size + size - 1] = 0.0;
    std::vector<double> w(size, 0.0), x;
    w[size - 1] = -1.0;
    int rank = 0;
    full_piv_solve(nB, size, w, x, rank);
    x.push_back((double)rank);
    return x;
  }

  void reset() {
    errs.clear();
    lastB.assign(1, 0.0);
    lastB_dim = 1;
  }

  std::vector<double> compute(Gpu& g, const double* err, size_t len) {
    std::vector<double> weights;
    const int it = (int)errs.size() + 1;
    if (!use) return weights;
    if (it > max) errs.pop_front();
    double* nb = errs.push();
    g.copy(err, nb, len);
    if (it == 1) {
      lastB.assign(1, g.dot(nb, nb, len));
      lastB_dim = 1;
    }
    if (it > 1) {
      const int lim = std::min(it, max), dim = lim + 1;
      std::vector<double> B((size_t)dim * dim, 0.0);
      const int start = it > lim ? 1 : 0;
      for (int i = 0; i < lim - 1; ++i) {
        for (int j = i; j < lim - 1; ++j)
          B[(size_t)i * dim + j] = B[(size_t)j * dim + i] = lastB[(size_t)(i + start) * lastB_dim + j + start];
        B[(size_t)lim * dim + i] = B[(size_t)i * dim + lim] = -1.0;
      }
      for (int i = 0; i < lim; ++i) {
        double v = g.dot(errs[i], errs[lim - 1], len);
        B[(size_t)(lim - 1) * dim + i] = B[(size_t)i * dim + lim - 1] = v;
      }
      B[(size_t)lim * dim + lim - 1] = B[(size_t)(lim - 1) * dim + lim] = -1.0;
      lastB = B;
      lastB_dim = dim;
      weights = solve(B, dim, 0);
      int rank = (int)weights.back();
      int st = 1;
      while (rank < (lim - st + 1) && st < lim) {
        weights = solve(B, dim, st++);
        rank = (int)weights.back();
      }
      weights.resize(weights.size() - 2);
    }
    return weights;
  }
};

}  // namespace

int scf_rhf(jk_engine* e, const jk_scf_options* o, jk_scf_result* r) {
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  const int n = e->obs.n_final, nocc = o->nocc;
  const size_t nn = (size_t)n * n;
  if (nocc <= 0 || nocc > n) return set_error(e, JK_ERR_ARG, "scf: nocc out of range");
  if (o->df && (e->df.k0 != 0 || (e->df.k1 >= 0 && e->df.k1 != e->aux.n_final)))
    return set_error(e, JK_ERR_STATE, "scf: the DF SCF needs the whole fitting range (jk_df_set_range)");
  if (o->df && !e->df.ready && !e->tiled.metric_ready) {
    // tiled storage with FP64 builds only needs the metric; mixed builds
    // build the fitted tensor on their first call
    int rc = (o->prec_mode == 0 && df_use_tiled(e)) ? df_tiled_metric(e) : df_setup(e);
    if (rc) return rc;
  }
  cudaStream_t s = e->stream;
  cublasSetStream(e->cublas, s);
  Gpu g{e, s, n};
  DevBuf<double> S, T, V, H, X, F, Fm, Finc, D, Dd, Dold, C, W, Wt, eps, J, K, t1, t2, err, work, Delta;
  DevBuf<double> Cal, Cprev, Um, Vm, Wm;  // orbital alignment of the mixed phase
  DevBuf<double> Dref, Gref, Ud, Cpm, lamd;  // FP64 anchor and low-rank density change (prec_mode 2)
  DevBuf<int> info;
  cudaError_t st = cudaSuccess;
  for (auto* b : {&S, &T, &V, &H, &X, &F, &Fm, &Finc, &D, &Dd, &Dold, &C, &W, &Wt, &J, &K, &t1, &t2, &err, &Delta,
                  &Cal, &Cprev, &Um, &Vm, &Wm})
    if (st == cudaSuccess) st = b->alloc(nn);
  if (st == cudaSuccess) st = eps.alloc(n);
  if (st == cudaSuccess) st = info.alloc(1);
  if (st == cudaSuccess && o->df && o->prec_mode == 2) {
    for (auto* b : {&Dref, &Gref, &Ud, &Cpm})
      if (st == cudaSuccess) st = b->alloc(nn);
    if (st == cudaSuccess) st = lamd.alloc(n);
  }
  if (st != cudaSuccess) return check_cuda(e, st, "scf allocation");
  int rc = one_body_device(e, S.p, T.p, V.p, s);
  if (rc) return rc;
  g.copy(T.p, H.p, nn);
  g.axpy(1.0, V.p, H.p, nn);
  // eigensolvers: divide and conquer (syevd), and Jacobi (syevj) warm-started
  // on the Fock matrix expressed in the previous eigenvectors, which is nearly
  // diagonal once the SCF settles (eig_mode 1)
  int lwork = 0, lwork_j = 0;
  syevjInfo_t jinfo = nullptr;
  cusolverDnCreateSyevjInfo(&jinfo);
  cusolverDnXsyevjSetTolerance(jinfo, 1e-14);
  cusolverDnXsyevjSetMaxSweeps(jinfo, 50);
  cusolverDnDsyevd_bufferSize(e->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, W.p, n, eps.p, &lwork);
  cusolverDnDsyevj_bufferSize(e->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, W.p, n, eps.p,
                              &lwork_j, jinfo);
  struct JinfoGuard {
    syevjInfo_t p;
    ~JinfoGuard() {
      if (p) cusolverDnDestroySyevjInfo(p);
    }
  } jguard{jinfo};
  if ((st = work.alloc(std::max(std::max(lwork, lwork_j), 1))) != cudaSuccess)
    return check_cuda(e, st, "eigensolver workspace");
  auto syev = [&](const double* A, double* vecs, double* vals) -> bool {
    g.copy(A, vecs, nn);
    return cusolverDnDsyevd(e->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, vecs, n, vals, work.p,
                            lwork, info.p) == CUSOLVER_STATUS_SUCCESS;
  };
  auto syevj_inplace = [&](double* A, double* vals) -> bool {
    return cusolverDnDsyevj(e->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A, n, vals, work.p,
                            lwork_j, info.p, jinfo) == CUSOLVER_STATUS_SUCCESS;
  };
  // S^-1/2 = U lambda^-1/2 U^T (Fock::formOrthog, src/fock.cpp:124-142)
  std::vector<double> lam(n);
  if (!syev(S.p, W.p, eps.p)) return set_error(e, JK_ERR_CUDA, "syevd(S)");
  cudaMemcpyAsync(lam.data(), eps.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  // lindep > 0: canonical orthogonalisation X = U diag(d) with the directions
  // of S eigenvalues <= lindep dropped (d = 0) and their Fock diagonal raised
  // to LINDEP_SHIFT so that they are never occupied; lindep = 0: molecular2's
  // symmetric S^-1/2 over every direction
  constexpr double LINDEP_SHIFT = 1e4;
  std::vector<double> shift(n, 0.0);
  int ndrop = 0;
  for (int i = 0; i < n; ++i) {
    if (!(lam[i] > 0.0) && !(o->lindep > 0.0))
      return set_error(e, JK_ERR_ARG, "overlap matrix is not positive definite");
    if (o->lindep > 0.0 && lam[i] <= o->lindep) {
      lam[i] = 0.0;
      shift[i] = LINDEP_SHIFT;
      ++ndrop;
    } else {
      lam[i] = 1.0 / std::sqrt(lam[i]);
    }
  }
  if (nocc > n - ndrop) return set_error(e, JK_ERR_ARG, "scf: lindep leaves fewer orbitals than nocc");
  DevBuf<double> dshift;
  if (ndrop > 0 && (st = dshift.upload(shift, s)) != cudaSuccess) return check_cuda(e, st, "scf lindep shift");
  g.copy(W.p, t1.p, nn);
  {
    DevBuf<double> dl;
    dl.upload(lam, s);
    cublasDdgmm(e->cublas, CUBLAS_SIDE_RIGHT, n, n, t1.p, n, dl.p, 1, t1.p, n);  // U diag
    if (o->lindep > 0.0)
      g.copy(t1.p, X.p, nn);              // canonical: U diag
    else
      g.mm(false, true, t1.p, W.p, X.p);  // symmetric: (U diag) U^T
    cudaStreamSynchronize(s);
  }
  double jk_ms = 0.0, diag_ms = 0.0;
  int builds = 0, mixed_builds = 0, corrected_builds = 0;
  // Mixed precision (DF only): split-BF16 builds until ||dD|| < mixed_switch
  // or the density change stalls (no halving over three iterations: the floor
  // set by the mixed builds' own error), FP64 builds after that.  With
  // mixed_refresh > 0 the later iterations instead use Gmixed(D) + Delta, where
  // Delta = G64 - Gmixed is taken from one FP64 and one mixed build at the same
  // density at the switch and then every mixed_refresh iterations (the DIIS
  // history restarts with each new Delta), and the reported energy comes from
  // a final FP64 build at the converged density: the energy is stationary in
  // D, so the density error the corrected builds leave enters it squared.
  // Convergence needs two corrected iterations after the last refresh.
  const bool incremental = o->df && o->prec_mode == 2;
  const bool mixed = o->df && (o->prec_mode == 1 || incremental);
  const double mixed_switch = o->mixed_switch > 0.0 ? o->mixed_switch : 1e-3;
  const int refresh_every = o->mixed_refresh > 0 ? o->mixed_refresh : 0;
  const bool corrected = mixed && !incremental && refresh_every > 0;
  // prec_mode 2: after the mixed phase an FP64 anchor build G64(D_ref), then
  // F = H + G64(D_ref) + Gmixed(D - D_ref) with D - D_ref = 2 (C+ C+^T - C- C-^T)
  // from its eigenvectors (rank <= 2 nocc), so the mixed error scales with
  // ||D - D_ref||.  A new anchor is taken at the current density when the
  // density change stalls where the noise of Gmixed(D - D_ref) dominates (no
  // 15% gain on the best ||dD|| since the anchor after four incremental
  // builds, with ||dD|| below 2% of ||D - D_ref||),
  // or when ||dD|| < densconverge while ||D - D_ref|| >= 100 densconverge;
  // a run converges only with ||D - D_ref|| < 100 densconverge.
  bool have_anchor = false, want_anchor = false;
  int anchors = 0, since_anchor = 0;
  double ref_norm = 0.0, dd_best = 1e300;
  constexpr int MAX_ANCHORS = 8;
  std::vector<double> hlam(incremental ? n : 0), hscale(incremental ? n : 0);
  DevBuf<double> dscale;
  if (incremental && (st = dscale.alloc(n)) != cudaSuccess) return check_cuda(e, st, "scf scale");
  int fp64_after_switch = 0;
  bool switched = !mixed, have_delta = false;
  int build_kind = 0;  // of the last Fock build (trace)
  int since_refresh = 0, refreshes = 0;
  double dd_hist[3] = {1e300, 1e300, 1e300};
  cudaEvent_t ev_a, ev_b;
  cudaEventCreate(&ev_a);
  cudaEventCreate(&ev_b);
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evguard{ev_a, ev_b};
  const double enuc = o->enuc;
  // state of Fock (src/fock.cpp:32-74)
  bool started_incremental = false, reset_incremental = false, have_dens = false;
  double next_reset = 0.0, rms_error = 1.0;
  const double incremental_threshold = 1e-5;
  int last_reset = 0, fock_iter = 0;
  const int MAX = o->maxdiis > 0 ? o->maxdiis : 8;
  Ring focks;
  Diis diis;
  diis.max = MAX;
  diis.use = o->diis != 0;
  if ((st = focks.init(MAX, nn)) != cudaSuccess || (st = diis.errs.init(MAX, nn)) != cudaSuccess)
    return check_cuda(e, st, "scf DIIS history");
  auto transform = [&](const double* Fa) {  // Fm = X^T F X (+ the shift of dropped directions)
    g.mm(false, false, Fa, X.p, t1.p);
    g.mm(true, false, X.p, t1.p, Fm.p);
    if (ndrop > 0) launch_add_diag(Fm.p, dshift.p, n, s);
  };
  bool have_W = false;  // W holds the eigenvectors of the previous Fm
  auto diagonalise = [&]() -> bool {
    cudaEventRecord(ev_a, s);
    bool ok;
    if (o->eig_mode == 1 && have_W) {
      g.mm(false, false, Fm.p, W.p, t1.p);
      g.mm(true, false, W.p, t1.p, Wt.p);  // W^T Fm W
      ok = syevj_inplace(Wt.p, eps.p);
      if (ok) {
        g.mm(false, false, W.p, Wt.p, t1.p);
        g.copy(t1.p, W.p, nn);
      }
    } else {
      ok = syev(Fm.p, W.p, eps.p);
    }
    have_W = ok;
    ok = ok && g.mm(false, false, X.p, W.p, C.p);
    cudaEventRecord(ev_b, s);
    cudaEventSynchronize(ev_b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev_a, ev_b);
    diag_ms += ms;
    return ok;
  };
  auto make_dens = [&]() {
    if (have_dens) {
      g.copy(D.p, Dd.p, nn);
      g.scal(-1.0, Dd.p, nn);
    }
    g.gemm(false, true, n, n, nocc, 2.0, C.p, n, C.p, n, 0.0, D.p, n);
    if (!have_dens)
      g.copy(D.p, Dd.p, nn);
    else
      g.axpy(1.0, D.p, Dd.p, nn);
    have_dens = true;
  };
  // Occupied orbitals for the DF build.  In the corrected mixed phase they are
  // rotated to the set closest to the previous build's (polar factor U of
  // Cocc^T S Cprev, by Newton-Schulz iterations U <- 1.5 U - 0.5 U U^T U):
  // J and K depend only on Cocc Cocc^T, so they are unchanged, while the
  // split-BF16 rounding, which depends on the coefficients themselves, now
  // changes only as much as the density does.
  const double* Cuse = C.p;
  bool have_prev = false;
  std::vector<double> hU((size_t)nocc * nocc);
  auto align = [&]() {
    Cuse = C.p;
    const size_t no = (size_t)n * nocc, oo = (size_t)nocc * nocc;
    if (!have_prev) {
      g.copy(C.p, Cprev.p, no);
      have_prev = true;
      return;
    }
    g.gemm(false, false, n, nocc, n, 1.0, S.p, n, Cprev.p, n, 0.0, t1.p, n);
    g.gemm(true, false, nocc, nocc, n, 1.0, C.p, n, t1.p, n, 0.0, Um.p, nocc);
    for (int k = 0; k < 12; ++k) {
      g.gemm(true, false, nocc, nocc, nocc, 1.0, Um.p, nocc, Um.p, nocc, 0.0, Wm.p, nocc);
      g.copy(Um.p, Vm.p, oo);
      g.gemm(false, false, nocc, nocc, nocc, -0.5, Um.p, nocc, Wm.p, nocc, 1.5, Vm.p, nocc);
      std::swap(Um.p, Vm.p);
    }
    g.gemm(true, false, nocc, nocc, nocc, 1.0, Um.p, nocc, Um.p, nocc, 0.0, Wm.p, nocc);
    cudaMemcpyAsync(hU.data(), Wm.p, oo * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double dev = 0.0;
    for (int i = 0; i < nocc; ++i)
      for (int j = 0; j < nocc; ++j) dev = std::max(dev, std::fabs(hU[(size_t)j * nocc + i] - (i == j ? 1.0 : 0.0)));
    if (dev < 1e-12) {  // a rotation: use it
      g.gemm(false, false, n, nocc, nocc, 1.0, C.p, n, Um.p, nocc, 0.0, Cal.p, n);
      Cuse = Cal.p;
    }
    g.copy(Cuse, Cprev.p, no);
  };
  // G = J - 1/2 K (direct, w.r.t. P) or 2J - K (DF, w.r.t. the occupied C)
  auto jk = [&](const double* P, double* G, int mode) -> int {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    int rc2;
    if (o->df) {
      rc2 = df_jk_device(e, Cuse, nocc, mode, J.p, K.p, s);
      if (mode == 1) ++mixed_builds;
      if (!rc2) {
        g.copy(J.p, G, nn);
        g.scal(2.0, G, nn);
        g.axpy(-1.0, K.p, G, nn);
      }
    } else {
      rc2 = direct_jk_device(e, P, o->precision, 1.0, J.p, K.p, s);
      if (!rc2) {
        g.copy(J.p, G, nn);
        g.axpy(-0.5, K.p, G, nn);
      }
    }
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    jk_ms += ms;
    ++builds;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc2;
  };
  // G = G64(D_ref) + Gmixed(D - D_ref) through two mixed DF builds of the
  // scaled eigenvectors of D - D_ref (positive and negative parts)
  auto incremental_fock = [&](double* G) -> int {
    g.copy(D.p, t1.p, nn);
    g.axpy(-1.0, Dref.p, t1.p, nn);
    if (!syev(t1.p, Ud.p, lamd.p)) return set_error(e, JK_ERR_CUDA, "syevd(D - D_ref)");
    cudaMemcpyAsync(hlam.data(), lamd.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double lmax = 0.0;
    for (int i = 0; i < n; ++i) lmax = std::max(lmax, std::fabs(hlam[i]));
    const double thr = std::max(1e-10 * lmax, 1e-14);
    int rm = 0, rp = 0;  // ascending eigenvalues: negative ones first, positive ones last
    while (rm < n && rm < nocc && hlam[rm] < -thr) ++rm;
    while (rp < n - rm && rp < nocc && hlam[n - 1 - rp] > thr) ++rp;
    g.copy(Gref.p, G, nn);
    for (int part = 0; part < 2; ++part) {
      const int r = part ? rp : rm, c0 = part ? n - rp : 0;
      if (r == 0) continue;
      for (int j = 0; j < r; ++j) hscale[j] = std::sqrt(0.5 * std::fabs(hlam[c0 + j]));
      cudaMemcpyAsync(dscale.p, hscale.data(), sizeof(double) * r, cudaMemcpyHostToDevice, s);
      launch_scale_columns(Ud.p + (size_t)c0 * n, n, r, dscale.p, Cpm.p, s);
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, s);
      int rc2 = df_jk_device(e, Cpm.p, r, 1, J.p, K.p, s);
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      jk_ms += ms;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      ++builds;
      ++mixed_builds;
      if (rc2) return rc2;
      const double sg = part ? 1.0 : -1.0;  // G(D+) - G(D-)
      g.axpy(2.0 * sg, J.p, G, nn);
      g.axpy(-sg, K.p, G, nn);
    }
    return JK_OK;
  };
  auto make_fock = [&]() -> int {
    if (!o->df) {
      g.copy(Finc.p, F.p, nn);
      if (!started_incremental && rms_error < incremental_threshold) {
        started_incremental = true;
        reset_incremental = false;
        next_reset = rms_error / 1e1;
        last_reset = fock_iter - 1;
      }
      if (reset_incremental || !started_incremental) {
        g.copy(H.p, F.p, nn);
        g.copy(D.p, Dd.p, nn);
      }
      if (reset_incremental && started_incremental) {
        reset_incremental = false;
        last_reset = fock_iter;
        next_reset = rms_error / 1e1;
      }
      int rc2 = jk(Dd.p, t2.p, 0);
      if (rc2) return rc2;
      g.axpy(1.0, t2.p, F.p, nn);
      g.copy(F.p, Finc.p, nn);
    } else {
      int rc2 = JK_OK;
      if (corrected && switched) align();
      if (!switched) {
        build_kind = 1;
        rc2 = jk(nullptr, t2.p, 1);
      } else if (incremental && (!have_anchor || want_anchor)) {
        build_kind = 0;  // FP64 anchor
        if ((rc2 = jk(nullptr, Gref.p, 0))) return rc2;
        g.copy(D.p, Dref.p, nn);
        g.copy(Gref.p, t2.p, nn);
        have_anchor = true;
        ++anchors;
        since_anchor = 0;
        dd_best = 1e300;
        focks.clear();  // Fock matrices built around the old reference
        diis.reset();
        fock_iter = 0;
      } else if (incremental) {
        build_kind = 4;
        if ((rc2 = incremental_fock(t2.p))) return rc2;
        ++since_anchor;
      } else if (corrected && (!have_delta || since_refresh >= refresh_every)) {
        build_kind = 3;
        if ((rc2 = jk(nullptr, Delta.p, 1))) return rc2;
        if ((rc2 = jk(nullptr, t2.p, 0))) return rc2;
        g.scal(-1.0, Delta.p, nn);
        g.axpy(1.0, t2.p, Delta.p, nn);  // Delta = G64 - Gmixed
        have_delta = true;
        since_refresh = 0;
        ++refreshes;
        // the Fock matrices in the DIIS history lack this correction
        focks.clear();
        diis.reset();
        fock_iter = 0;
      } else if (corrected) {
        build_kind = 2;
        if ((rc2 = jk(nullptr, t2.p, 1))) return rc2;
        g.axpy(1.0, Delta.p, t2.p, nn);
        ++corrected_builds;
        ++since_refresh;
      } else {
        build_kind = 0;
        rc2 = jk(nullptr, t2.p, 0);
        if (mixed) ++fp64_after_switch;
      }
      if (rc2) return rc2;
      g.copy(H.p, F.p, nn);
      g.axpy(1.0, t2.p, F.p, nn);
    }
    if (o->diis) {
      if (fock_iter >= MAX) focks.pop_front();
      g.copy(F.p, focks.push(), nn);
      ++fock_iter;
    }
    return JK_OK;
  };
  auto calc_err = [&]() {  // X^T (F D S - S D F) X
    g.mm(false, false, D.p, S.p, t1.p);
    g.mm(false, false, F.p, t1.p, err.p);
    g.mm(false, false, D.p, F.p, t1.p);
    g.mm(false, false, S.p, t1.p, err.p, -1.0, 1.0);
    g.mm(false, false, err.p, X.p, t1.p);
    g.mm(true, false, X.p, t1.p, err.p);
  };
  double energy = 0.0, last_energy = 0.0;
  auto calc_e = [&]() {  // 1/2 tr(D (H + F)) + Enuc
    last_energy = energy;
    g.copy(H.p, t1.p, nn);
    g.axpy(1.0, F.p, t1.p, nn);
    energy = 0.5 * g.dot(D.p, t1.p, nn) + enuc;
  };
  auto average = [&](const std::vector<double>& w) {
    if (o->diis && fock_iter > 2) {
      const int off = (int)focks.size() - (int)w.size();
      cudaMemsetAsync(F.p, 0, nn * sizeof(double), s);
      for (int i = off; i < (int)focks.size(); ++i) g.axpy(w[i - off], focks[i], F.p, nn);
    }
  };
  auto cleanup = [&]() {};
  // guess (Fock::transform(true)): core Hamiltonian, or a caller-supplied AO Fock
  if (o->guess_fock) {
    cudaMemcpyAsync(F.p, o->guess_fock, nn * sizeof(double), cudaMemcpyHostToDevice, s);
  } else {
    g.copy(H.p, F.p, nn);
  }
  g.copy(F.p, Finc.p, nn);
  transform(F.p);
  if (!diagonalise()) return cleanup(), set_error(e, JK_ERR_CUDA, "syevd(F)");
  make_dens();
  g.copy(D.p, Dold.p, nn);
  if ((rc = make_fock())) return cleanup(), rc;
  calc_err();
  std::vector<double> weights = diis.compute(g, err.p, nn);
  calc_e();
  average(weights);
  transform(F.p);
  int it = 1;
  bool converged = false;
  double dd = 0.0, delta = 0.0;
  while (!converged && it < o->maxiter) {
    if (!diagonalise()) return cleanup(), set_error(e, JK_ERR_CUDA, "syevd(F)");
    make_dens();
    g.copy(D.p, t1.p, nn);
    g.axpy(-1.0, Dold.p, t1.p, nn);
    dd = g.nrm2(t1.p, nn);
    if (incremental && have_anchor) {
      g.copy(D.p, t1.p, nn);
      g.axpy(-1.0, Dref.p, t1.p, nn);
      ref_norm = g.nrm2(t1.p, nn);
      const bool stall = since_anchor >= 4 && dd > 0.85 * dd_best && dd < 0.02 * ref_norm;
      const bool settle = dd < o->densconverge && ref_norm >= 100.0 * o->densconverge;
      want_anchor = (stall || settle) && anchors < MAX_ANCHORS;
      dd_best = std::min(dd_best, dd);
    }
    if (!switched) {  // takes effect in this iteration's build
      const double best = std::min(dd_hist[0], std::min(dd_hist[1], dd_hist[2]));
      if (dd < mixed_switch || (it >= 6 && dd > 0.5 * best)) switched = true;
      dd_hist[it % 3] = dd;
    }
    g.copy(D.p, Dold.p, nn);
    if ((rc = make_fock())) return cleanup(), rc;
    calc_err();
    rms_error = g.nrm2(err.p, nn) / (double)nn;
    if (rms_error < next_reset || it - last_reset > 8) reset_incremental = true;
    if (it > 2) weights = diis.compute(g, err.p, nn);
    calc_e();
    delta = std::fabs(energy - last_energy);
    if (it > 2) average(weights);
    transform(F.p);
    // a mixed run converges only on FP64 (or FP64-corrected) builds
    if (incremental && build_kind == 0) ref_norm = 0.0;  // this iteration's build was the anchor at D
    const bool precise = !mixed || (incremental ? (have_anchor && ref_norm < 100.0 * o->densconverge)
                                                : corrected ? (have_delta && since_refresh >= 2)
                                                            : fp64_after_switch >= 2);
    converged = dd < o->densconverge && delta < o->enconverge && precise;
    if (o->out_trace && it < o->maxiter) {
      double* tr = o->out_trace + (size_t)5 * it;
      tr[0] = energy;
      tr[1] = dd;
      tr[2] = rms_error;
      tr[3] = build_kind;
      tr[4] = g.nrm2(D.p, nn);
    }
    ++it;
  }
  if (mixed) {
    int rc2 = df_mixed_error(e);
    if (rc2) return cleanup(), rc2;
    if (corrected) {  // energy of the converged density with an FP64 Fock build
      if ((rc2 = jk(nullptr, t2.p, 0))) return cleanup(), rc2;
      g.copy(H.p, F.p, nn);
      g.axpy(1.0, t2.p, F.p, nn);
      calc_e();
    }
  }
  if (!diagonalise()) return cleanup(), set_error(e, JK_ERR_CUDA, "syevd(F)");
  st = cudaStreamSynchronize(s);
  cleanup();
  if (st != cudaSuccess) return check_cuda(e, st, "scf");
  r->energy = energy;
  r->iterations = it;
  r->converged = converged ? 1 : 0;
  r->jk_builds = builds;
  r->jk_ms = jk_ms;
  r->last_delta_e = delta;
  r->last_delta_d = dd;
  r->mixed_builds = mixed_builds;
  r->diag_ms = diag_ms;
  r->lindep_dropped = ndrop;
  if (o->out_density) cudaMemcpy(o->out_density, D.p, nn * sizeof(double), cudaMemcpyDeviceToHost);
  if (o->out_coeffs) cudaMemcpy(o->out_coeffs, C.p, nn * sizeof(double), cudaMemcpyDeviceToHost);
  if (o->out_eps) cudaMemcpy(o->out_eps, eps.p, n * sizeof(double), cudaMemcpyDeviceToHost);
  r->total_ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  return converged ? JK_OK : JK_ERR_NOT_CONVERGED;
}

}  // namespace m2

extern "C" int jk_scf_rhf(jk_engine* e, const jk_scf_options* o, jk_scf_result* r) {
  if (!e || !o || !r) return JK_ERR_ARG;
  std::memset(r, 0, sizeof(*r));
  return m2::scf_rhf(e, o, r);
}
