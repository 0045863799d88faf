// Internal engine state shared by the .cu translation units (not part of the C ABI).
#pragma once
#include <cublas_v2.h>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/jk_engine.h"

namespace m2 {

constexpr int MAX_L_OBS = 2;  // orbital shells up to d
constexpr int MAX_L_AUX = 3;  // fitting shells up to f
constexpr int NPAIRCLASS = (MAX_L_OBS + 1) * (MAX_L_OBS + 2) / 2;

inline int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }  // la >= lb

// Host copy of a normalised basis in the engine's layout.
struct HostBasis {
  int nshell = 0;
  std::vector<int> l, nprim, prim_off, atom, pure;
  std::vector<double> exps, coefs, xyz;   // coefs normalised (libint2 Shell semantics)
  std::vector<int> off_final, off_cart;   // per shell (+1 entry): function offsets
  int n_final = 0, n_cart = 0;
  int max_l = 0;
};

// Device array with RAII.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    if (count == n && p) return cudaSuccess;
    reset();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    return e;
  }
  cudaError_t upload(const std::vector<T>& v, cudaStream_t s) {
    cudaError_t e = alloc(v.size());
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
  }
};

// Shell data on the device (one basis).
struct DevBasis {
  DevBuf<int> l, cart_off, final_off, nprim, prim_off, atom, pure;
  DevBuf<double> x, y, z, exps, coefs;
  DevBuf<double> sph;       // packed solid-harmonic blocks, l = 0..SPH_LMAX (sph_off)
  DevBuf<int> cart_shell, cart_comp, final_shell, final_comp;  // per function
};

// Shell pairs of one angular class (la >= lb), sorted by Schwarz bound (descending).
struct PairClassHost {
  int la = 0, lb = 0;
  std::vector<int> sa, sb, prim_off, nprim;
  std::vector<double> Q;
};
struct PairClassDev {
  int la = 0, lb = 0, npair = 0;
  DevBuf<int> sa, sb, prim_off, nprim;
  DevBuf<double> Q;
};

struct DFState {
  bool ready = false;
  int naux = 0;             // fitted functions held here (k1 - k0)
  int k0 = 0, k1 = -1;      // fitted-index range kept in HBM (k1 < 0: all)
  DevBuf<double> B64;      // [x][K][y] unpacked, FP64
  DevBuf<double> L;        // Cholesky factor of the metric (naux x naux, col-major)
  DevBuf<double> Linv;     // L^-1 (naux x naux, col-major, strict upper triangle zero)
  DevBuf<double> X64;      // [x][K][i]
  DevBuf<double> gamma;    // naux
};

// Split-BF16 copies and scratch of the tensor-core (mixed) DF path.
struct MixedState {
  bool ready = false;
  int ldb = 0;                       // padded row length of Bh/Bl (multiple of 64)
  int NP = 0;                        // nocc padded to a multiple of 16
  int NP_cap = 0;                    // NP the scratch below was allocated for
  DevBuf<__nv_bfloat16> Bh, Bl;      // [x][K][y], ld = ldb
  DevBuf<__nv_bfloat16> Ch, Cl;      // [i][y] (NP x ldb)
  DevBuf<float> Cx;                  // [x][i] (n x NP), C for the gamma contraction
  DevBuf<__nv_bfloat16> Xh, Xl;      // [x][K][i] (n x naux*NP)
  DevBuf<double> Kt;                 // n x n partial K (lower-triangle tiles)
  DevBuf<int> err;                   // pipeline error word
  CUtensorMap maps[6];               // Bh, Bl, Ch, Cl, Xh, Xl
};

// Large-system DF storage: the fitted tensor B_K (symmetric in x, y) kept
// only on and below the diagonal, in 128 x 128 function tiles, as split BF16
// [K][tile pair][r][c]; the FP64 build streams (P|mn) tile pairs instead of
// keeping them.
struct TiledDF {
  bool ready = false;                // fitted tensor built (jk_df_setup)
  bool metric_ready = false;         // metric factor, its inverse and the tile lists
  int nt = 0, npt = 0, npad = 0;     // tile rows, stored tile pairs, padded n
  std::vector<long long> list_off;   // [tile pair][class] offsets into plist (+1 entry)
  DevBuf<int> plist;                 // pair indices (into the class lists) touching each tile pair
  DevBuf<__nv_bfloat16> Bh, Bl;      // [K][t][r][c]
  // mixed-build scratch
  int NPX = 0, waux = 0, nocc = 0;   // X row length per K (nhalf * 160), aux block, occupied count
  int wstride = 0;                   // X row stride in fitted functions (waux rounded up to even)
  int NPX_cap = 0;                   // NPX the mixed scratch was allocated for
  int waux_max = 0, oc_max = 0;      // caps on the aux block and the FP64 occupied slice (0: memory decides)
  DevBuf<__nv_bfloat16> Ch, Cl;      // [i][y], NPX x npad
  DevBuf<float> Cx;                  // [x][i], npad x NPX, C for the gamma contraction
  DevBuf<__nv_bfloat16> Xh, Xl;      // [x][K_local][i], npad x waux x NPX
  DevBuf<double> Kt;                 // n x n lower-tile K
  DevBuf<int> err;
  CUtensorMap maps[8];               // Bh/Bl K-major, Bh/Bl MN-major, Ch, Cl, Xh, Xl
};

}  // namespace m2

struct jk_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  // side streams of the per-class kernel launches (direct J/K, gradient):
  // forked from and joined back to the call's stream with events
  // bra-pair partition of the public direct J/K and gradient calls (rank r of
  // nranks takes the pairs r, r + nranks, ... of every class); internal callers
  // (SCF, SOAD) always build the whole
  int part_rank = 0, part_size = 1;
  bool part_active = false;
  static constexpr int NCLS_STREAMS = 8;
  cudaStream_t cls_stream[NCLS_STREAMS] = {};
  cudaEvent_t cls_fork = nullptr, cls_join[NCLS_STREAMS] = {};
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  std::string err;

  int natom = 0;
  std::vector<double> atom_xyz, Z;

  m2::HostBasis obs, aux;
  bool has_aux = false;
  m2::DevBasis dobs, daux;

  // shell pairs (orbital basis)
  m2::PairClassDev pcls[m2::NPAIRCLASS];
  m2::DevBuf<double> pp_p, pp_x, pp_y, pp_z, pp_K, pp_a;  // primitive pairs (pp_a: exponent of shell a)
  m2::DevBuf<double> ap_p, ap_x, ap_y, ap_z, ap_K;         // fitting primitives as (P, unit) pairs
  m2::DevBuf<int> aux_prim_off;                           // per fitting shell
  m2::DevBuf<int> aux_by_l[m2::MAX_L_AUX + 1];             // fitting shells grouped by l
  int aux_by_l_count[m2::MAX_L_AUX + 1] = {0, 0, 0, 0};
  std::vector<double> schwarz_host;                  // nshell x nshell, row-major (symmetric)
  m2::DevBuf<double> schwarz_dev;                    // nshell x nshell
  double Qmax = 0.0;

  m2::DevBuf<double> boys;                           // Boys table

  // scratch for J/K builds
  m2::DevBuf<double> Dcart, Jcart, Kcart, Dnorm, Dmax, Dfinal, Jfinal, Kfinal;
  m2::DFState df;
  m2::MixedState mixed;
  m2::TiledDF tiled;
  int df_storage = 0;     // jk_df_set_storage: 0 auto, 1 unpacked FP64, 2 tiled
  // quartet counter of the last direct build (engine scratch or the fixed
  // array of jk_direct_noalloc), read by jk_last_quartets
  const unsigned long long* last_counter = nullptr;
  // per (bra, ket) pair class of the last direct build: quartets, bra
  // primitive pairs and primitive quartets evaluated (the work model's counts)
  m2::DevBuf<unsigned long long> class_work;
  bool class_work_valid = false;
  // optional per-stage CUDA-event timing of the DF build (jk_set_profiling)
  bool profiling = false;
  static constexpr int NSTAGE_EV = 8;
  cudaEvent_t ev[NSTAGE_EV] = {};
  int nev_used = 0;
  // tiled mixed builds time each kernel launch (per fitted-function block:
  // GEMM1 start, GEMM2 start, GEMM2 end; then J end and finalize end)
  std::vector<cudaEvent_t> kev;
  int kev_blocks = 0;
};

namespace m2 {
// engine.cu
int set_error(jk_engine* e, int code, const std::string& msg);
int check_cuda(jk_engine* e, cudaError_t st, const char* what);
int build_basis(const jk_basis* b, bool allow_pure, int lmax, HostBasis& out, std::string& err);
int upload_basis(jk_engine* e, const HostBasis& hb, DevBasis& db);
// jk_direct.cu
int build_pairs(jk_engine* e);
int direct_jk_device(jk_engine* e, const double* dD, double precision, double mult, double* dJ, double* dK,
                     cudaStream_t s);
// df.cu
int prepare_aux(jk_engine* e);
int compute_V(jk_engine* e, double* V, cudaStream_t s);
int df_setup(jk_engine* e);
int df_jk_device(jk_engine* e, const double* dC, int nocc, int mode, double* dJ, double* dK, cudaStream_t s);
cudaError_t df_syrk_X(jk_engine* e, const double* X, int n, long long len, double* K, cudaStream_t s);
int one_body_device(jk_engine* e, double* S, double* T, double* V, cudaStream_t s);
void stage_mark(jk_engine* e, int k, cudaStream_t s);
// df_mixed.cu
int df_mixed_device(jk_engine* e, const double* dC, int nocc, double* dJ, double* dK, cudaStream_t s);
int df_mixed_error(jk_engine* e);
bool make_map(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint32_t box_cols, uint32_t box_rows);
// Cx[x][i] = C[x][i] in FP32 for x < n, i < nocc, zero in the padding (rows
// up to nrow, columns up to NP)
cudaError_t launch_rows_C(int n, int nocc, int NP, int nrow, const double* C, float* Cx, cudaStream_t s);
cudaError_t launch_split_C(int n, int nocc, int NP, int ld, const double* C, __nv_bfloat16* Ch, __nv_bfloat16* Cl,
                           cudaStream_t s);
cudaError_t launch_gemm2(const CUtensorMap& tXh, const CUtensorMap& tXl, int n, int kblocks, double* Kt, int* err,
                         int nsm, cudaStream_t s);
cudaError_t launch_finalize_mixed(int n, const double* Kt, double* J, double* K, cudaStream_t s);
// df_tiled.cu
int df_tiled_setup(jk_engine* e);
int df_tiled_metric(jk_engine* e);
int tiled_xprime_pass(jk_engine* e, const double* Cp, int i0, int ocur, double* X, double* Tt, cudaStream_t s,
                      const std::function<int(int, int, int)>& hook);
void launch_pad_rows(int n, int npad, int nocc, const double* C, double* Cp, cudaStream_t s);
int df_tiled_device(jk_engine* e, const double* dC, int nocc, int mode, double* dJ, double* dK, cudaStream_t s);
bool df_use_tiled(jk_engine* e);
int df_tiled_error(jk_engine* e);
// transforms (cart <-> final) and norms
void launch_final_to_cart(const jk_engine* e, const double* Dfinal, double* Dcart, cudaStream_t s);
void launch_cart_to_final_sym(const jk_engine* e, const double* Xcart, double scale, double* Xfinal, cudaStream_t s);
void launch_shell_norms(const jk_engine* e, const double* Dfinal, double* Dnorm, double* Dmax, cudaStream_t s);
void launch_add(const double* a, const double* b, double* c, size_t n, cudaStream_t s);  // c = a + b

// Makes the engine's bra-pair partition apply for the lifetime of the object
// (the public direct J/K and gradient entry points).
struct PartitionScope {
  jk_engine* e;
  explicit PartitionScope(jk_engine* e_) : e(e_) { e->part_active = true; }
  ~PartitionScope() { e->part_active = false; }
};
// First bra pair and stride of this rank's share, and how many of the npair
// pairs of a class that is.
inline void bra_share(const jk_engine* e, int npair, int& bra0, int& step, int& count) {
  bra0 = e->part_active ? e->part_rank : 0;
  step = e->part_active ? e->part_size : 1;
  count = npair > bra0 ? (npair - bra0 + step - 1) / step : 0;
}

// Per-class launches on side streams: ClassStreams cs(e, s) makes every side
// stream wait for the work already queued on s; cs.next(cost) picks the side
// stream with the least estimated cost queued so far (longest-first order
// packs best); cs.join() makes s wait for all of them.
struct ClassStreams {
  jk_engine* e;
  cudaStream_t s;
  double load[jk_engine::NCLS_STREAMS] = {};
  ClassStreams(jk_engine* e_, cudaStream_t s_);
  cudaStream_t next(double cost);
  void join();
};
int direct_jk_uhf_device(jk_engine* e, const double* dDa, const double* dDb, double precision, double mult,
                         double* dJa, double* dJb, double* dKa, double* dKb, cudaStream_t s);
}  // namespace m2
