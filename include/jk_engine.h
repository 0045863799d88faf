/* jk_engine.h — C ABI of the B200 J/K Fock-build engine.
 *
 * Drop-in for the two-electron part of molecular2's Fock / IntegralEngine
 * (rashaw1/molecular2).  Every entry point below names the reference
 * interface it replaces (path:line inside molecular2).  Plain pointers and
 * sizes only: no C++ or torch types cross this boundary.
 *
 * Conventions
 *  - Matrices are column-major like molecular2's `Matrix` (Eigen::MatrixXd,
 *    inc/eigen_wrapper.hpp:8).  D, J, K, S, T, V are symmetric n x n; Cocc is
 *    n x nocc column-major.
 *  - Basis functions follow shell order; inside a shell libint2's order:
 *    Cartesian x^a y^b z^c for a = l..0, b = l-a..0; pure (spherical) shells
 *    m = -l..l.  Pure applies to shells with l >= 2 whose `pure` flag is set.
 *  - `coefs` are the coefficients as printed in the basis library (for
 *    normalised primitives); the engine normalises them as libint2::Shell
 *    does (src/basis.cpp:49-61 constructs those shells).
 *  - Coordinates are bohr.
 *  - Return value: 0 on success, else a JK_ERR_* code; jk_last_error() gives
 *    the message.  Nothing aborts, throws across the boundary or traps on the
 *    device (molecular2 throws Error(code,msg), inc/error.hpp:25-29).
 *  - One engine = one CUDA device + one stream.  Calls on one engine are not
 *    re-entrant; different engines are independent.
 *  - `*_device` variants take device pointers and a cudaStream_t (as void*,
 *    NULL = the engine's stream) and do not synchronise the host.
 */
#ifndef M2_JK_ENGINE_H
#define M2_JK_ENGINE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  JK_OK = 0,
  JK_ERR_ARG = 1,         /* bad argument (null pointer, size, unsupported l) */
  JK_ERR_CUDA = 2,        /* CUDA / cuBLAS / cuSOLVER failure */
  JK_ERR_NOT_PD = 3,      /* fitting metric (P|Q) not positive definite */
  JK_ERR_STATE = 4,       /* call order (e.g. jk_df before jk_df_setup) */
  JK_ERR_NOMEM = 5,       /* device allocation failed */
  JK_ERR_NOT_CONVERGED = 6
};

/* Struct-of-arrays Gaussian basis.  Replaces std::vector<libint2::Shell>
 * built by Basis::addShell (src/basis.cpp:33-66). */
typedef struct jk_basis {
  int nshell;
  const int* l;          /* angular momentum per shell */
  const int* nprim;      /* primitives per shell */
  const int* prim_off;   /* offset of the shell's primitives in exps/coefs */
  const double* exps;    /* exponents */
  const double* coefs;   /* contraction coefficients (as printed) */
  const double* xyz;     /* 3 * nshell centre coordinates, bohr */
  const int* pure;       /* per shell: 1 = spherical for l >= 2 (NULL: all Cartesian) */
  const int* atom;       /* per shell: owning atom (NULL allowed when no gradient is needed) */
} jk_basis;

typedef struct jk_engine jk_engine;

/* Create an engine for an orbital basis and (optionally, NULL) a fitting
 * basis; natom point charges Z at atom_xyz (3*natom) for one-body and
 * gradient terms.  Computes the Schwarz bounds of all shell pairs.
 * Replaces the IntegralEngine constructor's prescreen step
 * (src/integrals.cpp:42-124, compute_schwarz_ints at :95). */
int jk_create(const jk_basis* obs, const jk_basis* aux, int natom, const double* atom_xyz, const double* Z,
              int device, jk_engine** out);
void jk_destroy(jk_engine* e);
const char* jk_last_error(const jk_engine* e);

/* Basis sizes: n (orbital), naux (fitting, 0 if none), nshell (orbital). */
int jk_sizes(const jk_engine* e, int* n, int* naux, int* nshell);

/* Schwarz matrix Q(s1,s2) = sqrt(max_i |(ab|ab)_ii|), nshell x nshell.
 * Replaces IntegralEngine::compute_schwarz_ints (src/integrals.cpp:472-513). */
int jk_schwarz(const jk_engine* e, double* Q);

/* Integral-direct J[D] and K[D] (both w.r.t. the full D passed in, scaled by
 * `multiplier`), FP64, Schwarz x density screening at `precision`:
 * Fock::formJKdirect(Schwarz, D, multiplier) (src/fockbuild.cpp:64-164);
 * the caller forms jkints = J - 0.5 K as :163 does. Host pointers. */
int jk_direct(jk_engine* e, const double* D, double precision, double multiplier, double* J, double* K);
int jk_direct_device(jk_engine* e, const double* dD, double precision, double multiplier, double* dJ,
                     double* dK, void* stream);

/* Unrestricted (UHF) integral-direct J and K: J[Da], J[Db], K[Da], K[Db] from
 * one pass over the shell quartets, screened with the shell-block norms of
 * Da + Db, every integral batch digested into both densities.  Each result is
 * w.r.t. its full spin density and scaled by `multiplier`; the caller forms
 * J - K per spin as molecular2 does.  Replaces
 * UnrestrictedFock::formJKdirect(Schwarz, Da, Db, multiplier)
 * (src/fockbuild.cpp:266-362). */
int jk_direct_uhf(jk_engine* e, const double* Da, const double* Db, double precision, double multiplier, double* Ja,
                  double* Jb, double* Ka, double* Kb);
int jk_direct_uhf_device(jk_engine* e, const double* dDa, const double* dDb, double precision, double multiplier,
                         double* dJa, double* dJb, double* dKa, double* dKb, void* stream);

/* Integral-direct J and K exactly as jk_direct_device, for callers that must
 * not allocate device memory while building a Fock matrix: for example a
 * service that reserves all device memory for a caching allocator at start-up
 * and may not take more, or code running next to latency-sensitive streams,
 * where cudaMalloc/cudaFree (which can synchronise the whole device) would
 * stall them.  This call allocates nothing: its scratch is one fixed array in
 * device memory that every GPU loading this library keeps until the process
 * exits, which limits the basis to at most 512 Cartesian functions and 256
 * shells (larger bases return JK_ERR_ARG; use jk_direct_device).  The engine
 * itself is still created by jk_create, which does allocate.  The first call on
 * a device looks up the array's device address, so make one call before any
 * stream capture.  All calls share the array: calls whose GPU work overlaps
 * (other streams, other engines on the same device) race and give wrong
 * results; serialise them.  Call it with the engine's device current
 * (JK_ERR_ARG otherwise): the array's address differs per GPU.  No
 * counterpart in molecular2. */
int jk_direct_noalloc(jk_engine* e, const double* dD, double precision, double multiplier, double* dJ,
                      double* dK, void* stream);

/* Share the direct builds and the four-index gradient over nranks processes:
 * every later jk_direct*, jk_direct_uhf* and jk_grad_rhf call on this engine
 * evaluates only the bra shell pairs rank, rank + nranks, ... of every pair
 * class (the Schwarz-sorted class lists interleave large and small pairs, so
 * the shares carry nearly equal work) and returns this rank's partial J, K or
 * gradient; the sum over ranks (one all-reduce of J and K, or of the 3 natom
 * gradient) is the whole.  The one-body and nuclear-repulsion gradient terms
 * go to rank 0 only.  The SCF driver and the SOAD guess always build the
 * whole.  Default rank 0 of 1.  The loops split are those of
 * src/fockbuild.cpp:88-158 and src/rhfgrad.cpp:454-590 (serial in molecular2). */
int jk_direct_set_partition(jk_engine* e, int rank, int nranks);

/* Number of shell quartets the last direct build (jk_direct, jk_direct_device
 * or jk_direct_noalloc) evaluated; -1 before the first build. */
long long jk_last_quartets(const jk_engine* e);

/* Work counts of the last jk_direct / jk_direct_device / jk_direct_uhf build
 * per (bra, ket) shell-pair class, classes ordered ss, ps, pp, ds, dp, dd:
 * out[3 (bra * 6 + ket) + k] for k = 0 quartets, 1 bra primitive pairs summed
 * over them, 2 primitive quartets; up to nmax values, count in *nwritten.
 * JK_ERR_STATE after jk_direct_noalloc (it keeps no counters).  molecular2
 * has no counterpart; these give the flop model of the roofline. */
int jk_last_class_work(const jk_engine* e, long long* out, int nmax, int* nwritten);

/* Three-index integrals (P|mn) in molecular2's packed layout: column-major
 * (n(n+1)/2) x naux, row x(x+1)/2 + y for x >= y.
 * Replaces IntegralEngine::compute_eris_3index(obs, auxbs, Matrix&)
 * (src/eris.cpp:89-156). */
int jk_eri3(jk_engine* e, double* T);

/* Two-index metric (P|Q), naux x naux.
 * Replaces IntegralEngine::compute_eris_2index (src/eris.cpp:304-356). */
int jk_eri2(jk_engine* e, double* V);

/* First-call part of compute_2body_fock_df (src/fockbuild.cpp:598-619):
 * (P|mn), (P|Q), the Cholesky factor V = L L^T and B = (mn|P) L^-T, kept in
 * HBM.  Returns JK_ERR_NOT_PD when the metric is not positive definite. */
int jk_df_setup(jk_engine* e);

/* Keep only the fitted functions k0 <= K < k1 of B (call before jk_df_setup):
 * jk_df then returns this slice's partial J and K, and the sum over slices
 * that cover 0..naux is the full build (one all-reduce per build when ranks
 * hold the slices).  Every slice still computes the full (P|mn) and the
 * Cholesky factor once at set-up.  The DF SCF and jk_grad_df need the whole
 * range (JK_ERR_STATE otherwise).  Replaces nothing in molecular2, whose DF
 * build is serial (src/fockbuild.cpp:621-659). */
int jk_df_set_range(jk_engine* e, int k0, int k1);

/* Unrestricted (UHF) DF J and K: the jk_df build for the alpha occupied
 * orbitals Ca (n x na) and for the beta ones Cb (n x nb) over the same fitted
 * tensor, all four scaled by `multiplier` (nb = 0 gives zero beta matrices).
 * Replaces UnrestrictedFock::formJKdf(ca_occ, cb_occ, multiplier)
 * (src/fockbuild.cpp:365-372). */
int jk_df_uhf(jk_engine* e, const double* Ca, int na, const double* Cb, int nb, int prec_mode, double multiplier,
              double* Ja, double* Jb, double* Ka, double* Kb);
int jk_df_uhf_device(jk_engine* e, const double* dCa, int na, const double* dCb, int nb, int prec_mode,
                     double multiplier, double* dJa, double* dJb, double* dKa, double* dKb, void* stream);

/* Density-fitted MP2 correlation energy for the canonical orbitals C (n x nmo
 * column-major, host) with orbital energies eps (nmo): the nfrozen lowest of
 * the nocc occupied orbitals are frozen, the nmo - nocc above them are the
 * virtuals.  (ia|jb) comes from the fitted tensor of jk_df_setup (unpacked
 * storage; run first if needed), E = sum (ia|jb)[2(ia|jb) - (ib|ja)] /
 * (e_i + e_j - e_a - e_b) in FP64.  Replaces MP2::dfmp2 (src/mp2.cpp:477-583),
 * which inverts (P|Q) explicitly where this uses its Cholesky factor. */
int jk_df_mp2(jk_engine* e, const double* C, const double* eps, int nmo, int nocc, int nfrozen, double* emp2);

/* Failure-detection check of the bounded mbarrier wait every tensor-core
 * kernel uses: one launch waits `polls` times on a barrier that nothing
 * completes (*timed_out = 1 when the wait gave up and the kernel returned)
 * and on one that has completed (*completed_timed_out = 0).  No molecular2
 * counterpart; the engine's device must be current. */
int jk_wait_selftest(jk_engine* e, unsigned polls, int* timed_out, int* completed_timed_out);

/* Layout of the fitted tensor, chosen before jk_df_setup (molecular2 keeps one
 * packed FP64 (n(n+1)/2) x naux matrix, src/fockbuild.cpp:598-619, which
 * stops fitting in device memory near n = 2600, naux = 9600):
 *   1  unpacked FP64 B[x][K][y] plus its split-BF16 copy (small systems);
 *   2  tiled: B_K kept on and below the diagonal of a 128 x 128 function
 *      tiling, split BF16 only (half the bytes of the packed FP64 matrix);
 *      the FP64 build (prec_mode 0) then recomputes the three-index
 *      integrals per build instead of reading B;
 *   0  automatic (default): tiled when the unpacked path would not fit.
 * jk_df_storage reports the layout in use (0 before set-up). */
int jk_df_set_storage(jk_engine* e, int mode);
int jk_df_storage(const jk_engine* e);

/* Device bytes of the fitted tensor as stored (tiled: the split-BF16 tiles;
 * unpacked: FP64 B plus its split-BF16 copy once a mixed build made it); 0
 * before jk_df_setup.  Measurement only; no molecular2 counterpart. */
long long jk_df_tensor_bytes(const jk_engine* e);

/* Tiled storage only: caps on the block of fitted functions a mixed build
 * contracts at once (its X block) and on the occupied slice of one FP64
 * integral pass (0 = size them from free device memory, the default).  Small
 * caps run the multi-block and multi-pass schedules on small systems. */
int jk_df_set_tiled_blocks(jk_engine* e, int waux_max, int oc_max);

/* Per-iteration part of compute_2body_fock_df (src/fockbuild.cpp:621-659):
 * J and K with respect to Cocc Cocc^T (the caller forms mult*(2J - K) as
 * Fock::formJKdf does at :173).  prec_mode 0 = FP64.  Host pointers. */
int jk_df(jk_engine* e, const double* Cocc, int nocc, int prec_mode, double* J, double* K);
int jk_df_device(jk_engine* e, const double* dCocc, int nocc, int prec_mode, double* dJ, double* dK, void* stream);

/* Per-stage device timing of DF builds (CUDA events on the launch stream;
 * molecular2 only has wall-clock timers, src/logger.cpp:35-40).
 * jk_stage_ms writes up to nmax stage durations of the last build (ms) and
 * their count to *nwritten.  Unpacked FP64 stages: X = B C, K = X X^T,
 * gamma, J; unpacked mixed: GEMM1, GEMM2, J, finalize; tiled mixed: GEMM1
 * total, GEMM2 total, J, finalize and (as a float) the number of
 * fitted-function blocks; tiled FP64: first integral pass, its Y = L^-1 X',
 * its K update, the remaining passes. */
int jk_set_profiling(jk_engine* e, int on);
int jk_stage_ms(jk_engine* e, float* ms, int nmax, int* nwritten);

/* Two-electron Fock contribution of a density D given in a second basis dbs
 * (n_d x n_d, column-major; shell-diagonal blocks only when shelldiag != 0):
 *   G(1,2) = sum_{3,4 in dbs} 2 D(3,4) (12|34) - D(3,4) (13|24),  n x n over obs,
 * screened at `precision`.  Replaces Fock::compute_2body_fock_general
 * (src/fockbuild.cpp:477-583) as used by the SOAD guess
 * (Fock::compute_soad_guess, src/fock.cpp:174-225, with dbs = STO-3G and D the
 * spherically averaged atomic occupations times 0.5).  Needs no engine: it
 * builds a temporary one on `device` for the union of both bases. */
int jk_fock_general(const jk_basis* obs, const jk_basis* dbs, const double* D, int shelldiag, double precision,
                    int device, double* G);

/* Overlap, kinetic and nuclear-attraction matrices (point charges of
 * jk_create): IntegralEngine::compute_1body_ints (src/integrals.cpp:394-449). */
int jk_one_body(jk_engine* e, double* S, double* T, double* V);

/* RHF SCF with every n x n matrix in HBM: SCF::rhf (src/scf.cpp:90-185) with
 * DIISEngine (src/diis.cpp:22-116), the incremental direct Fock build of
 * Fock::makeFock (src/fockbuild.cpp:176-222) and Fock::formJKdf for df != 0.
 * Converged when ||D - D_old||_F < densconverge and |dE| < enconverge (:156).
 * Returns JK_ERR_NOT_CONVERGED (result still filled) after maxiter. */
typedef struct jk_scf_options {
  int nocc;
  int df;                  /* 0 = integral-direct J/K, 1 = density-fitted */
  int prec_mode;           /* DF only: 0 = FP64; 1 = split-BF16 tensor-core builds while
                              ||D - D_old||_F >= mixed_switch and still falling, FP64
                              builds to convergence after that (or, with mixed_refresh,
                              corrected mixed builds); 2 = the same mixed phase, then an FP64
                              anchor build G64(D_ref) and mixed builds of the low-rank change
                              D - D_ref only (error proportional to ||D - D_ref||); a new anchor
                              when ||D - D_old||_F stalls, or falls below densconverge while
                              ||D - D_ref||_F >= 100 densconverge (at most 8); converged only
                              with ||D - D_ref||_F < 100 densconverge */
  double mixed_switch;     /* default 1e-3; the switch also happens when ||dD|| stalls */
  int mixed_refresh;       /* 0 (default): FP64 builds after the switch.  k > 0: mixed builds
                              plus the correction G64 - Gmixed refreshed every k iterations,
                              energy from a final FP64 build */
  int eig_mode;            /* 0 = cuSOLVER syevd every iteration; 1 = Jacobi (syevj) on the
                              Fock matrix in the previous eigenvectors after the first */
  int maxiter;             /* molecular2 default 40 */
  int maxdiis;             /* default 8 */
  int diis;                /* 1 = on */
  double precision;        /* Schwarz x density screening threshold, default 1e-12 */
  double enconverge;       /* default 1e-7 */
  double densconverge;     /* default 1e-4 */
  double enuc;             /* nuclear repulsion energy added to E */
  const double* guess_fock;  /* host n x n AO Fock for the first diagonalisation, NULL = core Hamiltonian */
  double* out_density;     /* optional host n x n */
  double* out_coeffs;      /* optional host n x n (MO coefficients, columns) */
  double* out_eps;         /* optional host n */
  double* out_trace;       /* optional host maxiter x 5, per iteration: energy, ||D - D_old||_F, rms of the
                              DIIS error, build kind (0 FP64, 1 mixed, 2 mixed + correction, 3 correction
                              refresh: mixed and FP64 builds, 4 FP64 anchor + mixed build of D - D_ref),
                              ||D||_F */
  double lindep;           /* 0 (default): symmetric S^-1/2 over all directions as molecular2
                              (src/fock.cpp:124-142); > 0: canonical orthogonalisation dropping the
                              directions whose overlap eigenvalue is <= lindep */
} jk_scf_options;

typedef struct jk_scf_result {
  double energy;
  int iterations;
  int converged;
  int jk_builds;
  double jk_ms;            /* device time inside J/K builds */
  double total_ms;         /* host wall time of the whole call */
  double last_delta_e;
  double last_delta_d;
  int mixed_builds;        /* J/K builds done in mixed precision */
  double diag_ms;          /* device time in the Fock diagonalisations */
  int lindep_dropped;      /* directions removed by jk_scf_options.lindep */
} jk_scf_result;

int jk_scf_rhf(jk_engine* e, const jk_scf_options* opt, jk_scf_result* res);

/* RHF nuclear gradient dE/dx (natom x 3, atom-major) for the full density D
 * and the energy-weighted density W = Cocc diag(eps_occ) Cocc^T (host, n x n):
 * Fock::compute_forces (src/rhfgrad.cpp:15-89) = (T' + V') . D - 2 S' . W
 * + 1/4 G'(D) . D + nuclear repulsion, with G' = compute_2body_fock_deriv<1>
 * (src/rhfgrad.cpp:419-598) screened at `precision` over the overlap-screened
 * shell-pair list.  The two-electron part alone is also written to grad2e
 * when it is not NULL.  Needs jk_basis.atom. */
int jk_grad_rhf(jk_engine* e, const double* D, const double* W, double precision, double* grad, double* grad2e);

/* RHF nuclear gradient of the density-fitted energy (the energy whose Fock
 * matrix jk_df / Fock::formJKdf builds, src/fockbuild.cpp:585-660) for the
 * occupied orbitals Cocc (host, n x nocc column-major) with energies eps_occ:
 * (T' + V') . D - 2 S' . W + nuclear repulsion as Fock::compute_forces
 * (src/rhfgrad.cpp:15-89), with D = 2 Cocc Cocc^T and W = Cocc diag(eps_occ)
 * Cocc^T, plus the derivative of the fitted two-electron energy,
 *   sum (mn|P)^x [c_P D_mn - 2 (C d^P C^T)_mn] + sum (P|Q)^x [d^P . d^Q - c_P c_Q / 2],
 * c = V^-1 (P|mn) D_mn, d^P_ij = V^-1 (Q|ij).  The two-electron part alone
 * goes to grad2e when it is not NULL.  Runs jk_df_setup first if needed; needs
 * jk_basis.atom on both bases.  molecular2 has no DF gradient (its
 * compute_forces differentiates the 4-index energy); this is the gradient
 * the DF SCF energy needs. */
int jk_grad_df(jk_engine* e, const double* Cocc, int nocc, const double* eps_occ, double* grad, double* grad2e);

#ifdef __cplusplus
}
#endif
#endif
