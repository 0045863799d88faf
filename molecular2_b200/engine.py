"""ctypes binding of ``libm2jk.so`` shaped like molecular2's ``IntegralEngine`` / ``Fock``.

The product path is the CUDA library; there is no CPU fallback.  Importing
works without a GPU, but creating an engine needs the built library and a
CUDA device and raises otherwise.

Reference surface mirrored here (molecular2 paths):
  * ``IntegralEngine.getPrescreen`` / ``compute_schwarz_ints`` (src/integrals.cpp:95, 472-513)
  * ``Fock.formJKdirect(Schwarz, D, multiplier)``   (src/fockbuild.cpp:64-164)
  * ``Fock.getJ / getK / getJK``                     (inc/fock.hpp:141-143)
"""
import ctypes
import os

import numpy as np

from .basis import BasisSet

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libm2jk.so")

JK_ERRORS = {1: "JK_ERR_ARG", 2: "JK_ERR_CUDA", 3: "JK_ERR_NOT_PD", 4: "JK_ERR_STATE", 5: "JK_ERR_NOMEM",
             6: "JK_ERR_NOT_CONVERGED"}

_lib = None

# exported symbols and their C signatures (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
SIGNATURES = {
    "jk_create": (_I, [_P, _P, _I, _P, _P, _I, ctypes.POINTER(_P)]),
    "jk_destroy": (None, [_P]),
    "jk_last_error": (ctypes.c_char_p, [_P]),
    "jk_sizes": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "jk_schwarz": (_I, [_P, _P]),
    "jk_direct": (_I, [_P, _P, _D, _D, _P, _P]),
    "jk_direct_device": (_I, [_P, _P, _D, _D, _P, _P, _P]),
    "jk_direct_noalloc": (_I, [_P, _P, _D, _D, _P, _P, _P]),
    "jk_direct_uhf": (_I, [_P, _P, _P, _D, _D, _P, _P, _P, _P]),
    "jk_direct_uhf_device": (_I, [_P, _P, _P, _D, _D, _P, _P, _P, _P, _P]),
    "jk_df_uhf": (_I, [_P, _P, _I, _P, _I, _I, _D, _P, _P, _P, _P]),
    "jk_df_uhf_device": (_I, [_P, _P, _I, _P, _I, _I, _D, _P, _P, _P, _P, _P]),
    "jk_last_quartets": (ctypes.c_longlong, [_P]),
    "jk_direct_set_partition": (_I, [_P, _I, _I]),
    "jk_last_class_work": (_I, [_P, _P, _I, ctypes.POINTER(_I)]),
    "jk_eri3": (_I, [_P, _P]),
    "jk_eri2": (_I, [_P, _P]),
    "jk_df_setup": (_I, [_P]),
    "jk_df_set_range": (_I, [_P, _I, _I]),
    "jk_df_set_storage": (_I, [_P, _I]),
    "jk_df_mp2": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "jk_wait_selftest": (_I, [_P, ctypes.c_uint, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "jk_df_storage": (_I, [_P]),
    "jk_df_tensor_bytes": (ctypes.c_longlong, [_P]),
    "jk_df_set_tiled_blocks": (_I, [_P, _I, _I]),
    "jk_df": (_I, [_P, _P, _I, _I, _P, _P]),
    "jk_df_device": (_I, [_P, _P, _I, _I, _P, _P, _P]),
    "jk_one_body": (_I, [_P, _P, _P, _P]),
    "jk_scf_rhf": (_I, [_P, _P, _P]),
    "jk_grad_rhf": (_I, [_P, _P, _P, _D, _P, _P]),
    "jk_fock_general": (_I, [_P, _P, _P, _I, _D, _I, _P]),
    "jk_grad_df": (_I, [_P, _P, _I, _P, _P, _P]),
    "jk_set_profiling": (_I, [_P, _I]),
    "jk_stage_ms": (_I, [_P, _P, _I, ctypes.POINTER(_I)]),
}


class SCFOptions(ctypes.Structure):
    """ctypes image of ``jk_scf_options``; defaults are molecular2's (src/ProgramController.cpp:296-307)."""
    _fields_ = [("nocc", _I), ("df", _I), ("prec_mode", _I), ("mixed_switch", _D), ("mixed_refresh", _I),
                ("eig_mode", _I),
                ("maxiter", _I), ("maxdiis", _I), ("diis", _I),
                ("precision", _D), ("enconverge", _D), ("densconverge", _D), ("enuc", _D),
                ("guess_fock", _P), ("out_density", _P), ("out_coeffs", _P), ("out_eps", _P),
                ("out_trace", _P), ("lindep", _D)]


class SCFResult(ctypes.Structure):
    _fields_ = [("energy", _D), ("iterations", _I), ("converged", _I), ("jk_builds", _I), ("jk_ms", _D),
                ("total_ms", _D), ("last_delta_e", _D), ("last_delta_d", _D), ("mixed_builds", _I),
                ("diag_ms", _D), ("lindep_dropped", _I)]


class JKError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{JK_ERRORS.get(code, code)}: {msg}")
        self.code = code


def load_library(path=LIBPATH):
    """Load the engine; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: run `python -m molecular2_b200.build` first")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _bp(basis):
    return ctypes.cast(ctypes.pointer(basis.struct()), ctypes.c_void_p)


def fock_general(obs: BasisSet, dbs: BasisSet, D, shelldiag=True, precision=1e-12, device=0):
    """Fock::compute_2body_fock_general (src/fockbuild.cpp:477-583): G over obs
    from the density D given in basis dbs."""
    lib = load_library()
    n = obs.nbf
    D = np.asfortranarray(D, dtype=np.float64)
    if D.shape != (dbs.nbf, dbs.nbf):
        raise ValueError("D must be dbs.nbf x dbs.nbf")
    G = np.zeros((n, n), order="F")
    rc = lib.jk_fock_general(_bp(obs), _bp(dbs), _p(D), 1 if shelldiag else 0, precision, device, _p(G))
    if rc:
        raise JKError(rc, "jk_fock_general failed")
    return G


class IntegralEngine:
    """Owns one ``jk_engine``: the device basis, shell pairs, Schwarz bounds and scratch."""

    def __init__(self, obs: BasisSet, aux: BasisSet = None, device=0):
        self.lib = load_library()
        self.obs = obs
        self.aux = aux
        mol = obs.mol
        self._Z = np.ascontiguousarray(mol.Z, dtype=np.float64)
        self._xyz = np.ascontiguousarray(mol.xyz.reshape(-1), dtype=np.float64)
        h = ctypes.c_void_p()
        rc = self.lib.jk_create(_bp(obs), _bp(aux) if aux is not None else None, mol.natom, _p(self._xyz),
                                _p(self._Z), device, ctypes.byref(h))
        self.h = h
        if rc:
            msg = self.lib.jk_last_error(h).decode() if h else "allocation failed"
            self.close()
            raise JKError(rc, msg)
        n, na, ns = _I(), _I(), _I()
        self.lib.jk_sizes(self.h, ctypes.byref(n), ctypes.byref(na), ctypes.byref(ns))
        self.n, self.naux, self.nshell = n.value, na.value, ns.value

    def _check(self, rc):
        if rc:
            raise JKError(rc, self.lib.jk_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.jk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def getPrescreen(self):
        Q = np.zeros((self.nshell, self.nshell))
        self._check(self.lib.jk_schwarz(self.h, _p(Q)))
        return Q

    compute_schwarz_ints = getPrescreen

    def last_class_work(self):
        """(6 x 6 x 3) array over (bra class, ket class) of the last direct build:
        quartets, bra primitive pairs, primitive quartets (classes ss, ps, pp, ds, dp, dd)."""
        out = np.zeros(108, dtype=np.int64)
        nw = ctypes.c_int(0)
        self._check(self.lib.jk_last_class_work(self.h, _p(out), 108, ctypes.byref(nw)))
        return out.reshape(6, 6, 3)

    def last_quartets(self):
        return int(self.lib.jk_last_quartets(self.h))

    # -- direct J/K ----------------------------------------------------------
    def jk_direct(self, D, precision=1e-12, multiplier=1.0):
        n = self.n
        D = np.asfortranarray(D, dtype=np.float64)
        J = np.zeros((n, n), order="F")
        K = np.zeros((n, n), order="F")
        self._check(self.lib.jk_direct(self.h, _p(D), precision, multiplier, _p(J), _p(K)))
        return J, K

    def jk_direct_device(self, dD, dJ, dK, precision=1e-12, multiplier=1.0, stream=None):
        """Device-pointer variant (ints from e.g. torch ``data_ptr()``)."""
        self._check(self.lib.jk_direct_device(self.h, ctypes.c_void_p(dD), precision, multiplier,
                                              ctypes.c_void_p(dJ), ctypes.c_void_p(dK),
                                              ctypes.c_void_p(stream) if stream else None))

    def jk_direct_uhf(self, Da, Db, precision=1e-12, multiplier=1.0):
        """UnrestrictedFock::formJKdirect (src/fockbuild.cpp:266-362): (Ja, Jb, Ka, Kb)."""
        n = self.n
        Da = np.asfortranarray(Da, dtype=np.float64)
        Db = np.asfortranarray(Db, dtype=np.float64)
        out = [np.zeros((n, n), order="F") for _ in range(4)]
        self._check(self.lib.jk_direct_uhf(self.h, _p(Da), _p(Db), precision, multiplier, *[_p(o) for o in out]))
        return tuple(out)

    def jk_df_uhf(self, Ca, Cb, prec_mode=0, multiplier=1.0):
        """UnrestrictedFock::formJKdf (src/fockbuild.cpp:365-372): (Ja, Jb, Ka, Kb)
        w.r.t. Ca Ca^T and Cb Cb^T."""
        n = self.n
        Ca = np.asfortranarray(Ca, dtype=np.float64).reshape(n, -1)
        Cb = np.asfortranarray(Cb, dtype=np.float64).reshape(n, -1)
        out = [np.zeros((n, n), order="F") for _ in range(4)]
        self._check(self.lib.jk_df_uhf(self.h, _p(Ca), Ca.shape[1], _p(Cb), Cb.shape[1], prec_mode, multiplier,
                                       *[_p(o) for o in out]))
        return tuple(out)

    # -- density fitting -----------------------------------------------------
    def compute_eris_3index(self):
        """(P|mn) in molecular2's packed layout: (n(n+1)/2) x naux, column-major."""
        n = self.n
        T = np.zeros((n * (n + 1) // 2, self.naux), order="F")
        self._check(self.lib.jk_eri3(self.h, _p(T)))
        return T

    def compute_eris_2index(self):
        V = np.zeros((self.naux, self.naux), order="F")
        self._check(self.lib.jk_eri2(self.h, _p(V)))
        return V

    def df_setup(self):
        self._check(self.lib.jk_df_setup(self.h))

    def df_mp2(self, C, eps, nocc, nfrozen=0):
        """MP2::dfmp2 (src/mp2.cpp:477-583): DF-MP2 correlation energy for canonical
        orbitals C (n x nmo) and energies eps; the nfrozen lowest occupied are frozen."""
        C = np.asfortranarray(C, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        e = ctypes.c_double(0.0)
        self._check(self.lib.jk_df_mp2(self.h, _p(C), _p(eps), C.shape[1], nocc, nfrozen, ctypes.byref(e)))
        return e.value

    def set_direct_partition(self, rank, nranks):
        """Later direct J/K builds and four-index gradients evaluate only this
        rank's share of the bra shell pairs (rank, rank + nranks, ... of every
        class) and return partial results that sum over ranks to the whole."""
        self._check(self.lib.jk_direct_set_partition(self.h, int(rank), int(nranks)))

    def wait_selftest(self, polls=1024):
        """Bounded-wait check: (gave up on a barrier nothing completes,
        gave up on a completed barrier) -- (True, False) when the waits work."""
        a, b = _I(-1), _I(-1)
        self._check(self.lib.jk_wait_selftest(self.h, polls, ctypes.byref(a), ctypes.byref(b)))
        return bool(a.value), bool(b.value)

    DF_STORAGE = {"auto": 0, "unpacked": 1, "tiled": 2}

    def set_df_storage(self, mode):
        """Layout of the fitted tensor (before df_setup): "unpacked" FP64
        B[x][K][y], "tiled" symmetric 128 x 128 tiles in split BF16 with the
        FP64 build streaming the integrals, or "auto" (tiled when the unpacked
        tensor would not fit on the device)."""
        self._check(self.lib.jk_df_set_storage(self.h, self.DF_STORAGE[mode]))

    def set_tiled_blocks(self, waux_max=0, oc_max=0):
        """Caps on the mixed build's fitted-function block and the FP64 build's
        occupied slice for tiled storage (0: sized from free device memory)."""
        self._check(self.lib.jk_df_set_tiled_blocks(self.h, waux_max, oc_max))

    @property
    def df_storage(self):
        return {0: None, 1: "unpacked", 2: "tiled"}[int(self.lib.jk_df_storage(self.h))]

    @property
    def df_tensor_bytes(self):
        """Device bytes of the fitted tensor as stored (0 before df_setup)."""
        return int(self.lib.jk_df_tensor_bytes(self.h))

    @property
    def df_range(self):
        return getattr(self, "_df_range", (0, self.naux))

    def set_df_range(self, k0, k1):
        """Keep only fitted functions k0 <= K < k1 (before df_setup); jk_df then
        gives this slice's partial J, K.  An empty range builds nothing."""
        if k0 == k1:
            self._df_range = (k0, k1)
            return
        self._check(self.lib.jk_df_set_range(self.h, k0, k1))
        self._df_range = (k0, k1)

    def jk_df(self, Cocc, prec_mode=0):
        """J, K with respect to Cocc Cocc^T (compute_2body_fock_df)."""
        n = self.n
        C = np.asfortranarray(Cocc, dtype=np.float64)
        J = np.zeros((n, n), order="F")
        K = np.zeros((n, n), order="F")
        self._check(self.lib.jk_df(self.h, _p(C), C.shape[1], prec_mode, _p(J), _p(K)))
        return J, K

    def jk_df_device(self, dC, nocc, dJ, dK, prec_mode=0, stream=None):
        self._check(self.lib.jk_df_device(self.h, ctypes.c_void_p(dC), nocc, prec_mode, ctypes.c_void_p(dJ),
                                          ctypes.c_void_p(dK), ctypes.c_void_p(stream) if stream else None))

    # -- gradient --------------------------------------------------------------
    def compute_forces(self, D, W, precision=1e-12):
        """Fock::compute_forces: (gradient natom x 3, two-electron part natom x 3)."""
        na = self.obs.mol.natom
        D = np.asfortranarray(D, dtype=np.float64)
        W = np.asfortranarray(W, dtype=np.float64)
        g = np.zeros(3 * na)
        g2 = np.zeros(3 * na)
        self._check(self.lib.jk_grad_rhf(self.h, _p(D), _p(W), precision, _p(g), _p(g2)))
        return g.reshape(na, 3), g2.reshape(na, 3)

    def compute_forces_df(self, Cocc, eps_occ):
        """Gradient of the density-fitted RHF energy for occupied orbitals
        Cocc (n x nocc) and their energies: (gradient natom x 3, two-electron
        part natom x 3)."""
        na = self.obs.mol.natom
        C = np.asfortranarray(Cocc, dtype=np.float64)
        eps = np.ascontiguousarray(eps_occ, dtype=np.float64)
        if eps.shape != (C.shape[1],):
            raise ValueError("eps_occ must have one entry per occupied orbital")
        g = np.zeros(3 * na)
        g2 = np.zeros(3 * na)
        self._check(self.lib.jk_grad_df(self.h, _p(C), C.shape[1], _p(eps), _p(g), _p(g2)))
        return g.reshape(na, 3), g2.reshape(na, 3)

    def set_profiling(self, on=True):
        self._check(self.lib.jk_set_profiling(self.h, 1 if on else 0))

    def stage_ms(self, nmax=8):
        """Device durations (ms) of the stages of the last DF build."""
        buf = (ctypes.c_float * nmax)()
        cnt = _I()
        self._check(self.lib.jk_stage_ms(self.h, ctypes.cast(buf, ctypes.c_void_p), nmax, ctypes.byref(cnt)))
        return [buf[i] for i in range(cnt.value)]

    # -- one-body and SCF ------------------------------------------------------
    def one_body(self):
        n = self.n
        S, T, V = (np.zeros((n, n), order="F") for _ in range(3))
        self._check(self.lib.jk_one_body(self.h, _p(S), _p(T), _p(V)))
        return S, T, V

    def soad_fock(self, precision=1e-12):
        """Fock::compute_soad_guess (src/fock.cpp:174-225): H + G[D_SOAD], with
        D_SOAD the STO-3G atomic occupations of the molecule."""
        from .basis import sto3g_density
        mol = self.obs.mol
        _, T, V = self.one_body()
        G = fock_general(self.obs, BasisSet(mol, "sto-3g", spherical=False), sto3g_density(mol),
                         shelldiag=True, precision=precision)
        return T + V + G

    def scf_rhf(self, nocc, enuc, df=False, prec_mode=0, maxiter=40, maxdiis=8, diis=True, precision=1e-12,
                enconverge=1e-7, densconverge=1e-4, guess_fock=None, want=False, mixed_switch=1e-3, eig_mode=0,
                mixed_refresh=0, guess="core", lindep=0.0):
        """SCF::rhf on the device; returns (SCFResult, extras dict).  guess is
        "core" (core Hamiltonian) or "soad" (SOAD Fock, the reference default);
        an explicit guess_fock overrides it."""
        n = self.n
        if guess_fock is None and guess == "soad":
            guess_fock = self.soad_fock(precision)
        elif guess not in ("core", "soad"):
            raise ValueError("guess must be 'core' or 'soad'")
        o = SCFOptions()
        o.nocc, o.df, o.prec_mode, o.maxiter, o.maxdiis, o.diis = nocc, int(df), prec_mode, maxiter, maxdiis, int(diis)
        o.mixed_switch, o.eig_mode, o.mixed_refresh = mixed_switch, eig_mode, mixed_refresh
        o.precision, o.enconverge, o.densconverge, o.enuc = precision, enconverge, densconverge, enuc
        o.lindep = lindep
        keep = []
        if guess_fock is not None:
            gf = np.asfortranarray(guess_fock, dtype=np.float64)
            keep.append(gf)
            o.guess_fock = gf.ctypes.data
        extras = {}
        trace = np.zeros((max(1, maxiter), 5))
        o.out_trace = trace.ctypes.data
        if want:
            extras = {"D": np.zeros((n, n), order="F"), "C": np.zeros((n, n), order="F"), "eps": np.zeros(n)}
            o.out_density, o.out_coeffs, o.out_eps = (extras[k].ctypes.data for k in ("D", "C", "eps"))
        r = SCFResult()
        rc = self.lib.jk_scf_rhf(self.h, ctypes.byref(o), ctypes.byref(r))
        if rc not in (0, 6):
            self._check(rc)
        extras["trace"] = trace[:max(0, min(r.iterations, maxiter))]
        return r, extras


class Fock:
    """The J/K part of molecular2's ``Fock`` on the GPU engine."""

    def __init__(self, engine: IntegralEngine, precision=1e-12):
        self.integrals = engine
        self.precision = precision
        self.jints = self.kints = self.jkints = None

    def formJKdirect(self, Schwarz, D, multiplier=1.0):
        """src/fockbuild.cpp:64-164 — the Schwarz argument is the engine's own
        (computed on the device at creation); passing None keeps it."""
        J, K = self.integrals.jk_direct(D, self.precision, multiplier)
        self.jints, self.kints = J, K
        self.jkints = J - 0.5 * K
        return self.jkints

    def getJ(self):
        return self.jints

    def getK(self):
        return self.kints

    def getJK(self):
        return self.jkints
