"""CPU FP64 oracle for the J/K engine — TEST INFRASTRUCTURE ONLY.

The parity checker for ``molecular2_b200``: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs may import
it, and the product never does.  ``oracle.cpp`` restates molecular2's J/K,
DF, Schwarz, SOAD and gradient loops in scalar C++ (citations in that file);
``scf.py`` restates ``SCF::rhf`` with DIIS and the incremental Fock build.

Pinned against molecular2's recorded outputs (tests/test_oracle_pins.py):
``test/h2otest.out_1`` and ``test/benzene.out_1`` RHF energies and the
analytic s-type ERIs of ``test/cdthe.ints``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_SRC = os.path.join(_HERE, "oracle.cpp")
_lib = None


def build(force=False):
    """Compile oracle.cpp into liboracle.so beside it (g++ only)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(_SRC):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", _SO, _SRC, "-lpthread"])
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        P = ctypes.c_void_p
        d = ctypes.c_double
        i = ctypes.c_int
        sig = {
            "orc_boys": (None, [i, d, P]),
            "orc_nbf": (i, [P]),
            "orc_normalised_coefs": (None, [P, P]),
            "orc_solid_harmonics": (None, [i, P]),
            "orc_eri_quartet": (None, [P, i, i, i, i, P]),
            "orc_eri_full": (None, [P, P]),
            "orc_schwarz": (None, [P, P]),
            "orc_shellblock_norm": (None, [P, P, P]),
            "orc_jk_direct": (ctypes.c_long, [P, P, P, d, d, P, P, i]),
            "orc_jk_direct_rows": (ctypes.c_long, [P, P, P, d, i, i, P, P]),
            "orc_jk_direct_uhf": (ctypes.c_long, [P, P, P, P, d, d, P, P, P, P, i]),
            "orc_fock_general": (None, [P, P, P, i, P]),
            "orc_eri3": (None, [P, P, P]),
            "orc_eri2": (None, [P, P]),
            "orc_cholesky": (i, [i, P, P]),
            "orc_df_B": (i, [i, i, P, P, P, i]),
            "orc_df_jk": (None, [i, i, i, P, P, P, P, i, i, i]),
            "orc_one_body": (None, [P, i, P, P, P, P, P]),
            "orc_one_body_deriv": (None, [P, P, i, P, P, P, P, P]),
            "orc_shellpair_list": (None, [P, d, P]),
            "orc_grad2e": (None, [P, P, i, P, P, d, P, P, i]),
            "orc_eri3_deriv_block": (None, [P, P, i, i, i, i, i, P]),
            "orc_eri4_deriv_block": (None, [P, i, i, i, i, i, i, P]),
            "orc_df_grad_contract": (None, [P, P, P, P, i, P, P, P, i]),
            "orc_grad2e_rows": (None, [P, P, i, P, P, d, i, i, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _bp(basis):
    return ctypes.cast(ctypes.pointer(basis.struct()), ctypes.c_void_p)


def F(a):
    """Column-major (Eigen Matrix) contiguous float64 copy."""
    return np.asfortranarray(a, dtype=np.float64)


def boys(mmax, T):
    out = np.zeros(mmax + 1)
    lib().orc_boys(mmax, float(T), _p(out))
    return out


def solid_harmonics(l):
    out = np.zeros((2 * l + 1, (l + 1) * (l + 2) // 2))
    lib().orc_solid_harmonics(l, _p(out))
    return out


def normalised_coefs(basis):
    out = np.zeros_like(basis.coefs)
    lib().orc_normalised_coefs(_bp(basis), _p(out))
    return out


def eri_quartet(basis, s1, s2, s3, s4):
    n = [basis.bf_off[s + 1] - basis.bf_off[s] for s in (s1, s2, s3, s4)]
    out = np.zeros(int(np.prod(n)))
    lib().orc_eri_quartet(_bp(basis), s1, s2, s3, s4, _p(out))
    return out.reshape(n)


def eri_full(basis):
    n = basis.nbf
    out = np.zeros((n, n, n, n))
    lib().orc_eri_full(_bp(basis), _p(out))
    return out


def schwarz(basis):
    ns = basis.nshell
    Q = np.zeros((ns, ns))
    lib().orc_schwarz(_bp(basis), _p(Q))
    return Q


def shellblock_norm(basis, D):
    D = F(D)
    out = np.zeros((basis.nshell, basis.nshell))
    lib().orc_shellblock_norm(_bp(basis), _p(D), _p(out))
    return out


def jk_direct(basis, D, Q=None, precision=1e-12, multiplier=1.0, nthreads=None):
    """Fock::formJKdirect: returns (J[D], K[D], n_quartets)."""
    n = basis.nbf
    D = F(D)
    J = np.zeros((n, n), order="F")
    K = np.zeros((n, n), order="F")
    Qc = None if Q is None else np.ascontiguousarray(Q, dtype=np.float64)
    nt = nthreads or os.cpu_count() or 1
    cnt = lib().orc_jk_direct(_bp(basis), _p(Qc), _p(D), precision, multiplier, _p(J), _p(K), nt)
    return J, K, cnt


def jk_direct_uhf(basis, Da, Db, Q=None, precision=1e-12, multiplier=1.0, nthreads=None):
    """UnrestrictedFock::formJKdirect: (Ja, Jb, Ka, Kb, quartets)."""
    n = basis.nbf
    Qc = None if Q is None else np.ascontiguousarray(Q, dtype=np.float64)
    Da, Db = F(Da), F(Db)
    out = [np.zeros((n, n), order="F") for _ in range(4)]
    nt = nthreads or os.cpu_count() or 1
    cnt = lib().orc_jk_direct_uhf(_bp(basis), _p(Qc) if Qc is not None else None, _p(Da), _p(Db), precision,
                                  multiplier, *[_p(o) for o in out], nt)
    return (*out, cnt)


def jk_direct_rows(basis, D, Q, precision, s1_begin, s1_end):
    n = basis.nbf
    D = F(D)
    J = np.zeros((n, n), order="F")
    K = np.zeros((n, n), order="F")
    Qc = np.ascontiguousarray(Q, dtype=np.float64)
    cnt = lib().orc_jk_direct_rows(_bp(basis), _p(Qc), _p(D), precision, s1_begin, s1_end, _p(J), _p(K))
    return J, K, cnt


def fock_general(obs, dbs, D, shelldiag=True):
    n = obs.nbf
    D = F(D)
    G = np.zeros((n, n), order="F")
    lib().orc_fock_general(_bp(obs), _bp(dbs), _p(D), 1 if shelldiag else 0, _p(G))
    return G


def eri3(obs, aux):
    n = obs.nbf
    T = np.zeros((n * (n + 1) // 2, aux.nbf), order="F")
    lib().orc_eri3(_bp(obs), _bp(aux), _p(T))
    return T


def eri2(aux):
    V = np.zeros((aux.nbf, aux.nbf), order="F")
    lib().orc_eri2(_bp(aux), _p(V))
    return V


def df_B(T, V, nthreads=None):
    T = F(T)
    V = F(V)
    npair, naux = T.shape
    B = np.zeros((npair, naux), order="F")
    st = lib().orc_df_B(npair, naux, _p(T), _p(V), _p(B), nthreads or os.cpu_count() or 1)
    if st:
        raise np.linalg.LinAlgError(f"metric not positive definite at column {st - 1}")
    return B


def df_jk(B, Cocc, k_range=None, nthreads=None):
    """Per-iteration compute_2body_fock_df: (J, K) w.r.t. C C^T."""
    B = F(B)
    C = F(Cocc)
    n, nocc = C.shape
    naux = B.shape[1]
    kb, ke = (0, naux) if k_range is None else k_range
    J = np.zeros((n, n), order="F")
    K = np.zeros((n, n), order="F")
    lib().orc_df_jk(n, naux, nocc, _p(B), _p(C), _p(J), _p(K), kb, ke, nthreads or os.cpu_count() or 1)
    return J, K


def one_body(basis):
    n = basis.nbf
    mol = basis.mol
    S = np.zeros((n, n), order="F")
    T = np.zeros((n, n), order="F")
    V = np.zeros((n, n), order="F")
    Z = np.ascontiguousarray(mol.Z)
    xyz = np.ascontiguousarray(mol.xyz.reshape(-1))
    lib().orc_one_body(_bp(basis), mol.natom, _p(Z), _p(xyz), _p(S), _p(T), _p(V))
    return S, T, V


def one_body_deriv(basis):
    n = basis.nbf
    mol = basis.mol
    na = mol.natom
    S1 = np.zeros((3 * na, n, n))
    T1 = np.zeros((3 * na, n, n))
    V1 = np.zeros((3 * na, n, n))
    Z = np.ascontiguousarray(mol.Z)
    xyz = np.ascontiguousarray(mol.xyz.reshape(-1))
    atom = np.ascontiguousarray(basis.atom, dtype=np.int32)
    lib().orc_one_body_deriv(_bp(basis), _p(atom), na, _p(Z), _p(xyz), _p(S1), _p(T1), _p(V1))
    # stored column-major per coordinate; transpose into numpy row-major views
    return S1.transpose(0, 2, 1), T1.transpose(0, 2, 1), V1.transpose(0, 2, 1)


def grad2e(basis, D, Q, precision=1e-12, want_G1=False, nthreads=None):
    """compute_2body_fock_deriv<1> + the 0.25*G1.D contraction of compute_forces."""
    n = basis.nbf
    na = basis.mol.natom
    D = F(D)
    Qc = np.ascontiguousarray(Q, dtype=np.float64)
    grad = np.zeros(3 * na)
    G1 = np.zeros((3 * na, n, n)) if want_G1 else None
    atom = np.ascontiguousarray(basis.atom, dtype=np.int32)
    lib().orc_grad2e(_bp(basis), _p(atom), na, _p(D), _p(Qc), precision, _p(G1), _p(grad),
                     nthreads or os.cpu_count() or 1)
    return (grad.reshape(na, 3), G1) if want_G1 else grad.reshape(na, 3)


def grad2e_rows(basis, D, Q, precision, s1_begin, s1_step):
    """Time-bounded compute_2body_fock_deriv<1> for the CPU baseline: the
    two-electron gradient terms of the shell rows s1_begin, s1_begin + s1_step,
    ... only (one thread), natom x 3."""
    D = F(D)
    na = basis.mol.natom
    grad = np.zeros(3 * na)
    atom = np.ascontiguousarray(basis.atom, dtype=np.int32)
    Qc = np.ascontiguousarray(Q, dtype=np.float64)
    lib().orc_grad2e_rows(_bp(basis), _p(atom), na, _p(D), _p(Qc), precision, s1_begin, s1_step, _p(grad))
    return grad.reshape(na, 3)


def eri4_deriv_block(basis, s1, s2, s3, s4, center, xyz):
    n = [basis.bf_off[s + 1] - basis.bf_off[s] for s in (s1, s2, s3, s4)]
    out = np.zeros(int(np.prod(n)))
    lib().orc_eri4_deriv_block(_bp(basis), s1, s2, s3, s4, center, xyz, _p(out))
    return out.reshape(n)


def eri3_deriv_block(obs, aux, sa, s2, s3, center, xyz):
    n = [aux.bf_off[sa + 1] - aux.bf_off[sa], obs.bf_off[s2 + 1] - obs.bf_off[s2],
         obs.bf_off[s3 + 1] - obs.bf_off[s3]]
    out = np.zeros(int(np.prod(n)))
    lib().orc_eri3_deriv_block(_bp(obs), _bp(aux), sa, s2, s3, center, xyz, _p(out))
    return out.reshape(n)


def df_grad2e(obs, aux, Cocc, nthreads=None):
    """Two-electron part of the gradient of the density-fitted RHF energy
    (the DF J/K of compute_2body_fock_df, src/fockbuild.cpp:585-660, with
    D = 2 C C^T), natom x 3.  With T = (P|mn), V = (P|Q), d = T.D,
    c = V^-1 d, W_P,ij = sum_Q V^-1_PQ (Q|ij) and
    G_P,mn = sum_ij C_mi C_nj W_P,ij:
      E_J = 1/2 d^T V^-1 d,  E_K = -sum_ij (ij|ij)_fit,
      dE = sum (P|mn)' [c_P D_mn - 2 G_P,mn] + sum (P|Q)' [-1/2 c_P c_Q + sum_ij W_P,ij W_Q,ij],
    the derivative integrals from the oracle's Obara-Saika/HGP derivative
    blocks (orc_df_grad_contract)."""
    n, naux = obs.nbf, aux.nbf
    C = np.asarray(Cocc, dtype=np.float64)
    Tp = eri3(obs, aux)                                   # packed (n(n+1)/2) x naux
    T = np.zeros((naux, n, n))
    iu = np.tril_indices(n)
    T[:, iu[0], iu[1]] = Tp.T
    T[:, iu[1], iu[0]] = Tp.T
    V = eri2(aux)
    D = 2.0 * C @ C.T
    d = np.einsum("pmn,mn->p", T, D)
    c = np.linalg.solve(V, d)
    Tij = np.einsum("mi,pmn,nj->pij", C, T, C)
    W = np.linalg.solve(V, Tij.reshape(naux, -1)).reshape(Tij.shape)
    G = np.einsum("mi,pij,nj->pmn", C, W, C)
    M3 = np.ascontiguousarray(c[:, None, None] * D[None, :, :] - 2.0 * G)
    Wf = W.reshape(naux, -1)
    M2 = np.ascontiguousarray(-0.5 * np.outer(c, c) + Wf @ Wf.T)
    natom = obs.mol.natom
    ob_atom = np.ascontiguousarray(obs.atom, dtype=np.int32)
    ax_atom = np.ascontiguousarray(aux.atom, dtype=np.int32)
    g = np.zeros(3 * natom)
    lib().orc_df_grad_contract(_bp(obs), _bp(aux), _p(ob_atom), _p(ax_atom), natom, _p(M3), _p(M2), _p(g),
                               nthreads or os.cpu_count() or 1)
    return g.reshape(natom, 3)


def df_mp2(obs, aux, C, eps, nocc, nfrozen=0):
    """MP2::dfmp2 (src/mp2.cpp:477-583): the explicit inverse metric (P|Q)^-1
    (:498), the two-step MO transform of the packed (P|mn) (:526-552), and the
    energy sum over i, a, j, b with (ia|jb) = B_ia (P|Q)^-1 B_jb (:554-581),
    vectorised over a, b."""
    n = obs.nbf
    Tp = eri3(obs, aux)                       # (n(n+1)/2) x naux, row x(x+1)/2 + y
    Vinv = np.linalg.inv(eri2(aux))
    x, y = np.tril_indices(n)
    T = np.zeros((n, n, Tp.shape[1]))
    T[x, y] = Tp[x * (x + 1) // 2 + y]
    T[y, x] = Tp[x * (x + 1) // 2 + y]
    Co, Cv = C[:, nfrozen:nocc], C[:, nocc:]
    B = np.einsum("mi,mnP,na->iaP", Co, T, Cv, optimize=True)
    BV = B @ Vinv
    eo, ev = eps[nfrozen:nocc], eps[nocc:C.shape[1]]
    E = 0.0
    for i in range(Co.shape[1]):
        for j in range(Co.shape[1]):
            v = B[i] @ BV[j].T                    # (ia|jb) over (a, b)
            E += np.sum(v * (2.0 * v - v.T) / (eo[i] + eo[j] - ev[:, None] - ev[None, :]))
    return E
