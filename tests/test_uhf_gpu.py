"""Unrestricted (UHF) J/K: UnrestrictedFock::formJKdirect and ::formJKdf
(molecular2 src/fockbuild.cpp:266-372).

The direct build digests both spin densities from one pass over the screened
quartets (screen on Da + Db) and is compared elementwise (1e-10) with the
oracle's restatement, quartet count included; it must also equal two RHF-style
builds when the screen admits the same quartets (Da = Db).  The DF build is
compute_2body_fock_df per spin over the same fitted tensor, compared with the
oracle (1e-10 FP64; the mixed build within 1e-4 of the largest element, for
core-Hamiltonian orbitals), for an open-shell case with na != nb and for
nb = 0.
"""
import numpy as np
import pytest

from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet, Molecule

pytestmark = pytest.mark.gpu


def _orbitals(n, no, seed):
    C, _ = np.linalg.qr(np.random.default_rng(seed).normal(size=(n, no)))
    return C


def test_uhf_direct_matches_oracle():
    import oracle
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water_cluster(2, 5.0, seed=3)
    b = BasisSet(mol, "cc-pvdz")
    n = b.nbf
    Ca, Cb = _orbitals(n, 11, 1), _orbitals(n, 9, 2)
    Da, Db = Ca @ Ca.T, Cb @ Cb.T
    eng = IntegralEngine(b)
    out = eng.jk_direct_uhf(Da, Db, 1e-12, 1.0)
    q = eng.last_quartets()
    *ref, cnt = oracle.jk_direct_uhf(b, Da, Db, oracle.schwarz(b), 1e-12, 1.0)
    errs = [np.max(np.abs(x - y)) for x, y in zip(out, ref)]
    print("UHF direct vs oracle (Ja, Jb, Ka, Kb):", " ".join(f"{e:.2e}" for e in errs), "quartets", q, cnt)
    assert max(errs) < 1e-10
    assert q == cnt
    # equal spin densities: the same quartets as an RHF build of that density
    Ja, Jb, Ka, Kb = eng.jk_direct_uhf(Da, Da, 1e-12, 1.0)
    J2, K2 = eng.jk_direct(2 * Da, 1e-12)
    assert np.max(np.abs(Ja + Jb - J2)) < 1e-10 and np.max(np.abs(Ka + Kb - K2)) < 1e-10
    eng.close()


@pytest.mark.parametrize("storage", ["unpacked", "tiled"])
def test_uhf_df_matches_oracle(storage):
    import oracle
    from molecular2_b200.engine import IntegralEngine
    # OH radical pair: an open shell with na = nb + 1 per radical
    mol = Molecule(["o", "h", "o", "h"], [[0, 0, 0], [0, 0, 0.97], [2.8, 0.3, 0.2], [2.9, 0.4, 1.15]])
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    n = obs.nbf
    na, nb = 9, 7
    eng = IntegralEngine(obs, aux)
    eng.set_df_storage(storage)
    eng.df_setup()
    # core-Hamiltonian orbitals (physical, unlike random orthonormal columns
    # whose X = B C cancels to far below the split-BF16 product error)
    import scipy.linalg as sl
    S, T, V = eng.one_body()
    _, C = sl.eigh(T + V, S)
    Ca, Cb = C[:, :na], C[:, :nb]
    B = oracle.df_B(oracle.eri3(obs, aux), oracle.eri2(aux))
    refa, refb = oracle.df_jk(B, Ca), oracle.df_jk(B, Cb)
    Ja, Jb, Ka, Kb = eng.jk_df_uhf(Ca, Cb, 0, multiplier=0.5)
    errs = [np.max(np.abs(x - 0.5 * y)) for x, y in zip((Ja, Ka, Jb, Kb), (*refa, *refb))]
    print(f"UHF DF ({storage}) vs oracle:", " ".join(f"{e:.2e}" for e in errs))
    assert max(errs) < 1e-10
    Ja, Jb, Ka, Kb = eng.jk_df_uhf(Ca, Cb, 1)
    rel = max(np.max(np.abs(x - y)) / np.max(np.abs(y)) for x, y in zip((Ja, Ka, Jb, Kb), (*refa, *refb)))
    assert rel < 1e-4
    Ja, Jb, Ka, Kb = eng.jk_df_uhf(Ca, Cb[:, :0], 0)
    assert np.max(np.abs(Ja - refa[0])) < 1e-10 and not Jb.any() and not Kb.any()
    eng.close()
