"""Density-fitted RHF gradient on the B200 (jk_grad_df): the derivative of
the DF energy that jk_df's Fock matrix defines, checked against central
differences of the converged GPU DF-SCF energy, for translational
invariance, and against the 4-index gradient (the two differ only by the
fitting error).

Bars: central differences (step 1e-4 bohr) within 1e-6 Eh/bohr; the sum over
atoms within 1e-9; DF vs 4-index gradient within 1e-3 Eh/bohr; the
two-electron part against the oracle's restatement (oracle.df_grad2e, analytic
derivative integrals) within 1e-9 Eh/bohr.
"""
import numpy as np
import pytest

from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu

CONV = dict(df=True, densconverge=1e-9, enconverge=1e-11, maxiter=100)


def _scf(mol, obs="cc-pvdz", aux="vdz-jkfit"):
    from molecular2_b200.engine import IntegralEngine
    b, a = BasisSet(mol, obs), BasisSet(mol, aux)
    eng = IntegralEngine(b, a)
    r, ex = eng.scf_rhf(mol.nocc, mol.enuc(), want=True, **CONV)
    assert r.converged
    return eng, r, ex


@pytest.mark.parametrize("k,obs,aux", [(1, "cc-pvdz", "vdz-jkfit"), (2, "cc-pvdz", "vdz-jkfit"),
                                       (1, "aug-cc-pvdz", "avdz-jkfit")])
def test_df_gradient_central_differences(k, obs, aux):
    mol = geometry.water() if k == 1 else geometry.water_cluster(k, 5.0, seed=3)
    eng, r, ex = _scf(mol, obs, aux)
    o = mol.nocc
    g, g2 = eng.compute_forces_df(ex["C"][:, :o], ex["eps"][:o])
    assert np.max(np.abs(g.sum(axis=0))) < 1e-9
    h = 1e-4
    coords = [(0, 0), (1, 2), (2, 1)] if k == 1 else [(0, 0), (1, 2), (4, 1), (5, 0)]
    for a, x in coords:
        Es = []
        for sgn in (1, -1):
            m2 = mol.displaced(a, x, sgn * h)
            _, r2, _ = _scf(m2, obs, aux)
            Es.append(r2.energy)
        fd = (Es[0] - Es[1]) / (2 * h)
        assert abs(fd - g[a, x]) < 1e-6, (a, x, fd, g[a, x])


def test_df_gradient_close_to_4index():
    mol = geometry.water_cluster(2, 5.0, seed=3)
    eng, r, ex = _scf(mol)
    o = mol.nocc
    g_df, _ = eng.compute_forces_df(ex["C"][:, :o], ex["eps"][:o])
    C = ex["C"][:, :o]
    W = C @ np.diag(ex["eps"][:o]) @ C.T
    g_4, _ = eng.compute_forces(ex["D"], W)
    assert np.max(np.abs(g_df - g_4)) < 1e-3


@pytest.mark.parametrize("k,obs,aux,storage", [(1, "cc-pvdz", "vdz-jkfit", "unpacked"),
                                               (2, "cc-pvdz", "vdz-jkfit", "unpacked"),
                                               (2, "cc-pvdz", "vdz-jkfit", "tiled"),
                                               (1, "aug-cc-pvdz", "avdz-jkfit", "tiled")])
def test_df_gradient_2e_matches_oracle(k, obs, aux, storage):
    import oracle
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water() if k == 1 else geometry.water_cluster(k, 5.0, seed=3)
    b, a = BasisSet(mol, obs), BasisSet(mol, aux)
    eng = IntegralEngine(b, a)
    eng.set_df_storage(storage)
    r, ex = eng.scf_rhf(mol.nocc, mol.enuc(), want=True, **CONV)
    assert r.converged
    o = mol.nocc
    _, g2 = eng.compute_forces_df(ex["C"][:, :o], ex["eps"][:o])
    g2_ref = oracle.df_grad2e(b, a, ex["C"][:, :o])
    err = np.max(np.abs(g2 - g2_ref))
    print(f"(H2O){k} {obs} {storage}: DF two-electron gradient vs oracle {err:.2e}")
    assert err < 1e-9
