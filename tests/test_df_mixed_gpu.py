"""Split-BF16 tensor-core DF J/K (prec_mode 1) against the FP64 path.

The FP64 GPU path is pinned to the oracle elementwise (test_df_gpu.py); the
mixed path is checked against it.  Stated bar: every element of J and K
within 1e-4 of the largest element (the split products carry ~16 bits per
operand with FP32 accumulation), and the SCF energy of a mixed run (mixed
builds, then FP64 builds to convergence) within 1e-6 Eh of the FP64 SCF.
"""
import numpy as np
import pytest

from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu

REL = 1e-4


def _engine(obs, aux):
    from molecular2_b200.engine import IntegralEngine
    return IntegralEngine(obs, aux)


def _occ(n, o, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, o)))
    return C


@pytest.mark.parametrize("k,box,seed", [(2, 5.0, 3), (16, 9.0, 16)])
def test_mixed_jk_matches_fp64(k, box, seed):
    mol = geometry.water_cluster(k, box, seed=seed)
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    eng = _engine(obs, aux)
    eng.df_setup()
    C = _occ(obs.nbf, mol.nocc, 7)
    J64, K64 = eng.jk_df(C, 0)
    J, K = eng.jk_df(C, 1)
    ej = np.max(np.abs(J - J64)) / np.max(np.abs(J64))
    ek = np.max(np.abs(K - K64)) / np.max(np.abs(K64))
    print(f"(H2O){k}: mixed vs FP64 max rel err J {ej:.2e} K {ek:.2e}")
    assert ej < REL and ek < REL
    # a second call reuses the split copies and must agree with the first
    J2, K2 = eng.jk_df(C, 1)
    assert np.max(np.abs(J2 - J)) < 1e-6 * np.max(np.abs(J64))
    assert np.max(np.abs(K2 - K)) < 1e-6 * np.max(np.abs(K64))


def test_mixed_scf_energy_within_1e6():
    mol = geometry.water_cluster(4, 6.0, seed=5)
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    eng = _engine(obs, aux)
    r64, _ = eng.scf_rhf(mol.nocc, mol.enuc(), df=True, densconverge=1e-7, enconverge=1e-9, maxiter=80)
    rmx, _ = eng.scf_rhf(mol.nocc, mol.enuc(), df=True, prec_mode=1, densconverge=1e-7, enconverge=1e-9,
                         maxiter=80)
    print(f"SCF FP64 {r64.energy:.10f} ({r64.iterations} it), mixed {rmx.energy:.10f} "
          f"({rmx.iterations} it, {rmx.mixed_builds} mixed builds)")
    assert r64.converged and rmx.converged
    assert rmx.mixed_builds > 0
    assert abs(rmx.energy - r64.energy) < 1e-6
