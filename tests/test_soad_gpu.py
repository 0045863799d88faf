"""SOAD guess on the B200: jk_fock_general against the oracle's restatement of
Fock::compute_2body_fock_general (src/fockbuild.cpp:477-583), and the SCF
started from the SOAD Fock (the reference's default guess, src/fock.cpp:174-225)
against the core-Hamiltonian start.

Bars: G elementwise within 1e-10; energies within 1e-10 Eh.
"""
import numpy as np
import pytest

import oracle
from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet, sto3g_density

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("basis,spherical,k", [("cc-pvdz", True, 1), ("cc-pvdz", False, 1), ("6-311g**", True, 2)])
def test_fock_general_matches_oracle(basis, spherical, k):
    from molecular2_b200.engine import fock_general
    mol = geometry.water() if k == 1 else geometry.water_cluster(k, 5.0, seed=3)
    obs = BasisSet(mol, basis, spherical=spherical)
    mb = BasisSet(mol, "sto-3g", spherical=False)
    D = sto3g_density(mol)
    G = fock_general(obs, mb, D)
    Gr = oracle.fock_general(obs, mb, D, shelldiag=True)
    assert np.max(np.abs(G - Gr)) < 1e-10
    assert np.max(np.abs(G - G.T)) < 1e-12


def test_fock_general_full_density():
    """shelldiag = 0: a general (not shell-diagonal) density."""
    from molecular2_b200.engine import fock_general
    mol = geometry.water()
    obs = BasisSet(mol, "cc-pvdz")
    mb = BasisSet(mol, "sto-3g", spherical=False)
    rng = np.random.default_rng(5)
    A = rng.normal(size=(mb.nbf, mb.nbf))
    D = A @ A.T / mb.nbf
    G = fock_general(obs, mb, D, shelldiag=False)
    Gr = oracle.fock_general(obs, mb, D, shelldiag=False)
    assert np.max(np.abs(G - Gr)) < 1e-10


def test_scf_soad_guess():
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water_cluster(2, 5.0, seed=3)
    b = BasisSet(mol, "cc-pvdz")
    eng = IntegralEngine(b)
    conv = dict(densconverge=1e-9, enconverge=1e-10, maxiter=80)
    r_core, _ = eng.scf_rhf(mol.nocc, mol.enuc(), **conv)
    r_soad, _ = eng.scf_rhf(mol.nocc, mol.enuc(), guess="soad", **conv)
    assert r_core.converged and r_soad.converged
    assert abs(r_core.energy - r_soad.energy) < 1e-10
    assert r_soad.iterations <= r_core.iterations
