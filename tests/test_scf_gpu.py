"""Whole RHF SCF on the B200 against the oracle's SCF and molecular2's recorded energy.

Bars: FP64 energies to 1e-8 Eh.  The GPU J/K accumulate with FP64 atomics,
whose order varies from run to run, so the energy carries ~1e-12 Eh of noise:
the convergence thresholds stay above it (|dE| < 1e-10 Eh).
"""
CONV = dict(densconverge=1e-9, enconverge=1e-10, maxiter=80)
import json
import os

import numpy as np
import pytest

import oracle
from oracle.scf import RHF
from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet, Molecule

pytestmark = pytest.mark.gpu

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))


def _engine(obs, aux=None):
    from molecular2_b200.engine import IntegralEngine
    return IntegralEngine(obs, aux)


def test_direct_scf_reproduces_h2otest_energy():
    """test/h2otest.out_1:124 (Cartesian cc-pVDZ) through the GPU J/K and SCF."""
    g = PINS["h2otest_geometry_bohr"]
    mol = Molecule([x[0] for x in g], [x[1:] for x in g], angstrom=False)
    b = BasisSet(mol, "cc-pvdz", spherical=False)
    r, _ = _engine(b).scf_rhf(mol.nocc, mol.enuc(), **CONV)
    assert r.converged
    assert abs(r.energy - PINS["h2otest_energy"]) < 1e-8


def test_direct_scf_matches_oracle_water():
    mol = geometry.water()
    b = BasisSet(mol, "cc-pvdz")
    r, _ = _engine(b).scf_rhf(mol.nocc, mol.enuc(), **CONV)
    ref = RHF(b, guess="hcore", **CONV)
    E = ref.run()
    assert r.converged and ref.converged
    assert abs(r.energy - E) < 1e-8


def test_df_scf_matches_oracle_water_dimer():
    mol = geometry.water_cluster(2, 5.0, seed=3)
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    r, _ = _engine(obs, aux).scf_rhf(mol.nocc, mol.enuc(), df=True, **CONV)
    B = oracle.df_B(oracle.eri3(obs, aux), oracle.eri2(aux))
    ref = RHF(obs, guess="hcore", df=lambda C: oracle.df_jk(B, C), **CONV)
    E = ref.run()
    assert r.converged and ref.converged
    assert abs(r.energy - E) < 1e-8
