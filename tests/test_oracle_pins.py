"""The oracle against molecular2's recorded outputs and against mathematics.

molecular2 has no test suite; its only expected values are the hand-run
outputs in test/ (copied into tests/golden/reference_pins.json by
tests/golden/make_golden.py).  These pin the CPU oracle that every GPU
parity test compares with.
"""
import json
import os

import numpy as np
import pytest

import oracle
from oracle.scf import RHF
from molecular2_b200.basis import BasisSet, Molecule

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))


def _mol(key, angstrom):
    g = PINS[key]
    return Molecule([x[0] for x in g], [x[1:] for x in g], angstrom=angstrom)


def test_boys_against_mpmath():
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 40
    for T in [0.0, 1e-8, 0.3, 1.7, 7.5, 19.9, 39.9, 40.1, 75.0, 400.0]:
        F = oracle.boys(12, T)
        for m in range(13):
            if T == 0.0:
                ref = mpmath.mpf(1) / (2 * m + 1)
            else:
                ref = mpmath.quad(lambda t: t ** (2 * m) * mpmath.exp(-T * t * t), [0, 1])
            assert abs(F[m] - float(ref)) <= 2e-14 * float(ref), (T, m)


def test_solid_harmonics_orthonormal():
    # rows are unit-normalised and mutually orthogonal in the x^l-normalised
    # Cartesian metric
    from math import prod

    def dfact(n):
        return prod(range(n, 0, -2)) if n > 0 else 1

    for l in range(2, 5):
        R = oracle.solid_harmonics(l)
        comps = [(a, b, l - a - b) for a in range(l, -1, -1) for b in range(l - a, -1, -1)]
        M = np.zeros((len(comps), len(comps)))
        for i, ci in enumerate(comps):
            for j, cj in enumerate(comps):
                s = [ci[k] + cj[k] for k in range(3)]
                if all(x % 2 == 0 for x in s):
                    M[i, j] = dfact(s[0] - 1) * dfact(s[1] - 1) * dfact(s[2] - 1) / dfact(2 * l - 1)
        np.testing.assert_allclose(R @ M @ R.T, np.eye(2 * l + 1), atol=1e-13)


def test_overlap_diagonal_is_one():
    mol = _mol("h2otest_geometry_bohr", False)
    for sph in (False, True):
        S, _, _ = oracle.one_body(BasisSet(mol, "aug-cc-pvdz", spherical=sph))
        d = np.diag(S)
        if sph:
            np.testing.assert_allclose(d, 1.0, atol=1e-13)
        else:
            assert np.all(d <= 1.0 + 1e-13) and np.max(d) == pytest.approx(1.0)


def test_cdthe_known_answers():
    """test/cdthe.ints: He with 5 uncontracted s functions, printed by
    IntegralEngine::printERI with its symmetry weights (src/integrals.cpp:203-233)."""
    mol = Molecule(["he"], [[0, 0, 0]], angstrom=False)
    b = BasisSet(mol, "test")
    eri = oracle.eri_full(b)
    for c1, c2, c3, c4, printed in PINS["cdthe_weighted_eris"]:
        c1, c2, c3, c4 = c1 - 1, c2 - 1, c3 - 1, c4 - 1
        w = 0.125
        if c1 != c2:
            w *= 2
        if c3 != c4:
            w *= 2
        if (c1 + c2) != (c3 + c4):
            w *= 2
        elif c1 != c3 and c1 != c4:
            w *= 2
        elif c2 != c3 and c2 != c4:
            w *= 2
        val = w * eri[c4, c3, c2, c1]
        assert val == pytest.approx(printed, rel=6e-6, abs=1e-6), (c1, c2, c3, c4)


def test_h2otest_energy_cartesian():
    """test/h2otest.out_1:124: RHF/cc-pVDZ (Cartesian d) = -75.990178761701 Eh."""
    mol = _mol("h2otest_geometry_bohr", False)
    b = BasisSet(mol, "cc-pvdz", spherical=False)
    r = RHF(b, minbasis=BasisSet(mol, "sto-3g"), densconverge=1e-10, enconverge=1e-12, maxiter=60)
    E = r.run()
    assert r.converged
    assert abs(E - PINS["h2otest_energy"]) < 1e-8


def test_h2otest_gradient_weak_pin_and_fd():
    """test/h2otest.opt: gradient printed by the optimiser (spherical cc-pVDZ,
    energy -75.9898).  Printed to ~6 digits from a loosely converged run, so the
    pin is 3e-5; the analytic gradient is checked tightly against central
    differences of the oracle energy."""
    mol = _mol("h2otest_geometry_bohr", False)
    b = BasisSet(mol, "cc-pvdz", spherical=True)
    r = RHF(b, minbasis=BasisSet(mol, "sto-3g"), densconverge=1e-10, enconverge=1e-12, maxiter=60)
    r.run()
    g = r.forces()
    ref = PINS["h2otest_gradient_first"]
    for a in range(3):
        for k, c in enumerate("XYZ"):
            assert abs(g[a, k] - ref[f"{c}{a}"]) < 3e-5
    h = 1e-4
    for a, x in [(0, 1), (1, 0), (2, 1)]:
        Es = []
        for s in (1, -1):
            m2 = mol.displaced(a, x, s * h)
            r2 = RHF(b.with_geometry(m2), minbasis=BasisSet(m2, "sto-3g"), densconverge=1e-11,
                     enconverge=1e-13, maxiter=80)
            Es.append(r2.run())
        assert abs((Es[0] - Es[1]) / (2 * h) - g[a, x]) < 5e-7


def test_benzene_energy_cartesian():
    """test/benzene.out_1:104: RHF/cc-pVDZ benzene (Cartesian d) = -230.723052736 Eh."""
    mol = _mol("benzene_geometry_angstrom", True)
    b = BasisSet(mol, "cc-pvdz", spherical=False)
    r = RHF(b, minbasis=BasisSet(mol, "sto-3g"), densconverge=1e-8, enconverge=1e-10)
    E = r.run()
    assert r.converged
    assert abs(E - PINS["benzene_energy"]) < 2e-9
