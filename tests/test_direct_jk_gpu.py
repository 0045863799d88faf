"""Direct J/K on the B200 against the FP64 CPU oracle (formJKdirect restated).

Bar: J and K elementwise to 1e-10 (FP64 path), quartet screening identical.
"""
import numpy as np
import pytest

import oracle
from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet, Molecule

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _engine(b):
    from molecular2_b200.engine import IntegralEngine
    return IntegralEngine(b)


def _rand_density(n, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(size=(n, max(1, n // 4)))
    D = C @ C.T / n
    return 0.5 * (D + D.T)


@pytest.mark.parametrize("spherical", [True, False])
def test_schwarz_matches_oracle(spherical):
    mol = geometry.water()
    b = BasisSet(mol, "cc-pvdz", spherical=spherical)
    eng = _engine(b)
    np.testing.assert_allclose(eng.getPrescreen(), oracle.schwarz(b), rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("basis,spherical", [("cc-pvdz", True), ("cc-pvdz", False), ("6-311g**", True),
                                             ("aug-cc-pvdz", True)])
def test_direct_jk_water(basis, spherical):
    mol = geometry.water()
    b = BasisSet(mol, basis, spherical=spherical)
    D = _rand_density(b.nbf, 1)
    eng = _engine(b)
    J, K = eng.jk_direct(D, 1e-12)
    Jr, Kr, cnt = oracle.jk_direct(b, D, oracle.schwarz(b), 1e-12)
    assert np.max(np.abs(J - Jr)) < TOL
    assert np.max(np.abs(K - Kr)) < TOL
    assert eng.last_quartets() == cnt


def test_direct_jk_water_dimer_screened():
    mol = geometry.water_cluster(2, 5.0, seed=3)
    b = BasisSet(mol, "cc-pvdz")
    D = _rand_density(b.nbf, 2) * 1e-3  # small density: screening removes quartets
    eng = _engine(b)
    Q = oracle.schwarz(b)
    for prec in (1e-12, 1e-8):
        J, K = eng.jk_direct(D, prec)
        Jr, Kr, cnt = oracle.jk_direct(b, D, Q, prec)
        assert np.max(np.abs(J - Jr)) < TOL
        assert np.max(np.abs(K - Kr)) < TOL
        assert eng.last_quartets() == cnt


def test_direct_jk_multiplier_and_zero_density():
    mol = geometry.water()
    b = BasisSet(mol, "cc-pvdz")
    eng = _engine(b)
    J, K = eng.jk_direct(np.zeros((b.nbf, b.nbf)))
    assert not J.any() and not K.any()
    D = _rand_density(b.nbf, 5)
    J1, K1 = eng.jk_direct(D, 1e-12, 1.0)
    J2, K2 = eng.jk_direct(D, 1e-12, -0.5)
    np.testing.assert_allclose(J2, -0.5 * J1, atol=1e-14)
    np.testing.assert_allclose(K2, -0.5 * K1, atol=1e-14)


def test_direct_partition_sums_to_full_build():
    """Bra-pair partition of the direct build and the four-index gradient
    (jk_direct_set_partition): three ranks' partial J, K, UHF J/K and
    gradients, computed on one GPU one after another, sum to the whole, the
    quartet counts add up, and the interleaved shares carry nearly equal work."""
    mol = geometry.water_cluster(8, 7.0, seed=8)
    b = BasisSet(mol, "cc-pvdz")
    eng = _engine(b)
    D = _rand_density(b.nbf, 3)
    Db = _rand_density(b.nbf, 4)
    J, K = eng.jk_direct(D, 1e-12)
    q_full = eng.last_quartets()
    Ja, Jb, Ka, Kb = eng.jk_direct_uhf(D, Db, 1e-12)
    W = 0.3 * D
    g_full, _ = eng.compute_forces(D, W)
    R = 3
    sJ, sK, sq = np.zeros_like(J), np.zeros_like(K), []
    su = [np.zeros_like(J) for _ in range(4)]
    sg = np.zeros_like(g_full)
    for r in range(R):
        eng.set_direct_partition(r, R)
        j, k = eng.jk_direct(D, 1e-12)
        sJ += j
        sK += k
        sq.append(eng.last_quartets())
        for acc, part in zip(su, eng.jk_direct_uhf(D, Db, 1e-12)):
            acc += part
        g, _ = eng.compute_forces(D, W)
        sg += g
    eng.set_direct_partition(0, 1)
    scale = max(np.max(np.abs(J)), np.max(np.abs(K)))
    assert np.max(np.abs(sJ - J)) < 1e-11 * scale and np.max(np.abs(sK - K)) < 1e-11 * scale
    for acc, full in zip(su, (Ja, Jb, Ka, Kb)):
        assert np.max(np.abs(acc - full)) < 1e-11 * scale
    assert np.max(np.abs(sg - g_full)) < 1e-10
    assert sum(sq) == q_full
    print(f"quartets per rank {sq} of {q_full}")
    assert max(sq) < 1.1 * q_full / R
    # the SCF and the whole-build calls are not partitioned
    J2, K2 = eng.jk_direct(D, 1e-12)
    assert np.max(np.abs(J2 - J)) < 1e-12 * scale
