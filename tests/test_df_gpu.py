"""DF integrals, DF J/K and one-body matrices on the B200 against the oracle.

Bars: (P|mn), (P|Q), S, T, V elementwise 1e-11; DF J, K elementwise 1e-10
(FP64 path, B = (mn|P) L^-T as compute_2body_fock_df builds it).
"""
import numpy as np
import pytest

import oracle
from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu


def _engine(obs, aux=None):
    from molecular2_b200.engine import IntegralEngine
    return IntegralEngine(obs, aux)


def _occ(n, o, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, o)))
    return C


@pytest.mark.parametrize("obs_name,aux_name", [("cc-pvdz", "vdz-jkfit"), ("aug-cc-pvdz", "avdz-jkfit")])
def test_eri3_eri2_water(obs_name, aux_name):
    mol = geometry.water()
    obs, aux = BasisSet(mol, obs_name), BasisSet(mol, aux_name)
    eng = _engine(obs, aux)
    T = eng.compute_eris_3index()
    Tr = oracle.eri3(obs, aux)
    assert np.max(np.abs(T - Tr)) < 1e-11
    V = eng.compute_eris_2index()
    assert np.max(np.abs(V - oracle.eri2(aux))) < 1e-11


def test_df_jk_water_dimer():
    mol = geometry.water_cluster(2, 5.0, seed=3)
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    eng = _engine(obs, aux)
    eng.df_setup()
    B = oracle.df_B(oracle.eri3(obs, aux), oracle.eri2(aux))
    C = _occ(obs.nbf, mol.nocc, 4)
    J, K = eng.jk_df(C)
    Jr, Kr = oracle.df_jk(B, C)
    assert np.max(np.abs(J - Jr)) < 1e-10
    assert np.max(np.abs(K - Kr)) < 1e-10


def test_df_before_setup_is_a_state_error():
    from molecular2_b200.engine import JKError
    mol = geometry.water()
    eng = _engine(BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit"))
    with pytest.raises(JKError) as ei:
        eng.jk_df(_occ(eng.n, 5, 1))
    assert ei.value.code == 4


@pytest.mark.parametrize("spherical", [True, False])
def test_one_body(spherical):
    mol = geometry.water_cluster(2, 5.0, seed=3)
    b = BasisSet(mol, "aug-cc-pvdz", spherical=spherical)
    eng = _engine(b)
    S, T, V = eng.one_body()
    Sr, Tr, Vr = oracle.one_body(b)
    for X, Xr in ((S, Sr), (T, Tr), (V, Vr)):
        assert np.max(np.abs(X - Xr)) < 1e-11


def test_one_body_on_reused_memory():
    """One-body matrices are complete on device memory that held other data:
    shell pairs with no significant primitive product are written as zeros."""
    import torch
    from molecular2_b200.engine import IntegralEngine
    junk = torch.full((1 << 27,), float("nan"), dtype=torch.float64, device="cuda")
    del junk
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    mol = geometry.water_cluster(8, 7.0, seed=8)
    b = BasisSet(mol, "cc-pvdz")
    S, T, V = IntegralEngine(b).one_body()
    So, To, Vo = oracle.one_body(b)
    assert np.max(np.abs(S - So)) < 1e-12
    assert np.max(np.abs(T - To)) < 1e-11
    assert np.max(np.abs(V - Vo)) < 1e-10


@pytest.mark.parametrize("prec_mode", [0, 1])
def test_df_slices_sum_to_full_build(prec_mode):
    """jk_df_set_range: the partial J, K of fitted-index slices covering the
    fitting basis add up to the one-engine build (the aux-sharded build that
    bench.py runs over ranks, here two slices on one GPU)."""
    from molecular2_b200.engine import IntegralEngine
    from molecular2_b200.sharding import aux_ranges
    mol = geometry.water_cluster(2, 5.0, seed=3)
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    rng = np.random.default_rng(2)
    C = np.linalg.qr(rng.normal(size=(obs.nbf, mol.nocc)))[0]
    full = IntegralEngine(obs, aux)
    full.df_setup()
    J1, K1 = full.jk_df(C, prec_mode)
    J2, K2 = np.zeros_like(J1), np.zeros_like(K1)
    for k0, k1 in aux_ranges(aux.nbf, 2):
        e = IntegralEngine(obs, aux)
        e.set_df_range(k0, k1)
        e.df_setup()
        J, K = e.jk_df(C, prec_mode)
        J2 += J
        K2 += K
    tol = 1e-11 if prec_mode == 0 else 5e-5 * np.abs(K1).max()
    assert np.max(np.abs(J2 - J1)) < tol
    assert np.max(np.abs(K2 - K1)) < tol
