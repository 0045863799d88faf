"""Tiled DF storage (the layout that carries (H2O)64 / aug-cc-pVDZ): B_K on and
below the diagonal of a 128 x 128 function tiling in split BF16, the FP64
build streaming (P|mn) tile pairs.

Checks, on aug-cc-pVDZ + AVDZ-JKFIT water clusters with two and three tile
rows (so that off-diagonal tiles and the transposed, MN-major operand path are
exercised):
  * the FP64 build against the oracle's compute_2body_fock_df restatement,
    every element of J and K within 1e-10;
  * the FP64 build against the unpacked FP64 path, 1e-10;
  * the mixed build against the FP64 build, every element within 1e-4 of the
    largest (the bar of the unpacked mixed path), and repeatable;
  * an SCF on tiled storage reaching the unpacked SCF energy within 1e-8 Eh.
"""
import numpy as np
import pytest

from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu

REL = 1e-4


def _occ(n, o, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, o)))
    return C


def _engine(mol, storage):
    from molecular2_b200.engine import IntegralEngine
    obs, aux = BasisSet(mol, "aug-cc-pvdz"), BasisSet(mol, "avdz-jkfit")
    eng = IntegralEngine(obs, aux)
    eng.set_df_storage(storage)
    eng.df_setup()
    assert eng.df_storage == storage
    return eng, obs, aux


def test_tiled_fp64_matches_oracle():
    import oracle
    mol = geometry.water_cluster(4, 6.0, seed=4)          # n = 164: two tile rows
    eng, obs, aux = _engine(mol, "tiled")
    C = _occ(obs.nbf, mol.nocc, 3)
    J, K = eng.jk_df(C, 0)
    B = oracle.df_B(oracle.eri3(obs, aux), oracle.eri2(aux))
    Jr, Kr = oracle.df_jk(B, C)
    ej, ek = np.max(np.abs(J - Jr)), np.max(np.abs(K - Kr))
    print(f"(H2O)4 aug tiled FP64 vs oracle: J {ej:.2e} K {ek:.2e}")
    assert ej < 1e-10 and ek < 1e-10
    Jm, Km = eng.jk_df(C, 1)
    em = max(np.max(np.abs(Jm - Jr)) / np.max(np.abs(Jr)), np.max(np.abs(Km - Kr)) / np.max(np.abs(Kr)))
    print(f"(H2O)4 aug tiled mixed vs oracle: max rel {em:.2e}")
    assert em < REL
    eng.close()


def test_tiled_matches_unpacked_and_mixed_is_repeatable():
    mol = geometry.water_cluster(8, 7.0, seed=8)          # n = 328: three tile rows
    et, obs, _ = _engine(mol, "tiled")
    eu, _, _ = _engine(mol, "unpacked")
    C = _occ(obs.nbf, mol.nocc, 5)
    Jt, Kt = et.jk_df(C, 0)
    Ju, Ku = eu.jk_df(C, 0)
    assert np.max(np.abs(Jt - Ju)) < 1e-10 and np.max(np.abs(Kt - Ku)) < 1e-10
    Jm, Km = et.jk_df(C, 1)
    ej = np.max(np.abs(Jm - Ju)) / np.max(np.abs(Ju))
    ek = np.max(np.abs(Km - Ku)) / np.max(np.abs(Ku))
    print(f"(H2O)8 aug tiled mixed vs FP64: J {ej:.2e} K {ek:.2e}")
    assert ej < REL and ek < REL
    Jm2, Km2 = et.jk_df(C, 1)
    assert np.max(np.abs(Jm2 - Jm)) < 1e-6 * np.max(np.abs(Ju))
    assert np.max(np.abs(Km2 - Km)) < 1e-6 * np.max(np.abs(Ku))
    et.close()
    eu.close()


def test_tiled_scf_matches_unpacked():
    mol = geometry.water_cluster(4, 6.0, seed=5)
    et, _, _ = _engine(mol, "tiled")
    eu, _, _ = _engine(mol, "unpacked")
    kw = dict(df=True, densconverge=1e-7, enconverge=1e-9, maxiter=80)
    rt, _ = et.scf_rhf(mol.nocc, mol.enuc(), **kw)
    ru, _ = eu.scf_rhf(mol.nocc, mol.enuc(), **kw)
    print(f"SCF tiled {rt.energy:.10f} ({rt.iterations} it), unpacked {ru.energy:.10f} ({ru.iterations} it)")
    assert rt.converged and ru.converged
    assert abs(rt.energy - ru.energy) < 1e-8
    et.close()
    eu.close()


def test_tiled_multiblock_schedules_match_oracle():
    """Several fitted-function blocks in the mixed build and several occupied
    slices (integral passes) in the FP64 build, on a system small enough for
    the oracle."""
    import oracle
    mol = geometry.water_cluster(4, 6.0, seed=4)
    eng, obs, aux = _engine(mol, "tiled")
    eng.set_tiled_blocks(waux_max=130, oc_max=7)          # 5 blocks of <= 130 of 600, 3 slices of 20
    C = _occ(obs.nbf, mol.nocc, 11)
    B = oracle.df_B(oracle.eri3(obs, aux), oracle.eri2(aux))
    Jr, Kr = oracle.df_jk(B, C)
    J, K = eng.jk_df(C, 0)
    assert np.max(np.abs(J - Jr)) < 1e-10 and np.max(np.abs(K - Kr)) < 1e-10
    Jm, Km = eng.jk_df(C, 1)
    em = max(np.max(np.abs(Jm - Jr)) / np.max(np.abs(Jr)), np.max(np.abs(Km - Kr)) / np.max(np.abs(Kr)))
    print(f"(H2O)4 aug tiled, 5 blocks / 3 slices: mixed max rel {em:.2e}")
    assert em < REL
    eng.close()


def test_tiled_gradient_matches_unpacked():
    """The DF gradient streamed from tiled storage (metric only, no fitted
    tensor kept) equals the unpacked DF gradient, which the finite-difference
    tests pin."""
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water_cluster(3, 5.5, seed=2)
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    eu = IntegralEngine(obs, aux)
    eu.set_df_storage("unpacked")
    r, ex = eu.scf_rhf(mol.nocc, mol.enuc(), df=True, densconverge=1e-8, enconverge=1e-10, maxiter=80, want=True)
    assert r.converged
    C = ex["C"][:, :mol.nocc]
    eps = ex["eps"][:mol.nocc]
    gu = eu.compute_forces_df(C, eps)
    et = IntegralEngine(obs, aux)
    et.set_df_storage("tiled")
    et.set_tiled_blocks(oc_max=6)                          # two occupied slices
    gt = et.compute_forces_df(C, eps)
    gu, gt = np.asarray(gu[0] if isinstance(gu, tuple) else gu), np.asarray(gt[0] if isinstance(gt, tuple) else gt)
    err = np.max(np.abs(gt - gu))
    print(f"tiled vs unpacked DF gradient: max |dg| {err:.2e}")
    assert err < 1e-9
    eu.close()
    et.close()


def test_tiled_odd_blocks():
    """An odd fitted-function block with one 160-orbital half (X rows that end
    inside a 64-wide k block) against the FP64 build."""
    mol = geometry.water_cluster(4, 6.0, seed=4)
    eng, obs, _ = _engine(mol, "tiled")
    C = _occ(obs.nbf, mol.nocc, 13)
    J64, K64 = eng.jk_df(C, 0)
    eng.set_tiled_blocks(waux_max=127)                      # blocks of 127, 127, 127, 127, 92 of 600
    Jm, Km = eng.jk_df(C, 1)
    em = max(np.max(np.abs(Jm - J64)) / np.max(np.abs(J64)), np.max(np.abs(Km - K64)) / np.max(np.abs(K64)))
    assert em < REL
    eng.close()
