"""DF-MP2 correlation energy (MP2::dfmp2, molecular2 src/mp2.cpp:477-583)
against the oracle's restatement (explicit inverse metric, two-step MO
transform, energy loop), at the DF-SCF orbitals, all-electron and with the
oxygen 1s orbitals frozen (molecular2's withcore = false), within 1e-10 Eh."""
import numpy as np
import pytest

from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k,nfrozen_per_water", [(1, 0), (2, 1), (4, 1)])
def test_df_mp2_matches_oracle(k, nfrozen_per_water):
    import oracle
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water() if k == 1 else geometry.water_cluster(k, 5.0 + k, seed=k)
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    eng = IntegralEngine(obs, aux)
    eng.set_df_storage("unpacked")
    r, ex = eng.scf_rhf(mol.nocc, mol.enuc(), df=True, densconverge=1e-8, enconverge=1e-10, maxiter=80, want=True)
    assert r.converged
    nf = nfrozen_per_water * k
    e_gpu = eng.df_mp2(ex["C"], ex["eps"], mol.nocc, nf)
    e_ref = oracle.df_mp2(obs, aux, ex["C"], ex["eps"], mol.nocc, nf)
    print(f"(H2O){k} DF-MP2 (frozen {nf}): GPU {e_gpu:.12f} oracle {e_ref:.12f} diff {e_gpu - e_ref:.2e}")
    assert e_gpu < 0.0
    assert abs(e_gpu - e_ref) < 1e-10
    eng.close()
