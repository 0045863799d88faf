"""Failure detection of the tensor-core kernels: every mbarrier wait gives up
after a bounded number of polls, records the failure and returns, and the
context stays usable.  jk_wait_selftest runs that wait on a barrier that
nothing completes (it must give up) and on one that has completed (it must
not), then a normal DF build runs on the same engine."""
import numpy as np
import pytest

from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives():
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water()
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    eng = IntegralEngine(obs, aux)
    for polls in (1, 64, 4096):
        gave_up, completed_gave_up = eng.wait_selftest(polls)
        assert gave_up and not completed_gave_up
    eng.df_setup()
    rng = np.random.default_rng(1)
    C, _ = np.linalg.qr(rng.normal(size=(obs.nbf, mol.nocc)))
    J64, K64 = eng.jk_df(C, 0)
    J, K = eng.jk_df(C, 1)
    assert np.max(np.abs(K - K64)) < 1e-4 * np.max(np.abs(K64))
    eng.close()
