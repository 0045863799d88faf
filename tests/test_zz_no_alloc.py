"""jk_direct_noalloc: the direct J/K build for callers that cannot allocate
device memory during a Fock build (its scratch is a fixed device array kept by
the library).  Its J and K must equal those of jk_direct_device within the
FP64 tolerance of the other direct J/K tests, on two calls in a row (the
second call finds the first call's data in the shared array and must clear
it).  This file is collected last so that a run stopping at the first failure
has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _density(n, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(size=(n, max(1, n // 4)))
    return C @ C.T / n


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water_cluster(2, 5.0, seed=3)
    b = BasisSet(mol, "cc-pvdz")
    eng = IntegralEngine(b)
    n = eng.n
    dev = torch.device("cuda", 0)
    dD = torch.from_numpy(np.asfortranarray(_density(n, 11)).T.copy()).to(dev)
    Jref = torch.empty((n, n), dtype=torch.float64, device=dev)
    Kref = torch.empty_like(Jref)
    eng.jk_direct_device(dD.data_ptr(), Jref.data_ptr(), Kref.data_ptr(), 1e-12, 1.0)
    torch.cuda.synchronize()
    for _ in range(2):
        J = torch.full((n, n), float("nan"), dtype=torch.float64, device=dev)
        K = torch.full_like(J, float("nan"))
        rc = eng.lib.jk_direct_noalloc(eng.h, ctypes.c_void_p(dD.data_ptr()), 1e-12, 1.0,
                                       ctypes.c_void_p(J.data_ptr()), ctypes.c_void_p(K.data_ptr()), None)
        assert rc == 0, eng.lib.jk_last_error(eng.h).decode()
        torch.cuda.synchronize()
        assert float((J - Jref).abs().max()) < TOL
        assert float((K - Kref).abs().max()) < TOL
    eng.close()


def test_noalloc_rejects_a_basis_beyond_its_scratch():
    import torch
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.c20h42()
    b = BasisSet(mol, "6-311g**")          # 632 Cartesian functions > 512
    eng = IntegralEngine(b)
    n = eng.n
    dD = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    out = torch.empty_like(dD)
    rc = eng.lib.jk_direct_noalloc(eng.h, ctypes.c_void_p(dD.data_ptr()), 1e-12, 1.0,
                                   ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert "too large" in eng.lib.jk_last_error(eng.h).decode()
    eng.close()
