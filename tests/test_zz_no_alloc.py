"""jk_direct_noalloc: the direct J/K build for callers that cannot allocate
device memory during a Fock build (its scratch is a fixed device array kept by
the library).

On a fresh engine the no-alloc build runs before anything else has allocated
the engine's own direct-build scratch, and device free memory must not move
across its calls.  Its J and K must equal those of jk_direct_device within the
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


def _noalloc(eng, dD, J, K):
    return eng.lib.jk_direct_noalloc(eng.h, ctypes.c_void_p(dD.data_ptr()), 1e-12, 1.0,
                                     ctypes.c_void_p(J.data_ptr()), ctypes.c_void_p(K.data_ptr()), None)


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from molecular2_b200.engine import IntegralEngine
    mol = geometry.water_cluster(2, 5.0, seed=3)
    b = BasisSet(mol, "cc-pvdz")
    eng = IntegralEngine(b)                 # fresh engine: no direct-build scratch yet
    n = eng.n
    dev = torch.device("cuda", 0)
    dD = torch.from_numpy(np.asfortranarray(_density(n, 11)).T.copy()).to(dev)
    outs = [(torch.full((n, n), float("nan"), dtype=torch.float64, device=dev),
             torch.full((n, n), float("nan"), dtype=torch.float64, device=dev)) for _ in range(3)]
    torch.cuda.synchronize()
    # The first call on a device makes the CUDA driver load the library's code
    # modules it launches (lazy loading), which maps their memory; that is the
    # driver's one-time cost, not an allocation of this entry point.
    assert _noalloc(eng, dD, *outs[0]) == 0, eng.lib.jk_last_error(eng.h).decode()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    for J, K in outs[1:]:
        rc = _noalloc(eng, dD, J, K)
        assert rc == 0, eng.lib.jk_last_error(eng.h).decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0, "jk_direct_noalloc changed device free memory"
    q_noalloc = eng.last_quartets()
    assert q_noalloc > 0
    # the allocating build on the same engine, afterwards
    Jref = torch.empty((n, n), dtype=torch.float64, device=dev)
    Kref = torch.empty_like(Jref)
    eng.jk_direct_device(dD.data_ptr(), Jref.data_ptr(), Kref.data_ptr(), 1e-12, 1.0)
    torch.cuda.synchronize()
    assert eng.last_quartets() == q_noalloc
    for J, K in outs[1:]:
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
    rc = _noalloc(eng, dD, out, out)
    assert rc == 1
    assert "too large" in eng.lib.jk_last_error(eng.h).decode()
    eng.close()
