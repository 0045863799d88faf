"""Host side of the aux-sharded DF J/K build on two gloo ranks (CPU): the
fitted-index ranges cover the fitting basis without overlap, and the sum of
the per-rank partial J, K over the all-reduce equals the one-rank build.
The partial builds here are the oracle's restatement of compute_2body_fock_df
(src/fockbuild.cpp:621-659) over each rank's K range, standing in for the GPU
engine; the GPU slice itself is checked in test_df_gpu.py."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from molecular2_b200.sharding import aux_ranges, allreduce_jk


def test_aux_ranges_cover():
    for naux, world in [(1856, 2), (1856, 8), (928, 3), (10, 4), (7, 1)]:
        r = aux_ranges(naux, world)
        assert r[0][0] == 0 and r[-1][1] == naux
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        assert all(k0 % 4 == 0 or k0 == naux for k0, _ in r)
        sizes = [k1 - k0 for k0, k1 in r]
        assert max(sizes) - min(sizes) <= 4


def _worker(rank, world, port, B, C, out):
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        k0, k1 = aux_ranges(B.shape[1], world)[rank]
        J, K = oracle.df_jk(B, C, (k0, k1), nthreads=1)
        J, K = torch.from_numpy(np.ascontiguousarray(J)), torch.from_numpy(np.ascontiguousarray(K))
        allreduce_jk(J, K)
        if rank == 0:
            np.save(out, np.stack([J.numpy(), K.numpy()]))
    finally:
        dist.destroy_process_group()


def test_sharded_jk_two_gloo_ranks(tmp_path):
    import oracle
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    mol = geometry.water()
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    B = oracle.df_B(oracle.eri3(obs, aux), oracle.eri2(aux))
    rng = np.random.default_rng(1)
    C = np.asfortranarray(np.linalg.qr(rng.normal(size=(obs.nbf, mol.nocc)))[0])
    out = str(tmp_path / "jk.npy")
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_worker, args=(2, port, B, C, out), nprocs=2, start_method="spawn")
    J2, K2 = np.load(out)
    J1, K1 = oracle.df_jk(B, C, nthreads=1)
    assert np.max(np.abs(J2 - J1)) < 1e-12
    assert np.max(np.abs(K2 - K1)) < 1e-12


# ---------------------------------------------------------------- direct J/K and gradient
class _OracleDirectEngine:
    """Duck-typed stand-in for IntegralEngine on CPU: its partial direct build
    is the oracle's restatement of Fock::formJKdirect over the shell rows s1 of
    this rank's interleaved share (the GPU engine shares the bra pairs of every
    class the same way; its partial builds are checked on the GPU in
    test_direct_jk_gpu.py)."""

    def __init__(self, basis):
        import oracle
        self.basis, self.Q = basis, oracle.schwarz(basis)
        self.rank, self.world = 0, 1

    def set_direct_partition(self, rank, world):
        self.rank, self.world = rank, world

    def jk_direct(self, D, precision=1e-12, multiplier=1.0):
        import oracle
        from molecular2_b200.sharding import interleaved_share
        n = self.basis.nbf
        J, K = np.zeros((n, n)), np.zeros((n, n))
        for s1 in interleaved_share(self.Q.shape[0], self.rank, self.world):
            j, k, _ = oracle.jk_direct_rows(self.basis, D, self.Q, precision, s1, s1 + 1)
            J += j
            K += k
        return multiplier * J, multiplier * K


def _direct_worker(rank, world, port, D, out):
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    from molecular2_b200.sharding import direct_jk_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        eng = _OracleDirectEngine(BasisSet(geometry.water(), "cc-pvdz"))
        J, K = direct_jk_sharded(eng, D)
        if rank == 0:
            np.save(out, np.stack([J, K]))
    finally:
        dist.destroy_process_group()


def test_interleaved_share_cover():
    from molecular2_b200.sharding import interleaved_share
    for n, world in [(10, 3), (7, 7), (3, 5), (100, 8)]:
        got = sorted(i for r in range(world) for i in interleaved_share(n, r, world))
        assert got == list(range(n))
    with pytest.raises(ValueError):
        interleaved_share(5, 2, 2)


def test_direct_jk_sharded_two_gloo_ranks(tmp_path):
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    basis = BasisSet(geometry.water(), "cc-pvdz")
    rng = np.random.default_rng(2)
    C = np.linalg.qr(rng.normal(size=(basis.nbf, 5)))[0]
    D = np.asfortranarray(2.0 * C @ C.T)
    out = str(tmp_path / "djk.npy")
    port = 29700 + os.getpid() % 1000
    mp.start_processes(_direct_worker, args=(2, port, D, out), nprocs=2, start_method="spawn")
    J2, K2 = np.load(out)
    J1, K1 = _OracleDirectEngine(basis).jk_direct(D)
    assert np.max(np.abs(J2 - J1)) < 1e-12
    assert np.max(np.abs(K2 - K1)) < 1e-12
    assert np.max(np.abs(J1)) > 1e-3


class _SplitGradientEngine:
    """Duck-typed engine whose partial gradient is the rank's share of a fixed
    per-row decomposition of a known gradient (the GPU partition itself is
    checked in test_direct_jk_gpu.py)."""

    def __init__(self, parts):
        self.parts = parts  # rows x natom x 3
        self.rank, self.world = 0, 1

    def set_direct_partition(self, rank, world):
        self.rank, self.world = rank, world

    def compute_forces(self, D, W):
        from molecular2_b200.sharding import interleaved_share
        g = sum(self.parts[i] for i in interleaved_share(len(self.parts), self.rank, self.world))
        return g, g


def _gradient_worker(rank, world, port, parts, out):
    from molecular2_b200.sharding import gradient_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = gradient_sharded(_SplitGradientEngine(parts), None, None)
        if rank == 0:
            np.save(out, g)
    finally:
        dist.destroy_process_group()


def test_gradient_sharded_three_gloo_ranks(tmp_path):
    parts = np.random.default_rng(3).normal(size=(10, 4, 3))
    out = str(tmp_path / "g.npy")
    port = 29900 + os.getpid() % 100
    mp.start_processes(_gradient_worker, args=(3, port, parts, out), nprocs=3, start_method="spawn")
    assert np.max(np.abs(np.load(out) - parts.sum(axis=0))) < 1e-12
