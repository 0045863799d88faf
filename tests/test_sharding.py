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
