"""J/K builds and gradients sharded over ranks (one process per GPU).

Density fitting:
The fitted three-index tensor B[x][K][y] = sum_P (xy|P) (L^-T)_PK splits
along the fitted index K with no coupling between slices:

    J = sum_K B_K gamma_K,  gamma_K = sum_xy B_K D/2,   K = sum_K X_K X_K^T,

so rank r keeps only the columns K in its range (its share of HBM), builds
the partial J_r, K_r of its slice with the same kernels as the one-GPU build,
and one all-reduce (sum) of J and K, 2 n^2 doubles, completes the build
(the exchange step of compute_2body_fock_df split by K; molecular2 itself is
serial, src/fockbuild.cpp:621-659).  No rank needs another rank's slice.
"""
import torch
import torch.distributed as dist


def aux_ranges(naux, world, align=4):
    """Contiguous fitted-function ranges [k0, k1), one per rank, as even as
    possible with every boundary a multiple of `align` or equal to naux (the
    split-BF16 path tiles naux * nocc_padded in blocks of 64 with nocc_padded a
    multiple of 16).  With more ranks than units the last ranges are empty."""
    if world < 1 or naux < 1:
        raise ValueError("need world >= 1 and naux >= 1")
    units = -(-naux // align)
    base, extra = divmod(units, world)
    out, k = [], 0
    for r in range(world):
        k1 = min(naux, k + (base + (1 if r < extra else 0)) * align)
        out.append((k, k1))
        k = k1
    return out


def allreduce_jk(J, K, group=None):
    """Sum the partial J and K of every rank in place (torch tensors on the
    process group's device: CUDA for NCCL, CPU for gloo)."""
    dist.all_reduce(J, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(K, op=dist.ReduceOp.SUM, group=group)
    return J, K


def df_jk_sharded(engine, dC, nocc, dJ, dK, prec_mode=0, stream=None, group=None):
    """One sharded DF J/K build: the engine was created with this rank's K
    range (IntegralEngine.set_df_range before df_setup); dC, dJ, dK are CUDA
    tensors.  The partial build and the all-reduce run on `stream` (a
    torch.cuda.Stream, default the current one)."""
    s = stream or torch.cuda.current_stream()
    if engine.df_range[0] == engine.df_range[1]:   # nothing on this rank: contribute zeros
        with torch.cuda.stream(s):
            dJ.zero_()
            dK.zero_()
            allreduce_jk(dJ, dK, group)
        return dJ, dK
    engine.jk_df_device(dC.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), prec_mode, stream=s.cuda_stream)
    with torch.cuda.stream(s):
        allreduce_jk(dJ, dK, group)
    return dJ, dK


# ---------------------------------------------------------------- direct J/K and gradient
# The unique shell quartets of the direct build are (bra pair, ket pair) with
# the bra pairs of every angular class sorted by their Schwarz bound.  Rank r
# of R takes the bra pairs r, r + R, r + 2R, ... of every class
# (IntegralEngine.set_direct_partition), so each rank gets pairs from the whole
# range of bounds and nearly the same work; J, K (and the gradient) are sums
# over quartets, so one all-reduce completes them (the loops of
# src/fockbuild.cpp:88-158 and src/rhfgrad.cpp:454-590 split over ranks).

def interleaved_share(n, rank, world):
    """Indices rank, rank + world, ... below n: a rank's share of a sorted list."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return list(range(rank, n, world))


def direct_jk_sharded(engine, D, precision=1e-12, multiplier=1.0, group=None):
    """One sharded direct J/K build from a host density D (numpy): this rank's
    partial J and K, then the all-reduce; returns the whole (J, K) as numpy
    arrays on every rank.  The process group may be NCCL (the partials are
    moved to this rank's GPU) or gloo (CPU)."""
    import numpy as np
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    engine.set_direct_partition(rank, world)
    J, K = engine.jk_direct(D, precision, multiplier)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    tJ = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    tK = torch.from_numpy(np.ascontiguousarray(K)).to(dev)
    allreduce_jk(tJ, tK, group)
    return tJ.cpu().numpy(), tK.cpu().numpy()


def gradient_sharded(engine, D, W, group=None):
    """Sharded four-index RHF gradient: this rank's share of the two-electron
    quartets (rank 0 adds the one-body and nuclear terms), then one all-reduce
    of the 3 natom vector; returns the whole gradient (natom x 3)."""
    import numpy as np
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    engine.set_direct_partition(rank, world)
    g, _ = engine.compute_forces(D, W)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(g)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()
