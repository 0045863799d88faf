"""Density-fitted J/K sharded over ranks (one process per GPU).

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
