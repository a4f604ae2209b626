"""Multi-GPU path stage: one process per GPU, paths sharded across ranks, rows summed with one all-reduce.

The paths of a job are independent; the only exchange is the final sum of every rank's partial rows (rows x NK FP64,
e.g. 2 x 401 x 8 B per absorber pair).  ``shard`` splits a path list across ranks by cost (longest-processing-time
first over the ranks, deterministic); ``chi_reduce_all_ranks`` evaluates each rank's share with the fused stage and
sums the exact row sums over the process group as 64-bit integers (NCCL on GPUs, gloo elsewhere) before the rows are
formed, so the rows are bit for bit those of one process over all the paths; ``allreduce_rows`` sums finished FP64
partial rows instead.  Both are differentiable: every rank computes the loss from the same summed rows, so the
gradient reaching each rank's paths is the upstream gradient itself.  Gradients of positions shared by all ranks (an
RMC model) are then summed with ``allreduce_grad``.

The reference runs multi-GPU jobs as independent processes per MD-frame shard (``src/feffgpu/parallel/__init__.py:
78-133``); this module adds the path-level split with one collective.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def path_cost(nleg: np.ndarray) -> np.ndarray:
    """Relative cost of a path by its leg count (the scattering-matrix chain grows linearly with the legs)."""
    nleg = np.asarray(nleg)
    return np.where(nleg == 2, 0.45, nleg - 1.0)


def shard(nleg: np.ndarray, world: int, cost=None) -> np.ndarray:
    """Rank of every path: longest-processing-time-first assignment of the path costs (default: by leg count; pass
    roofline.path_flops for the FLOP cost over all energies) to the least-loaded rank, by the library's host routine
    fg_shard_lpt (a heap over the ranks' loads).  Deterministic for a given input."""
    from . import _lib
    nleg = np.asarray(nleg)
    cost = np.ascontiguousarray(path_cost(nleg) if cost is None else np.asarray(cost, float), dtype=np.float64)
    owner = np.zeros(len(nleg), np.int32)
    lib = _lib.load()
    _lib.check(lib.fg_shard_lpt(cost.ctypes.data, len(cost), int(world), owner.ctypes.data))
    return owner.astype(np.int64)


def split_groups(groups, world: int, rank: int, lmax=None):
    """The rank's share of a list of path groups (coords, ipots, deg, row) as returned for PathBatch; with the
    stage's lmax table (E, nph+1) the split balances algorithmic FLOPs over all energies."""
    nl = np.concatenate([np.full(len(g[0]), np.asarray(g[0]).shape[1]) for g in groups]) if groups else np.zeros(0)
    cost = None
    if lmax is not None and len(nl):
        from .roofline import path_flops
        nmax = int(nl.max())
        ip = np.concatenate([np.pad(np.asarray(g[1]), ((0, 0), (0, nmax - np.asarray(g[1]).shape[1]))) for g in groups])
        cost = path_flops(nl, ip, lmax)
    owner = shard(nl, world, cost)
    out, off = [], 0
    for g in groups:
        n = len(g[0])
        sel = np.nonzero(owner[off:off + n] == rank)[0]
        off += n
        if len(sel) == 0:
            continue
        gg = [np.asarray(g[0])[sel], np.asarray(g[1])[sel]]
        gg.append(None if len(g) < 3 or g[2] is None else np.asarray(g[2])[sel])
        gg.append(None if len(g) < 4 or g[3] is None else np.asarray(g[3])[sel])
        out.append(tuple(gg))
    return out


class _AllReduceSum(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, group):
        y = x.detach().clone()
        dist.all_reduce(y, op=dist.ReduceOp.SUM, group=group)
        return y

    @staticmethod
    def backward(ctx, g):
        # every rank holds the same loss of the summed rows: its partial rows receive the upstream gradient
        return g, None


class _ChiReduceAllRanks(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, sigma2, q, S, stage, batch, prec, group):
        need = ctx.needs_input_grad[0] or (sigma2 is not None and ctx.needs_input_grad[1])
        words, cchi, reff = stage._chi_reduce_words(batch, coords, sigma2, q, S, prec, save=need)
        if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
            dist.all_reduce(words, op=dist.ReduceOp.SUM, group=group)     # 64-bit integers: exact, any order
        if need:
            ctx.save_for_backward(coords, sigma2, q, S, cchi, reff)
        ctx.stage, ctx.batch, ctx.prec = stage, batch, prec
        return stage.rows_from_words(words)

    @staticmethod
    def backward(ctx, g):
        # every rank holds the same loss of the summed rows: its paths receive the upstream gradient
        coords, sigma2, q, S, cchi, reff = ctx.saved_tensors
        want_s2 = sigma2 is not None and ctx.needs_input_grad[1]
        gc, gs = ctx.stage._chi_reduce_backward(ctx.batch, coords, sigma2, q, S, ctx.prec, g, cchi, reff, want_s2)
        return (gc if ctx.needs_input_grad[0] else None), (gs if want_s2 else None), None, None, None, None, None, None


def chi_reduce_all_ranks(stage, batch, q, S=None, coords=None, sigma2=None, dtype=None, group=None) -> torch.Tensor:
    """The rows of every rank's paths: each rank evaluates its own batch (its share of the paths, e.g. from
    split_groups) with the fused stage, the exact row sums are summed over the ranks as 64-bit integers, and the rows
    are formed from the total -- bit for bit the rows one process computes over all the paths, whatever the number of
    ranks or the split.  Same arguments as GPUPathStage.chi_reduce; differentiable in coords and sigma2 (each rank
    receives the gradient of its own paths).  One all-reduce of 2 x nrows x NK int64 per call."""
    crd, s2, qt, Sd, prec = stage._reduce_args(batch, q, S, coords, sigma2, dtype)
    return _ChiReduceAllRanks.apply(crd, s2, qt, Sd, stage, batch, prec, group)


def allreduce_rows(rows: torch.Tensor, group=None) -> torch.Tensor:
    """Sum of the ranks' partial rows, differentiable (identity backward)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return rows
    return _AllReduceSum.apply(rows, group)


def allreduce_grad(t: torch.Tensor, group=None) -> torch.Tensor:
    """In-place sum over ranks of a gradient of parameters that every rank holds (shared positions)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t
