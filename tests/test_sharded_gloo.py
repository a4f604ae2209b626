"""Multi-process sharding of the path stage on CPU ranks (gloo, world size 2): the partition covers every path once
and balances the cost, the all-reduced rows equal the one-process sum, and gradients through the differentiable
all-reduce match the one-process gradient.  Each rank evaluates its shard with the CPU oracle (the GPU stage is the
same computation; this tests the multi-rank logic)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from feffgpu_b200.sharded import allreduce_grad, allreduce_rows, shard, split_groups


def test_shard_covers_every_path_and_balances():
    rng = np.random.default_rng(0)
    nleg = rng.integers(2, 9, 5000)
    for world in (1, 2, 3, 8):
        owner = shard(nleg, world)
        assert owner.min() >= 0 and owner.max() < world and len(owner) == len(nleg)
        cost = np.where(nleg == 2, 0.45, nleg - 1.0)
        loads = np.bincount(owner, weights=cost, minlength=world)
        assert loads.max() - loads.min() <= cost.max() + 1e-9
        assert np.array_equal(owner, shard(nleg, world))    # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rows_of(groups, P, q, nrows):
    from oracle import oracle as O
    orc = O.Oracle(P)
    S = orc.linear_matrix(q)
    rows = np.zeros((nrows, len(q)))
    for coords, ipots, deg, row in groups:
        cc, rf = orc.cchi(coords, ipots, nthreads=1)
        chi = deg[:, None] * O.chi_fine(cc, rf, q, S)
        np.add.at(rows, row, chi)
    return rows


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from tests.fixtures import groups, phase
        P = phase("case_L001")
        gs = [(c, i, d, np.arange(len(c)) % 2) for c, i, d in groups("case_L001").values()]
        q = np.arange(1, 201) * 0.1
        mine = split_groups(gs, world, rank)
        part = torch.tensor(_rows_of(mine, P, q, 2))
        # differentiable all-reduce: a scale factor per rank's partial rows stands for the rank's parameters
        a = torch.ones((), dtype=torch.float64, requires_grad=True)
        total = allreduce_rows(part * a)
        loss = (total ** 2).sum()
        loss.backward()
        g = allreduce_grad(a.grad.clone())
        n_mine = sum(len(x[0]) for x in mine)
        out[rank] = (total.detach().numpy(), float(g), float((2 * total * part).sum()), n_mine)
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_one_process():
    from tests.fixtures import groups, phase
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    P = phase("case_L001")
    gs = [(c, i, d, np.arange(len(c)) % 2) for c, i, d in groups("case_L001").values()]
    q = np.arange(1, 201) * 0.1
    ref = _rows_of(gs, P, q, 2)
    assert out[0][3] + out[1][3] == sum(len(g[0]) for g in gs)
    for r in range(world):
        np.testing.assert_allclose(out[r][0], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    # d loss / d a with a scaling every rank's part: sum over ranks of 2 total . part = 2 total . total
    np.testing.assert_allclose(out[0][1], 2 * (ref ** 2).sum(), rtol=1e-10)
    np.testing.assert_allclose(out[0][1], out[0][2] + out[1][2], rtol=1e-10)


def test_flop_balanced_split():
    """With the FLOP cost (roofline.path_flops over all energies) every rank gets a near-equal share of the work."""
    from feffgpu_b200.roofline import path_flops
    from feffgpu_b200.sharded import shard, split_groups
    rng = np.random.default_rng(3)
    lmax = rng.integers(5, 24, size=(60, 4))
    groups = []
    for n, m in ((2, 40), (3, 300), (5, 500), (8, 60)):
        ip = rng.integers(1, 4, size=(m, n))
        ip[:, 0] = 0
        groups.append((rng.normal(size=(m, n, 3)), ip, None, None))
    nl = np.concatenate([np.full(len(g[0]), g[0].shape[1]) for g in groups])
    ipp = np.concatenate([np.pad(g[1], ((0, 0), (0, 8 - g[1].shape[1]))) for g in groups])
    cost = path_flops(nl, ipp, lmax)
    owner = shard(nl, 4, cost)
    load = np.bincount(owner, weights=cost, minlength=4)
    assert load.max() / load.min() < 1.01
    parts = [split_groups(groups, 4, r, lmax=lmax) for r in range(4)]
    assert sum(len(g[0]) for p in parts for g in p) == len(nl)
