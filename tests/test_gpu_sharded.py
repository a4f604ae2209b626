"""The multi-GPU split on the CUDA stage: two ranks (processes with gloo as the collective backend, both on cuda:0 --
their kernels never wait on each other) each evaluate their FLOP-balanced share of FEFF's L001 path list with the
fused stage, sum the rows with the differentiable all-reduce and back-propagate a loss of the summed rows.  The summed
rows equal the oracle's (FP64 form, 1e-12 of the largest value) and every path's coordinate gradient equals the one
the whole list gives in one process (the adjoint of a path does not depend on which rank evaluates it)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

Q = np.arange(1, 201) * 0.1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _groups():
    from tests.fixtures import groups
    return [(c, i, d, np.arange(len(c)) % 2) for c, i, d in groups("case_L001").values()]


def _weights():
    return np.random.default_rng(4).normal(size=(2, len(Q)))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from feffgpu_b200 import GPUPathStage, PathBatch
        from feffgpu_b200.sharded import allreduce_rows, split_groups
        from tests.fixtures import phase
        st = GPUPathStage(phase("case_L001"), device="cuda:0", dtype=torch.complex128)
        mine = split_groups(_groups(), world, rank, lmax=st.lmax.cpu().numpy())
        b = PathBatch(mine, nrows=2, device="cuda:0")
        cg = b.coords.clone().requires_grad_(True)
        total = allreduce_rows(st.chi_reduce(b, Q, coords=cg).cpu())
        (total * torch.tensor(_weights())).sum().backward()
        out[rank] = (total.detach().numpy(), cg.grad.cpu().numpy(), b.nleg.cpu().numpy(), b.n)
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_the_cuda_stage_equal_one_process():
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.sharded import shard
    from oracle import oracle as O
    from tests.fixtures import phase
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    gs = _groups()
    P = phase("case_L001")
    orc = O.Oracle(P)
    S = orc.linear_matrix(Q)
    ref = np.zeros((2, len(Q)))
    for c, i, d, r in gs:
        cc, rf = orc.cchi(c, i)
        np.add.at(ref, r, d[:, None] * O.chi_fine(cc, rf, Q, S))
    for r in range(world):
        assert np.abs(out[r][0] - ref).max() <= 1e-12 * np.abs(ref).max()
    assert out[0][3] + out[1][3] == sum(len(g[0]) for g in gs) and min(out[0][3], out[1][3]) > 0
    # the same loss in one process: per-path gradients, matched to the ranks' shares through the split itself
    st = GPUPathStage(P, device="cuda:0", dtype=torch.complex128)
    b = PathBatch(gs, nrows=2, device="cuda:0")
    cg = b.coords.clone().requires_grad_(True)
    (st.chi_reduce(b, Q, coords=cg).cpu() * torch.tensor(_weights())).sum().backward()
    full = cg.grad.cpu().numpy()
    nl = b.nleg.cpu().numpy()
    from feffgpu_b200.roofline import path_flops
    ip = b.ipots.cpu().numpy()
    owner = shard(nl, world, path_flops(nl, ip, st.lmax.cpu().numpy()))
    for r in range(world):
        mine = np.nonzero(owner == r)[0]          # split_groups keeps every group's paths in order
        assert np.array_equal(out[r][2], nl[mine])
        np.testing.assert_allclose(out[r][1], full[mine], rtol=0, atol=1e-12 * np.abs(full).max())


def _worker_exact(rank, world, port, out, dtype_name):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from feffgpu_b200 import GPUPathStage, PathBatch
        from feffgpu_b200.sharded import chi_reduce_all_ranks, split_groups
        from tests.fixtures import phase
        st = GPUPathStage(phase("case_L001"), device="cuda:0", dtype=getattr(torch, dtype_name))
        mine = split_groups(_groups(), world, rank, lmax=st.lmax.cpu().numpy())
        b = PathBatch(mine, nrows=2, device="cuda:0")
        cg = b.coords.clone().requires_grad_(True)
        s2 = torch.full((b.n,), 0.003, dtype=torch.float64, device="cuda:0", requires_grad=True)
        total = chi_reduce_all_ranks(st, b, Q, coords=cg, sigma2=s2)
        (total * torch.tensor(_weights(), device="cuda:0")).sum().backward()
        out[rank] = (total.detach().cpu().numpy(), cg.grad.cpu().numpy(), s2.grad.cpu().numpy(), b.nleg.cpu().numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dtype_name", ["complex64", "complex128"])
def test_two_ranks_exact_rows_equal_one_process_bit_for_bit(dtype_name):
    """chi_reduce_all_ranks: the ranks' exact row sums are summed as 64-bit integers before the rows are formed, so
    the rows of two ranks equal one process's chi_reduce over all the paths bit for bit (mixed and FP64 forms), and
    every path's coordinate and sigma^2 gradient equals the one-process one."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.roofline import path_flops
    from feffgpu_b200.sharded import shard
    from tests.fixtures import phase
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_worker_exact, args=(r, world, port, out, dtype_name)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    gs = _groups()
    st = GPUPathStage(phase("case_L001"), device="cuda:0", dtype=getattr(torch, dtype_name))
    b = PathBatch(gs, nrows=2, device="cuda:0")
    cg = b.coords.clone().requires_grad_(True)
    s2 = torch.full((b.n,), 0.003, dtype=torch.float64, device="cuda:0", requires_grad=True)
    rows = st.chi_reduce(b, Q, coords=cg, sigma2=s2)
    (rows * torch.tensor(_weights(), device="cuda:0")).sum().backward()
    ref = rows.detach().cpu().numpy()
    for r in range(world):
        assert np.array_equal(out[r][0], ref), r          # bit for bit
    nl = b.nleg.cpu().numpy()
    owner = shard(nl, world, path_flops(nl, b.ipots.cpu().numpy(), st.lmax.cpu().numpy()))
    full_c, full_s = cg.grad.cpu().numpy(), s2.grad.cpu().numpy()
    for r in range(world):
        mine = np.nonzero(owner == r)[0]
        assert np.array_equal(out[r][3], nl[mine])
        assert np.array_equal(out[r][1], full_c[mine]) and np.array_equal(out[r][2], full_s[mine])
