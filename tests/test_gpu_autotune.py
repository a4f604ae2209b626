"""Autotuned launch shapes on a B200: every candidate gives bit-identical results (fixed-order sums, per-path
gradients), the tuner returns one of the candidates with its timings, and autotune=True changes nothing but speed."""
import numpy as np
import pytest
import torch

from feffgpu_b200 import workloads as W
from tests.fixtures import cfg2_phase

pytestmark = pytest.mark.gpu

Q = np.arange(401) * 0.05


def _batch(seed=3):
    from feffgpu_b200 import PathBatch
    pos, lab, box = W.random_packing(600, 0.08, 1.8, seed=seed)
    ab = int(W.central_atom(pos, box, lab, "Fe", 1)[0])
    ipot_of = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    paths = W.random_paths(pos, box, ab, {2: 20, 3: 200, 4: 300, 5: 300, 6: 200, 7: 40}, rmax=7.0, seed=9,
                           ipot_of=ipot_of)
    return PathBatch([(c, ip, None, np.arange(len(c)) % 2) for c, ip, _ in paths.values()], nrows=2, device="cuda")


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_shapes_bit_identical_and_tuner_choice(dtype, tmp_path):
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200.autotune import BWD_WARPS, FWD_SHAPES, Autotuner
    st = GPUPathStage(cfg2_phase(), device="cuda", dtype=dtype)
    b = _batch()
    S = st.linear_matrix(Q)
    s2 = torch.full((b.n,), 0.002, dtype=torch.float64, device="cuda")
    w = torch.randn(b.nrows, len(Q), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    ref = None
    shapes = [(fw, 4, r, t_) for fw, r, t_ in FWD_SHAPES] + [(4, bw, 0, 0) for bw in BWD_WARPS]
    for shape in shapes:                         # every forward shape, every adjoint shape
        st.set_launch(*shape)
        x = b.coords.clone().requires_grad_(True)
        s = s2.clone().requires_grad_(True)
        rows = st.chi_reduce(b, Q, S, coords=x, sigma2=s)
        (rows * w).sum().backward()
        out = (rows.detach(), x.grad, s.grad)
        if ref is None:
            ref = out
        else:
            assert all(torch.equal(a, r) for a, r in zip(out, ref)), shape
    t = Autotuner(tmp_path / "tune.json")
    st.set_launch(0, 0)
    fw, bw, r, t_ = st.tune(b, Q, S, backward=True, tuner=t)
    assert (fw, r, t_) in FWD_SHAPES and bw in BWD_WARPS and st._launch == (fw, bw, r, t_)
    assert len(t.log) == len(FWD_SHAPES) + len(BWD_WARPS) and all(ms > 0 for *_, ms in t.log)
    print(f"{dtype}: tuned fwd {fw}/{r}/{t_} bwd {bw}; " + ", ".join(f"{k}{w_}={ms:.3f}ms" for _, k, w_, ms in t.log))
    # a stage that tunes itself on first use returns the same numbers
    auto = GPUPathStage(cfg2_phase(), device="cuda", dtype=dtype, autotune=True)
    import feffgpu_b200.autotune as A
    A._default = Autotuner(tmp_path / "tune2.json")
    x = b.coords.clone().requires_grad_(True)
    s = s2.clone().requires_grad_(True)
    rows = auto.chi_reduce(b, Q, S, coords=x, sigma2=s)
    (rows * w).sum().backward()
    assert auto._launch != (0, 0, 0, 0)
    assert torch.equal(rows.detach(), ref[0]) and torch.equal(x.grad, ref[1]) and torch.equal(s.grad, ref[2])
    A._default = None
