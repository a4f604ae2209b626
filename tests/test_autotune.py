"""Autotuner host logic (CPU): candidate choice, persistence, signatures, and the stratified timing sample."""
import numpy as np
import torch

from feffgpu_b200 import autotune as A
from feffgpu_b200.batch import PathBatch


class _Stage:
    device = torch.device("cpu")
    ilinit, E = 1, 59


def _batch(counts, seed=0):
    rng = np.random.default_rng(seed)
    groups = []
    for nleg, n in counts.items():
        c = rng.normal(size=(n, nleg, 3)) * 2
        c[:, 0] = 0
        groups.append((c, np.zeros((n, nleg), int), None, np.arange(n) % 2))
    return PathBatch(groups, device="cpu")


def test_choice_and_persistence(tmp_path, monkeypatch):
    monkeypatch.setattr(A, "gpu_name", lambda d: "FakeGPU")
    calls = []

    def timer(kind, stage, batch, q, S, prec, w):
        calls.append((kind, w))
        return {("fwd", 1): 3.0, ("fwd", 2): 2.0, ("fwd", 4): 2.5, ("bwd", 1): 9.0, ("bwd", 2): 9.5,
                ("bwd", 4): 9.05}[(kind, w)]

    b = _batch({2: 10, 5: 30, 8: 4})
    q = torch.arange(401) * 0.05
    t = A.Autotuner(tmp_path / "t.json", timer=timer)
    assert t.tune(_Stage(), b, q, None, 0, backward=True) == (2, 4)     # near-ties go to the wider shape
    assert len(calls) == 6
    # a second tuner reads the file: no timing
    t2 = A.Autotuner(tmp_path / "t.json", timer=timer)
    assert t2.tune(_Stage(), b, q, None, 0, backward=True) == (2, 4)
    assert len(calls) == 6
    # forward-only entries are completed when the adjoint is asked for later
    b2 = _batch({3: 20})
    assert t2.tune(_Stage(), b2, q, None, 0, backward=False) == (2, 0)
    assert t2.lookup(A.signature(_Stage(), b2, 401, 0), backward=True) is None
    assert t2.tune(_Stage(), b2, q, None, 0, backward=True) == (2, 4)


def test_signature_separates_workloads(monkeypatch):
    monkeypatch.setattr(A, "gpu_name", lambda d: "FakeGPU")
    s = _Stage()
    a = A.signature(s, _batch({2: 10, 5: 30}), 401, 0)
    assert a == A.signature(s, _batch({2: 10, 5: 30}, seed=1), 401, 0)
    assert a != A.signature(s, _batch({2: 10, 5: 30}), 401, 1)          # precision
    assert a != A.signature(s, _batch({2: 10, 5: 30}), 201, 0)          # k grid
    assert a != A.signature(s, _batch({2: 30, 5: 10}), 401, 0)          # leg mix
    assert a != A.signature(s, _batch({2: 10, 5: 30, 7: 1}), 401, 0)    # longest path


def test_sample_is_stratified():
    b = _batch({2: 100, 4: 300, 8: 50})
    s = b.sample(45)
    assert s.n <= 45 and s.nleg_max == 8
    for k, v in b.counts.items():
        assert abs(s.counts[k] / s.n - v / b.n) < 0.05
    assert b.sample(10_000) is b
    # the sampled rows are rows of the batch
    full = {tuple(np.round(c.numpy(), 12).ravel()) for c in b.coords}
    assert all(tuple(np.round(c.numpy(), 12).ravel()) in full for c in s.coords)
