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
    fwd_ms = {(1, 0, 0): 3.0, (2, 0, 0): 2.0, (4, 0, 0): 2.5, (1, 1, 0): 2.6, (2, 1, 0): 1.995, (4, 1, 0): 2.9,
              (1, 0, 1): 3.3, (2, 0, 1): 2.8, (4, 0, 1): 3.1}

    def timer(kind, stage, batch, q, S, prec, shape):
        calls.append((kind, shape))
        if kind == "fwd":
            return fwd_ms[shape]
        return {1: 9.0, 2: 9.5, 4: 9.05}[shape]

    b = _batch({2: 10, 5: 30, 8: 4})
    q = torch.arange(401) * 0.05
    t = A.Autotuner(tmp_path / "t.json", timer=timer)
    # near-ties go to the default variant, then to the wider shape
    assert t.tune(_Stage(), b, q, None, 0, backward=True) == (2, 4, 0, 0)
    assert len(calls) == len(A.FWD_SHAPES) + len(A.BWD_WARPS)
    # a second tuner reads the file: no timing
    t2 = A.Autotuner(tmp_path / "t.json", timer=timer)
    assert t2.tune(_Stage(), b, q, None, 0, backward=True) == (2, 4, 0, 0)
    assert len(calls) == len(A.FWD_SHAPES) + len(A.BWD_WARPS)
    # forward-only entries are completed when the adjoint is asked for later, without timing the forward again
    b2 = _batch({3: 20})
    fwd_ms[(4, 0, 1)] = 1.0                      # a clear winner off the default variant is taken
    assert t2.tune(_Stage(), b2, q, None, 0, backward=False) == (4, 0, 0, 1)
    assert t2.lookup(A.signature(_Stage(), b2, 401, 0), backward=True) is None
    n = len(calls)
    assert t2.tune(_Stage(), b2, q, None, 0, backward=True) == (4, 4, 0, 1)
    assert len(calls) == n + len(A.BWD_WARPS)


def test_reads_entries_of_warps_only(tmp_path, monkeypatch):
    """A cache entry holding the forward warps alone (no variant) reads as the default variant."""
    import json
    monkeypatch.setattr(A, "gpu_name", lambda d: "FakeGPU")
    b = _batch({3: 20})
    sig = A.signature(_Stage(), b, 401, 0)
    (tmp_path / "t.json").write_text(json.dumps({sig: {"fwd": 2, "bwd": 1, "ms_fwd": {"2": 1.0}}}))
    t = A.Autotuner(tmp_path / "t.json", timer=None)
    assert t.lookup(sig, backward=True) == (2, 1, 0, 0)


def test_signature_separates_workloads(monkeypatch):
    monkeypatch.setattr(A, "gpu_name", lambda d: "FakeGPU")
    s = _Stage()
    a = A.signature(s, _batch({2: 10, 5: 30}), 401, 0)
    assert a == A.signature(s, _batch({2: 10, 5: 30}, seed=1), 401, 0)
    assert a != A.signature(s, _batch({2: 10, 5: 30}), 401, 1)          # precision
    assert a != A.signature(s, _batch({2: 10, 5: 30}), 201, 0)          # k grid
    assert a != A.signature(s, _batch({2: 30, 5: 10}), 401, 0)          # leg mix
    assert a != A.signature(s, _batch({2: 10, 5: 30, 7: 1}), 401, 0)    # longest path
    s3 = _Stage()
    s3.iorder = 3
    assert a != A.signature(s3, _batch({2: 10, 5: 30}), 401, 0)         # lambda-set order


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
