"""The R-space transform matrix reproduces the reference's conventions (padded FFT, compare.py's R-factor), and the
misfit kernel matches it with its gradient (the kernel part on a B200)."""
import numpy as np
import pytest
import torch

from feffgpu_b200.rspace import FitWindow, RSpaceMisfit, transform_matrix
from oracle import oracle as O

K = 0.05 * np.arange(401)
WIN = FitWindow(kmin=3.0, kmax=19.0, dk=1.0, kweight=2, rmin=1.0, rmax=6.0)


def _signals():
    rng = np.random.default_rng(0)
    target = np.sin(2 * 2.4 * K) * np.exp(-0.01 * K ** 2) * K / 10
    model = target + 0.01 * rng.normal(size=K.size)
    return target, model


def _misfit_np(F, target, x):
    tr = F @ target
    d = F @ x - tr
    norm = float((np.abs(tr) ** 2).sum())
    return float((np.abs(d) ** 2).sum() / norm), 2.0 / norm * (np.conj(d)[:, None] * F).real.sum(0)


def test_matrix_equals_r_factor_and_gradient():
    F, r = transform_matrix(len(K), WIN)
    target, model = _signals()
    v, g = _misfit_np(F, target, model)
    ref = O.r_factor(K, target, model, kmin=3.0, kmax=19.0, rmin=1.0, rmax=6.0, kweight=2, dk=1.0)
    assert abs(v - ref) < 1e-12 * ref
    for i in (100, 200, 300):
        h = 1e-6
        xp, xm = model.copy(), model.copy()
        xp[i] += h
        xm[i] -= h
        fd = (O.r_factor(K, target, xp, kmin=3, kmax=19, rmin=1, rmax=6) -
              O.r_factor(K, target, xm, kmin=3, kmax=19, rmin=1, rmax=6)) / (2 * h)
        assert abs(g[i] - fd) < 1e-6 * abs(fd) + 1e-12


@pytest.mark.gpu
def test_misfit_kernel_and_gradient():
    target, model = _signals()
    mis = RSpaceMisfit(len(K), target, WIN, device="cuda")
    F, _ = transform_matrix(len(K), WIN)
    rows = np.stack([model, target, 2 * model])
    x = torch.tensor(rows, device="cuda", requires_grad=True)
    v = mis(x)
    w = torch.tensor([1.0, -0.5, 0.25], device="cuda", dtype=torch.float64)
    (v * w).sum().backward()
    for b in range(3):
        val, g = _misfit_np(F, target, rows[b])
        assert abs(float(v[b]) - val) <= 1e-12 * max(val, 1e-30) + 1e-15
        assert np.abs(x.grad[b].cpu().numpy() - float(w[b]) * g).max() <= 1e-10 * np.abs(g).max() + 1e-15
    assert float(v[1]) < 1e-28


def _fixture_windows():
    z = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "rspace_ref.npz")
    out = []
    for i in range(3):
        w = z[f"win_{i}"]
        out.append((i, FitWindow(w[0], w[1], w[2], int(w[3]), w[4], w[5])))
    return z, out


def test_misfit_pinned_to_the_reference_losses():
    """The R window, the loss and its gradient equal the reference's own R-space losses (tests/golden/rspace_ref.npz,
    generated from its source): r_factor_torch (transform.py:130-145) with the FP64 k grid, and PathSpectra.misfit
    (exafs/forward.py:165-168) with its FP32 k grid and window.  Both keep the R points of the FP32 R grid
    (transform.py:125-127) -- one window's lower limit falls on a grid point the FP32 grid drops.  Tolerances: 1e-12
    relative for the FP64 form; 1e-7 for the FP32-grid form (its window values are FP32 cosines, equal to the
    reference's to an FP32 rounding)."""
    from feffgpu_b200.rspace import r_window
    z, wins = _fixture_windows()
    for i, win in wins:
        assert np.array_equal(r_window(win), z[f"keep_{i}"])
        for kd, key, tol in ((np.float64, "", 1e-12), (np.float32, "32", 1e-7)):
            F, _ = transform_matrix(401, win, kd)
            for b in range(z["models"].shape[0]):
                v, g = _misfit_np(F, z["data"], z["models"][b])
                ref_v, ref_g = z[f"R{key}_{i}"][b], z[f"grad{key}_{i}"][b]
                assert abs(v - ref_v) <= tol * ref_v, (i, key, b)
                assert np.abs(g - ref_g).max() <= tol * np.abs(ref_g).max(), (i, key, b)


@pytest.mark.gpu
def test_misfit_kernel_pinned_to_the_reference_losses():
    """The misfit kernel (value and gradient) against the reference's losses of the fixture, both k-grid forms."""
    z, wins = _fixture_windows()
    for i, win in wins:
        for kd, key, tol in ((np.float64, "", 1e-12), (np.float32, "32", 1e-7)):
            mis = RSpaceMisfit(401, z["data"], win, device="cuda", k_dtype=kd)
            x = torch.tensor(z["models"], device="cuda", requires_grad=True)
            v = mis(x)
            v.sum().backward()
            ref_v, ref_g = z[f"R{key}_{i}"], z[f"grad{key}_{i}"]
            np.testing.assert_allclose(v.detach().cpu().numpy(), ref_v, rtol=tol, atol=0)
            assert np.abs(x.grad.cpu().numpy() - ref_g).max() <= tol * np.abs(ref_g).max()
