"""The R-space misfit equals the reference's conventions (padded FFT, compare.py's R-factor) and is differentiable."""
import numpy as np
import torch

from feffgpu_b200.rspace import FitWindow, RSpaceMisfit
from oracle import oracle as O


def test_misfit_equals_r_factor_and_gradient():
    k = 0.05 * np.arange(401)
    rng = np.random.default_rng(0)
    target = np.sin(2 * 2.4 * k) * np.exp(-0.01 * k ** 2) * k / 10
    model = target + 0.01 * rng.normal(size=k.size)
    win = FitWindow(kmin=3.0, kmax=19.0, dk=1.0, kweight=2, rmin=1.0, rmax=6.0)
    mis = RSpaceMisfit(len(k), target, win, device="cpu")
    x = torch.tensor(model[None], requires_grad=True)
    v = mis(x)
    ref = O.r_factor(k, target, model, kmin=3.0, kmax=19.0, rmin=1.0, rmax=6.0, kweight=2, dk=1.0)
    assert abs(float(v[0]) - ref) < 1e-12 * max(ref, 1e-30) + 1e-15
    v.sum().backward()
    # central differences on a few entries
    for i in (100, 200, 300):
        h = 1e-6
        xp, xm = model.copy(), model.copy()
        xp[i] += h
        xm[i] -= h
        fd = (O.r_factor(k, target, xp, kmin=3, kmax=19, rmin=1, rmax=6) -
              O.r_factor(k, target, xm, kmin=3, kmax=19, rmin=1, rmax=6)) / (2 * h)
        assert abs(float(x.grad[0, i]) - fd) < 1e-6 * abs(fd) + 1e-12
