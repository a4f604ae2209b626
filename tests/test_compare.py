"""The package's R-factor (rspace.r_factor, the dense restricted transform) equals the oracle's restatement of the
reference's compare.py (a padded FFT) on the uniform k grid from zero."""
import numpy as np

from feffgpu_b200.rspace import FitWindow, r_factor
from oracle import oracle as O


def test_r_factor_matches():
    k = np.arange(0, 401) * 0.05
    rng = np.random.default_rng(0)
    a = np.sin(2 * 2.5 * k) * np.exp(-k / 10) + 0.01 * rng.normal(size=k.size)
    b = a + 1e-3 * rng.normal(size=k.size)
    for kw in (dict(kmin=3, kmax=19, rmin=1, rmax=6), dict(kmin=2, kmax=14, rmin=1.2, rmax=5.5)):
        ours = r_factor(a, b, FitWindow(**kw))
        assert abs(ours - O.r_factor(k, a, b, **kw)) <= 1e-12 * ours
    assert r_factor(a, a) == 0.0
