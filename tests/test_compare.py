"""The package's R-factor equals the oracle's restatement of the reference's compare.py."""
import numpy as np

from feffgpu_b200 import r_factor
from oracle import oracle as O


def test_r_factor_matches():
    k = np.arange(0, 401) * 0.05
    rng = np.random.default_rng(0)
    a = np.sin(2 * 2.5 * k) * np.exp(-k / 10) + 0.01 * rng.normal(size=k.size)
    b = a + 1e-3 * rng.normal(size=k.size)
    assert r_factor(k, a, b, kmin=3, kmax=19) == O.r_factor(k, a, b, kmin=3, kmax=19)
    assert r_factor(k, a, a) == 0.0
