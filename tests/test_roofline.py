"""The roofline's FLOP model (feffgpu_b200.roofline; no GPU): the tabulated counts of the reference's literal loops
at L = 21 and 25 reproduced exactly, affine in L, per-path costs that add up to the batch total the benchmark
divides by the launch time, and a per-energy mean over the scatterers' partial-wave limits."""
import numpy as np

from feffgpu_b200.roofline import _L21, _L25, batch_flops, flops_per_energy, path_flops


def test_table_is_reproduced_and_affine_in_L():
    for n in range(2, 9):
        assert flops_per_energy(n, 25) == _L25[n] and flops_per_energy(n, 21) == _L21[n]
        assert abs(flops_per_energy(n, 23) - 0.5 * (_L25[n] + _L21[n])) < 1e-9
    for L in (6, 15, 25):
        assert all(flops_per_energy(n + 1, L) > flops_per_energy(n, L) for n in range(2, 9))


def test_path_costs_add_up_to_the_batch_total():
    rng = np.random.default_rng(0)
    lmax = rng.integers(4, 25, size=(401, 4))
    nleg = rng.integers(2, 10, size=500)
    ipots = np.zeros((500, 9), int)
    for b, n in enumerate(nleg):
        ipots[b, 1:n] = rng.integers(1, 4, size=n - 1)
    per = path_flops(nleg, ipots, lmax)
    assert per.shape == (500,) and np.all(per > 0)
    assert abs(per.sum() - batch_flops(nleg, ipots, lmax)) <= 1e-9 * per.sum()


def test_mean_over_scatterers_per_energy():
    lmax = np.array([[0, 9, 19], [0, 4, 24]])                 # two energies, potentials 0..2
    ipots = np.array([[0, 1, 2, 0]])                          # a three-leg path through potentials 1 and 2
    want = flops_per_energy(3, (10 + 20) / 2) + flops_per_energy(3, (5 + 25) / 2)
    assert abs(path_flops([3], ipots, lmax)[0] - want) < 1e-6
