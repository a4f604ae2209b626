"""Pair tables on a B200 against the reference's PairTables (tests/golden/pairs_nio.npz, a cubic periodic box, and
pairs_nio_tri.npz, a triclinic cell) and the oracle.

Tables: every 25th row against the reference's (FP64 stage here, FP32 copies there: 1e-6 of the largest entry; the
mixed form to 2e-5).  Histogram of chosen absorbers: the reference's to 1e-9 (weights summed in 2^-32 fixed point),
the same count of short pairs, bit-identical on a repeat.  All-pairs spectrum and its position gradient: the
reference's (FP32 positions and tables there) to 1e-5 and 1e-4 of the largest value, the oracle's (FP64) to 1e-10 and
1e-9; the gradient bit-identical on a repeat and against central differences of the spectrum.
"""
import numpy as np
import pytest
import torch

from oracle import pairs as OP
from tests.fixtures import npz, phase
from tests.test_oracle_pairs import pairs_case

CASES = ["pairs_nio", "pairs_nio_tri"]

pytestmark = pytest.mark.gpu


def _tables(dtype=torch.complex128, name="pairs_nio"):
    from feffgpu_b200.pairs import PairTables
    z, box, r0, dr, rmax = pairs_case(name)
    pt = PairTables(phase("cfg5_nik_phase"), z["k"], np.zeros(len(z["k"])), 0.0, box=box,
                    rmax=rmax, r_min=r0, dr=dr, device="cuda", dtype=dtype)
    pt.ipot = torch.tensor(z["ipot"])
    return pt, z, box


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-6), (torch.complex64, 2e-5)])
def test_tables_equal_reference(dtype, tol):
    pt, z, _ = _tables(dtype)
    assert pt.nr == int(z["nr"])
    for p, t in pt.tables.items():
        ref = z[f"table_{p}"]
        assert np.abs(t.cpu().numpy()[::25] - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("name", CASES)
def test_histogram_equals_reference_and_repeats(name):
    pt, z, box = _tables(name=name)
    h1, s1 = pt.histogram(z["pos"][0], z["absorbers"], z["ipot"], box=box)
    h2, s2 = pt.histogram(z["pos"][0], z["absorbers"], z["ipot"], box=box)
    assert torch.equal(h1, h2) and s1 == s2 == int(z["short"])
    assert np.abs(h1.cpu().numpy() - z["hist"]).max() <= 1e-9


@pytest.mark.parametrize("name", CASES)
def test_single_scattering_and_gradient(name):
    pt, z, box = _tables(name=name)
    w = torch.tensor(z["w"], device="cuda")
    out = []
    for _ in range(2):
        x = torch.tensor(z["pos"], device="cuda", requires_grad=True)
        chi = pt.single_scattering(x)
        (chi * w).sum().backward()
        out.append((chi.detach(), x.grad))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    chi, grad = out[0][0].cpu().numpy(), out[0][1].cpu().numpy()
    assert np.abs(chi - z["chi"]).max() <= 1e-5 * np.abs(z["chi"]).max()
    assert np.abs(grad - z["grad"]).max() <= 1e-4 * np.abs(z["grad"]).max()
    T = pt.T.cpu().numpy()
    oc, og = OP.single_scattering(z["pos"], box, z["ipot"], T, pt.r0, pt.dr, pt.rmax, w=z["w"])
    assert np.abs(chi - oc).max() <= 1e-10 * np.abs(oc).max()
    assert np.abs(grad - og).max() <= 1e-9 * np.abs(og).max()
    # central differences on the largest gradient entries
    with torch.no_grad():
        for idx in np.argsort(-np.abs(grad).ravel())[:4]:
            c, i, q = np.unravel_index(idx, grad.shape)
            h = 1e-5
            xp, xm = z["pos"].copy(), z["pos"].copy()
            xp[c, i, q] += h
            xm[c, i, q] -= h
            fd = float(((pt.single_scattering(torch.tensor(xp, device="cuda")) -
                         pt.single_scattering(torch.tensor(xm, device="cuda"))) * w).sum()) / (2 * h)
            assert abs(fd - grad[c, i, q]) <= 1e-6 * np.abs(grad).max(), (idx, fd, grad[c, i, q])
