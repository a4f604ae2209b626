"""The pair-table oracle (oracle/pairs.py) against the reference's PairTables (tests/golden/pairs_nio.npz: a cubic
periodic box; pairs_nio_tri.npz: a triclinic cell)."""
import numpy as np
import pytest

from oracle import pairs as OP
from tests.fixtures import npz, phase


def pairs_case(name):
    """(fixture, box: the cubic length or the 3 x 3 cell, r_min, dr, rmax)."""
    z = npz(name)
    box = z["cell"] if "cell" in z else float(z["box"])
    return z, box, float(z["r_min"]), float(z["dr"]), float(z["rmax"])


@pytest.mark.parametrize("name", ["pairs_nio", "pairs_nio_tri"])
def test_tables_histogram_spectrum_gradient(name):
    z, box, r0, dr, rmax = pairs_case(name)
    P = phase("cfg5_nik_phase")
    T = OP.tables(P, z["k"], r0, rmax, dr)
    nr = int(z["nr"])
    assert T.shape == (P.nph, nr, len(z["k"]))
    for p in range(1, P.nph + 1):
        if f"table_{p}" not in z:
            continue
        ref = z[f"table_{p}"]
        # the reference's tables are FP32 copies of its FP64 stage
        assert np.abs(T[p - 1, ::25] - ref).max() <= 1e-6 * np.abs(ref).max()
    h, short = OP.histogram(z["pos"][0], z["absorbers"], z["ipot"], box, r0, dr, nr, rmax, P.nph)
    assert short == int(z["short"])
    assert np.abs(h - z["hist"]).max() <= 1e-9
    # the reference's spectrum and gradient come from FP32 positions and tables
    chi, grad = OP.single_scattering(z["pos"].astype(np.float32).astype(float), box, z["ipot"],
                                     T.astype(np.float32).astype(float), r0, dr, rmax, w=z["w"])
    assert np.abs(chi - z["chi"]).max() <= 1e-5 * np.abs(z["chi"]).max()
    assert np.abs(grad - z["grad"]).max() <= 1e-4 * np.abs(z["grad"]).max()
