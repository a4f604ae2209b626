"""The oracle's feffNNNN.dat columns (oracle.columns, the reference's genfmt.py:449-461) against FEFF's own
feff0001..0008.dat of the W case, to the precision FEFF prints (5 significant digits)."""
import numpy as np

from oracle import oracle as O
from tests.fixtures import npz, phase


def test_columns_equal_feff_files():
    z = npz("feffdat_W")
    orc = O.Oracle(phase("case_W"))
    for i in range(1, 9):
        cols = z[f"cols_{i}"]
        cc, rf = orc.cchi(z[f"coords_{i}"][None], z[f"ipots_{i}"][None])
        assert abs(float(rf[0]) - float(z[f"reff_{i}"])) <= 1e-4
        c = O.columns(orc, cc[0], rf[0])
        assert len(c["k"]) == len(cols)
        assert np.abs(c["k"] - cols[:, 0]).max() <= 1e-9
        for key, j, tol in (("real_phc", 1, 1e-3), ("phase", 3, 2e-3), ("red_fact", 4, 1e-3), ("rep", 6, 1e-3)):
            assert np.abs(c[key] - cols[:, j]).max() <= tol, (i, key)
        for key, j in (("mag", 2), ("lam", 5)):
            assert np.abs(c[key] - cols[:, j]).max() <= 3e-4 * np.abs(cols[:, j]).max(), (i, key)
