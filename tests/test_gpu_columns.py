"""FEFF's feffNNNN.dat columns on a B200 (GPUPathStage.columns, fg_path_columns) against the oracle (FP64 form to
1e-10 relative magnitude and 1e-9 rad phase, mixed form to 2e-5 and 2e-4 rad) and against FEFF's own feff0001..0008.dat
of the W case to the precision FEFF prints."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.fixtures import npz, phase

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,tm,tp", [(torch.complex128, 1e-10, 1e-9), (torch.complex64, 2e-5, 2e-4)])
def test_columns(dtype, tm, tp):
    from feffgpu_b200 import GPUPathStage
    z = npz("feffdat_W")
    P = phase("case_W")
    st = GPUPathStage(P, device="cuda", dtype=dtype)
    orc = O.Oracle(P)
    for i in range(1, 9):
        c, ip, cols = z[f"coords_{i}"], z[f"ipots_{i}"], z[f"cols_{i}"]
        cc, rf = st.cchi(torch.tensor(c[None]), torch.tensor(ip[None]))
        col = st.columns(cc, rf)
        occ, orf = orc.cchi(c[None], ip[None])
        ref = O.columns(orc, occ[0], orf[0])
        mag, ph = col["mag"][0].cpu().numpy(), col["phase"][0].cpu().numpy()
        assert np.abs(mag - ref["mag"]).max() <= tm * np.abs(ref["mag"]).max(), i
        assert np.abs(ph - ref["phase"]).max() <= tp, i
        for key in ("k", "real_phc", "red_fact", "lam", "rep"):
            assert np.allclose(col[key], ref[key], rtol=1e-12, atol=1e-12), key
        # FEFF's printed columns
        assert np.abs(mag - cols[:, 2]).max() <= 3e-4 * np.abs(cols[:, 2]).max()
        assert np.abs(ph - cols[:, 3]).max() <= 2e-3
