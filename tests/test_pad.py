"""The phase-file boundary: PhaseData fields, the packed-ASCII reader, npz round trip, resampling."""

import numpy as np
import pytest

from feffgpu_b200.pad import PhaseData, load_phase, phase_from_npz, phase_to_arrays, read_phase_pad, resample_phase
from oracle import oracle as O
from tests.fixtures import GOLDEN, npz, phase


def test_reader_matches_the_reference_tables():
    """read_phase_pad on FEFF's L001 phase.pad gives the tables of the reference's reader (trimmed as stored)."""
    src = GOLDEN / "L001_phase.pad"
    P = read_phase_pad(src)
    Q = phase("case_L001")
    E = Q.ne1
    lt = Q.ltot
    assert P.ne1 == Q.ne1 and P.nph == Q.nph and P.ihole == Q.ihole and P.edge == Q.edge
    assert np.array_equal(P.em[:E], Q.em) and np.array_equal(P.eref[:E], Q.eref) and np.array_equal(P.rkk[:E], Q.rkk)
    assert np.array_equal(P.ph[:E, P.ltot - lt:P.ltot + lt + 1], Q.ph)
    assert np.array_equal(P.lmax[:E], Q.lmax)


def test_lmax_xk_ck_follow_rdxsph():
    for name in ("case_W", "case_A009"):
        P = phase(name)
        lm, xk, ck = O.phase_tables(P)
        assert np.array_equal(P.lmax[:P.ne1], lm)
        assert np.array_equal(P.xk[:P.ne1], xk) and np.array_equal(P.ck[:P.ne1], ck)


def test_npz_round_trip(tmp_path):
    P = phase("case_A014")
    f = tmp_path / "p.npz"
    np.savez(f, **phase_to_arrays(P, trim=False))
    Q = load_phase(f)
    assert isinstance(Q, PhaseData)
    for k in ("em", "eref", "ph", "rkk", "lmax0", "iz"):
        assert np.array_equal(getattr(P, k), getattr(Q, k))
    assert load_phase(P) is P


def test_load_phase_errors(tmp_path):
    with pytest.raises(FileNotFoundError):
        load_phase(tmp_path / "missing.pad")


def test_resample_keeps_the_grid_values():
    """On the file's own k points the resampled tables equal the originals; lmax follows the tables."""
    P = phase("case_L001")
    k = P.xk[:P.ne1] / 0.52917721067
    sel = k >= 0
    Q = resample_phase(P, k[sel])
    assert np.allclose(Q.ph, P.ph[:P.ne1][sel], atol=1e-14)
    assert np.allclose(Q.rkk, P.rkk[:P.ne1][sel], atol=1e-14)
    assert np.allclose(Q.xk, P.xk[:P.ne1][sel], rtol=1e-12, atol=1e-12)
    Q2 = resample_phase(P, np.arange(401) * 0.05)
    assert Q2.ne1 == 401 and Q2.ph.shape[0] == 401 and Q2.lmax.shape == (401, P.nph + 1)
