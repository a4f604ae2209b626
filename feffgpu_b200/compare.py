"""The R-space R-factor between two chi(k) (the reference's ``src/feffgpu/compare.py:6-27``, same conventions):
FT of k^kweight chi with a Hanning window whose sills are centred on kmin and kmax and dk wide, then
sum |FT(fit) - FT(data)|^2 / sum |FT(data)|^2 over rmin..rmax.  This is the parity metric of the stage."""
from __future__ import annotations

import math

import numpy as np


def hanning(k, kmin, kmax, dk=1.0):
    """Hanning window with sills centred on kmin and kmax, dk wide (dk = 0: rectangular)."""
    k = np.asarray(k, float)
    if dk <= 0:
        return ((k >= kmin) & (k <= kmax)).astype(float)
    rise = 0.5 * (1 - np.cos(np.pi * np.clip((k - (kmin - dk / 2)) / dk, 0, 1)))
    fall = 0.5 * (1 + np.cos(np.pi * np.clip((k - (kmax - dk / 2)) / dk, 0, 1)))
    return rise * fall


def r_factor(k, data, fit, kmin=3.0, kmax=23.0, rmin=1.0, rmax=6.0, kweight=2, nfft=2048, dk=1.0):
    k, data, fit = (np.asarray(v, float) for v in (k, data, fit))
    step = k[1] - k[0]
    win = hanning(k, kmin, kmax, dk)

    def ft(c):
        return np.fft.fft(c * k ** kweight * win, n=nfft)[: nfft // 2] * step / math.sqrt(math.pi)

    r = np.arange(nfft // 2) * math.pi / (nfft * step)
    keep = (r >= rmin) & (r <= rmax)
    d, m = ft(data)[keep], ft(fit)[keep]
    return float(np.sum(np.abs(m - d) ** 2) / np.sum(np.abs(d) ** 2))
