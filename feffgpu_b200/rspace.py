"""R-space misfit of chi(k) rows against a target, differentiable (the loss of the adjoint and RMC workloads).

Conventions of the reference's ``src/feffgpu/exafs/transform.py:24-145`` (xraylarch's): uniform k grid from zero with
step 0.05 1/A, Hanning window with sills centred on kmin and kmax and dk wide, chi(R) = (kstep / sqrt(pi)) FFT of
k^kweight chi(k) window zero-padded to 2048 points, R = pi / (kstep 2048) * arange(1024), and the R-factor
sum |chi_R(model) - chi_R(target)|^2 / sum |chi_R(target)|^2 over rmin <= R <= rmax (real and imaginary parts).

The transform is the restriction of that FFT to the R window, applied as one dense (NR, NK) complex matrix in FP64:
the same numbers as the padded FFT, one small matrix product per evaluation, deterministic.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

KSTEP = 0.05
NFFT = 2048
RSTEP = math.pi / (KSTEP * NFFT)


@dataclass(frozen=True)
class FitWindow:
    kmin: float = 3.0
    kmax: float = 14.0
    dk: float = 1.0
    kweight: int = 2
    rmin: float = 1.0
    rmax: float = 6.0


def hanning(k: np.ndarray, kmin: float, kmax: float, dk: float = 1.0) -> np.ndarray:
    k = np.asarray(k, float)
    if dk <= 0:
        return ((k >= kmin) & (k <= kmax)).astype(float)
    up = 0.5 * (1 - np.cos(np.pi * np.clip((k - (kmin - dk / 2)) / dk, 0, 1)))
    down = 0.5 * (1 + np.cos(np.pi * np.clip((k - (kmax - dk / 2)) / dk, 0, 1)))
    return up * down


class RSpaceMisfit:
    """R-factor of rows chi (B, NK) on k = KSTEP * arange(NK) against a target (NK,)."""

    def __init__(self, nk: int, target, window: FitWindow = FitWindow(), device="cuda"):
        k = KSTEP * np.arange(nk)
        r = RSTEP * np.arange(NFFT // 2)
        keep = (r >= window.rmin) & (r <= window.rmax)
        self.r = r[keep]
        w = hanning(k, window.kmin, window.kmax, window.dk) * k ** window.kweight
        # FFT restricted to the kept R: sum_n x_n exp(-2 pi i m n / NFFT), m = index of R
        m = np.nonzero(keep)[0]
        F = np.exp(-2j * np.pi * np.outer(m, np.arange(nk)) / NFFT) * (KSTEP / math.sqrt(math.pi)) * w[None, :]
        self.F = torch.tensor(F, dtype=torch.complex128, device=device)          # (NR, NK)
        self.set_target(target)

    def set_target(self, target):
        t = torch.as_tensor(np.asarray(target, float) if not torch.is_tensor(target) else target,
                            dtype=torch.float64, device=self.F.device)
        self.target_r = self.F @ t.to(torch.complex128)
        self.norm = float((self.target_r.abs() ** 2).sum())

    def transform(self, chi: torch.Tensor) -> torch.Tensor:
        """chi(R) on the kept R, (B, NR) complex."""
        return chi.to(torch.complex128) @ self.F.T

    def __call__(self, chi: torch.Tensor) -> torch.Tensor:
        """(B,) R-factors of the rows of chi (B, NK), differentiable."""
        d = self.transform(chi) - self.target_r[None]
        return (d.real ** 2 + d.imag ** 2).sum(1) / self.norm
