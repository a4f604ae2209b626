"""R-space misfit of chi(k) rows against a target, differentiable (the loss of the adjoint and RMC workloads).

Conventions of the reference's ``src/feffgpu/exafs/transform.py:24-145`` (xraylarch's): uniform k grid from zero with
step 0.05 1/A, Hanning window with sills centred on kmin and kmax and dk wide, chi(R) = (kstep / sqrt(pi)) FFT of
k^kweight chi(k) window zero-padded to 2048 points, R = pi / (kstep 2048) * arange(1024), and the R-factor
sum |chi_R(model) - chi_R(target)|^2 / sum |chi_R(target)|^2 over rmin <= R <= rmax (real and imaginary parts).

The transform restricted to the R window is one dense (NR, NK) complex matrix (``transform_matrix``): the same numbers
as the padded FFT.  The misfit and its gradient are one CUDA kernel (``fg_rspace_misfit``, one block per row, FP64,
fixed-order sums): the forward pass already holds dR/dchi, so the backward is a scaling.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

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


def transform_matrix(nk: int, window: FitWindow = FitWindow()):
    """(F (NR, NK) complex128, R (NR,)): chi_R = F chi restricted to rmin <= R <= rmax."""
    k = KSTEP * np.arange(nk)
    r = RSTEP * np.arange(NFFT // 2)
    keep = (r >= window.rmin) & (r <= window.rmax)
    w = hanning(k, window.kmin, window.kmax, window.dk) * k ** window.kweight
    # FFT restricted to the kept R: sum_n x_n exp(-2 pi i m n / NFFT), m = index of R
    m = np.nonzero(keep)[0]
    F = np.exp(-2j * np.pi * np.outer(m, np.arange(nk)) / NFFT) * (KSTEP / math.sqrt(math.pi)) * w[None, :]
    return F, r[keep]


class RSpaceMisfit:
    """R-factor of rows chi (B, NK) on k = KSTEP * arange(NK) against a target (NK,), on a CUDA device."""

    def __init__(self, nk: int, target, window: FitWindow = FitWindow(), device="cuda"):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("feffgpu_b200 evaluates the misfit on CUDA devices only (no CPU path)")
        F, self.r = transform_matrix(nk, window)
        self.nk = nk
        self.F = torch.tensor(F, dtype=torch.complex128, device=self.device).contiguous()     # (NR, NK)
        self._lib = _lib.load()
        self.set_target(target)

    def set_target(self, target):
        t = torch.as_tensor(np.asarray(target, float) if not torch.is_tensor(target) else target,
                            dtype=torch.float64, device=self.F.device)
        self.target_r = (self.F @ t.to(torch.complex128)).contiguous()
        self.norm = float((self.target_r.abs() ** 2).sum())

    def transform(self, chi: torch.Tensor) -> torch.Tensor:
        """chi(R) on the kept R, (B, NR) complex."""
        return chi.to(torch.complex128) @ self.F.T

    def __call__(self, chi: torch.Tensor) -> torch.Tensor:
        """(B,) R-factors of the rows of chi (B, NK), differentiable."""
        return _Misfit.apply(chi, self)

    def _run(self, x: torch.Tensor, want_grad: bool):
        B, NK = x.shape
        R = torch.empty(B, device=self.device, dtype=torch.float64)
        g = torch.empty(B, NK, device=self.device, dtype=torch.float64) if want_grad else None
        _lib.check(self._lib.fg_rspace_misfit(B, NK, int(self.F.shape[0]), x.data_ptr(), self.F.data_ptr(),
                                              self.target_r.data_ptr(), 1.0 / self.norm, R.data_ptr(),
                                              None if g is None else g.data_ptr(),
                                              torch.cuda.current_stream(self.device).cuda_stream))
        return R, g


class _Misfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, chi, mis):
        x = chi.detach().to(torch.float64).contiguous()
        if x.shape[-1] != mis.nk:
            raise ValueError(f"rows must have {mis.nk} k points")
        R, g = mis._run(x, want_grad=ctx.needs_input_grad[0])
        ctx.save_for_backward(g if g is not None else R)
        ctx.dtype = chi.dtype
        return R

    @staticmethod
    def backward(ctx, gR):
        (g,) = ctx.saved_tensors
        return (gR[:, None] * g).to(ctx.dtype), None
