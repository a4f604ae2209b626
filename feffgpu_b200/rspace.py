"""R-space misfit of chi(k) rows against a target, differentiable (the loss of the adjoint and RMC workloads).

Conventions of the reference's ``src/feffgpu/exafs/transform.py:24-145`` (xraylarch's): uniform k grid from zero with
step 0.05 1/A, Hanning window with sills centred on kmin and kmax and dk wide, chi(R) = (kstep / sqrt(pi)) FFT of
k^kweight chi(k) window zero-padded to 2048 points, R = pi / (kstep 2048) * arange(1024), and the R-factor
sum |chi_R(model) - chi_R(target)|^2 / sum |chi_R(target)|^2 over rmin <= R <= rmax (real and imaginary parts), the R
window taken on the reference's FP32 R grid.

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
    """Hanning window with sills centred on kmin and kmax, dk wide (dk = 0: rectangular), in k's precision."""
    k = np.asarray(k)
    if not np.issubdtype(k.dtype, np.floating):
        k = k.astype(float)
    if dk <= 0:
        return ((k >= kmin) & (k <= kmax)).astype(k.dtype)
    t = k.dtype.type
    rise = t(0.5) * (t(1) - np.cos(t(np.pi) * np.clip((k - t(kmin - dk / 2)) / t(dk), 0, 1)))
    fall = t(0.5) * (t(1) + np.cos(t(np.pi) * np.clip((k - t(kmax - dk / 2)) / t(dk), 0, 1)))
    return rise * fall


def r_window(window: FitWindow) -> np.ndarray:
    """Indices of the R points rmin <= R <= rmax.  The reference forms its R grid in FP32
    (``transform.py:125-127``) and compares it with the window's limits in FP32; so does this mask, so that a limit
    that falls on a grid point keeps or drops that point as the reference does."""
    r = (np.float32(RSTEP) * np.arange(NFFT // 2, dtype=np.float32)).astype(np.float32)
    return np.nonzero((r >= np.float32(window.rmin)) & (r <= np.float32(window.rmax)))[0]


def transform_matrix(nk: int, window: FitWindow = FitWindow(), k_dtype=np.float64):
    """(F (NR, NK) complex128, R (NR,)): chi_R = F chi restricted to rmin <= R <= rmax.

    k_dtype float64: the k grid and window of ``r_factor_torch`` (``transform.py:130-145``); float32: those of
    ``PathSpectra.misfit`` (``exafs/forward.py:87-90, 165-168``), which holds k and forms the window in FP32 and
    widens both to FP64 for the transform."""
    k = (KSTEP * np.arange(nk)).astype(k_dtype)
    m = r_window(window)
    w = hanning(k, window.kmin, window.kmax, window.dk).astype(np.float64)
    k = k.astype(np.float64)
    w = w * k ** window.kweight
    # FFT restricted to the kept R: sum_n x_n exp(-2 pi i m n / NFFT), m = index of R
    F = np.exp(-2j * np.pi * np.outer(m, np.arange(nk)) / NFFT) * (KSTEP / math.sqrt(math.pi)) * w[None, :]
    return F, RSTEP * m


def r_factor(data, fit, window: FitWindow = FitWindow()) -> float:
    """R-factor of one spectrum ``fit`` against ``data``, both on k = KSTEP * arange(NK) (numpy, host):
    sum |chi_R(fit) - chi_R(data)|^2 / sum |chi_R(data)|^2 over the R window -- the comparison of the reference's
    ``compare.py:17-27`` and ``r_factor_torch`` with the transform of ``transform_matrix``."""
    data, fit = np.asarray(data, float), np.asarray(fit, float)
    F, _ = transform_matrix(data.shape[-1], window)
    d = F @ data
    return float(np.sum(np.abs(F @ fit - d) ** 2) / np.sum(np.abs(d) ** 2))


class RSpaceMisfit:
    """R-factor of rows chi (B, NK) on k = KSTEP * arange(NK) against a target (NK,), on a CUDA device."""

    def __init__(self, nk: int, target, window: FitWindow = FitWindow(), device="cuda", k_dtype=np.float64):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("feffgpu_b200 evaluates the misfit on CUDA devices only (no CPU path)")
        F, self.r = transform_matrix(nk, window, k_dtype)
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
