"""Single scattering of whole configurations from tabulated two-leg signals: the reference's ``PairTables``
(``src/feffgpu/exafs/forward.py:178-320``) on the B200.

For every scatterer potential the two-leg chi(q) is tabulated on a distance grid r_min + dr i (i < nr); the
single-scattering spectrum of a configuration is the histogram of its absorber-neighbour distances (linear
interpolation between grid points, so it is differentiable in the positions) times the table.  Here

* the tables are one fused-stage call (``GPUPathStage.chi_reduce``): every grid point of every potential a two-leg
  path along z with its own row;
* the histogram is a CUDA kernel (``fg_pair_histogram``): a block per absorber, weights summed in 2^-32 fixed point
  with integer atomics (exact, so the result repeats bit for bit);
* ``single_scattering(pos)`` (every atom of every copy an absorber) is the histogram times the tables (a plain
  matrix product), differentiable through its own backward: D = T g per potential, then a kernel
  (``fg_pair_ss_grad``) that gives each atom a block visiting every pair it belongs to.

The reference's constructor also builds its multiple-scattering front end (``ms=True``, a PathSpectra); that part is
the path finder and the path stage of this package, so ``ms`` must be False here.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .batch import PathBatch
from .cell import as_cell, cell_words, min_width
from .stage import GPUPathStage

ETOK = 0.2624684236075176   # 2 m_e / hbar^2 in 1/(eV A^2): k^2 = ETOK (E - E0) (exafs/transform.py:22)


def _box_args(box, device):
    """(cubic length or -1, cell words (18,) FP64 on the device or None) of a box in any of the reference's forms."""
    cell = as_cell(box)
    if isinstance(cell, np.ndarray):
        return -1.0, torch.as_tensor(cell_words(cell, np.float64), device=device)
    return (cell if cell is not None else -1.0), None


def _ptr(t):
    return t.data_ptr() if t is not None else None


class PairTables:
    """The reference's constructor arguments: phase, k (1/A), target (kept for the caller), e0 (eV), window,
    r_range, box, rmax, r_min, dr, ms, nlegmax, critpw, chunk, device, dtype, kweight, dk.  The tables are built
    at q = sign(k^2 - e0 ETOK) sqrt(|k^2 - e0 ETOK|) (forward.py:79-81) with the stage's linear interpolation."""

    def __init__(self, phase, k, target=None, e0=0.0, window=(3.0, 23.0), r_range=(1.0, 8.0), box=None, rmax=9.4,
                 r_min=1.5, dr=0.002, ms=False, nlegmax=4, critpw=0.5, chunk=2048, device="cuda",
                 dtype=torch.complex64, kweight=2, dk=1.0):
        if ms:
            raise NotImplementedError("multiple scattering is the path finder and the path stage of this package "
                                      "(feffgpu_b200.pathfinder, GPUPathStage.chi_reduce); build PairTables with ms=False")
        width = min_width(as_cell(box))
        if width < 2 * float(rmax):
            # the reference refuses such a cell in the same place (its PathSpectra, exafs/forward.py:71-73)
            raise ValueError(f"the periodic cell (smallest width {width:.2f} A) is narrower than twice the cutoff "
                             f"({float(rmax)} A): a pair would have more than one image within it; use a larger "
                             f"supercell or a smaller cutoff")
        self.device = torch.device(device)
        self.stage = phase if isinstance(phase, GPUPathStage) else GPUPathStage(phase, device=device, dtype=dtype)
        self.device = self.stage.device
        self.box, self.rmax = box, float(rmax)
        self.k = np.asarray(k, float)
        self.target, self.e0, self.window, self.r_range = target, float(e0), window, r_range
        en = self.k ** 2 - self.e0 * ETOK
        self.q = np.sign(en) * np.sqrt(np.abs(en))
        self.r0, self.dr = float(r_min), float(dr)
        self.nr = int(round((self.rmax - self.r0) / self.dr)) + 1
        self.nph = int(self.stage.P.nph)
        self._lib = _lib.load()
        # every grid point of every potential: a two-leg path along z, its own row
        r = self.r0 + self.dr * np.arange(self.nr)
        groups = []
        for p in range(1, self.nph + 1):
            coords = np.zeros((self.nr, 2, 3))
            coords[:, 1, 2] = r
            ip = np.tile(np.array([[0, p]]), (self.nr, 1))
            groups.append((coords, ip, None, (p - 1) * self.nr + np.arange(self.nr)))
        batch = PathBatch(groups, nrows=self.nph * self.nr, device=self.device)
        with torch.no_grad():
            rows = self.stage.chi_reduce(batch, self.q)                        # (nph nr, NK) FP64
        self.T = rows.reshape(self.nph, self.nr, -1).contiguous()
        self.tables = {p: self.T[p - 1] for p in range(1, self.nph + 1)}
        self.ipot = None

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _ipot(self, ipot, n):
        ip = torch.as_tensor(ipot if ipot is not None else np.ones(n, np.int32), device=self.device).to(torch.int32)
        if ip.shape != (n,):
            raise ValueError("ipot must give one potential per atom")
        if n and (int(ip.min()) < 0 or int(ip.max()) > self.nph):
            raise IndexError(f"scatterer potentials must be within 0..{self.nph}")
        return ip.contiguous()

    # -- histogram of chosen absorbers (forward.py:248-289) --------------------------------------------------------
    @torch.no_grad()
    def histogram(self, pos, absorbers, ipot, box=None, batch=None):
        """(hist (nph + 1, nr) FP64, pairs closer than r_min) of the absorbers of one configuration pos (n, 3)."""
        pos = torch.as_tensor(pos, device=self.device, dtype=torch.float64).contiguous()
        n = int(pos.shape[0])
        ab = torch.as_tensor(absorbers, device=self.device, dtype=torch.int64).reshape(-1).contiguous()
        if ab.numel() and (int(ab.min()) < 0 or int(ab.max()) >= n):
            raise IndexError("absorber index out of range")
        ip = self._ipot(ipot, n)
        hist = torch.empty(self.nph + 1, self.nr, device=self.device, dtype=torch.float64)
        short = torch.empty(1, device=self.device, dtype=torch.int64)
        bl, cw = _box_args(box, self.device)
        _lib.check(self._lib.fg_pair_histogram(pos.data_ptr(), 1, n, bl, _ptr(cw), ab.data_ptr(), int(ab.numel()),
                                               ip.data_ptr(), self.nph, self.r0, self.dr, self.nr, self.rmax,
                                               hist.data_ptr(), short.data_ptr(), self._stream()))
        return hist, int(short.item())

    def table_stack(self, potentials=None, dtype=torch.float64):
        """The two-leg tables of the given scatterer potentials (default all), stacked: (P, nr, NK)."""
        potentials = sorted(self.tables) if potentials is None else list(potentials)
        return torch.stack([self.tables[p].to(dtype) for p in potentials])

    # -- single scattering over all pairs (forward.py:303-319) ------------------------------------------------------
    def single_scattering(self, pos):
        """The single-scattering chi (NK,) FP64 of pos (C, n, 3), every atom of every copy an absorber, averaged
        over C n.  Differentiable in pos.  Potentials: ``self.ipot`` (n,) if set, else 1 for every atom."""
        x = torch.as_tensor(pos, device=self.device)
        if x.dim() == 2:
            x = x[None]
        ip = self._ipot(self.ipot, int(x.shape[1]))
        return _SingleScattering.apply(x, self, ip)

    def _hist_all(self, pos64, ip):
        C, n, _ = pos64.shape
        hist = torch.empty(self.nph + 1, self.nr, device=self.device, dtype=torch.float64)
        short = torch.empty(1, device=self.device, dtype=torch.int64)
        bl, cw = _box_args(self.box, self.device)
        _lib.check(self._lib.fg_pair_histogram(pos64.data_ptr(), C, n, bl, _ptr(cw), None, 0, ip.data_ptr(),
                                               self.nph, self.r0, self.dr, self.nr, self.rmax, hist.data_ptr(),
                                               short.data_ptr(), self._stream()))
        return hist


class _SingleScattering(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, pt, ip):
        pos64 = pos.detach().to(torch.float64).contiguous()
        C, n, _ = pos64.shape
        hist = pt._hist_all(pos64, ip)
        chi = torch.einsum("pr,prk->k", hist[1:], pt.T) / (C * n)
        ctx.save_for_backward(pos64)
        ctx.pt, ctx.ip, ctx.dtype = pt, ip, pos.dtype
        return chi

    @staticmethod
    def backward(ctx, g):
        (pos64,) = ctx.saved_tensors
        pt = ctx.pt
        C, n, _ = pos64.shape
        D = torch.einsum("prk,k->pr", pt.T, g.to(torch.float64)).contiguous()          # (nph, nr)
        grad = torch.empty_like(pos64)
        bl, cw = _box_args(pt.box, pt.device)
        _lib.check(pt._lib.fg_pair_ss_grad(pos64.data_ptr(), C, n, bl, _ptr(cw), ctx.ip.data_ptr(), pt.nph,
                                           D.data_ptr(), pt.r0, pt.dr, pt.nr, pt.rmax, 1.0 / (C * n), grad.data_ptr(),
                                           pt._stream()))
        return grad.to(ctx.dtype), None, None
