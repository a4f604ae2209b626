"""The path stage on a B200: a drop-in for the reference's ``GPUPathStage`` (``src/feffgpu/stage.py:96-388``).

Same constructor, methods, attributes and tensor layouts as the reference, so that ``feffgpu.chain.run``, the
MD-EXAFS and RMC-EXAFS front ends and their forward model (``src/feffgpu/exafs/forward.py``) call it unchanged:

* ``GPUPathStage(phase, device="cuda", dtype=torch.complex64, iorder=2)``; ``dtype`` complex64 selects the mixed
  form (FP32 scattering-matrix chain, FP64 geometry, 2kR + phase argument and sums), complex128 the plain FP64 form;
* ``cchi(coords, ipots) -> (cchi (B, E) complex, reff (B,) A)``, differentiable in ``coords`` through the hand-written
  adjoint (a plain ``backward()`` works; the reference needs ``checkpoint(use_reentrant=False)``, which also works);
* ``linear_matrix(q)``, ``spline_matrix(q)``, ``unwrap(phase)``, ``chi_fine(cchi, reff, q, S=None, convention)``,
  ``geometry(coords_bohr) -> (ri, beta, eta)``;
* attributes ``P``, ``E``, ``rdtype``, ``cdtype``, ``device``, ``iorder``, ``L1``, ``lmax``, ``xk``, ``ck``.

New beside them: ``chi_reduce(batch, q, ...)``, the fused stage: every path of a ``PathBatch`` (mixed leg counts,
one persistent launch), the fine-grid signal, an optional per-path exp(-2 sigma^2 q^2) and the degeneracy-weighted
sum into FP64 rows (exact integer sums of the terms rounded to 2^-64: deterministic), differentiable in the
coordinates and in sigma^2.

All computation runs in the CUDA library (``_build/libfeffgpu_b200.so``); there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from .pad import BOHR, load_phase, read_phase_pad


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _tspan_of(S: torch.Tensor) -> torch.Tensor:
    """(E, 2) int32 [lo, hi) of each column's non-zero rows (the transposed interpolation's ranges)."""
    return _span_of(S.t())


def _span_of(S: torch.Tensor) -> torch.Tensor:
    """(NK, 2) int32 [lo, hi) of each row's non-zero columns (rows without any: [0, 0))."""
    nz = S != 0
    E = S.shape[1]
    any_ = nz.any(1)
    lo = torch.argmax(nz.to(torch.int8), 1)
    hi = E - torch.argmax(nz.flip(1).to(torch.int8), 1)
    lo = torch.where(any_, lo, torch.zeros_like(lo))
    hi = torch.where(any_, hi, torch.zeros_like(hi))
    return torch.stack([lo, hi], 1).to(torch.int32).contiguous()


class GPUPathStage:
    """FEFF's path stage for one phase file on a B200 (see the module docstring)."""

    def __init__(self, phase, device="cuda", dtype=torch.complex64, iorder=2, autotune=False):
        P = read_phase_pad(phase) if isinstance(phase, str) else load_phase(phase)
        if P.nsp != 1:
            raise NotImplementedError("spin-dependent phase files are not ported")
        self.P, self.iorder, self.device, self.cdtype = P, iorder, torch.device(device), dtype
        if self.device.type != "cuda":
            raise RuntimeError("feffgpu_b200 evaluates the path stage on CUDA devices only (no CPU path)")
        if dtype not in (torch.complex64, torch.complex128):
            raise ValueError("dtype must be torch.complex64 or torch.complex128")
        self.rdtype = torch.float32 if dtype == torch.complex64 else torch.float64
        self.prec = _lib.FG_MIXED if dtype == torch.complex64 else _lib.FG_FP64
        E = self.E = int(P.ne1)
        self._lib = _lib.load()
        dev_index = self.device.index if self.device.index is not None else torch.cuda.current_device()
        self.device = torch.device("cuda", dev_index)
        # host arrays that the library copies into its device tables
        ph = np.ascontiguousarray(np.asarray(P.ph)[:E, :, 0, :], dtype=np.complex128)
        em = np.ascontiguousarray(np.asarray(P.em)[:E], dtype=np.complex128)
        eref = np.ascontiguousarray(np.asarray(P.eref)[:E, 0], dtype=np.complex128)
        rkk = np.ascontiguousarray(np.asarray(P.rkk)[:E, :, 0], dtype=np.complex128)
        lmax0 = np.ascontiguousarray(np.asarray(P.lmax0), dtype=np.int32)
        desc = _lib.PhaseDesc(E, int(P.nph), int(P.ltot), int(P.nsp), int(P.ihole), int(iorder), float(P.edge),
                              lmax0.ctypes.data, em.ctypes.data, eref.ctypes.data, ph.ctypes.data, rkk.ctypes.data)
        handle = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.fg_stage_create(C.byref(desc), dev_index, C.byref(handle)))
        self._h = handle
        info = _lib.StageInfo()
        _lib.check(self._lib.fg_stage_get_info(self._h, C.byref(info)))
        self.L1 = int(info.L1)
        self.kinit, self.ilinit = int(info.kinit), int(info.ilinit)
        lm = np.zeros((E, P.nph + 1), np.int32)
        _lib.check(self._lib.fg_stage_lmax(self._h, lm.ctypes.data))
        xk = np.zeros(E, np.float64)
        _lib.check(self._lib.fg_stage_xk(self._h, xk.ctypes.data))
        self.lmax = torch.tensor(lm, device=self.device)
        self._xk = xk
        self.xk = torch.tensor(xk, device=self.device, dtype=self.rdtype)
        self.ck = torch.tensor(np.sqrt(2 * (em - eref)), device=self.device, dtype=dtype)
        self._span_cache: dict = {}
        # launch shape (warps per CTA of the forward and adjoint kernels; 0 = the library default), per workload
        # when autotuning (feffgpu_b200.autotune)
        self.autotune = bool(autotune)
        self._launch = (0, 0, 0, 0)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.fg_stage_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- per-path signal ------------------------------------------------------------------------------------
    def _check_ipots(self, ipots: torch.Tensor) -> None:
        if ipots.numel():
            lo, hi = (int(v) for v in torch.stack(torch.aminmax(ipots)).cpu())    # one synchronisation
            if lo < 0 or hi > self.P.nph:
                raise IndexError(f"potential index out of range 0..{self.P.nph}")

    def cchi(self, coords, ipots):
        """coords (B, nleg, 3) A, absorber first; ipots (B, nleg) long with the absorber 0.  Returns cchi (B, E) of
        ``cdtype`` and reff (B,) of ``rdtype`` in A; differentiable in coords."""
        coords = torch.as_tensor(coords)
        if coords.dim() != 3 or coords.shape[2] != 3:
            raise ValueError("coords must be (B, nleg, 3)")
        ipots = torch.as_tensor(ipots).to(self.device, torch.int64)
        return _Cchi.apply(coords.to(self.device, self.rdtype), ipots, self)

    def _cchi_forward(self, coords: torch.Tensor, ipots: torch.Tensor):
        B, nleg, _ = coords.shape
        if not 2 <= nleg <= 9:
            raise ValueError("paths have 2 to 9 legs")
        if ipots.shape != (B, nleg):
            raise ValueError("ipots must be (B, nleg)")
        self._check_ipots(ipots)
        coords = coords.contiguous()
        ipots = ipots.contiguous()
        out = torch.empty(B, self.E, device=self.device, dtype=self.cdtype)
        reff = torch.empty(B, device=self.device, dtype=self.rdtype)
        _lib.check(self._lib.fg_cchi(self._h, self.prec, B, nleg, coords.data_ptr(), int(coords.dtype == torch.float64),
                                     ipots.data_ptr(), out.data_ptr(), reff.data_ptr(), None, _stream(self.device)))
        return out, reff

    def _cchi_backward(self, coords, ipots, g_cchi, g_reff):
        B, nleg, _ = coords.shape
        coords = coords.contiguous()
        g_cchi = (g_cchi if g_cchi is not None else torch.zeros(B, self.E, device=self.device, dtype=self.cdtype))
        g_cchi = g_cchi.to(self.cdtype).contiguous()
        g_reff = None if g_reff is None else g_reff.to(self.rdtype).contiguous()
        grad = torch.empty(B, nleg, 3, device=self.device, dtype=self.rdtype)
        ws_n = int(self._lib.fg_cchi_backward_workspace(self._h, B, nleg))
        ws = torch.empty(max(ws_n, 1), device=self.device, dtype=torch.uint8)
        _lib.check(self._lib.fg_cchi_backward(self._h, self.prec, B, nleg, coords.data_ptr(),
                                              int(coords.dtype == torch.float64), ipots.contiguous().data_ptr(),
                                              g_cchi.data_ptr(), _ptr(g_reff), grad.data_ptr(), ws.data_ptr(), ws_n,
                                              _stream(self.device)))
        return grad

    # -- fine grid ------------------------------------------------------------------------------------------
    def spline_matrix(self, q):
        """Cubic-spline interpolation matrix (len(q), E) (scipy UnivariateSpline s=0, as Larch), q clamped."""
        from scipy.interpolate import UnivariateSpline
        kf = self._xk / BOHR
        qn = np.clip(np.asarray(q, float), kf[0], kf[-1])
        S = np.zeros((len(qn), self.E))
        for j in range(self.E):
            y = np.zeros(self.E)
            y[j] = 1.0
            S[:, j] = UnivariateSpline(kf, y, s=0, k=3)(qn)
        return torch.tensor(S, device=self.device, dtype=self.rdtype)

    def linear_matrix(self, q):
        """FEFF's linear interpolation of amplitude and phase from the real-axis grid (ff2gen's terp1) as a dense
        (len(q), E) map; q beyond the grid is clamped."""
        kf = self._xk / BOHR
        qn = np.clip(np.asarray(q, float), kf[0], kf[-1])
        S = np.zeros((len(qn), self.E))
        j = np.clip(np.searchsorted(kf, qn, side="right") - 1, 0, self.E - 2)
        f = (qn - kf[j]) / (kf[j + 1] - kf[j])
        S[np.arange(len(qn)), j] = 1 - f
        S[np.arange(len(qn)), j + 1] = f
        return torch.tensor(S, device=self.device, dtype=self.rdtype)

    @staticmethod
    def unwrap(phase):
        """Unwrap along the last axis (differences brought into (-pi, pi])."""
        d = torch.diff(phase, dim=-1)
        d = d - 2 * math.pi * torch.round(d / (2 * math.pi))
        return torch.cat([phase[..., :1], phase[..., :1] + torch.cumsum(d, -1)], -1)

    def _span(self, S: torch.Tensor, transposed: bool = False) -> torch.Tensor:
        key = (S.data_ptr(), tuple(S.shape), S.dtype, S._version, transposed)
        sp = self._span_cache.get(key)
        if sp is None:
            if len(self._span_cache) > 32:
                self._span_cache.clear()
            sp = _tspan_of(S) if transposed else _span_of(S)
            self._span_cache[key] = sp
        return sp

    def chi_fine(self, cchi, reff, q, S=None, convention="feff"):
        """chi(q) = a(q) sin(phi(q) + 2 q reff) per path, a and the unwrapped phase phi of cchi interpolated by S
        (linear_matrix for "feff", spline_matrix for "larch").  Returns (B, len(q)) of S's dtype; differentiable in
        cchi and reff."""
        if S is None:
            S = self.linear_matrix(q) if convention == "feff" else self.spline_matrix(q)
        cdt = torch.complex128 if cchi.dtype == torch.complex128 else torch.complex64
        rdt = torch.float64 if cdt == torch.complex128 else torch.float32
        Sd = S.to(self.device, rdt).contiguous()
        qt = torch.as_tensor(q, device=self.device, dtype=rdt).contiguous()
        out = _ChiFine.apply(cchi.to(self.device, cdt), reff.to(self.device, rdt), qt, Sd, self)
        return out.to(S.dtype)

    def _chi_fine_forward(self, cchi, reff, q, S):
        B, NK = cchi.shape[0], q.shape[0]
        prec = _lib.FG_FP64 if cchi.dtype == torch.complex128 else _lib.FG_MIXED
        cchi, reff = cchi.contiguous(), reff.contiguous()
        out = torch.empty(B, NK, device=self.device, dtype=reff.dtype)
        _lib.check(self._lib.fg_chi_fine(self._h, prec, B, cchi.data_ptr(), reff.data_ptr(), NK, q.data_ptr(),
                                         S.data_ptr(), self._span(S).data_ptr(), out.data_ptr(), _stream(self.device)))
        return out

    def _chi_fine_backward(self, cchi, reff, q, S, g):
        B, NK = cchi.shape[0], q.shape[0]
        prec = _lib.FG_FP64 if cchi.dtype == torch.complex128 else _lib.FG_MIXED
        gc = torch.empty_like(cchi)
        gr = torch.empty_like(reff)
        g = g.to(reff.dtype).contiguous()
        _lib.check(self._lib.fg_chi_fine_backward(self._h, prec, B, cchi.contiguous().data_ptr(),
                                                  reff.contiguous().data_ptr(), NK, q.data_ptr(), S.data_ptr(),
                                                  self._span(S).data_ptr(), self._span(S, True).data_ptr(),
                                                  g.data_ptr(), gc.data_ptr(), gr.data_ptr(), _stream(self.device)))
        return gc, gr

    # -- feffNNNN.dat columns ------------------------------------------------------------------------------
    def _energy_columns(self):
        """Per energy: k, real[2 phc], red factor, lambda, real[p] (FEFF's units) and the (E, 4) device table of
        fg_path_columns.  phc is the absorber's phase shift in the channel l = l_init + 1 (kappa > 0: l = l_init,
        as FEFF's fdtarr.f picks it); its doubled real part is unwrapped along the energies."""
        if getattr(self, "_ecols", None) is None:
            P, E = self.P, self.E
            ll = self.ilinit if self.kinit > 0 else -self.ilinit
            caps = np.asarray(P.ph)[:E, ll + P.ltot, 0, 0]
            ck = np.sqrt(2 * (np.asarray(P.em)[:E] - np.asarray(P.eref)[:E, 0]))
            red = np.exp(-2 * caps.imag)
            raw = 2 * caps.real
            cdelt = raw.copy()
            for i in range(1, E):                      # sequential unwrap of 2 pi jumps (FEFF's pijump)
                d = raw[i] - cdelt[i - 1]
                cdelt[i] = cdelt[i - 1] + d - 2 * np.pi * np.round(d / (2 * np.pi))
            lam = np.where(np.abs(ck.imag) > 1e-16, 1 / np.where(np.abs(ck.imag) > 1e-16, ck.imag, 1.0), 1e10)
            shift = cdelt + self.ilinit * np.pi
            table = np.stack([np.abs(self._xk), 2 / lam, 1 / red, shift], 1)
            self._ecols = ({"k": self._xk / BOHR, "real_phc": shift, "red_fact": red, "lam": lam * BOHR,
                            "rep": ck.real / BOHR}, torch.tensor(table, device=self.device, dtype=torch.float64))
        return self._ecols

    def geometry(self, coords_bohr):
        """ri (B, nleg), beta (B, nleg), eta (B, nleg) for legs 1..nleg of paths coords (B, nleg, 3) in bohr, absorber
        first -- the reference's GPUPathStage.geometry (stage.py:170-206), with its branch choices: FP64 on the
        device (fg_path_geometry), returned in the coordinates' dtype, differentiable in the coordinates."""
        x = torch.as_tensor(coords_bohr)
        if x.dim() != 3 or x.shape[2] != 3:
            raise ValueError("coords must be (B, nleg, 3)")
        return _Geometry.apply(x, self)

    def columns(self, cchi, reff) -> dict:
        """FEFF's feffNNNN.dat columns of paths from their signals (the reference's PathStage._columns,
        genfmt.py:449-461): cchi (B, E) and reff (B,) A as cchi() returns them.  Per path mag (B, E) (A) and phase
        (B, E) on the device; per energy k, real_phc, red_fact, lam, rep (numpy)."""
        shared, table = self._energy_columns()
        cc = torch.as_tensor(cchi, device=self.device)
        if cc.dim() == 1:
            cc = cc[None]
        prec = _lib.FG_FP64 if cc.dtype == torch.complex128 else _lib.FG_MIXED
        cc = cc.to(torch.complex128 if prec == _lib.FG_FP64 else torch.complex64).contiguous()
        rf = torch.as_tensor(reff, device=self.device).reshape(-1).to(
            torch.float64 if prec == _lib.FG_FP64 else torch.float32).contiguous()
        B = int(cc.shape[0])
        if cc.shape[1] != self.E or rf.shape[0] != B:
            raise ValueError("cchi must be (B, E) and reff (B,)")
        mag = torch.empty(B, self.E, device=self.device, dtype=torch.float64)
        phase = torch.empty_like(mag)
        _lib.check(self._lib.fg_path_columns(B, self.E, prec, cc.data_ptr(), rf.data_ptr(), table.data_ptr(),
                                             mag.data_ptr(), phase.data_ptr(), _stream(self.device)))
        return dict(shared, mag=mag, phase=phase)

    # -- launch shape ---------------------------------------------------------------------------------------
    def set_launch(self, fwd_warps: int = 0, bwd_warps: int = 0, regs_alt: int = 0, stage_t: int = 0) -> None:
        """Warps per CTA of this stage's forward and adjoint kernels (0 = the library default), and the fused
        forward's register budget (1: three CTAs of 128 threads per SM) and t-matrix staging (1: through shared
        memory)."""
        want = (int(fwd_warps), int(bwd_warps), int(regs_alt), int(stage_t))
        if want != self._launch:
            _lib.check(self._lib.fg_stage_set_launch(self._h, want[0], want[1]))
            _lib.check(self._lib.fg_stage_set_fused_variant(self._h, want[2], want[3]))
            self._launch = want

    def tune(self, batch: "PathBatch", q, S=None, backward: bool = True, dtype=None, tuner=None):
        """Times the launch shapes on (a sample of) batch, applies and returns the fastest
        (fwd_warps, bwd_warps, regs_alt, stage_t)."""
        from .autotune import default_tuner
        if S is None:
            S = self.linear_matrix(q)
        Sd = torch.as_tensor(S).to(self.device, torch.float64).contiguous()
        qt = torch.as_tensor(q, device=self.device, dtype=torch.float64).contiguous()
        prec = self.prec if dtype is None else (_lib.FG_FP64 if dtype == torch.complex128 else _lib.FG_MIXED)
        choice = (tuner or default_tuner()).tune(self, batch, qt, Sd, prec, backward)
        batch._tuned[(id(self), prec, int(qt.shape[0]))] = choice
        self.set_launch(*choice)
        return choice

    def _pick_launch(self, batch, qt, Sd, prec, backward: bool) -> None:
        if not self.autotune:
            return
        from .autotune import default_tuner, signature
        key = (id(self), prec, int(qt.shape[0]))
        choice = batch._tuned.get(key)
        if choice is None or (backward and choice[1] == 0):
            tuner = default_tuner()
            choice = tuner.lookup(signature(self, batch, int(qt.shape[0]), prec), backward)
            if choice is None and not torch.cuda.is_current_stream_capturing():
                choice = tuner.tune(self, batch, qt, Sd, prec, backward)
            if choice is None:
                return
            batch._tuned[key] = choice
        self.set_launch(*choice)

    # -- fused stage ----------------------------------------------------------------------------------------
    def chi_reduce(self, batch: "PathBatch", q, S=None, coords=None, sigma2=None, dtype=None):
        """rows (nrows, len(q)) FP64: sum over the batch's paths of deg exp(-2 sigma2 q^2) chi_path(q) into each
        path's row, exact in the terms (the result does not depend on the evaluation order).  ``coords`` (n, nleg_max, 3) A replaces the batch's coordinates (same
        paths, new positions); ``sigma2`` (n,) A^2 per path.  Differentiable in coords and sigma2.  ``dtype``
        complex64 / complex128 overrides the stage's precision for this call."""
        if S is None:
            S = self.linear_matrix(q)
        Sd = torch.as_tensor(S).to(self.device, torch.float64).contiguous()
        qt = torch.as_tensor(q, device=self.device, dtype=torch.float64).contiguous()
        crd = batch.coords if coords is None else coords
        crd = crd.to(self.device, torch.float64)
        s2 = None if sigma2 is None else torch.as_tensor(sigma2).to(self.device, torch.float64)
        prec = self.prec if dtype is None else (_lib.FG_FP64 if dtype == torch.complex128 else _lib.FG_MIXED)
        if batch.max_ipot > self.P.nph:
            raise IndexError(f"potential index {batch.max_ipot} out of range 0..{self.P.nph}")
        grad = torch.is_grad_enabled() and (crd.requires_grad or (s2 is not None and s2.requires_grad))
        self._pick_launch(batch, qt, Sd, prec, backward=grad)
        if s2 is None:
            return _ChiReduce.apply(crd, qt, Sd, self, batch, prec)
        return _ChiReduceS2.apply(crd, s2, qt, Sd, self, batch, prec)

    def _reduce_args(self, batch, q, S, coords, sigma2, dtype):
        """chi_reduce's argument preparation: (coords, sigma2, q, S, prec) on the device."""
        if S is None:
            S = self.linear_matrix(q)
        Sd = torch.as_tensor(S).to(self.device, torch.float64).contiguous()
        qt = torch.as_tensor(q, device=self.device, dtype=torch.float64).contiguous()
        crd = (batch.coords if coords is None else coords).to(self.device, torch.float64)
        s2 = None if sigma2 is None else torch.as_tensor(sigma2).to(self.device, torch.float64)
        prec = self.prec if dtype is None else (_lib.FG_FP64 if dtype == torch.complex128 else _lib.FG_MIXED)
        if batch.max_ipot > self.P.nph:
            raise IndexError(f"potential index {batch.max_ipot} out of range 0..{self.P.nph}")
        grad = torch.is_grad_enabled() and (crd.requires_grad or (s2 is not None and s2.requires_grad))
        self._pick_launch(batch, qt, Sd, prec, backward=grad)
        return crd, s2, qt, Sd, prec

    def _paths_struct(self, batch, coords, sigma2):
        return _lib.Paths(batch.n, batch.nleg_max, batch.nrows, coords.data_ptr(), batch.ipots.data_ptr(),
                          batch.nleg.data_ptr(), batch.deg.data_ptr(), _ptr(sigma2), batch.row.data_ptr(),
                          batch.order.data_ptr())

    def rows_from_words(self, words: torch.Tensor) -> torch.Tensor:
        """rows (nrows, NK) FP64 from exact row-sum words (2, nrows, NK) int64 as chi_reduce_words leaves them, or
        their integer sum over ranks (fg_rows_from_words)."""
        w = words.contiguous()
        if w.dim() != 3 or w.shape[0] != 2 or w.dtype != torch.int64:
            raise ValueError("words must be (2, nrows, NK) int64")
        rows = torch.empty(int(w.shape[1]), int(w.shape[2]), device=w.device, dtype=torch.float64)
        _lib.check(self._lib.fg_rows_from_words(int(w.shape[1]), int(w.shape[2]), w.data_ptr(), rows.data_ptr(),
                                                _stream(self.device)))
        return rows

    def _chi_reduce_words(self, batch, coords, sigma2, q, S, prec, save: bool):
        """The fused forward with its exact row sums left as words (2, nrows, NK) int64 (fg_chi_reduce_words)."""
        coords = coords.contiguous()
        NK = q.shape[0]
        ps = self._paths_struct(batch, coords, sigma2)
        words = torch.empty(2, batch.nrows, NK, device=self.device, dtype=torch.int64)
        ws = batch.workspace(256)
        cchi = reff = None
        if save:
            cchi = torch.empty(batch.n, self.E, device=self.device,
                               dtype=torch.complex128 if prec == _lib.FG_FP64 else torch.complex64)
            reff = torch.empty(batch.n, device=self.device, dtype=torch.float64)
        _lib.check(self._lib.fg_chi_reduce_words(self._h, prec, C.byref(ps), NK, q.data_ptr(), S.data_ptr(),
                                                 self._span(S).data_ptr(), words.data_ptr(), _ptr(cchi), _ptr(reff),
                                                 ws.data_ptr(), 256, _stream(self.device)))
        return words, cchi, reff

    def _chi_reduce_forward(self, batch, coords, sigma2, q, S, prec, save: bool):
        coords = coords.contiguous()
        NK = q.shape[0]
        ps = self._paths_struct(batch, coords, sigma2)
        rows = torch.empty(batch.nrows, NK, device=self.device, dtype=torch.float64)
        ws_n = int(self._lib.fg_chi_reduce_workspace(self._h, C.byref(ps), NK))
        ws = batch.workspace(ws_n)
        cchi = reff = None
        if save:
            cchi = torch.empty(batch.n, self.E, device=self.device,
                               dtype=torch.complex128 if prec == _lib.FG_FP64 else torch.complex64)
            reff = torch.empty(batch.n, device=self.device, dtype=torch.float64)
        _lib.check(self._lib.fg_chi_reduce(self._h, prec, C.byref(ps), NK, q.data_ptr(), S.data_ptr(),
                                           self._span(S).data_ptr(), rows.data_ptr(), _ptr(cchi), _ptr(reff),
                                           ws.data_ptr(), ws_n, _stream(self.device)))
        return rows, cchi, reff

    def _chi_reduce_backward(self, batch, coords, sigma2, q, S, prec, g_rows, cchi, reff, want_s2: bool):
        choice = batch._tuned.get((id(self), prec, int(q.shape[0]))) if self.autotune else None
        if choice is not None:
            self.set_launch(*choice)
        coords = coords.contiguous()
        NK = q.shape[0]
        ps = self._paths_struct(batch, coords, sigma2)
        gc = torch.empty_like(coords)
        gs = torch.empty(batch.n, device=self.device, dtype=torch.float64) if want_s2 else None
        ws_n = int(self._lib.fg_chi_reduce_backward_workspace(self._h, C.byref(ps), NK))
        ws = batch.workspace(ws_n, backward=True)
        _lib.check(self._lib.fg_chi_reduce_backward(self._h, prec, C.byref(ps), NK, q.data_ptr(), S.data_ptr(),
                                                    self._span(S).data_ptr(), self._span(S, True).data_ptr(),
                                                    g_rows.contiguous().data_ptr(),
                                                    cchi.data_ptr(), reff.data_ptr(), gc.data_ptr(), _ptr(gs),
                                                    ws.data_ptr(), ws_n, _stream(self.device)))
        return gc, gs


class _Cchi(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, ipots, stage):
        out, reff = stage._cchi_forward(coords, ipots)
        ctx.save_for_backward(coords, ipots)
        ctx.stage = stage
        return out, reff

    @staticmethod
    def backward(ctx, g_cchi, g_reff):
        coords, ipots = ctx.saved_tensors
        if not ctx.needs_input_grad[0]:
            return None, None, None
        return ctx.stage._cchi_backward(coords, ipots, g_cchi, g_reff), None, None


class _Geometry(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, stage):
        x64 = x.detach().to(stage.device, torch.float64).contiguous()
        B, nleg = int(x64.shape[0]), int(x64.shape[1])
        ri, beta, eta = (torch.empty(B, nleg, device=stage.device, dtype=torch.float64) for _ in range(3))
        _lib.check(stage._lib.fg_path_geometry(B, nleg, x64.data_ptr(), ri.data_ptr(), beta.data_ptr(),
                                               eta.data_ptr(), _stream(stage.device)))
        ctx.save_for_backward(x64)
        ctx.stage, ctx.dtype, ctx.in_device = stage, x.dtype, x.device
        return ri.to(x.dtype), beta.to(x.dtype), eta.to(x.dtype)

    @staticmethod
    def backward(ctx, g_ri, g_beta, g_eta):
        (x64,) = ctx.saved_tensors
        if not ctx.needs_input_grad[0]:
            return None, None
        B, nleg = int(x64.shape[0]), int(x64.shape[1])
        gs = [torch.zeros(B, nleg, device=x64.device, dtype=torch.float64) if g is None
              else g.to(torch.float64).contiguous() for g in (g_ri, g_beta, g_eta)]
        grad = torch.empty_like(x64)
        st = ctx.stage
        _lib.check(st._lib.fg_path_geometry_backward(B, nleg, x64.data_ptr(), gs[0].data_ptr(), gs[1].data_ptr(),
                                                     gs[2].data_ptr(), grad.data_ptr(), _stream(st.device)))
        return grad.to(ctx.in_device, ctx.dtype), None


class _ChiFine(torch.autograd.Function):
    @staticmethod
    def forward(ctx, cchi, reff, q, S, stage):
        out = stage._chi_fine_forward(cchi, reff, q, S)
        ctx.save_for_backward(cchi, reff, q, S)
        ctx.stage = stage
        return out

    @staticmethod
    def backward(ctx, g):
        cchi, reff, q, S = ctx.saved_tensors
        gc, gr = ctx.stage._chi_fine_backward(cchi, reff, q, S, g)
        return (gc if ctx.needs_input_grad[0] else None), (gr if ctx.needs_input_grad[1] else None), None, None, None


class _ChiReduce(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, q, S, stage, batch, prec):
        need = ctx.needs_input_grad[0]
        rows, cchi, reff = stage._chi_reduce_forward(batch, coords, None, q, S, prec, save=need)
        if need:
            ctx.save_for_backward(coords, q, S, cchi, reff)
        ctx.stage, ctx.batch, ctx.prec = stage, batch, prec
        return rows

    @staticmethod
    def backward(ctx, g):
        coords, q, S, cchi, reff = ctx.saved_tensors
        gc, _ = ctx.stage._chi_reduce_backward(ctx.batch, coords, None, q, S, ctx.prec, g, cchi, reff, False)
        return gc, None, None, None, None, None


class _ChiReduceS2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, sigma2, q, S, stage, batch, prec):
        need = ctx.needs_input_grad[0] or ctx.needs_input_grad[1]
        rows, cchi, reff = stage._chi_reduce_forward(batch, coords, sigma2, q, S, prec, save=need)
        if need:
            ctx.save_for_backward(coords, sigma2, q, S, cchi, reff)
        ctx.stage, ctx.batch, ctx.prec = stage, batch, prec
        return rows

    @staticmethod
    def backward(ctx, g):
        coords, sigma2, q, S, cchi, reff = ctx.saved_tensors
        gc, gs = ctx.stage._chi_reduce_backward(ctx.batch, coords, sigma2, q, S, ctx.prec, g, cchi, reff, True)
        return (gc if ctx.needs_input_grad[0] else None), (gs if ctx.needs_input_grad[1] else None), None, None, \
            None, None, None
