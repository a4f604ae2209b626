"""FP64 CPU oracle of the path stage -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this module, and only as the
checker.  The product package ``feffgpu_b200`` never imports it.

It restates the reference's path stage on the CPU:

* ``cchi`` -- the per-path complex signal on the phase file's real-axis grid, from the C restatement in
  ``oracle/feff_oracle.c`` (FEFF GENFMT as ported in ``src/feffgpu/genfmt.py:279-447``).
* ``phase_tables`` -- ``lmax``, ``xk`` and ``ck`` of a phase file (``src/feffgpu/pad.py:93-121``).
* ``linear_matrix``, ``unwrap``, ``chi_fine`` -- the fine-grid signal (``src/feffgpu/stage.py:353-388``), numpy.
* ``chi_rows`` -- the degeneracy-weighted sum of paths into rows (``src/feffgpu/chain.py:48-49``,
  ``src/feffgpu/exafs/forward.py:162``), with the per-path factor exp(-2 sigma^2 q^2), a new input without a
  counterpart in the reference (sigma^2 = 0 gives the reference's sum).
* ``r_factor`` -- the parity metric (``src/feffgpu/compare.py:6-27``).
* ``columns`` -- the feffNNNN.dat columns (``src/feffgpu/genfmt.py:449-461``, with ``pijump_unwrap`` of
  ``genfmt.py:267-276``).
* ``fd_gradient`` -- central finite differences of any of the above with respect to the path coordinates.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libfeff_oracle.so"
BOHR = 0.52917721067
PHMIN = 1.0e-7
EPS = 1.0e-16


def build(force: bool = False) -> Path:
    """Compile the C oracle with the Makefile beside this file (gcc, pthreads)."""
    if force or not LIB.exists() or LIB.stat().st_mtime < (HERE / "feff_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        lib.fo_cchi.restype = ctypes.c_int
        lib.fo_cchi.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.fo_lambda.restype = ctypes.c_int
        lib.fo_lambda.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p]
        lib.fo_wigner_d.restype = None
        lib.fo_wigner_d.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
        lib.fo_geometry.restype = None
        lib.fo_geometry.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib = lib
    return _lib


class _Phase(ctypes.Structure):
    _fields_ = [("E", ctypes.c_int), ("nph", ctypes.c_int), ("ltot", ctypes.c_int), ("ihole", ctypes.c_int),
                ("iorder", ctypes.c_int), ("lmax", ctypes.c_void_p), ("ph", ctypes.c_void_p), ("xk", ctypes.c_void_p),
                ("ck", ctypes.c_void_p), ("rkk", ctypes.c_void_p)]


def phase_tables(P):
    """lmax (ne1, nph+1), xk (ne1,) bohr^-1 and ck (ne1,) complex of a phase-file object (pad.py:93-121)."""
    E = int(P.ne1)
    ph = np.asarray(P.ph)
    lmax = np.zeros((E, P.nph + 1), np.int32)
    for iph in range(P.nph + 1):
        for ie in range(E):
            lm = 0
            for l in range(int(P.lmax0[iph]), -1, -1):
                lm = l
                if abs(np.sin(ph[ie, l + P.ltot, 0, iph])) > PHMIN or abs(np.sin(ph[ie, l + P.ltot, P.nsp - 1, iph])) > PHMIN:
                    break
            lmax[ie, iph] = lm
    e = np.asarray(P.em).real[:E] - P.edge
    xk = np.sign(e) * np.sqrt(np.abs(2 * e))
    eref = np.asarray(P.eref)
    eref = eref[:, 0] if P.nsp == 1 else 0.5 * (eref[:, 0] + eref[:, -1])
    ck = np.sqrt(2 * (np.asarray(P.em)[:E] - eref[:E]))
    return lmax, xk, ck


class Oracle:
    """The oracle for one phase file."""

    def __init__(self, P, iorder: int = 2):
        if P.nsp != 1:
            raise NotImplementedError("spin-dependent phase files are not ported")
        self.P, self.iorder = P, iorder
        self.E = int(P.ne1)
        self.lmax, self.xk, self.ck = phase_tables(P)
        E = self.E
        self._ph = np.ascontiguousarray(np.asarray(P.ph)[:E, :, 0, :].astype(np.complex128))
        self._xk = np.ascontiguousarray(self.xk, np.float64)
        self._ck = np.ascontiguousarray(self.ck, np.complex128)
        self._rkk = np.ascontiguousarray(np.asarray(P.rkk)[:E, :, 0].astype(np.complex128))
        self._lmax = np.ascontiguousarray(self.lmax, np.int32)
        self._s = _Phase(E, int(P.nph), int(P.ltot), int(P.ihole), int(iorder), self._lmax.ctypes.data,
                         self._ph.ctypes.data, self._xk.ctypes.data, self._ck.ctypes.data, self._rkk.ctypes.data)

    def cchi(self, coords, ipots, nthreads: int | None = None):
        """coords (B, nleg, 3) A, absorber first; ipots (B, nleg). Returns cchi (B, E) complex128, reff (B,) A."""
        coords = np.ascontiguousarray(np.asarray(coords, np.float64))
        ipots = np.ascontiguousarray(np.asarray(ipots, np.int64))
        B, nleg, _ = coords.shape
        out = np.zeros((B, self.E), np.complex128)
        reff = np.zeros(B, np.float64)
        n = nthreads if nthreads else (os.cpu_count() or 1)
        rc = _load().fo_cchi(ctypes.byref(self._s), nleg, B, coords.ctypes.data, ipots.ctypes.data, out.ctypes.data,
                             reff.ctypes.data, int(n))
        if rc == -2:
            raise NotImplementedError("icalc >= 10 or an unknown hole")
        if rc:
            raise ValueError(f"oracle status {rc}")
        return out, reff

    # -- fine grid -------------------------------------------------------------------------------------------
    def kgrid(self):
        """The real-axis k grid in 1/A."""
        return self.xk / BOHR

    def linear_matrix(self, q):
        return linear_matrix(self.kgrid(), q)

    def chi_fine(self, cchi, reff, q, S=None):
        if S is None:
            S = self.linear_matrix(q)
        return chi_fine(cchi, reff, q, S)


def lambda_set(ihole: int, nsc: int, iorder: int = 2):
    """(mlam[1..], nlam[1..], lamx, laml0x, mmaxp1, nmax) of the C oracle's setlam."""
    m = np.zeros(16, np.int32)
    n = np.zeros(16, np.int32)
    s = np.zeros(4, np.int32)
    rc = _load().fo_lambda(ihole, iorder, nsc, m.ctypes.data, n.ctypes.data, s.ctypes.data)
    if rc:
        raise ValueError(rc)
    return m[1:s[0] + 1].tolist(), n[1:s[0] + 1].tolist(), *[int(v) for v in s]


def wigner_d(beta: float, lmax: int):
    """(lmax+1, 7, 7) d^l_{mn}(beta) for |m|,|n| <= 3."""
    d = np.zeros((lmax + 1, 7, 7), np.float64)
    _load().fo_wigner_d(float(beta), int(lmax), d.ctypes.data)
    return d


def geometry(coords):
    """Leg lengths (A), scattering angles and Euler sums of one path (nleg, 3)."""
    c = np.ascontiguousarray(np.asarray(coords, np.float64))
    nleg = c.shape[0]
    ri, beta, eta = np.zeros(nleg), np.zeros(nleg), np.zeros(nleg)
    _load().fo_geometry(nleg, c.ctypes.data, ri.ctypes.data, beta.ctypes.data, eta.ctypes.data)
    return ri, beta, eta


# -- fine grid and sums (stage.py:353-388) ------------------------------------------------------------------------
def linear_matrix(kf, q):
    """(len(q), E): FEFF's linear interpolation from the real-axis grid kf (1/A), q clamped to the grid."""
    kf = np.asarray(kf, float)
    E = len(kf)
    qn = np.clip(np.asarray(q, float), kf[0], kf[-1])
    S = np.zeros((len(qn), E))
    j = np.clip(np.searchsorted(kf, qn, side="right") - 1, 0, E - 2)
    f = (qn - kf[j]) / (kf[j + 1] - kf[j])
    S[np.arange(len(qn)), j] = 1 - f
    S[np.arange(len(qn)), j + 1] = f
    return S


def unwrap(phase):
    d = np.diff(phase, axis=-1)
    d = d - 2 * math.pi * np.round(d / (2 * math.pi))
    return np.concatenate([phase[..., :1], phase[..., :1] + np.cumsum(d, -1)], -1)


def chi_fine(cchi, reff, q, S):
    """(B, len(q)): amplitude and unwrapped phase interpolated by S, chi = a sin(phi + 2 q reff)."""
    cchi = np.asarray(cchi)
    amp = np.sqrt(cchi.real ** 2 + cchi.imag ** 2 + 1e-30)
    pha = unwrap(np.where(amp >= 1e-16, np.angle(cchi), 0.0))
    a = amp @ S.T
    ph = pha @ S.T
    q = np.asarray(q, float)
    return a * np.sin(ph + 2 * q[None, :] * np.asarray(reff, float)[:, None])


def chi_rows(chi_paths, deg, rows, nrows, q, sigma2=None):
    """sum over paths of deg * chi_path * exp(-2 sigma2 q^2) into rows (nrows, NK), FP64 with math.fsum per entry."""
    chi_paths = np.asarray(chi_paths, float)
    w = np.asarray(deg, float)[:, None] * chi_paths
    if sigma2 is not None:
        w = w * np.exp(-2 * np.asarray(sigma2, float)[:, None] * np.asarray(q, float)[None, :] ** 2)
    out = np.zeros((nrows, chi_paths.shape[1]))
    rows = np.asarray(rows)
    for r in range(nrows):
        sel = w[rows == r]
        if len(sel):
            out[r] = [math.fsum(col) for col in sel.T]
    return out


# -- parity metric (compare.py:6-27) --------------------------------------------------------------------------------
def hanning(k, kmin, kmax, dk=1.0):
    k = np.asarray(k, float)
    if dk <= 0:
        return ((k >= kmin) & (k <= kmax)).astype(float)
    up = 0.5 * (1 - np.cos(np.pi * np.clip((k - (kmin - dk / 2)) / dk, 0, 1)))
    down = 0.5 * (1 + np.cos(np.pi * np.clip((k - (kmax - dk / 2)) / dk, 0, 1)))
    return up * down


def r_factor(k, data, fit, kmin=3.0, kmax=23.0, rmin=1.0, rmax=6.0, kweight=2, nfft=2048, dk=1.0):
    k, data, fit = (np.asarray(v, float) for v in (k, data, fit))
    step = k[1] - k[0]
    win = hanning(k, kmin, kmax, dk)
    f = lambda c: np.fft.fft(c * k ** kweight * win, n=nfft)[: nfft // 2] * step / math.sqrt(math.pi)
    r = np.arange(nfft // 2) * math.pi / (nfft * step)
    keep = (r >= rmin) & (r <= rmax)
    d, m = f(data)[keep], f(fit)[keep]
    return float(np.sum(np.abs(m - d) ** 2) / np.sum(np.abs(d) ** 2))


# -- feffNNNN.dat columns (genfmt.py:267-276, 449-461) ---------------------------------------------------------------
def pijump_unwrap(ph):
    out = np.array(ph, float)
    for i in range(1, len(out)):
        d = out[i] - out[i - 1]
        jump = int((abs(d) + np.pi) / (2 * np.pi))
        cands = [d, d - jump * 2 * np.pi, d + jump * 2 * np.pi]
        out[i] = out[i - 1] + min(cands, key=abs)
    return out


def columns(oracle: Oracle, cchi, reff_A):
    """The seven feffNNNN.dat columns of one path's cchi (E,) and reff (A)."""
    P = oracle.P
    E = oracle.E
    ilinit = _ilinit(P.ihole)
    kinit = _kinit(P.ihole)
    ll = ilinit if kinit > 0 else -ilinit
    caps = np.asarray(P.ph)[:E, ll + P.ltot, 0, 0]
    xk, ck = oracle.xk, oracle.ck
    reff = reff_A / BOHR
    amff = np.abs(cchi)
    phff = pijump_unwrap(np.where(amff >= EPS, np.angle(cchi), 0.0))
    xlam = np.where(np.abs(ck.imag) > EPS, 1 / np.where(np.abs(ck.imag) > EPS, ck.imag, 1.0), 1e10)
    redfac = np.exp(-2 * caps.imag)
    cdelt = pijump_unwrap(2 * caps.real)
    cfms = amff * np.exp(1j * phff) * xk * reff ** 2 * np.exp(2 * reff / xlam) / redfac
    return {"k": xk / BOHR, "real_phc": cdelt + ilinit * np.pi, "mag": np.abs(cfms) * BOHR,
            "phase": phff - cdelt - ilinit * np.pi, "red_fact": redfac, "lam": xlam * BOHR, "rep": ck.real / BOHR}


_KAP = [((1, 2, 5, 10, 17, 24, 27), (-1, 0)), ((3, 6, 11, 18, 25, 30), (1, 1)), ((4, 7, 12, 19, 26), (-2, 1)),
        ((8, 13, 20, 27), (2, 2)), ((9, 14, 21, 28), (-3, 2)), ((15, 22), (3, 3)), ((16, 23), (-4, 3))]


def _kinit(ihole):
    for holes, (k, _l) in _KAP:
        if ihole in holes:
            return k
    raise ValueError(ihole)


def _ilinit(ihole):
    for holes, (_k, l) in _KAP:
        if ihole in holes:
            return l + 1
    raise ValueError(ihole)


# -- gradients --------------------------------------------------------------------------------------------------------
def fd_gradient(fn, coords, h=1e-4):
    """Central differences of a scalar fn(coords) over every coordinate (A); coords (B, nleg, 3)."""
    c = np.array(coords, float)
    g = np.zeros_like(c)
    it = np.nditer(c, flags=["multi_index"])
    for _ in it:
        idx = it.multi_index
        cp = c.copy(); cp[idx] += h
        cm = c.copy(); cm[idx] -= h
        g[idx] = (fn(cp) - fn(cm)) / (2 * h)
    return g
