"""Phase tables for the path stage: FEFF's ``phase.pad`` reader, the ``PhaseData`` container, and resampling.

``PhaseData``, ``read_phase_pad`` and ``load_phase`` keep the names, fields and units of the reference's phase-file
boundary (``src/feffgpu/pad.py:69-151, 249-280``): energies in hartree, lengths in bohr, ``ph[ie, l + ltot, isp,
iph]`` the complex phase shifts for l = -lmax0..lmax0 (the j = l -/+ 1/2 channels), ``rkk[ie, k, isp]`` the reduced
matrix elements.  ``lmax``, ``xk`` and ``ck`` are derived as FEFF's rdxsph and genfmt_prep derive them.

``resample_phase`` (no reference counterpart; the reference's energy mesh stops at 100 real-axis points) puts a
phase file on a uniform k grid so that a stage can run on, e.g., 401 k points from 0 to 20 1/A.
"""
from __future__ import annotations

import pickle
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

BOHR = 0.52917721067      # A per bohr (pad.py:13)
HART = 2.0 * 13.60569301  # eV per hartree
PHMIN = 1.0e-7            # a phase shift counts while |sin(delta)| exceeds this (rdxsph)

# FEFF's packed-ASCII encoding (COMMON/padlib.f): base-90 digits offset by 37, first character the decimal exponent
_IOFF, _IBASE, _IBAS2 = 37, 90, 45


def _unpack(bodies: list[str], npack: int) -> np.ndarray:
    """Decode fixed-width packed numbers; `bodies` are strings of npack characters each."""
    if not bodies:
        return np.zeros(0)
    a = np.frombuffer("".join(bodies).encode("latin-1"), dtype=np.uint8).reshape(-1, npack).astype(np.int64) - _IOFF
    expo = a[:, 0] - _IBAS2
    lead = a[:, 1]
    sign = np.where(lead % 2 == 1, 1.0, -1.0)
    mant = (lead // 2) / float(_IBASE * _IBASE)
    for i in range(npack, 2, -1):                 # least significant digit first, as padlib sums them
        mant = mant + a[:, i - 1] / float(_IBASE) ** i
    # powers of ten by the C library's pow, one per distinct exponent (numpy's vectorised power can differ by an ulp)
    uniq, inv = np.unique(expo, return_inverse=True)
    scale = np.array([10.0 ** int(v) for v in uniq])[inv]
    return 2.0 * sign * _IBASE * mant * scale


class _Reader:
    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.i = 0

    def line(self) -> str:
        s = self.lines[self.i]
        self.i += 1
        return s

    def _numbers(self, marker: str, width: int, count: int) -> list[str]:
        out: list[str] = []
        while len(out) < count:
            s = self.line().rstrip()
            if not s or s[0] != marker:
                raise ValueError(f"expected a packed line starting with {marker!r}, got {s[:20]!r}")
            body = s[1:]
            take = min(len(body) // width, count - len(out))
            out.extend(body[j * width:(j + 1) * width] for j in range(take))
        return out

    def reals(self, npack: int, count: int) -> np.ndarray:
        return _unpack(self._numbers("!", npack, count), npack)

    def complexes(self, npack: int, count: int) -> np.ndarray:
        pairs = self._numbers("$", 2 * npack, count)
        flat = []
        for p in pairs:
            flat.append(p[:npack])
            flat.append(p[npack:])
        v = _unpack(flat, npack)
        return v[0::2] + 1j * v[1::2]


@dataclass
class PhaseData:
    """Everything the path stage reads from a phase file (same fields as the reference's ``PhaseData``)."""
    nsp: int
    ne: int
    ne1: int
    ne3: int
    nph: int
    ihole: int
    ik0: int
    ixc: int
    rs: float
    vint: float
    rnrmav: float
    xmu: float
    edge: float
    em: np.ndarray
    eref: np.ndarray
    lmax0: np.ndarray
    iz: np.ndarray
    potlbl: list = field(default_factory=list)
    ph: np.ndarray = None
    rkk: np.ndarray = None
    ltot: int = 0

    @property
    def lmax(self) -> np.ndarray:
        """(ne, nph+1): the largest l whose phase shift is not negligible (rdxsph's rule)."""
        out = np.zeros((self.ne, self.nph + 1), int)
        s0 = np.abs(np.sin(self.ph[:, :, 0, :]))
        s1 = np.abs(np.sin(self.ph[:, :, self.nsp - 1, :]))
        big = (s0 > PHMIN) | (s1 > PHMIN)                 # (ne, 2 ltot + 1, nph+1)
        for iph in range(self.nph + 1):
            ls = np.arange(int(self.lmax0[iph]), -1, -1)
            hit = big[:, ls + self.ltot, iph]              # (ne, lmax0+1), l descending
            first = np.argmax(hit, axis=1)
            out[:, iph] = np.where(hit.any(axis=1), ls[first], 0)
        return out

    def phase(self, ie, l, iph, isp=0):
        return self.ph[ie, l + self.ltot, isp, iph]

    @property
    def xk(self) -> np.ndarray:
        """Real momentum relative to the edge (bohr^-1)."""
        e = np.asarray(self.em).real - self.edge
        return np.sign(e) * np.sqrt(np.abs(2 * e))

    @property
    def ck(self) -> np.ndarray:
        """Complex momentum p = sqrt(2 (E - E_ref)), spin averaged."""
        eref = self.eref[:, 0] if self.nsp == 1 else 0.5 * (self.eref[:, 0] + self.eref[:, -1])
        return np.sqrt(2 * (self.em - eref))


def read_phase_pad(filename) -> PhaseData:
    """FEFF 8.5L's phase.pad (COMMON/rdxsph.f layout) as a PhaseData."""
    text = Path(filename).read_text(encoding="latin-1")
    rd = _Reader(text)
    head = rd.line()
    nsp, ne, ne1, ne3, nph, ihole, ik0, npadx, ixc = (int(head[1 + 5 * j:5 + 5 * j]) for j in range(9))
    rs, vint = float(head[45:56]), float(head[56:67])
    rnrmav, xmu, edge = rd.reals(npadx, 3)
    em = rd.complexes(npadx, ne)
    eref = rd.complexes(npadx, ne * nsp).reshape(nsp, ne).T
    lmax0, iz, potlbl, blocks = [], [], [], []
    for _ in range(nph + 1):
        s = rd.line()
        lmax0.append(int(s[1:4])); iz.append(int(s[5:8])); potlbl.append(s[9:15].strip())
        nl = 2 * lmax0[-1] + 1
        blocks.append(np.stack([rd.complexes(npadx, ne * nl).reshape(ne, nl) for _ in range(nsp)], -1))
    ltot = max(lmax0)
    ph = np.zeros((ne, 2 * ltot + 1, nsp, nph + 1), complex)
    for iph, blk in enumerate(blocks):
        lo = ltot - lmax0[iph]
        ph[:, lo:lo + blk.shape[1], :, iph] = blk
    rkk = rd.complexes(npadx, ne * 8 * nsp).reshape(nsp, 8, ne).transpose(2, 1, 0)
    return PhaseData(nsp, ne, ne1, ne3, nph, ihole, ik0, ixc, rs, vint, float(rnrmav), float(xmu), float(edge), em, eref,
                     np.array(lmax0), np.array(iz), potlbl, ph, rkk, ltot)


def load_phase(phase) -> PhaseData:
    """A phase file: the object itself (anything with ``iz`` and ``ph``), a phase.pad, a pickle, or an ``.npz``
    written by ``save_phase``.  A pickle can run code when loaded: load only files you trust."""
    if isinstance(phase, PhaseData) or (hasattr(phase, "iz") and hasattr(phase, "ph")):
        return phase
    p = Path(phase)
    if not p.is_file():
        raise FileNotFoundError(f"no such phase file: {p}")
    if p.suffix.lower() == ".npz":
        return phase_from_npz(np.load(p, allow_pickle=False))
    with open(p, "rb") as f:
        head = f.read(1)
    if head == b"\x80" or p.suffix.lower() in (".pkl", ".pickle"):
        with open(p, "rb") as f:
            obj = pickle.load(f)
        if not (hasattr(obj, "iz") and hasattr(obj, "ph")):
            raise ValueError(f"{p}: the pickle does not hold a phase file (got {type(obj).__name__})")
        return obj
    return read_phase_pad(str(p))


_SCALARS = ("nsp", "ne", "ne1", "ne3", "nph", "ihole", "ik0", "ixc", "rs", "vint", "rnrmav", "xmu", "edge", "ltot")


def phase_to_arrays(P, prefix: str = "", trim: bool = True) -> dict:
    """The fields of a phase file as plain arrays (for np.savez).  trim keeps the first ne1 energies and the l the
    stage can reach (the largest lmax over those energies), which changes nothing the path stage computes."""
    ne = int(P.ne1) if trim else int(P.ne)
    ph = np.asarray(P.ph)[:ne]
    ltot, lmax0 = int(P.ltot), np.asarray(P.lmax0).copy()
    if trim:
        Q = PhaseData(P.nsp, ne, ne, 0, P.nph, P.ihole, P.ik0, P.ixc, P.rs, P.vint, P.rnrmav, P.xmu, P.edge,
                      np.asarray(P.em)[:ne], np.asarray(P.eref)[:ne], lmax0, np.asarray(P.iz), list(P.potlbl), ph,
                      np.asarray(P.rkk)[:ne], ltot)
        lt = int(Q.lmax.max())
        ph = ph[:, ltot - lt:ltot + lt + 1]
        ltot = lt
        lmax0 = np.minimum(lmax0, lt)
    out = {prefix + k: np.asarray(getattr(P, k)) for k in _SCALARS if k not in ("ne", "ne3", "ltot")}
    out.update({prefix + "ne": np.asarray(ne), prefix + "ne3": np.asarray(0 if trim else P.ne3), prefix + "ltot": np.asarray(ltot),
                prefix + "em": np.asarray(P.em)[:ne], prefix + "eref": np.asarray(P.eref)[:ne], prefix + "lmax0": lmax0,
                prefix + "iz": np.asarray(P.iz), prefix + "ph": ph, prefix + "rkk": np.asarray(P.rkk)[:ne],
                prefix + "potlbl": np.array([str(s) for s in P.potlbl])})
    if trim:
        out[prefix + "ne1"] = np.asarray(ne)
    return out


def phase_from_npz(z, prefix: str = "") -> PhaseData:
    g = lambda k: z[prefix + k]
    return PhaseData(int(g("nsp")), int(g("ne")), int(g("ne1")), int(g("ne3")), int(g("nph")), int(g("ihole")),
                     int(g("ik0")), int(g("ixc")), float(g("rs")), float(g("vint")), float(g("rnrmav")), float(g("xmu")),
                     float(g("edge")), np.asarray(g("em")), np.asarray(g("eref")), np.asarray(g("lmax0")),
                     np.asarray(g("iz")), [str(s) for s in g("potlbl")], np.asarray(g("ph")), np.asarray(g("rkk")),
                     int(g("ltot")))


def save_phase(P, filename) -> None:
    np.savez_compressed(filename, **phase_to_arrays(P))


def resample_phase(P, k) -> PhaseData:
    """The phase file on the real-axis grid k (1/A, ascending, from 0): phase shifts, energy reference and matrix
    elements are interpolated linearly in the file's own momentum grid (each clamped to its end values beyond the
    grid), em = edge + (k bohr)^2 / 2 + i Im(em) interpolated.  lmax follows from the interpolated phase shifts."""
    k = np.asarray(k, float)
    E = int(P.ne1)
    xk0 = np.asarray(P.xk)[:E]
    xk1 = k * BOHR
    order = np.argsort(xk0)
    xs = xk0[order]

    def interp(v):
        v = np.asarray(v)[:E][order]
        flat = v.reshape(E, -1)
        out = np.empty((len(xk1), flat.shape[1]), complex)
        for j in range(flat.shape[1]):
            out[:, j] = np.interp(xk1, xs, flat[:, j].real) + 1j * np.interp(xk1, xs, flat[:, j].imag)
        return out.reshape((len(xk1),) + v.shape[1:])

    em_im = np.interp(xk1, xs, np.asarray(P.em)[:E][order].imag)
    em = P.edge + np.sign(xk1) * xk1 ** 2 / 2 + 1j * em_im
    n = len(k)
    return PhaseData(P.nsp, n, n, 0, P.nph, P.ihole, P.ik0, P.ixc, P.rs, P.vint, P.rnrmav, P.xmu, P.edge, em,
                     interp(P.eref), np.asarray(P.lmax0).copy(), np.asarray(P.iz).copy(), list(P.potlbl),
                     interp(P.ph), interp(P.rkk), int(P.ltot))
