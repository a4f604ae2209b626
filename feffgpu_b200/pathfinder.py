"""FEFF's path finder on the B200: the reference's ``GPUPathFinder`` (``src/feffgpu/pathfinder.py``), batched over
absorbers.

Same constructor and ``enumerate(pos, box, absorber, ipot)`` output as the reference, so its front ends
(``chain.py:35-36``, ``exafs/forward.py:611-644``) can call it unchanged; ``enumerate_many`` runs every absorber of
every frame of an MD or RMC job in one set of launches.  The enumeration, the path geometry, the plane-wave
importance and the degeneracy keys are CUDA kernels (``csrc/fg_paths.cu``, C ABI ``fg_pf_*``); the merges and the
importance cut are index bookkeeping done here with torch on the device (sorts, unique, gathers), the greedy
length windows of the accidental-degeneracy merge on the host (``fg_pf_windows``).  A call for one absorber (how
the reference's front ends call it) is one library call, ``fg_pf_enumerate_one``: the same kernels driven from C++,
the merges and the cut on the host after one copy of the fields they read, with the same FP32 arithmetic and order
(a few hundred paths are not worth the dispatch latency of many small host-driven steps).

Algorithm (pathfinder.py:159-279): a path of nleg legs is a sequence of nleg - 1 intermediates (the absorber's
candidates -- atoms within rmax, minimum image, in atom order -- then the absorber itself), first and last a
candidate, no atom followed by itself, closed length at most 2 rmax; of a sequence and its reverse the smaller is
kept with degeneracy 2 (1 for a palindrome).  Single-scattering paths with the same distance to 1e-3 A, potential
and greedy 1e-3 A length window merge (pathfinder.py:102-132); multiple-scattering paths are filtered on the summed
degeneracy of their geometry class (pathfinder.py:134-157); the cut keeps paths whose degeneracy-weighted importance
is at least critpw percent of the shortest single-scattering path's (pathfinder.py:271-279).  All lengths are FP32,
as in the reference.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .cell import as_cell, cell_words
from .pad import BOHR, load_phase, read_phase_pad

NBETA = 40
NLEG_MAX = 9                # pathfinder.py:24, FEFF's npatx = 8 scatterers
PARTIAL_LIMIT = 30_000_000  # partial paths per absorber (pathfinder.py:25)


def _legendre_table(x: np.ndarray, lmax: int) -> np.ndarray:
    """P_l(x) for l = 0..lmax by the three-term recurrence (l+1) P_{l+1} = (2l+1) x P_l - l P_{l-1}."""
    out = np.zeros((lmax + 1,) + x.shape)
    out[0] = 1.0
    if lmax >= 1:
        out[1] = x
    for l in range(1, lmax):
        out[l + 1] = ((2 * l + 1) * x * out[l] - l * out[l - 1]) / (l + 1)
    return out


def fbeta_table(P) -> np.ndarray:
    """|f(beta)| (E, nph+1, 81) on cos(beta) = 0.025 k (ends -1 and 1): |sum over l <= lmax(e, iph) of
    t_l (2l+1) P_l(cos beta)|, t_l = (exp(2 i delta_{-l}) - 1) / 2i (pathfinder.py:47-57, FEFF's prcrit)."""
    E = int(P.ne1)
    lmax = np.asarray(P.lmax)[:E]
    cosb = 0.025 * np.arange(-NBETA, NBETA + 1)
    cosb[0], cosb[-1] = -1.0, 1.0
    pl = _legendre_table(cosb, int(lmax.max()))
    out = np.zeros((E, P.nph + 1, 2 * NBETA + 1))
    for iph in range(P.nph + 1):
        for ie in range(E):
            L = int(lmax[ie, iph])
            ls = np.arange(L + 1)
            delta = np.array([P.phase(ie, -l, iph) for l in ls])
            t = (np.exp(2j * delta) - 1) / 2j
            out[ie, iph] = np.abs(((t * (2 * ls + 1))[:, None] * pl[: L + 1]).sum(0))
    return out.astype(np.float32)


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


class GPUPathFinder:
    """The reference's constructor: phase file (PhaseData or a phase.pad path), device, rmax (A), nlegmax (2..9),
    critpw (percent), merge_degenerate."""

    def __init__(self, phase, device="cuda", rmax=9.4, nlegmax=4, critpw=0.1, merge_degenerate=True):
        P = read_phase_pad(phase) if isinstance(phase, str) else load_phase(phase)
        self.P, self.device = P, torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("feffgpu_b200 finds paths on CUDA devices only (no CPU path)")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.rmax, self.nlegmax, self.critpw = float(rmax), int(nlegmax), float(critpw)
        if not 2 <= self.nlegmax <= NLEG_MAX:
            raise ValueError(f"the largest number of legs must be between 2 and {NLEG_MAX}, FEFF's own limit "
                             f"(got {nlegmax})")
        self.merge_degenerate = merge_degenerate
        self._lib = _lib.load()
        E = int(P.ne1)
        ck = np.asarray(P.ck)[:E]
        dev = self.device
        self.fbeta = torch.tensor(fbeta_table(P), device=dev)
        self.cksp = torch.tensor(ck.real / BOHR, device=dev, dtype=torch.float32)
        safe = np.where(np.abs(ck.imag) > 1e-16, ck.imag, 1.0)
        self.xlam = torch.tensor(np.where(np.abs(ck.imag) > 1e-16, 1 / safe, 1e10) * BOHR, device=dev,
                                 dtype=torch.float32)
        self.ik0 = int(P.ik0) - 1
        x = ck.real[self.ik0:] / BOHR
        w = np.zeros(len(x))
        w[0] = x[1] - x[0]
        w[1:-1] = x[2:] - x[:-2]
        w[-1] = x[-1] - x[-2]
        self.trap = torch.tensor(w / 2, device=dev, dtype=torch.float32)
        self._tables = _lib.PfTables(E, P.nph + 1, self.ik0, self.fbeta.data_ptr(), self.cksp.data_ptr(),
                                     self.xlam.data_ptr(), self.trap.data_ptr())
        self._cells: dict = {}

    def _cell(self, box):
        """(cubic length or -1, the cell words on the device or None) of a box, kept per box: the reference's front
        ends pass the same box (often a device tensor) on every call, and converting it costs a synchronisation and a
        matrix inverse on the host.  A tensor is known by its identity and version counter (an in-place change makes a
        new entry); the entry holds the tensor, so its identity cannot pass to another one while it is cached."""
        if torch.is_tensor(box):
            key = ("t", id(box), box._version)
        elif box is None or np.isscalar(box):
            key = ("s", None if box is None else float(box))
        else:
            a = np.asarray(box, np.float64)
            key = ("a", a.shape, a.tobytes())
        hit = self._cells.get(key)
        if hit is None:
            cell = as_cell(box)
            cellw = (torch.as_tensor(cell_words(cell, np.float32), device=self.device)
                     if isinstance(cell, np.ndarray) else None)
            hit = (cell if isinstance(cell, float) else -1.0, cellw, box if torch.is_tensor(box) else None)
            if len(self._cells) > 32:
                self._cells.clear()
            self._cells[key] = hit
        return hit[0], hit[1]

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    # -- importance of given paths (the reference's importance(pts, ipots)) ----------------------------------------
    def importance(self, pts, ipots) -> torch.Tensor:
        """pts (B, m+1, 3) A with the absorber first, ipots (B, m+1): xport (B,) (pathfinder.py:75-100)."""
        dev = self.device
        pts = torch.as_tensor(pts, device=dev, dtype=torch.float32).contiguous()
        ipots = torch.as_tensor(ipots, device=dev, dtype=torch.int64)
        B, nleg, _ = pts.shape
        m = nleg - 1
        if B == 0:
            return torch.zeros(0, device=dev)
        # each path is its own slot whose candidates are its scatterers (relative to its absorber)
        rel = (pts[:, 1:] - pts[:, :1]).reshape(-1, 3).contiguous()
        off = torch.arange(0, B * m + 1, m, device=dev, dtype=torch.int64)
        seq = torch.arange(m, device=dev, dtype=torch.int32).repeat(B, 1).contiguous()
        slot = torch.arange(B, device=dev, dtype=torch.int32)
        cand_atom = torch.arange(B * m, device=dev, dtype=torch.int64)
        ipot_of = ipots[:, 1:].reshape(-1).contiguous()
        absorbers = torch.zeros(B, device=dev, dtype=torch.int64)
        out = self._describe(B, nleg, seq, slot, off, rel, cand_atom, ipot_of, absorbers, want_key=False)
        return out["xport"]

    @staticmethod
    def degenerate_total(coords, deg) -> torch.Tensor:
        """Summed degeneracy per geometry class: leg lengths and cos(beta) rounded to 1e-3, either direction
        (pathfinder.py:134-157)."""
        c = torch.as_tensor(coords, dtype=torch.float32)
        closed = torch.cat([c, c[:, :1]], 1)
        legs = closed[:, 1:] - closed[:, :-1]
        ri = torch.sqrt(legs[..., 0] * legs[..., 0] + legs[..., 1] * legs[..., 1] + legs[..., 2] * legs[..., 2])
        u = legs / ri.clamp_min(1e-12)[..., None]
        nx = torch.roll(u, -1, 1)
        cosb = u[..., 0] * nx[..., 0] + u[..., 1] * nx[..., 1] + u[..., 2] * nx[..., 2]
        n = ri.shape[1]
        kf = torch.round(torch.cat([ri, cosb], 1) * 1000).long()
        kr = torch.round(torch.cat([ri.flip(1), cosb[:, :n - 1].flip(1), cosb[:, n - 1:]], 1) * 1000).long()
        return _group_sum(_canonical(kf, kr), torch.as_tensor(deg, device=kf.device))

    # -- enumeration ---------------------------------------------------------------------------------------
    def enumerate(self, pos, box, absorber, ipot, chunk=256):
        """The reference's enumerate for one absorber: ({nleg: (coords (B, nleg, 3) relative to the absorber,
        ipots (B, nleg), deg (B,), xport (B,), atoms (B, nleg - 1))} after the importance cut, the reference
        importance).  One library call drives the whole search (fg_pf_enumerate_one): the reference's front ends call
        this once per absorber, and for a few hundred paths a sequence of small host-driven steps would be bound by
        its launch and dispatch latency.  The paths are those enumerate_many gives, bit for bit."""
        dev, lib, st = self.device, self._lib, self._stream()
        posd = torch.as_tensor(np.asarray(pos) if not torch.is_tensor(pos) else pos, device=dev,
                               dtype=torch.float32).contiguous()
        if posd.dim() == 3:
            if posd.shape[0] != 1:
                raise ValueError("enumerate takes one frame of positions (n, 3)")
            posd = posd[0]
        n = int(posd.shape[0])
        if not 0 <= int(absorber) < n:
            raise IndexError(f"absorber {int(absorber)} outside the {n} atoms")
        boxf, cellw = self._cell(box)
        ipot_of = (ipot.to(dev, torch.int64) if torch.is_tensor(ipot)
                   else torch.as_tensor(np.asarray(ipot), device=dev, dtype=torch.int64)).contiguous()
        h = C.c_void_p()
        counts = (C.c_int64 * (NLEG_MAX + 1))()
        ref = C.c_float()
        _lib.check(lib.fg_pf_enumerate_one(posd.data_ptr(), n, boxf, _ptr(cellw), int(absorber), ipot_of.data_ptr(),
                                           C.byref(self._tables), self.rmax, self.nlegmax, self.critpw,
                                           int(bool(self.merge_degenerate)), C.byref(h), counts, C.byref(ref), st))
        try:
            kept = {}
            for nleg in range(2, NLEG_MAX + 1):
                B = int(counts[nleg])
                if B < 0:
                    continue
                f32 = torch.empty(B * (3 * nleg + 2), device=dev, dtype=torch.float32)
                i64 = torch.empty(B * (2 * nleg - 1), device=dev, dtype=torch.int64)
                coords = f32[:3 * nleg * B].view(B, nleg, 3)
                deg, xport = f32[3 * nleg * B:(3 * nleg + 1) * B], f32[(3 * nleg + 1) * B:]
                ipots, atoms = i64[:nleg * B].view(B, nleg), i64[nleg * B:].view(B, nleg - 1)
                _lib.check(lib.fg_pf_result_gather(h, nleg, coords.data_ptr(), ipots.data_ptr(), deg.data_ptr(),
                                                   xport.data_ptr(), atoms.data_ptr(), st))
                kept[nleg] = (coords, ipots, deg, xport, atoms)
        finally:
            lib.fg_pf_result_destroy(h)
        return kept, float(ref.value)

    def enumerate_many(self, pos, box, absorbers, ipot):
        """Every path of every absorber of every frame in one set of launches.  pos (n, 3) A, or (F, n, 3) for F
        frames of the same atoms (an MD trajectory); box None, a cubic length, (3,) edges or a 3 x 3 cell (rows); absorbers (A,) atom indices, or
        (F, A) per frame; ipot (n,) potential per atom.  Returns {"paths": {nleg: (coords, ipots, deg, xport, atoms,
        slot)}, "ref": (slots,) reference importance}, slot = frame * A + absorber, paths grouped by slot in the
        reference's order, atoms as indices within the frame."""
        dev, lib, st = self.device, self._lib, self._stream()
        posd = torch.as_tensor(np.asarray(pos) if not torch.is_tensor(pos) else pos, device=dev,
                               dtype=torch.float32).contiguous()
        if posd.dim() == 2:
            posd = posd[None]
        F, n = int(posd.shape[0]), int(posd.shape[1])
        ab_np = np.asarray(absorbers.cpu() if torch.is_tensor(absorbers) else absorbers, np.int64)
        if ab_np.ndim == 1:
            ab_np = np.tile(ab_np, (F, 1))      # the same atoms in every frame
        if ab_np.shape[0] != F:
            raise ValueError("absorbers must be (A,) or (frames, A)")
        per_frame = max(int(ab_np.shape[1]), 1)
        boxf, cellw = self._cell(box)
        cptr = cellw.data_ptr() if cellw is not None else None
        ab = torch.as_tensor(ab_np.reshape(-1), device=dev).contiguous()
        A = int(ab.shape[0])
        ipot_of = (ipot.to(dev, torch.int64) if torch.is_tensor(ipot)
                   else torch.as_tensor(np.asarray(ipot), device=dev, dtype=torch.int64)).contiguous()
        # candidates
        cnt = torch.zeros(A, device=dev, dtype=torch.int32)
        if A == 0:
            return {"paths": {}, "ref": torch.ones(0, device=dev)}
        _lib.check(lib.fg_pf_candidates(posd.data_ptr(), n, boxf, cptr, ab.data_ptr(), A, per_frame, self.rmax,
                                        cnt.data_ptr(), None, None, None, st))
        off = torch.zeros(A + 1, device=dev, dtype=torch.int64)
        off[1:] = torch.cumsum(cnt.long(), 0)
        total = int(off[-1])
        cand_atom = torch.empty(max(total, 1), device=dev, dtype=torch.int64)
        cand_rel = torch.empty(max(total, 1), 3, device=dev, dtype=torch.float32)
        _lib.check(lib.fg_pf_candidates(posd.data_ptr(), n, boxf, cptr, ab.data_ptr(), A, per_frame, self.rmax, None,
                                        off.data_ptr(), cand_atom.data_ptr(), cand_rel.data_ptr(), st))
        slot = torch.repeat_interleave(torch.arange(A, device=dev, dtype=torch.int32), cnt.long(),
                                       output_size=total)          # the size is known: no synchronisation
        seq = (torch.arange(total, device=dev) - off[slot.long()]).to(torch.int32)[:, None].contiguous()
        cr = cand_rel[:total]
        length = torch.sqrt(cr[:, 0] * cr[:, 0] + cr[:, 1] * cr[:, 1] + cr[:, 2] * cr[:, 2]).contiguous()
        groups = {2: (seq, slot, torch.ones(total, device=dev))}
        # multiple scattering needs two candidates (pathfinder.py:237, 243, 262)
        grow = torch.nonzero(cnt[slot.long()] > 1).squeeze(1)         # one index vector: one sync for three gathers
        seq, slot, length = seq.index_select(0, grow), slot.index_select(0, grow), length.index_select(0, grow)
        two_r = float(np.float32(2 * self.rmax))
        for m in range(1, self.nlegmax - 1):
            P = int(seq.shape[0])
            if P == 0:
                break
            cc = torch.zeros(P, device=dev, dtype=torch.int32)
            _lib.check(lib.fg_pf_extend(P, m, seq.data_ptr(), length.data_ptr(), slot.data_ptr(), off.data_ptr(),
                                        cand_rel.data_ptr(), two_r, cc.data_ptr(), None, None, None, None, st))
            coff = torch.zeros(P + 1, device=dev, dtype=torch.int64)
            coff[1:] = torch.cumsum(cc.long(), 0)
            Cn = int(coff[-1])
            if Cn > PARTIAL_LIMIT * max(A, 1) or Cn * (4 * (m + 2) + 8) > (8 << 30):
                raise RuntimeError(f"{Cn} partial paths of {m + 2} legs within {self.rmax} A: lower the path cutoff or "
                                   f"the largest number of legs")
            cseq = torch.empty(max(Cn, 1), m + 1, device=dev, dtype=torch.int32)
            clen = torch.empty(max(Cn, 1), device=dev, dtype=torch.float32)
            cslot = torch.empty(max(Cn, 1), device=dev, dtype=torch.int32)
            _lib.check(lib.fg_pf_extend(P, m, seq.data_ptr(), length.data_ptr(), slot.data_ptr(), off.data_ptr(),
                                        cand_rel.data_ptr(), two_r, None, coff.data_ptr(), cseq.data_ptr(),
                                        clen.data_ptr(), cslot.data_ptr(), st))
            seq, length, slot = cseq[:Cn], clen[:Cn], cslot[:Cn]
            if Cn == 0:
                break
            keep = torch.empty(Cn, device=dev, dtype=torch.uint8)
            deg = torch.empty(Cn, device=dev, dtype=torch.float32)
            _lib.check(lib.fg_pf_terminal(Cn, m + 1, seq.data_ptr(), slot.data_ptr(), off.data_ptr(), keep.data_ptr(),
                                          deg.data_ptr(), st))
            k = torch.nonzero(keep).squeeze(1)
            groups[m + 2] = (seq.index_select(0, k), slot.index_select(0, k), deg.index_select(0, k))
        out = {}
        for nleg, (s, sl, dg) in groups.items():
            d = self._describe(int(s.shape[0]), nleg, s, sl, off, cand_rel, cand_atom, ipot_of, ab,
                               want_key=nleg > 2 and self.merge_degenerate)
            out[nleg] = dict(d, deg=dg, slot=sl)
        return self._merge_and_cut(out, A, off, cand_rel)

    def _describe(self, B, nleg, seq, slot, off, cand_rel, cand_atom, ipot_of, absorbers, want_key):
        dev, st = self.device, self._stream()
        coords = torch.empty(B, nleg, 3, device=dev, dtype=torch.float32)
        ipots = torch.empty(B, nleg, device=dev, dtype=torch.int64)
        atoms = torch.empty(B, nleg - 1, device=dev, dtype=torch.int64)
        rtot = torch.empty(B, device=dev, dtype=torch.float32)
        xport = torch.empty(B, device=dev, dtype=torch.float32)
        key = torch.empty(B, 2 * nleg, device=dev, dtype=torch.int64) if want_key else None
        if B:
            _lib.check(self._lib.fg_pf_describe(B, nleg, seq.data_ptr(), slot.data_ptr(), off.data_ptr(),
                                                cand_rel.data_ptr(), cand_atom.data_ptr(), ipot_of.data_ptr(),
                                                absorbers.data_ptr(), C.byref(self._tables), coords.data_ptr(),
                                                ipots.data_ptr(), atoms.data_ptr(), rtot.data_ptr(), xport.data_ptr(),
                                                _ptr(key), st))
        return {"coords": coords, "ipots": ipots, "atoms": atoms, "rtot": rtot, "xport": xport, "key": key}

    def _merge_and_cut(self, out, A, off, cand_rel):
        dev = self.device
        ss = out[2]
        c1 = ss["coords"][:, 1]
        d = torch.sqrt(c1[:, 0] * c1[:, 0] + c1[:, 1] * c1[:, 1] + c1[:, 2] * c1[:, 2])
        ref = torch.ones(A, device=dev, dtype=torch.float32)
        nonempty = (off[1:] - off[:-1]) > 0
        if not self.merge_degenerate or ss["slot"].shape[0] == 0:
            # the shortest candidate of each slot (first of equal ones)
            if ss["slot"].shape[0]:
                first = _first_min(d, ss["slot"].long(), A)
                ref = torch.where(nonempty, ss["xport"][first.clamp_min(0)], ref)
        multi = (off[1:] - off[:-1]) > 1
        if self.merge_degenerate and ss["slot"].shape[0]:
            win = self._windows(out, A)
            ss_win = win[2]
            # single scattering: sort by (slot, distance), group by (slot, rounded distance, potential, window) in
            # order of first appearance; the first member represents the group, its degeneracy is the group's size
            o = _stable_sort2(ss["slot"].long(), d)
            keys = torch.stack([ss["slot"].long()[o], torch.round(d[o] * 1000).long(), ss["ipots"][o, 1], ss_win[o]], 1)
            _, inv = torch.unique(keys, dim=0, return_inverse=True)
            G = int(inv.max()) + 1
            posn = torch.arange(len(o), device=dev)
            firstp = torch.full((G,), len(o), device=dev, dtype=torch.long).scatter_reduce(0, inv, posn, "amin")
            cnt = torch.bincount(inv, minlength=G).to(torch.float32)
            go = torch.argsort(firstp)
            rep = o[firstp[go]]
            merged = {k: (v[rep] if torch.is_tensor(v) and v.shape[0] == d.shape[0] else v) for k, v in ss.items()}
            merged["deg"] = cnt[go]
            out[2] = merged
            # the reference importance: the shortest merged path's, times its degeneracy (a slot with a single
            # candidate, which the reference does not merge, gives the same: degeneracy 1)
            mc = merged["coords"][:, 1]
            first = _first_min(torch.sqrt(mc[:, 0] * mc[:, 0] + mc[:, 1] * mc[:, 1] + mc[:, 2] * mc[:, 2]),
                               merged["slot"].long(), A)
            ref = torch.where(first >= 0, merged["xport"][first.clamp_min(0)] * merged["deg"][first.clamp_min(0)],
                              ref)
        paths, refs = {}, ref
        for nleg, v in sorted(out.items()):
            dg = v["deg"]
            if nleg > 2 and self.merge_degenerate and dg.shape[0]:
                key = torch.cat([v["slot"].long()[:, None], v["key"]], 1)
                dtot = _group_sum(key, dg)
                dtot = torch.where(multi[v["slot"].long()], dtot, dg)
            else:
                dtot = dg
            frac = 100 * dtot * v["xport"] / refs[v["slot"].long()]
            k = torch.nonzero(frac >= self.critpw).squeeze(1)
            paths[nleg] = tuple(t.index_select(0, k) for t in (v["coords"], v["ipots"], dg, v["xport"], v["atoms"],
                                                                v["slot"]))
        return {"paths": paths, "ref": refs}

    def _windows(self, out, A):
        """Greedy 1e-3 A windows over each slot's sorted closed lengths of every path (pathfinder.py:110-119):
        {nleg: window id per path}."""
        dev = self.device
        r = torch.cat([v["rtot"] for v in out.values()])
        sl = torch.cat([v["slot"].long() for v in out.values()])
        o = _stable_sort2(sl, r)
        sr = r[o].cpu().numpy().astype(np.float32)
        counts = torch.bincount(sl, minlength=A).cpu().numpy()
        seg = np.zeros(A + 1, np.int64)
        seg[1:] = np.cumsum(counts)
        win = np.zeros(len(sr), np.int64)
        _lib.check(self._lib.fg_pf_windows(sr.ctypes.data, seg.ctypes.data, A, float(np.float32(1e-3)),
                                           win.ctypes.data))
        w = torch.empty(len(sr), device=dev, dtype=torch.long)
        w[o] = torch.as_tensor(win, device=dev)
        res, s = {}, 0
        for nleg, v in out.items():
            nb = v["rtot"].shape[0]
            res[nleg] = w[s:s + nb]
            s += nb
        return res


def _stable_sort2(major: torch.Tensor, minor: torch.Tensor) -> torch.Tensor:
    """Permutation sorting by (major, minor), ties in index order."""
    o = torch.sort(minor, stable=True).indices
    return o[torch.sort(major[o], stable=True).indices]


def _first_min(values: torch.Tensor, slot: torch.Tensor, A: int) -> torch.Tensor:
    """Per slot the index of the first minimum of values (-1 for an empty slot)."""
    if values.shape[0] == 0:
        return torch.full((A,), -1, device=slot.device, dtype=torch.long)
    o = _stable_sort2(slot, values)
    s = slot[o]
    first = torch.full((A,), -1, device=slot.device, dtype=torch.long)
    is_first = torch.ones_like(s, dtype=torch.bool)
    is_first[1:] = s[1:] != s[:-1]
    first[s[is_first]] = o[is_first]
    return first


def _canonical(kf: torch.Tensor, kr: torch.Tensor) -> torch.Tensor:
    """Rows of kf or kr, whichever is lexicographically smaller."""
    less = torch.zeros(kf.shape[0], dtype=torch.bool, device=kf.device)
    undecided = torch.ones_like(less)
    for j in range(kf.shape[1]):
        less |= undecided & (kr[:, j] < kf[:, j])
        undecided &= kr[:, j] == kf[:, j]
    return torch.where(less[:, None], kr, kf)


def _group_sum(key: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
    """Per row the sum of w over the rows with the same key."""
    if key.shape[0] == 0:
        return w.clone()
    _, inv = torch.unique(key, dim=0, return_inverse=True)
    tot = torch.zeros(int(inv.max()) + 1, device=w.device, dtype=w.dtype).index_add_(0, inv, w)
    return tot[inv]
