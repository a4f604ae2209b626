"""CPU restatement of the reference's path finder (src/feffgpu/pathfinder.py) -- test infrastructure only.

Used by tests/ to check the CUDA path finder (feffgpu_b200/pathfinder.py, csrc/fg_paths.cu); never by the product.
Pinned against the reference finder's own outputs (tests/golden/finder_*.npz, made by tests/golden/make_golden.py).

Algorithm (FEFF's paths.f / pathsd.f / prcrit.f as the reference restates them), for one absorber:

* candidates: atoms within rmax of the absorber (minimum image), the absorber excluded (pathfinder.py:222-224);
  intermediates: the candidates followed by the absorber itself (an inner atom may be the absorber);
* a path of nleg legs is a sequence of nleg - 1 intermediates whose first and last are candidates, no atom followed
  by itself, closed length (absorber -> ... -> absorber) at most 2 rmax; of a sequence and its reverse the
  lexicographically smaller (in intermediate order) is kept, degeneracy 2, or 1 for a palindrome
  (pathfinder.py:233-271; the 3- and 4-leg rules i < j and i <= l are this rule for two and three atoms);
* importance (pathfinder.py:75-100): the trapezoid integral over the energies from ik0 of
  max(|cos beta_0|, 0.3) / rho_0 x prod_j |f_j(beta_j)| / rho_j x exp(-R / lambda), |f(beta)| tabulated on a
  cos(beta) grid of 0.025 (pathfinder.py:47-57), nearest grid point with FEFF's rounding (pathfinder.py:67-72);
* single-scattering merge (pathfinder.py:102-132): all paths sorted by closed length, cut into greedy 1e-3 A
  windows; single-scattering paths with the same distance to 1e-3 A, potential and window are one path (the
  shortest kept, degeneracy = count);
* multiple-scattering degeneracy totals (pathfinder.py:134-157): leg lengths and cos(beta) rounded to 1e-3,
  canonical direction (the smaller of the key and its reverse), summed degeneracy per key;
* filter (pathfinder.py:271-279): 100 x total degeneracy x importance / the shortest single-scattering path's
  (degeneracy-weighted) importance >= critpw.

Lengths and importances are FP32 as in the reference; distances here are direct differences, where the reference's
torch.cdist may use the |x|^2 + |y|^2 - 2 x.y form, so paths within ~1e-5 A of the cutoff may differ.
"""
from __future__ import annotations

import numpy as np

BOHR = 0.52917721067
NBETA = 40


def fbeta_table(P):
    """|f(beta)| (E, nph+1, 2 NBETA + 1) float32 on cos(beta) = 0.025 k, ends at -1 and 1 (pathfinder.py:47-57):
    sum over l <= lmax(e, iph) of t_l (2l+1) P_l(cos beta), t_l = (exp(2 i delta_{-l}) - 1) / 2i."""
    from scipy.special import eval_legendre
    E = int(P.ne1)
    lmax = np.asarray(P.lmax)[:E]
    cosb = 0.025 * np.arange(-NBETA, NBETA + 1)
    cosb[0], cosb[-1] = -1.0, 1.0
    out = np.zeros((E, P.nph + 1, 2 * NBETA + 1))
    for iph in range(P.nph + 1):
        for ie in range(E):
            f = np.zeros(len(cosb), complex)
            for l in range(int(lmax[ie, iph]) + 1):
                t = (np.exp(2j * P.phase(ie, -l, iph)) - 1) / 2j
                f += t * (2 * l + 1) * eval_legendre(l, cosb)
            out[ie, iph] = np.abs(f)
    return out.astype(np.float32)


class Finder:
    def __init__(self, P, rmax=9.4, nlegmax=4, critpw=0.1, merge_degenerate=True):
        self.P, self.rmax, self.nlegmax, self.critpw, self.merge = P, float(rmax), int(nlegmax), float(critpw), \
            merge_degenerate
        E = int(P.ne1)
        self.fbeta = fbeta_table(P)
        ck = np.asarray(P.ck)[:E]
        self.cksp = (ck.real / BOHR).astype(np.float32)
        self.xlam = (np.where(np.abs(ck.imag) > 1e-16, 1 / np.where(np.abs(ck.imag) > 1e-16, ck.imag, 1), 1e10)
                     * BOHR).astype(np.float32)
        self.ik0 = int(P.ik0) - 1
        x = ck.real[self.ik0:] / BOHR
        w = np.zeros(len(x))
        w[0] = x[1] - x[0]
        w[1:-1] = x[2:] - x[:-2]
        w[-1] = x[-1] - x[-2]
        self.trap = (w / 2).astype(np.float32)

    # -- importance (pathfinder.py:67-100) -------------------------------------------------------------------
    @staticmethod
    def indbet(cosb):
        a = np.abs(cosb).astype(np.float32)
        n = np.floor(a / np.float32(0.025))
        n = np.where(a - n * np.float32(0.025) > np.float32(0.0125), n + 1, n)
        n = np.where(cosb < 0, -n, n)
        return np.clip(n.astype(np.int64) + NBETA, 0, 2 * NBETA)

    def importance(self, coords, ipots):
        """coords (B, nleg, 3) absorber first (float32), ipots (B, nleg): xport (B,) float32."""
        c = np.asarray(coords, np.float32)
        closed = np.concatenate([c, c[:, :1]], 1)
        legs = closed[:, 1:] - closed[:, :-1]
        ri = np.sqrt((legs * legs).sum(-1)).astype(np.float32)
        rtot = ri.sum(1)
        u = legs / np.maximum(ri, np.float32(1e-12))[..., None]
        cos_sc = (u[:, :-1] * u[:, 1:]).sum(-1)
        cos_abs = (u[:, -1] * u[:, 0]).sum(-1)
        es = np.arange(self.ik0, self.fbeta.shape[0])
        k = self.cksp[es]
        crit = np.maximum(np.abs(cos_abs), np.float32(0.3))[:, None] / (ri[:, -1][:, None] * k[None])
        ib = self.indbet(cos_sc)
        for j in range(c.shape[1] - 1):
            f = self.fbeta[es][:, np.asarray(ipots)[:, j + 1], ib[:, j]].T
            crit = crit * f / (ri[:, j][:, None] * k[None])
        crit = crit * np.exp(-rtot[:, None] / self.xlam[None, es])
        return (np.abs(crit) * self.trap[None]).sum(1).astype(np.float32)

    # -- enumeration (pathfinder.py:159-271) -----------------------------------------------------------------
    def sequences(self, rel):
        """{nleg: (atoms (B, nleg - 1) as candidate positions / the absorber = nc, deg (B,))} before the filter,
        every nleg in one rule (see the module docstring).  rel: (nc, 3) float32 candidates relative to the
        absorber."""
        nc = len(rel)
        P = np.concatenate([rel, np.zeros((1, 3), np.float32)]).astype(np.float32)
        D = np.sqrt(((P[:, None] - P[None]) ** 2).sum(-1)).astype(np.float32)
        back = np.sqrt((P * P).sum(-1)).astype(np.float32)
        two_r = np.float32(2 * self.rmax)
        out = {2: (np.arange(nc)[:, None], np.ones(nc))}
        seq = np.arange(nc)[:, None]
        length = back[:nc].copy()
        ni = nc + 1
        for m in range(2, self.nlegmax):
            tot = length[:, None] + D[seq[:, -1]]
            ok = (tot + back[None, :] <= two_r) & (np.arange(ni)[None, :] != seq[:, -1:])
            i, j = np.nonzero(ok)
            seq = np.concatenate([seq[i], j[:, None]], 1)
            length = tot[i, j]
            if len(seq) == 0:
                break
            done = seq[seq[:, -1] != nc]
            if len(done) == 0:
                continue
            rev = done[:, ::-1]
            differ = done != rev
            first = np.argmax(differ, 1)
            pal = ~differ.any(1)
            rows = np.arange(len(done))
            keep = pal | (done[rows, first] < rev[rows, first])
            out[m + 1] = (done[keep], np.where(pal[keep], 1.0, 2.0))
        return out

    def enumerate(self, pos, box, absorber, ipot):
        """The reference's GPUPathFinder.enumerate on the CPU: {nleg: (coords (B, nleg, 3) float32 relative to the
        absorber, ipots (B, nleg), deg (B,), xport (B,), atoms (B, nleg - 1) atom indices)} after the filter,
        and the reference importance."""
        pos = np.asarray(pos, np.float32)
        rel = pos - pos[absorber]
        if box is not None and np.ndim(box) == 0:
            b = np.float32(box)
            rel = rel - b * np.round(rel / b)
        elif box is not None:
            # a cell (cell.py:11-35): (3,) edges -> the diagonal cell; f = rel inv(cell), rel = (f - round(f)) cell
            c = np.asarray(box, np.float32)
            c = np.diag(c) if c.shape == (3,) else c
            f = rel @ np.linalg.inv(c).astype(np.float32)
            rel = ((f - np.round(f)) @ c).astype(np.float32)
        d0 = np.sqrt((rel * rel).sum(-1)).astype(np.float32)
        n = len(pos)
        cl = np.nonzero((d0 <= np.float32(self.rmax)) & (np.arange(n) != absorber))[0]
        inter = np.concatenate([cl, [absorber]])
        ipot = np.asarray(ipot)
        seqs = self.sequences(rel[cl])
        out = {}
        for nleg, (s, deg) in seqs.items():
            atoms = inter[s]
            coords = np.concatenate([np.zeros((len(atoms), 1, 3), np.float32), rel[atoms]], 1)
            ip = np.concatenate([np.zeros((len(atoms), 1), int), np.where(atoms == absorber, 0, ipot[atoms])], 1)
            out[nleg] = [coords, ip, np.asarray(deg, np.float32), self.importance(coords, ip), atoms]
        ref = out[2][3][np.argmin(d0[cl])] if len(cl) else np.float32(1.0)
        if self.merge and len(cl) > 1:
            out = self.merge_single(out)
            i = int(np.argmin(np.linalg.norm(out[2][0][:, 1], axis=1)))
            ref = out[2][3][i] * out[2][2][i]
        kept = {}
        for nleg, (coords, ip, deg, xp, atoms) in out.items():
            dtot = self.degenerate_total(coords, deg) if (nleg > 2 and self.merge and len(deg)) else deg
            frac = np.float32(100) * dtot * xp / ref
            keep = frac >= np.float32(self.critpw)
            kept[nleg] = (coords[keep], ip[keep], deg[keep], xp[keep], atoms[keep])
        return kept, float(ref)

    @staticmethod
    def closed_length(coords):
        c = np.asarray(coords, np.float32)
        closed = np.concatenate([c, c[:, :1]], 1)
        return np.sqrt(((closed[:, 1:] - closed[:, :-1]) ** 2).sum(-1)).sum(1).astype(np.float32)

    def merge_single(self, out):
        """pathfinder.py:102-132: greedy 1e-3 A windows over the sorted closed lengths of every path; 2-leg paths
        with the same rounded distance, potential and window merge (the shortest first, degeneracy = count)."""
        allr = np.concatenate([self.closed_length(v[0]) for v in out.values()]).astype(np.float32)
        order = np.argsort(allr, kind="stable")
        sr = allr[order]
        window = np.zeros(len(sr), np.int64)
        i = w = 0
        while i < len(sr):
            j = max(int(np.searchsorted(sr, np.float32(sr[i] + np.float32(1e-3)), side="left")), i + 1)
            window[i:j] = w
            w += 1
            i = j
        win_of = np.empty(len(sr), np.int64)
        win_of[order] = window
        coords, ip, deg, xp, atoms = out[2]
        n2 = len(coords)
        d = np.sqrt((coords[:, 1] ** 2).sum(-1)).astype(np.float32)
        key = np.round(d * np.float32(1000)).astype(np.int64)
        groups: dict = {}
        for k in np.argsort(d, kind="stable"):
            groups.setdefault((int(key[k]), int(ip[k, 1]), int(win_of[k])), []).append(int(k))
        rep = np.array([g[0] for g in groups.values()], int)
        cnt = np.array([len(g) for g in groups.values()], np.float32)
        assert n2 == len(out[2][0])
        out[2] = [coords[rep], ip[rep], cnt, xp[rep], atoms[rep]]
        return out

    @staticmethod
    def degenerate_total(coords, deg):
        """pathfinder.py:134-157: summed degeneracy of the paths with the same rounded leg lengths and cos(beta) in
        either direction."""
        c = np.asarray(coords, np.float32)
        closed = np.concatenate([c, c[:, :1]], 1)
        legs = closed[:, 1:] - closed[:, :-1]
        ri = np.sqrt((legs * legs).sum(-1)).astype(np.float32)
        u = legs / np.maximum(ri, np.float32(1e-12))[..., None]
        cosb = (u * np.roll(u, -1, 1)).sum(-1)
        n = ri.shape[1]
        fwd = np.concatenate([ri, cosb], 1)
        rev = np.concatenate([ri[:, ::-1], cosb[:, :n - 1][:, ::-1], cosb[:, n - 1:]], 1)
        kf = np.round(fwd * np.float32(1000)).astype(np.int64)
        kr = np.round(rev * np.float32(1000)).astype(np.int64)
        key = np.empty_like(kf)
        for b in range(len(kf)):
            key[b] = kr[b] if tuple(kr[b]) < tuple(kf[b]) else kf[b]
        _, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        total = np.zeros(inv.max() + 1 if len(inv) else 0)
        np.add.at(total, inv, np.asarray(deg, float))
        return total[inv].astype(np.float32)
