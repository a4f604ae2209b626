"""Seeded synthetic structures and path lists with the shapes of the stage's benchmark configurations.

Path lists come from the path finder (``feffgpu_b200.pathfinder``) where a workload names one; ``random_paths``
draws closed scattering paths over a structure's atoms with a prescribed number of paths per leg count, legs no
longer than a cutoff and the half path length below ``rmax`` (test workloads of a chosen size), and
``bcc_site_paths`` / ``md_batch`` enumerate the 2- and 3-leg paths of a bcc lattice for the MD batch -- all in the
input layout of ``GPUPathStage.cchi`` (coordinates relative to the absorber, absorber first; potential indices
absorber 0).
"""
from __future__ import annotations

import numpy as np



def random_packing(n=3000, density=0.08, dmin=1.8, species=("Fe", "O", "Pt"), seed=2024, fractions=None):
    """Random sequential addition of n points at `density` (1/A^3) in a periodic cube, no two closer than dmin.
    Returns positions (n, 3) A, species labels (n,), box length A."""
    rng = np.random.default_rng(seed)
    box = (n / density) ** (1.0 / 3.0)
    ncell = max(1, int(box // dmin))
    cw = box / ncell
    cells: dict = {}
    pos = np.zeros((n, 3))
    k = 0
    tries = 0
    while k < n:
        cand = rng.random((4096, 3)) * box
        for c in cand:
            tries += 1
            ci = np.floor(c / cw).astype(int) % ncell
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((ci[0] + dx) % ncell, (ci[1] + dy) % ncell, (ci[2] + dz) % ncell)
                        for j in cells.get(key, ()):
                            d = pos[j] - c
                            d -= box * np.round(d / box)
                            if d @ d < dmin * dmin:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pos[k] = c
                cells.setdefault(tuple(ci), []).append(k)
                k += 1
                if k == n:
                    break
        if tries > 200 * n:
            raise RuntimeError("random packing did not converge")
    p = np.full(len(species), 1.0 / len(species)) if fractions is None else np.asarray(fractions, float)
    labels = rng.choice(np.asarray(species), size=n, p=p / p.sum())
    return pos, labels, box


def fcc_cluster(a=3.61, rcut=6.0):
    """fcc lattice points within rcut of the origin (absorber at the origin first)."""
    m = int(np.ceil(rcut / a)) + 1
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.array([[i, j, k] for i in range(-m, m + 1) for j in range(-m, m + 1) for k in range(-m, m + 1)], float)
    pts = (g[:, None, :] + base[None]).reshape(-1, 3) * a
    r = np.linalg.norm(pts, axis=1)
    pts = pts[r <= rcut + 1e-9]
    return pts[np.argsort(np.linalg.norm(pts, axis=1), kind="stable")]


def bcc_supercell(n=16, a=2.87):
    """bcc supercell n^3 conventional cells: positions (2 n^3, 3) A and the box length."""
    g = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    pts = np.concatenate([g, g + 0.5]) * a
    return pts, n * a


def rock_salt_supercell(n=8, a=4.177, species=("Ni", "O")):
    """rock-salt supercell n^3 conventional cells: positions (8 n^3, 3), labels, box length."""
    g = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    fa = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    fb = fa + np.array([0.5, 0, 0])
    pa = (g[:, None] + fa[None]).reshape(-1, 3) * a
    pb = (g[:, None] + fb[None]).reshape(-1, 3) * a
    pos = np.concatenate([pa, pb])
    lab = np.array([species[0]] * len(pa) + [species[1]] * len(pb))
    return pos, lab, n * a


def thermal(pos, sigma, seed):
    """Gaussian displacements of every coordinate with standard deviation sigma (A)."""
    return pos + np.random.default_rng(seed).normal(0.0, sigma, pos.shape)


def neighbors(pos, box, cutoff):
    """Minimum-image neighbour lists within cutoff: (offsets (n+1,), indices, vectors) in CSR form."""
    from scipy.spatial import cKDTree
    pos = np.asarray(pos, float)
    n = len(pos)
    if box is not None:
        tree = cKDTree(np.mod(pos, box), boxsize=box)
    else:
        tree = cKDTree(pos)
    pairs = tree.query_pairs(cutoff, output_type="ndarray")
    i = np.concatenate([pairs[:, 0], pairs[:, 1]])
    j = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    d = pos[j] - pos[i]
    if box is not None:
        d -= box * np.round(d / box)
    offs = np.concatenate([[0], np.cumsum(np.bincount(i, minlength=n))])
    return offs, j, d


def random_paths(pos, box, absorber, counts, rmax=8.0, leg_max=6.0, seed=0, ipot_of=None, batch=200000):
    """Closed paths absorber -> s_1 -> ... -> s_{nleg-1} -> absorber drawn at random: each leg joins minimum-image
    neighbours no farther apart than leg_max, consecutive atoms differ, the last scatterer is not the absorber, and
    the half path length is at most rmax; the scatterer-to-scatterer hops of an n-leg path are drawn among
    neighbours within min(leg_max, max(2.4, 2 rmax / n + 0.8 - 0.3 max(0, n - 6))) A.  counts: {nleg: number of paths}.  Returns {nleg: (coords (B, nleg, 3)
    relative to the absorber, ipots (B, nleg), atoms (B, nleg-1))}; ipot_of (n,) gives each atom's potential
    (default 1), the absorber gets 0."""
    rng = np.random.default_rng(seed)
    n = len(pos)
    ipot_of = np.ones(n, int) if ipot_of is None else np.asarray(ipot_of)
    offs0, nbr0, vec0 = neighbors(pos, box, leg_max)
    r0 = np.linalg.norm(vec0, axis=1)
    owner = np.repeat(np.arange(n), np.diff(offs0))
    out = {}
    for nleg, want in sorted(counts.items()):
        nsc = nleg - 1
        # hops no longer than about the mean leg that fits the length budget, so that long paths close often
        hop = min(leg_max, max(2.4, 2.0 * rmax / nleg + 0.8 - 0.3 * max(0, nleg - 6)))
        keep = r0 <= hop
        if not keep.any():
            raise ValueError(f"no scatterer-to-scatterer hop within {hop:.2f} A for {nleg}-leg paths: raise rmax")
        nbr, vec = nbr0[keep], vec0[keep]
        offs = np.concatenate([[0], np.cumsum(np.bincount(owner[keep], minlength=n))])
        deg = np.diff(offs)
        got_c, got_a = [], []
        have = 0
        guard = 0
        while have < want:
            guard += 1
            if guard > 2000:
                raise RuntimeError(f"could not draw {want} paths of {nleg} legs")
            cur = np.full(batch, absorber)
            disp = np.zeros((batch, 3))
            length = np.zeros(batch)
            atoms = np.zeros((batch, nsc), int)
            rel = np.zeros((batch, nsc, 3))
            ok = np.ones(batch, bool)
            for s in range(nsc):
                d = deg[cur]
                ok &= d > 0
                pick = offs[cur] + (rng.random(batch) * np.maximum(d, 1)).astype(int)
                pick = np.minimum(pick, offs[cur + 1] - 1)
                step = vec[pick]
                nxt = nbr[pick]
                disp = disp + step
                length += np.linalg.norm(step, axis=1)
                cur = np.where(ok, nxt, cur)
                atoms[:, s] = cur
                rel[:, s] = disp
            back = np.linalg.norm(disp, axis=1)
            length += back
            ok &= (atoms[:, -1] != absorber) & (back <= leg_max) & (back > 1e-6) & (length <= 2 * rmax)
            sel = np.nonzero(ok)[0][: want - have]
            got_c.append(rel[sel]); got_a.append(atoms[sel])
            have += len(sel)
        rel = np.concatenate(got_c)[:want]
        atoms = np.concatenate(got_a)[:want]
        coords = np.concatenate([np.zeros((want, 1, 3)), rel], 1)
        ip = np.concatenate([np.zeros((want, 1), int), ipot_of[atoms]], 1)
        ip[:, 1:][atoms == absorber] = 0
        ip[:, 0] = 0
        out[nleg] = (coords, ip, atoms)
    return out


def central_atom(pos, box, labels=None, species=None, k=1):
    """The k atoms of the given species closest to the centre of the box."""
    c = np.full(3, box / 2.0)
    d = np.linalg.norm(pos - c, axis=1)
    if labels is not None and species is not None:
        d = np.where(np.asarray(labels) == species, d, np.inf)
    return np.argsort(d, kind="stable")[:k]


def bcc_site_paths(n, a, rmax=5.5):
    """Every 2- and 3-leg path of an ideal bcc lattice (n^3 conventional cells of bcc_supercell) with half path
    length <= rmax, as site offsets: {2: (P2, 1, 3) int, 3: (P3, 2, 3) int} scatterer offsets in units of a/2 (bcc
    sites: all-even or all-odd half-lattice coordinates), i.e. the path finder's output for one absorber before
    degeneracy merging (MD frames break the symmetry, so every path is kept)."""
    m = int(np.ceil(2 * rmax / a)) + 1
    g = np.arange(-m, m + 1)
    v = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    v = v[((v[:, 0] % 2) == (v[:, 1] % 2)) & ((v[:, 1] % 2) == (v[:, 2] % 2)) & (np.abs(v).sum(1) > 0)]
    r = np.linalg.norm(v * a / 2, axis=1)
    v, r = v[r <= rmax + 1e-9], r[r <= rmax + 1e-9]
    v = v[np.lexsort((v[:, 2], v[:, 1], v[:, 0], np.round(r, 9)))]
    r = np.linalg.norm(v * a / 2, axis=1)
    d = np.linalg.norm((v[:, None] - v[None]) * a / 2, axis=2)
    i, j = np.nonzero((r[:, None] + d + r[None, :] <= 2 * rmax + 1e-9) & (d > 1e-9))
    return {2: v[:, None, :], 3: np.stack([v[i], v[j]], 1)}


def bcc_site_index(n, half):
    """Atom index in bcc_supercell(n) of half-lattice coordinates (..., 3) (wrapped periodically)."""
    h = np.mod(half, 2 * n)
    body = h[..., 0] % 2
    c = h // 2
    return body * n ** 3 + (c[..., 0] * n + c[..., 1]) * n + c[..., 2]


def md_batch(frames=500, absorbers=32, n=16, a=2.87, sigma=0.08, rmax=5.5, seed=0):
    """MD-EXAFS batch of bcc Fe: `frames` seeded thermal snapshots (Gaussian displacements sigma) of the n^3-cell
    supercell, `absorbers` random absorbers per frame, every 2- and 3-leg path within rmax of each (minimum-image
    coordinates relative to the absorber).  Returns groups for PathBatch with deg = 1/absorbers and row = frame (the
    frame's absorber average), and the number of paths per absorber."""
    base, box = bcc_supercell(n, a)
    half0 = np.rint(base / (a / 2)).astype(np.int64)
    sites = bcc_site_paths(n, a, rmax)
    rng = np.random.default_rng(seed)
    groups = {}
    for f in range(frames):
        pos = thermal(base, sigma, seed=seed * 100003 + f + 1)
        ab = rng.choice(len(base), size=absorbers, replace=False)
        for nleg, off in sites.items():
            idx = bcc_site_index(n, half0[ab][:, None, None, :] + off[None])          # (A, P, nleg-1)
            rel = pos[idx] - pos[ab][:, None, None, :]
            rel -= box * np.round(rel / box)
            B = idx.shape[0] * idx.shape[1]
            c = np.concatenate([np.zeros((B, 1, 3)), rel.reshape(B, nleg - 1, 3)], 1)
            groups.setdefault(nleg, []).append((c, np.full(B, f, np.int32)))
    out = []
    for nleg, parts in sorted(groups.items()):
        c = np.concatenate([p[0] for p in parts])
        row = np.concatenate([p[1] for p in parts])
        ip = np.ones((len(c), nleg), np.int64)
        ip[:, 0] = 0
        out.append((c, ip, np.full(len(c), 1.0 / absorbers), row))
    return out, sum(len(s) for s in sites.values())
