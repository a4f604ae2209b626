"""PathBatch: a fixed list of paths with mixed leg counts, laid out for the fused stage.

The reference evaluates one leg count at a time in chunks (``src/feffgpu/chain.py:45-49``,
``src/feffgpu/exafs/forward.py:670-685``) and sums the chunks into rows with ``index_add``.  A PathBatch holds every
path once, padded to the largest leg count, together with

* ``order``  -- the launch order of the persistent work queue: costliest paths (most legs) first, so that the last
  paths to start are the cheapest (longest-processing-time-first scheduling);
* ``row`` -- the output row of every path; the stage adds each path's terms to its row exactly (integer sums of the
  terms rounded to 2^-64), so the result does not depend on scheduling.

The layout is built once per path list (on the host) and reused: only the coordinates change from call to call
(``GPUPathStage.chi_reduce(batch, q, coords=...)``).
"""
from __future__ import annotations

import numpy as np
import torch


class PathBatch:
    """Paths for ``GPUPathStage.chi_reduce``.

    groups: iterable of (coords (B, nleg, 3) A absorber first, ipots (B, nleg), deg (B,) or None, row (B,) or None),
    one entry per leg count (or any grouping); nrows defaults to max(row) + 1.
    """

    def __init__(self, groups, nrows: int | None = None, device="cuda"):
        self.device = torch.device(device)
        cs, ips, nl, dg, rw = [], [], [], [], []
        nleg_max = 2
        groups = [tuple(g) + (None,) * (4 - len(g)) for g in groups]
        for coords, ipots, deg, row in groups:
            c = torch.as_tensor(coords).detach().to("cpu", torch.float64)
            if c.dim() != 3 or c.shape[2] != 3:
                raise ValueError("coords must be (B, nleg, 3)")
            nleg_max = max(nleg_max, c.shape[1])
        for coords, ipots, deg, row in groups:
            c = torch.as_tensor(coords).detach().to("cpu", torch.float64)
            B, nleg, _ = c.shape
            if not 2 <= nleg <= 9:
                raise ValueError("paths have 2 to 9 legs")
            ip = torch.as_tensor(ipots).detach().to("cpu", torch.int64)
            if ip.shape != (B, nleg):
                raise ValueError("ipots must be (B, nleg)")
            pc = torch.zeros(B, nleg_max, 3, dtype=torch.float64)
            pc[:, :nleg] = c
            pi = torch.zeros(B, nleg_max, dtype=torch.int64)
            pi[:, :nleg] = ip
            cs.append(pc); ips.append(pi)
            nl.append(torch.full((B,), nleg, dtype=torch.int32))
            dg.append(torch.ones(B, dtype=torch.float64) if deg is None else torch.as_tensor(deg).detach().to("cpu", torch.float64).reshape(B))
            rw.append(torch.zeros(B, dtype=torch.int32) if row is None else torch.as_tensor(row).detach().to("cpu", torch.int32).reshape(B))
        self.nleg_max = nleg_max
        coords = torch.cat(cs) if cs else torch.zeros(0, nleg_max, 3, dtype=torch.float64)
        ipots = torch.cat(ips) if ips else torch.zeros(0, nleg_max, dtype=torch.int64)
        nleg = torch.cat(nl) if nl else torch.zeros(0, dtype=torch.int32)
        deg = torch.cat(dg) if dg else torch.zeros(0, dtype=torch.float64)
        row = torch.cat(rw) if rw else torch.zeros(0, dtype=torch.int32)
        self.n = int(coords.shape[0])
        if self.n and int(row.min()) < 0:
            raise ValueError("rows must be non-negative")
        self.nrows = int(nrows) if nrows is not None else (int(row.max()) + 1 if self.n else 0)
        if self.n and int(row.max()) >= self.nrows:
            raise ValueError("row index beyond nrows")
        if self.n and int(ipots.min()) < 0:
            raise IndexError("negative potential index")
        self.max_ipot = int(ipots.max()) if self.n else 0
        # launch order: most legs first (stable), the persistent queue's LPT schedule
        nl_np = nleg.numpy()
        order = np.argsort(-nl_np, kind="stable").astype(np.int32)
        d = self.device
        self.coords = coords.to(d)
        self.ipots = ipots.to(d)
        self.nleg = nleg.to(d)
        self.deg = deg.to(d)
        self.row = row.to(d)
        self.order = torch.as_tensor(order).to(d)
        self.counts = {int(k): int(v) for k, v in zip(*np.unique(nl_np, return_counts=True))}
        self._ws = {}
        self._tuned = {}             # launch shapes chosen for this batch, per (stage, precision, k points)

    def sample(self, max_paths: int) -> "PathBatch":
        """A batch of at most max_paths of these paths: every k-th path in launch order, so every leg count keeps
        its share (the autotuner's timing sample).  The batch itself when it is small enough."""
        if self.n <= max_paths:
            return self
        step = -(-self.n // max_paths)
        idx = self.order[::step].long()
        nl = self.nleg[idx]
        groups = []
        for n in sorted(set(nl.tolist())):
            sel = idx[nl == n]
            groups.append((self.coords[sel, :n].cpu(), self.ipots[sel, :n].cpu(), self.deg[sel].cpu(),
                           self.row[sel].cpu()))
        return PathBatch(groups, nrows=self.nrows, device=self.device)

    def workspace(self, nbytes: int, backward: bool = False) -> torch.Tensor:
        """A cached device scratch buffer of at least nbytes (one per direction)."""
        key = "bwd" if backward else "fwd"
        ws = self._ws.get(key)
        if ws is None or ws.numel() < max(nbytes, 1):
            ws = torch.empty(max(nbytes, 1), device=self.device, dtype=torch.uint8)
            self._ws[key] = ws
        return ws

    def __len__(self) -> int:
        return self.n
