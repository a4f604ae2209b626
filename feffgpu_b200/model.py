"""Paths held as atom indices over a structure, evaluated by the fused stage at any positions (MD and RMC use).

The reference keeps path lists as global atom indices and rebuilds the coordinates from the current positions at
every evaluation (``src/feffgpu/exafs/forward.py:99-163, 664-725``): relative vectors to the absorber under the
minimum image, absorber first, then ``cchi`` + ``chi_fine`` per chunk and an ``index_add`` into one row per
absorber/copy.  ``PathModel`` does the same with one ``PathBatch`` and one fused call per evaluation: the gather of
the coordinates is a differentiable torch indexing (its backward scatters the per-path gradients onto the atoms),
the stage is ``GPUPathStage.chi_reduce``.  ``GraphedRefinement`` captures one refinement step -- model, R-space
misfit, backward and the Adam update -- in a CUDA graph and replays it (the RMC loop of
``src/feffgpu/rmc/refine.py:120-260``), re-enumerating the paths and capturing the step again every
``refresh_every`` steps as that loop does (``refine.py:176-179``).
"""
from __future__ import annotations

import time

import numpy as np
import torch

from .batch import PathBatch
from .cell import as_cell, cell_words


class MinImage:
    """The minimum image of a box in any of the reference's forms (None, a cubic length, (3,) edges, a 3 x 3 cell),
    with the cell and its inverse held on the device in FP64, so that applying it launches no copy (it runs inside
    captured CUDA graphs)."""

    def __init__(self, box, device):
        self.cell = as_cell(box)
        self.words = None
        if isinstance(self.cell, np.ndarray):
            w = torch.as_tensor(cell_words(self.cell, np.float64), device=device)
            self.words = (w[:9].reshape(3, 3), w[9:].reshape(3, 3))

    def __call__(self, rel: torch.Tensor) -> torch.Tensor:
        if self.cell is None:
            return rel
        if self.words is None:
            return rel - self.cell * torch.round(rel / self.cell)
        c, inv = self.words
        f = rel @ inv
        return (f - torch.round(f)) @ c


class PathModel:
    """groups: (atoms (B, nleg) global indices with the absorber first, ipots (B, nleg), deg (B,) or None,
    row (B,) or None) per leg count; positions (N, 3) A."""

    def __init__(self, stage, groups, positions, nrows=None, box=None):
        self.stage, self.box = stage, box
        dev = stage.device
        self.min_image = MinImage(box, dev)
        pos = torch.as_tensor(positions, dtype=torch.float64).to(dev)
        nleg_max = max(int(np.asarray(g[0]).shape[1]) for g in groups)
        atoms, bgroups = [], []
        for g in groups:
            a = torch.as_tensor(np.asarray(g[0]), dtype=torch.long)
            B, n = a.shape
            rel = self.min_image(pos[a.to(dev)] - pos[a[:, :1].to(dev)]).cpu().numpy()
            bgroups.append((rel, g[1], g[2] if len(g) > 2 else None, g[3] if len(g) > 3 else None))
            pad = torch.cat([a, a[:, :1].expand(B, nleg_max - n)], 1)
            atoms.append(pad)
        self.batch = PathBatch(bgroups, nrows=nrows, device=dev)
        self.atoms = torch.cat(atoms).to(dev)
        legs = torch.arange(nleg_max, device=dev)
        self.mask = (legs[None, :] < self.batch.nleg[:, None].long()).to(torch.float64)[:, :, None]

    def coords(self, pos: torch.Tensor) -> torch.Tensor:
        """(n, nleg_max, 3) relative coordinates of every path at positions pos (N, 3), differentiable."""
        rel = pos[self.atoms] - pos[self.atoms[:, :1]]
        return self.min_image(rel) * self.mask

    def rows(self, pos: torch.Tensor, q: torch.Tensor, S: torch.Tensor, sigma2=None) -> torch.Tensor:
        return self.stage.chi_reduce(self.batch, q, S, coords=self.coords(pos), sigma2=sigma2)


def finder_groups(finder, positions, box, absorbers, ipot_of, weight=None):
    """PathModel groups of every path the finder (``GPUPathFinder``) returns for the absorbers at positions (N, 3):
    atoms as global indices with the absorber first, degeneracy times ``weight`` (default 1 / the number of absorbers:
    the row is the absorbers' mean spectrum, as the reference's PathSpectra.spectra divides by them,
    ``exafs/forward.py:141-163``), row 0."""
    ab_np = np.asarray(absorbers, np.int64)
    w = 1.0 / max(len(ab_np), 1) if weight is None else float(weight)
    res = finder.enumerate_many(positions, box, ab_np, ipot_of)
    groups = []
    for nleg, (_c, ipots, deg, _xp, atoms, slot) in sorted(res["paths"].items()):
        ab = torch.as_tensor(ab_np, device=atoms.device)[slot.long()][:, None]
        groups.append((torch.cat([ab, atoms.long()], 1).cpu().numpy(), ipots.cpu().numpy(),
                       deg.double().cpu().numpy() * w, np.zeros(len(deg), int)))
    return groups


class GraphedRefinement:
    """One refinement step -- rows of every model, mean spectrum per model, R-space misfit summed over the models,
    backward, Adam -- captured once in a CUDA graph, then replayed.  models: list of (PathModel, q as a device
    tensor, S, misfit); the positions are shared by all models (several edges of one structure).  The warm-up steps
    that precede the capture (they allocate every buffer the step uses) are undone afterwards: the first replay
    is the first step from `positions` with a fresh optimiser state.

    rebuild(positions (N, 3) FP64 tensor, models) -> models, with refresh_every > 0: every refresh_every steps the
    path lists are found again at the current positions (the reference's loop re-enumerates every refresh_every
    steps, ``rmc/refine.py:176-179``) and the step is captured again; positions and optimiser state carry over.
    ``refreshes`` records (step, milliseconds of finding and capturing)."""

    def __init__(self, models, positions, lr=0.002, warmup=2, rebuild=None, refresh_every=0):
        self.models = models
        dev = models[0][0].stage.device
        self.dev = dev
        self.pos0 = torch.as_tensor(positions, dtype=torch.float64).to(dev).clone()
        self.pos = self.pos0.clone().requires_grad_(True)
        self.opt = torch.optim.Adam([self.pos], lr=lr, capturable=True)
        self.loss = torch.zeros((), dtype=torch.float64, device=dev)
        self.rebuild, self.refresh_every = rebuild, int(refresh_every)
        if self.refresh_every and rebuild is None:
            raise ValueError("refresh_every needs a rebuild function")
        self.nstep = 0
        self.refreshes: list = []
        self._capture(warmup)
        self.reset()

    def _capture(self, warmup):
        dev = self.dev
        s = torch.cuda.Stream(dev)
        s.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(s):
            for _ in range(max(1, warmup)):
                self._step()
        torch.cuda.current_stream(dev).wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        self.opt.zero_grad(set_to_none=False)
        with torch.cuda.graph(self.graph):
            self._step()

    @torch.no_grad()
    def refresh(self) -> None:
        """New path lists at the current positions and a new capture of the step; the positions, the optimiser state
        and the loss are kept (the warm-up before the capture runs on copies' behalf and is undone)."""
        torch.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        pos = self.pos.detach().clone()
        state = [{k: v.clone() for k, v in st.items() if torch.is_tensor(v)} for st in self.opt.state.values()]
        loss = self.loss.clone()
        self.models = self.rebuild(pos, self.models)
        del self.graph
        with torch.enable_grad():
            self._capture(1)
        self.pos.copy_(pos)
        for st, saved in zip(self.opt.state.values(), state):
            for k, v in saved.items():
                st[k].copy_(v)
        self.loss.copy_(loss)
        torch.cuda.synchronize(self.dev)
        self.refreshes.append((self.nstep, (time.perf_counter() - t0) * 1e3))

    @torch.no_grad()
    def reset(self, positions=None) -> None:
        """Back to `positions` (default: the initial ones) with a fresh optimiser state and step count, in place
        (the path lists stay those of the last refresh)."""
        self.nstep = 0
        self.pos.copy_(self.pos0 if positions is None else torch.as_tensor(positions, dtype=torch.float64))
        for st in self.opt.state.values():
            for v in st.values():
                if torch.is_tensor(v):
                    v.zero_()
        self.loss.zero_()

    def _loss(self):
        total = 0.0
        for model, q, S, misfit in self.models:
            rows = model.rows(self.pos, q, S)
            total = total + misfit(rows.mean(0, keepdim=True))[0]
        return total

    def _step(self):
        self.opt.zero_grad(set_to_none=False)
        loss = self._loss()
        loss.backward()
        self.opt.step()
        self.loss.copy_(loss.detach())

    def step(self) -> None:
        if self.refresh_every and self.nstep and self.nstep % self.refresh_every == 0:
            self.refresh()
        self.graph.replay()
        self.nstep += 1
