"""Paths held as atom indices over a structure, evaluated by the fused stage at any positions (MD and RMC use).

The reference keeps path lists as global atom indices and rebuilds the coordinates from the current positions at
every evaluation (``src/feffgpu/exafs/forward.py:99-163, 664-725``): relative vectors to the absorber under the
minimum image, absorber first, then ``cchi`` + ``chi_fine`` per chunk and an ``index_add`` into one row per
absorber/copy.  ``PathModel`` does the same with one ``PathBatch`` and one fused call per evaluation: the gather of
the coordinates is a differentiable torch indexing (its backward scatters the per-path gradients onto the atoms),
the stage is ``GPUPathStage.chi_reduce``.  ``GraphedRefinement`` captures one refinement step -- model, R-space
misfit, backward and the Adam update -- in a CUDA graph and replays it (the RMC loop of
``src/feffgpu/rmc/refine.py:120-260`` with a fixed path list).
"""
from __future__ import annotations

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

    def __init__(self, stage, groups, positions, nrows=None, box=None, chunk=256):
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
        self.batch = PathBatch(bgroups, nrows=nrows, device=dev, chunk=chunk)
        self.atoms = torch.cat(atoms).to(dev)
        legs = torch.arange(nleg_max, device=dev)
        self.mask = (legs[None, :] < self.batch.nleg[:, None].long()).to(torch.float64)[:, :, None]

    def coords(self, pos: torch.Tensor) -> torch.Tensor:
        """(n, nleg_max, 3) relative coordinates of every path at positions pos (N, 3), differentiable."""
        rel = pos[self.atoms] - pos[self.atoms[:, :1]]
        return self.min_image(rel) * self.mask

    def rows(self, pos: torch.Tensor, q: torch.Tensor, S: torch.Tensor, sigma2=None) -> torch.Tensor:
        return self.stage.chi_reduce(self.batch, q, S, coords=self.coords(pos), sigma2=sigma2)


class GraphedRefinement:
    """One refinement step -- rows of every model, mean spectrum per model, R-space misfit summed over the models,
    backward, Adam -- captured once in a CUDA graph, then replayed.  models: list of (PathModel, q as a device
    tensor, S, misfit); the positions are shared by all models (several edges of one structure).  The warm-up steps
    that precede the capture (they allocate every buffer the step uses) are undone afterwards: the first replay
    is the first step from `positions` with a fresh optimiser state."""

    def __init__(self, models, positions, lr=0.002, warmup=2):
        self.models = models
        dev = models[0][0].stage.device
        self.pos0 = torch.as_tensor(positions, dtype=torch.float64).to(dev).clone()
        self.pos = self.pos0.clone().requires_grad_(True)
        self.opt = torch.optim.Adam([self.pos], lr=lr, capturable=True)
        self.loss = torch.zeros((), dtype=torch.float64, device=dev)
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
        self.reset()

    @torch.no_grad()
    def reset(self, positions=None) -> None:
        """Back to `positions` (default: the initial ones) with a fresh optimiser state, in place."""
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
        self.graph.replay()
