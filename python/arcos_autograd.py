"""torch.autograd.Function over the arcos CDR density update (ctypes shim).

The C ABI (include/arcos_cdr.h) takes plain pointers and sizes; this module
moves torch tensors across it through numpy and wraps the discrete adjoint
(arcos_adj_forward / arcos_adj_backward) as the backward of K fused RK2
steps on one single-grid 2-D problem:

    n(T) = CdrSteps.apply(runner, dens0, mobility, diffusion, tables)

dens0      [species, nz + 4, nr + 4] float64: the initial densities (rz
           layout; ghost entries are ignored, the step refills them)
mobility   [species] float64: 1/mass (entries of immobile species are
           ignored and get a zero gradient)
diffusion  [] float64: diffusion_coeff
tables     [sum of (steps + 1)] float64: every reaction table's values,
           reaction after reaction

The first forward call of a runner records the step sizes from the CFL rule;
later calls (and the finite-difference checks) reuse them, so the map is the
same differentiable function every time.
"""
from __future__ import annotations

import os
import sys
from typing import Optional

import numpy as np
import torch

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from arcos_b200.adjoint import Adjoint  # noqa: E402
from arcos_b200.cdr import CdrTree  # noqa: E402
from arcos_b200.workloads import Problem  # noqa: E402


class CdrRunner:
    """A committed device context for one 2-D single-grid problem."""

    def __init__(self, pb: Problem, nsteps: int, ckpt_every: int = 8, h_attempt: float = 50.0,
                 h_seq: Optional[np.ndarray] = None):
        assert len(pb.specs) == 1 and pb.specs[0].ntheta == 1, "one 2-D grid"
        self.pb = pb
        self.nsteps, self.ckpt_every, self.h_attempt = nsteps, ckpt_every, h_attempt
        self.tree = CdrTree(pb.params, pb.model, pb.specs)
        self.tree.set_fixed_field(pb.fields)
        self.adj = Adjoint(self.tree)
        self.h_seq = None if h_seq is None else np.asarray(h_seq, dtype=np.float64).reshape(1, nsteps)
        self.sizes = [r.table.steps + 1 for r in pb.model.reactions]

    def apply(self, dens0: np.ndarray, mobility: np.ndarray, diffusion: float, tables: np.ndarray):
        t = self.tree
        for s in range(dens0.shape[0]):
            t.upload(0, "dens", dens0[s][None], s)
        for s, sp in enumerate(self.pb.model.species):
            if sp.mass > 0:
                t.set_species_mass(s, 1.0 / float(mobility[s]))
        t.set_diffusion(float(diffusion))
        o = 0
        for r, re in enumerate(self.pb.model.reactions):
            n = self.sizes[r]
            t.set_table_values(r, tables[o:o + n], re.table.underflow, re.table.overflow)
            o += n

    def run(self, dens0, mobility, diffusion, tables) -> np.ndarray:
        self.apply(dens0, mobility, diffusion, tables)
        hs = self.adj.forward(self.nsteps, self.ckpt_every, h=self.h_attempt, h_seq=self.h_seq)
        if self.h_seq is None:
            self.h_seq = hs.copy()
        ns = dens0.shape[0]
        return np.stack([self.tree.download(0, "dens", s)[0] for s in range(ns)])


class CdrSteps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, runner: CdrRunner, dens0, mobility, diffusion, tables):
        dev = dens0.device
        out = runner.run(dens0.detach().cpu().numpy().astype(np.float64),
                         mobility.detach().cpu().numpy().astype(np.float64),
                         float(diffusion.detach().cpu()),
                         tables.detach().cpu().numpy().astype(np.float64))
        ctx.runner = runner
        ctx.dev = dev
        return torch.from_numpy(out).to(dev)

    @staticmethod
    def backward(ctx, grad_out):
        runner: CdrRunner = ctx.runner
        g = grad_out.detach().cpu().numpy().astype(np.float64)
        ns = g.shape[0]
        for s in range(ns):
            lam = g[s].copy()
            lam[:2, :] = 0.0
            lam[-2:, :] = 0.0
            lam[:, :2] = 0.0
            lam[:, -2:] = 0.0
            runner.adj.set_cotangent(0, s, lam[None])
        gr = runner.adj.backward()
        d0 = np.stack([gr.dens0[0][s][0] for s in range(ns)])
        d0[:, :2, :] = 0.0
        d0[:, -2:, :] = 0.0
        d0[:, :, :2] = 0.0
        d0[:, :, -2:] = 0.0
        dev = ctx.dev
        gt = np.concatenate(gr.tables) if gr.tables else np.zeros(0)
        return (None, torch.from_numpy(d0).to(dev), torch.from_numpy(gr.mobility.copy()).to(dev),
                torch.tensor(gr.diffusion, dtype=torch.float64, device=dev), torch.from_numpy(gt).to(dev))


def cdr_steps(runner: CdrRunner, dens0, mobility, diffusion, tables):
    return CdrSteps.apply(runner, dens0, mobility, diffusion, tables)
