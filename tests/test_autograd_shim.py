"""The torch.autograd.Function shim (python/arcos_autograd.py) over the C ABI
adjoint: J.backward() against central finite differences of the same frozen
forward map."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "python"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def test_shim_imports_without_gpu():
    import arcos_autograd
    assert hasattr(arcos_autograd, "CdrSteps") and hasattr(arcos_autograd, "CdrRunner")


@pytest.mark.gpu
def test_shim_gradient_matches_fd(cuda_device):
    import torch
    import arcos_autograd
    from arcos_b200 import workloads
    from arcos_b200.adjoint import cell_volume

    pb = workloads.plain(nr=32, nz=64, ion_mass=0.0, noise=1e-3, seed=5)
    K = 12
    runner = arcos_autograd.CdrRunner(pb, nsteps=K, ckpt_every=4)
    spec = pb.specs[0]
    vol = torch.from_numpy(cell_volume(spec, pb.params.dr(0), pb.params.dz(0))[0])
    d0 = torch.from_numpy(np.stack([a[0] for a in pb.dens[0]])).requires_grad_(True)
    mu = torch.tensor([1.0, 0.0], dtype=torch.float64, requires_grad=True)
    D = torch.tensor(pb.params.diffusion_coeff, dtype=torch.float64, requires_grad=True)
    tab = torch.from_numpy(np.array(pb.model.reactions[0].table.values, dtype=np.float64)).requires_grad_(True)
    target = torch.from_numpy(np.stack([a[0] for a in pb.dens[0]])[0] * 0.9)

    def J(out):
        return 0.5 * torch.sum((out[0] - target) ** 2 * vol)

    out = arcos_autograd.cdr_steps(runner, d0, mu, D, tab)
    loss = J(out)
    loss.backward()
    from test_adjoint import smooth_field
    rng = np.random.default_rng(3)
    eps = 1e-6
    dd = np.zeros(d0.shape)
    for s in range(2):
        dd[s, 2:-2, 2:-2] = smooth_field(rng, spec.nz, spec.nr)
    dirs = [torch.from_numpy(dd), torch.tensor([rng.standard_normal(), 0.0], dtype=torch.float64),
            torch.tensor(rng.standard_normal(), dtype=torch.float64),
            torch.from_numpy(rng.standard_normal(tab.shape))]
    base = [d0.detach(), mu.detach(), D.detach(), tab.detach()]
    grads = [d0.grad, mu.grad, D.grad, tab.grad]

    def out_at(sign):
        args = [b * (1 + sign * eps * d) for b, d in zip(base, dirs)]
        with torch.no_grad():
            return arcos_autograd.cdr_steps(runner, *args)[0]

    a, b = out_at(1), out_at(-1)
    fd = float(0.5 * torch.sum(vol * (a - b) * (a + b - 2 * target))) / (2 * eps)
    pr = float(sum(torch.sum(g * b * d) for g, b, d in zip(grads, base, dirs)))
    assert abs(fd - pr) <= 1e-6 * abs(fd), (fd, pr)
