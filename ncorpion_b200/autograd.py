"""torch.autograd.Function over the differentiable leapfrog of libncgpu.

    from ncorpion_b200 import api, autograd
    api.init(n_max, api.default_params(G=1.0, softening_parameter=0.5, collision_bool=0))
    x = autograd.leapfrog(x0, v0, m, R, cm, dt=1e-3, nsteps=1000)   # differentiable in x0, v0, m
    loss = ((x - target) ** 2).sum(dim=1).mean()
    loss.backward()

The forward and the backward both run on the GPU through the C ABI
(ncgpu_leapfrog / ncgpu_leapfrog_vjp); tensors are float64, on any device
(they are staged through host memory, the library's own device state is
separate from torch's).  R (softening radii) and the central-mass record
are not differentiated.
"""
from __future__ import annotations

import numpy as np
import torch

from . import api


def _np(t):
    return t.detach().to("cpu", torch.float64).contiguous().numpy()


class LeapfrogFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, m, R, cm, dt, nsteps, checkpoint):
        xf, _ = api.leapfrog(_np(x0), _np(v0), _np(m), _np(R), _np(cm), dt, nsteps, checkpoint)
        ctx.save_for_backward(x0, v0, m, R, cm)
        ctx.cfg = (dt, nsteps, checkpoint)
        return torch.from_numpy(xf).to(x0.device)

    @staticmethod
    def backward(ctx, gx):
        x0, v0, m, R, cm = ctx.saved_tensors
        dt, nsteps, checkpoint = ctx.cfg
        gx0, gv0, gm = api.leapfrog_vjp(_np(x0), _np(v0), _np(m), _np(R), _np(cm), dt, nsteps, _np(gx), checkpoint)
        dev = x0.device
        return (torch.from_numpy(gx0).to(dev), torch.from_numpy(gv0).to(dev), torch.from_numpy(gm).to(dev), None, None,
                None, None, None)


def leapfrog(x0, v0, m, R, cm, dt, nsteps, checkpoint=32):
    """Final positions (n, 3) after the collisionless leapfrog, differentiable
    with respect to x0, v0 and m."""
    return LeapfrogFunction.apply(x0, v0, m, R, cm, float(dt), int(nsteps), int(checkpoint))
