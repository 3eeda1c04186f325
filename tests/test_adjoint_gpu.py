"""GPU: the differentiable leapfrog (ncgpu_leapfrog / ncgpu_leapfrog_vjp) and
its torch.autograd.Function.

Tolerances:
  forward     final positions vs the oracle's exact-FP64 integrator loop:
              max relative difference <= 1e-10 (the forward sums pairs with
              one FP64 rsqrt instead of the reference's sqrt and divisions);
  gradients   vs FP64 central finite differences of the same forward:
              relative error <= 1e-5 per checked coordinate.
"""
import numpy as np
import pytest

from conftest import make_params

pytestmark = pytest.mark.gpu


@pytest.fixture()
def lib_ready(lib):
    from ncorpion_b200 import api
    api.init(1024, make_params(softening_parameter=0.5))
    yield api
    api.finalize()


def disk(n, seed):
    from ncorpion_b200 import disks
    b = disks.gravity_disk(n, seed=seed)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    b, cm = disks.reduce_to_com(b, cm)
    return b, cm


def mse_loss(x, target):
    return float(np.mean(np.sum((x - target) ** 2, axis=1)))


def test_forward_matches_oracle_loop(lib_ready, port):
    api = lib_ready
    b, cm = disk(300, 1)
    dt, n = 1e-3, 40
    xf, vf = api.leapfrog(b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, dt, n)
    p = make_params(softening_parameter=0.5)
    ex = np.ones(len(b), np.int32)
    bb, cc = port.drift(b, ex, cm, dt / 2, p)
    for _ in range(n):
        bb, cc = port.kick(bb, ex, cc, dt, p)
        bb, cc = port.drift(bb, ex, cc, dt, p)
    x_ref = bb[:, :3] - dt / 2 * bb[:, 3:6]
    rel = np.abs(xf - x_ref).max() / np.abs(x_ref).max()
    assert rel <= 1e-10, rel
    assert np.abs(vf - bb[:, 3:6]).max() <= 1e-10 * np.abs(bb[:, 3:6]).max()


def _fd_check(api, b, cm, dt, nsteps, coords, seed, h=1e-6):
    rng = np.random.default_rng(seed)
    x0, v0, m, R = b[:, :3].copy(), b[:, 3:6].copy(), b[:, 6].copy(), b[:, 7].copy()
    xf, _ = api.leapfrog(x0, v0, m, R, cm, dt, nsteps)
    target = xf + rng.normal(0, 1e-4, xf.shape)
    n = len(b)
    adj = 2.0 * (xf - target) / n
    gx, gv, gm = api.leapfrog_vjp(x0, v0, m, R, cm, dt, nsteps, adj)

    def loss_of(x0_, v0_, m_):
        return mse_loss(api.leapfrog(x0_, v0_, m_, R, cm, dt, nsteps)[0], target)

    worst = 0.0
    for q in range(coords):
        kind = q % 3
        i = int(rng.integers(n))
        if kind == 2:  # mass: relative step
            hm = h * m[i]
            mp, mm = m.copy(), m.copy()
            mp[i] += hm
            mm[i] -= hm
            fd = (loss_of(x0, v0, mp) - loss_of(x0, v0, mm)) / (2 * hm)
            g = gm[i]
        else:
            d = int(rng.integers(3))
            arr = x0 if kind == 0 else v0
            ap, am = arr.copy(), arr.copy()
            ap[i, d] += h
            am[i, d] -= h
            if kind == 0:
                fd = (loss_of(ap, v0, m) - loss_of(am, v0, m)) / (2 * h)
                g = gx[i, d]
            else:
                fd = (loss_of(x0, ap, m) - loss_of(x0, am, m)) / (2 * h)
                g = gv[i, d]
        err = abs(g - fd) / max(abs(fd), 1e-300)
        worst = max(worst, err)
    return worst


def test_vjp_vs_finite_differences_small(lib_ready):
    b, cm = disk(200, 2)
    assert _fd_check(lib_ready, b, cm, 1e-3, 150, 18, seed=3) <= 1e-5


def test_vjp_checkpoint_independent(lib_ready):
    api = lib_ready
    b, cm = disk(128, 4)
    adj = np.random.default_rng(5).normal(size=(128, 3))
    r1 = api.leapfrog_vjp(b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, 1e-3, 70, adj, checkpoint=32)
    r2 = api.leapfrog_vjp(b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, 1e-3, 70, adj, checkpoint=7)
    for a, c in zip(r1, r2):
        assert np.array_equal(a, c)


def test_torch_autograd_function(lib_ready):
    import torch
    from ncorpion_b200 import autograd
    api = lib_ready
    b, cm = disk(96, 6)
    x0 = torch.tensor(b[:, :3], requires_grad=True)
    v0 = torch.tensor(b[:, 3:6], requires_grad=True)
    m = torch.tensor(b[:, 6], requires_grad=True)
    target = torch.tensor(b[:, :3]) + 1e-3
    x = autograd.leapfrog(x0, v0, m, torch.tensor(b[:, 7]), torch.tensor(cm), 1e-3, 50)
    loss = ((x - target) ** 2).sum(dim=1).mean()
    loss.backward()
    adj = (2.0 * (x.detach() - target) / len(b)).numpy()
    gx, gv, gm = api.leapfrog_vjp(b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, 1e-3, 50, adj)
    assert np.array_equal(x0.grad.numpy(), gx)
    assert np.array_equal(v0.grad.numpy(), gv)
    assert np.array_equal(m.grad.numpy(), gm)


def test_adjoint_disk_16384_1000_steps(lib):
    """The differentiable workload: N = 16,384 (log-uniform masses, softening
    0.5 (R_k + R_p)), 1,000 steps, dt = 1e-3, checkpoints every 32 steps;
    MSE loss to a seeded target; 64 coordinates (x, v, m) against FP64
    central differences with h = 1e-6."""
    from ncorpion_b200 import api
    api.init(16384, make_params(softening_parameter=0.5))
    try:
        b, cm = disk(16384, 0)
        assert _fd_check(api, b, cm, 1e-3, 1000, 64, seed=11) <= 1e-5
    finally:
        api.finalize()
