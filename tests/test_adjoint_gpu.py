"""GPU: the differentiable leapfrog (ncgpu_leapfrog / ncgpu_leapfrog_vjp) and
its torch.autograd.Function.

Tolerances:
  forward     final positions vs the oracle's exact-FP64 integrator loop:
              max relative difference <= 1e-10 (the forward sums pairs with
              one FP64 rsqrt instead of the reference's sqrt and divisions);
  x0, v0      vs FP64 central finite differences of the same forward (h = 1e-6):
              relative error <= 1e-5 per checked coordinate;
  m           vs the tangent-linear model (ncgpu_leapfrog_jvp, exact to
              rounding): relative error <= 1e-8.  FP64 finite differences of
              the masses (1e-9 .. 1e-6) drown in roundoff at h <= 1e-6 m; a
              Richardson-extrapolated difference with steps 0.1 m and 0.05 m is
              kept as a sanity check (<= 1e-3).
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


def _fd_check(api, b, cm, dt, nsteps, coords, seed, h=1e-6, richardson=False):
    """Worst relative error of the adjoint gradient of the MSE loss over
    `coords` random coordinates (x, v: finite differences; m: tangent model)."""
    rng = np.random.default_rng(seed)
    x0, v0, m, R = b[:, :3].copy(), b[:, 3:6].copy(), b[:, 6].copy(), b[:, 7].copy()
    xf, _ = api.leapfrog(x0, v0, m, R, cm, dt, nsteps)
    target = xf + rng.normal(0, 1e-4, xf.shape)
    n = len(b)
    adj = 2.0 * (xf - target) / n
    gx, gv, gm = api.leapfrog_vjp(x0, v0, m, R, cm, dt, nsteps, adj)

    def loss_of(x0_, v0_, m_):
        return mse_loss(api.leapfrog(x0_, v0_, m_, R, cm, dt, nsteps)[0], target)

    worst = {"x": 0.0, "v": 0.0, "m": 0.0, "m_fd": 0.0}
    zero3 = np.zeros((n, 3))
    for q in range(coords):
        kind = q % 3
        i = int(rng.integers(n))
        if kind == 2:
            em = np.zeros(n)
            em[i] = 1.0
            tan = api.leapfrog_jvp(x0, v0, m, R, cm, dt, nsteps, zero3, zero3, em)
            ref = float(np.sum(adj * tan))
            worst["m"] = max(worst["m"], abs(gm[i] - ref) / abs(ref))
            if richardson:
                def D(rel):
                    hm = rel * m[i]
                    mp, mm = m.copy(), m.copy()
                    mp[i] += hm
                    mm[i] -= hm
                    return (loss_of(x0, v0, mp) - loss_of(x0, v0, mm)) / (2 * hm)
                rich = (4 * D(0.05) - D(0.1)) / 3
                worst["m_fd"] = max(worst["m_fd"], abs(gm[i] - rich) / abs(rich))
        else:
            d = int(rng.integers(3))
            arr = x0 if kind == 0 else v0
            ap, am = arr.copy(), arr.copy()
            ap[i, d] += h
            am[i, d] -= h
            if kind == 0:
                fd = (loss_of(ap, v0, m) - loss_of(am, v0, m)) / (2 * h)
                g, key = gx[i, d], "x"
            else:
                fd = (loss_of(x0, ap, m) - loss_of(x0, am, m)) / (2 * h)
                g, key = gv[i, d], "v"
            worst[key] = max(worst[key], abs(g - fd) / max(abs(fd), 1e-300))
    return worst


def _assert_worst(w):
    assert w["x"] <= 1e-5 and w["v"] <= 1e-5, w
    assert w["m"] <= 1e-8, w
    assert w["m_fd"] <= 1e-3, w


def test_vjp_vs_finite_differences_small(lib_ready):
    b, cm = disk(200, 2)
    _assert_worst(_fd_check(lib_ready, b, cm, 1e-3, 150, 18, seed=3, richardson=True))


def test_adjoint_dot_product_identity(lib_ready):
    """<w, J d> = <J^T w, d> for random w and random directions d."""
    api = lib_ready
    b, cm = disk(300, 8)
    rng = np.random.default_rng(9)
    n = len(b)
    args = (b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, 1e-3, 120)
    dx, dv, dm = rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.normal(size=n) * b[:, 6]
    w = rng.normal(size=(n, 3))
    jd = api.leapfrog_jvp(*args, dx, dv, dm)
    gx, gv, gm = api.leapfrog_vjp(*args, w)
    lhs = float(np.sum(w * jd))
    rhs = float(np.sum(gx * dx) + np.sum(gv * dv) + np.sum(gm * dm))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


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
    # torch forms dL/dx_final itself (same values to rounding)
    assert np.allclose(x0.grad.numpy(), gx, rtol=1e-12, atol=0)
    assert np.allclose(v0.grad.numpy(), gv, rtol=1e-12, atol=0)
    assert np.allclose(m.grad.numpy(), gm, rtol=1e-12, atol=0)


def test_adjoint_disk_16384_1000_steps(lib):
    """The differentiable workload: N = 16,384 (log-uniform masses, R = 1e-2,
    softening 0.5 (R_k + R_p)), 1,000 steps, dt = 1e-3, checkpoints every 32
    steps; MSE loss to a seeded target; 64 coordinates: x and v against FP64
    central differences with h = 1e-6, m against the tangent-linear model."""
    from ncorpion_b200 import api, disks
    api.init(16384, make_params(softening_parameter=0.5))
    try:
        b, cm = disks.reduce_to_com(disks.adjoint_disk(16384, 0), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]))
        w = _fd_check(api, b, cm, 1e-3, 1000, 64, seed=11)
        print("adjoint 16384 x 1000 worst relative errors:", w)
        _assert_worst(w)
    finally:
        api.finalize()


def test_adjoint_chaotic_disk_dot_product(lib):
    """On the R = 1e-5 disk the 1,000-step map is chaotic (finite differences
    leave the linear regime), but the adjoint must still be the exact
    transpose of the tangent-linear model along the same trajectory:
    <w, J d> = <J^T w, d> for seeded w, d, to 1e-8 relative."""
    from ncorpion_b200 import api
    api.init(16384, make_params(softening_parameter=0.5))
    try:
        b, cm = disk(16384, 0)
        n = len(b)
        rng = np.random.default_rng(21)
        args = (b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, 1e-3, 1000)
        dx, dv, dm = rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.normal(size=n) * b[:, 6]
        w = rng.normal(size=(n, 3))
        jd = api.leapfrog_jvp(*args, dx, dv, dm)
        gx, gv, gm = api.leapfrog_vjp(*args, w)
        lhs = float(np.sum(w * jd))
        rhs = float(np.sum(gx * dx) + np.sum(gv * dv) + np.sum(gm * dm))
        print("chaotic disk <w, J d> =", lhs, " <J^T w, d> =", rhs)
        assert np.isfinite(lhs) and abs(lhs - rhs) <= 1e-8 * abs(lhs)
    finally:
        api.finalize()


def test_mixed_adjoint_disk_16384_1000_steps(lib):
    """The differentiable workload in the MIXED gravity mode (FP32 pair terms
    on tile-relative coordinates for far tile pairs, FP64 for near ones, FP64
    state): its gradients against the FP64 ones -- x and v against FP64
    central finite differences (h = 1e-6) of the FP64 forward, m against the
    FP64 tangent-linear model -- within 1e-5 relative on 64 coordinates of
    the 16,384-body, 1,000-step run."""
    from ncorpion_b200 import api, disks
    p64 = make_params(softening_parameter=0.5)
    pmx = make_params(softening_parameter=0.5, gravity_mode=api.GRAVITY_MIXED)
    api.init(16384, p64)
    try:
        b, cm = disks.reduce_to_com(disks.adjoint_disk(16384, 0), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]))
        dt, nsteps, n = 1e-3, 1000, len(b)
        rng = np.random.default_rng(11)
        x0, v0, m, R = b[:, :3].copy(), b[:, 3:6].copy(), b[:, 6].copy(), b[:, 7].copy()
        xf, _ = api.leapfrog(x0, v0, m, R, cm, dt, nsteps)
        api.set_params(pmx)
        xf_mx, _ = api.leapfrog(x0, v0, m, R, cm, dt, nsteps)
        print("mixed vs FP64 forward, max |dx| / max |x|:", np.abs(xf_mx - xf).max() / np.abs(xf).max())
        target = xf + rng.normal(0, 1e-4, xf.shape)
        adj = 2.0 * (xf - target) / n
        gx, gv, gm = api.leapfrog_vjp(x0, v0, m, R, cm, dt, nsteps, adj)
        api.set_params(p64)

        def loss_of(x0_, v0_):
            return mse_loss(api.leapfrog(x0_, v0_, m, R, cm, dt, nsteps)[0], target)

        worst = {"x": 0.0, "v": 0.0, "m": 0.0}
        zero3 = np.zeros((n, 3))
        h = 1e-6
        for q in range(64):
            kind = q % 3
            i = int(rng.integers(n))
            if kind == 2:
                em = np.zeros(n)
                em[i] = 1.0
                ref = float(np.sum(adj * api.leapfrog_jvp(x0, v0, m, R, cm, dt, nsteps, zero3, zero3, em)))
                worst["m"] = max(worst["m"], abs(gm[i] - ref) / abs(ref))
                continue
            d = int(rng.integers(3))
            arr = x0 if kind == 0 else v0
            ap, am = arr.copy(), arr.copy()
            ap[i, d] += h
            am[i, d] -= h
            if kind == 0:
                fd = (loss_of(ap, v0) - loss_of(am, v0)) / (2 * h)
                g, key = gx[i, d], "x"
            else:
                fd = (loss_of(x0, ap) - loss_of(x0, am)) / (2 * h)
                g, key = gv[i, d], "v"
            worst[key] = max(worst[key], abs(g - fd) / max(abs(fd), 1e-300))
        print("mixed adjoint 16384 x 1000 worst relative errors vs FP64:", worst)
        assert worst["x"] <= 1e-5 and worst["v"] <= 1e-5 and worst["m"] <= 1e-5, worst
    finally:
        api.finalize()


def test_mixed_adjoint_is_the_transpose_of_its_tangent(lib):
    """In the MIXED mode too the VJP and the JVP are transposes of each other
    along the same trajectory (dot-product identity, 1e-6 relative: both carry
    FP32 pair terms)."""
    from ncorpion_b200 import api
    api.init(1024, make_params(softening_parameter=0.5, gravity_mode=api.GRAVITY_MIXED))
    try:
        b, cm = disk(1000, 8)
        rng = np.random.default_rng(9)
        n = len(b)
        args = (b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, 1e-3, 120)
        dx, dv, dm = rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.normal(size=n) * b[:, 6]
        w = rng.normal(size=(n, 3))
        jd = api.leapfrog_jvp(*args, dx, dv, dm)
        gx, gv, gm = api.leapfrog_vjp(*args, w)
        lhs = float(np.sum(w * jd))
        rhs = float(np.sum(gx * dx) + np.sum(gv * dv) + np.sum(gm * dm))
        print("mixed <w, J d> =", lhs, " <J^T w, d> =", rhs)
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    finally:
        api.finalize()
