"""GPU parity of the tides raised on the central body (src/physics.c:496-542,
called by kick, src/rk4.c:88-90), through the C ABI, against the reference's
golden vectors and the oracle port.

The tides make the central body's rotation SideralOmega change body by body
(a sequential recurrence, one warp on the device); the fixtures use a long
time lag (Delta_t = 1) so that every body changes it.  Tolerance: the state,
the central mass and SideralOmega after every step bit-identical in the exact
gravity mode; in the mixed mode (same recurrence on mixed-precision
accelerations) SideralOmega within 1e-14 relative of the exact run.
"""
import numpy as np
import pytest

import oracle
from conftest import golden, make_params

pytestmark = pytest.mark.gpu

TIDES = dict(central_tides_bool=1, Delta_t=1.0)
J2F = dict(J2_bool=1, J2=0.0, sideral_omega=2.0 * np.pi / 25.0)


def _digest(a):
    import hashlib
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


@pytest.fixture()
def gpu(lib):
    from ncorpion_b200 import api

    def _init(n_max, **kw):
        api.init(n_max, make_params(**kw))
        return api

    yield _init
    api.finalize()


BF = [("tides_bf_steps", dict(softening_parameter=0.5, **TIDES)), ("tides_j2f_bf_steps", dict(**TIDES, **J2F))]


@pytest.mark.parametrize("name,kw", BF)
def test_tides_bf_steps_match_reference_golden(gpu, name, kw):
    g = golden(name)
    api = gpu(1024, **kw)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    assert api.get_sideral_omega() == g["omegas"][0]
    for s in range(int(g["nsteps"])):
        api.step_brute_force()
        assert api.get_sideral_omega() == g["omegas"][s + 1]
    b, ex, cm = api.download(1024)
    assert np.array_equal(b, g["out_bodies"]) and np.array_equal(ex, g["out_exists"])
    assert np.array_equal(cm, g["out_cm"])


def test_tides_mesh_steps_match_reference_golden(gpu):
    from ncorpion_b200 import api as A
    g = golden("tides_mesh_steps")
    api = gpu(16384, mesh_bool=1, brute_force_bool=0, collision_bool=0, collision_cube_cells=256, **TIDES, **J2F)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    gam = float(g["gam"])
    for s in range(int(g["nsteps"])):
        hm, tn = api.step_mesh(gam)
        gam = A.update_gamma(gam, tn, hm, 16.0, 4.4 / 256)
        assert gam == g["gams"][s]
        assert api.get_sideral_omega() == g["omegas"][s + 1]
    b, ex, cm = api.download(16384)
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])
    assert np.array_equal(cm, g["out_cm"])


@pytest.mark.parametrize("n", [1, 63, 64, 65, 3000])
def test_tides_kick_matches_port(gpu, port, n):
    """One kick with tides from a rotation set through the ABI, against the
    port's kick: velocities, central mass and the new rotation; sizes around
    the 64-body staging block of the recurrence."""
    from ncorpion_b200 import disks
    rng = np.random.default_rng(n)
    b = disks.gravity_disk(n, seed=n + 3)
    ex = (rng.random(n) > 0.1).astype(np.int32)
    ex[0] = 1
    cm = np.array([1e-6, -2e-6, 0.0, 1e-7, 0.0, -1e-7, 1.0, 1.0])
    kw = dict(softening_parameter=0.5, **TIDES)
    api = gpu(4096, **kw)
    api.upload(b, ex, cm)
    api.set_timestep(2e-3)
    api.set_sideral_omega(0.7)
    api.kick()
    bg, exg, cmg = api.download(4096)
    p = make_params(**kw)
    p.sideral_omega = 0.7
    b_ref, cm_ref = port.kick(b, ex, cm, 2e-3, p)
    live = ex == 1
    assert np.array_equal(bg[live], b_ref[live]) and np.array_equal(cmg, cm_ref)
    assert api.get_sideral_omega() == p.sideral_omega != 0.7


def test_tides_mixed_mode_close_to_exact(gpu):
    """The mixed gravity mode feeds the same recurrence with mixed-precision
    accelerations: the rotation stays within 1e-14 of the exact run."""
    from ncorpion_b200 import disks
    n = 4000
    b = disks.gravity_disk(n, seed=77)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    out = {}
    for mode in (0, 2):
        api = gpu(8192, gravity_mode=mode, softening_parameter=0.5, **TIDES)
        api.upload(b, ex, cm)
        api.set_timestep(1e-3)
        for _ in range(3):
            api.step_brute_force()
        out[mode] = api.get_sideral_omega()
        api.finalize()
    assert out[0] != 2.0 * np.pi / 3.556721809
    assert abs(out[2] - out[0]) <= 1e-14 * abs(out[0])


def test_tides_need_central_mass(lib):
    from ncorpion_b200 import api as A
    with pytest.raises(A.NcgpuError) as e:
        A.init(64, make_params(central_mass_bool=0, **TIDES))
    assert e.value.status == A.E_ARG
    A.finalize()


def test_tides_division_is_correctly_rounded(lib):
    """The recurrence's quotient (reciprocal + two residual corrections,
    Markstein) against correctly rounded division, bit for bit: random
    quotients, divisors in S's range (0.5, 1] and beyond, quotients next to
    exactly representable ones, zeros of both signs."""
    from ncorpion_b200 import api
    rng = np.random.default_rng(12)
    n = 1 << 21
    a = rng.standard_normal(n) * np.exp2(rng.integers(-60, 60, n).astype(np.float64))
    b = np.where(np.arange(n) % 2 == 0, rng.uniform(0.5, 1.0, n), rng.uniform(1e-3, 1e3, n))
    near = np.arange(n) % 4 == 3  # a = b * q0 one or two ulps off: quotients next to q0
    q0 = rng.uniform(-1, 1, n) * np.exp2(rng.integers(-30, 30, n).astype(np.float64))
    step = np.where(np.arange(near.sum()) % 2 == 0, np.inf, -np.inf)
    a[near] = np.nextafter(np.nextafter(b[near] * q0[near], step), step)
    a[:4] = [0.0, -0.0, 1.0, -3.0]
    out = np.empty(n)
    api.check(lib.ncgpu_probe_div(api.ptr(a), api.ptr(b), api.ptr(out), n), "ncgpu_probe_div")
    assert np.array_equal(out.view(np.int64), (a / b).view(np.int64))
