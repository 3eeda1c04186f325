"""GPU parity of the brute-force collision sweep, the collision resolutions
and end_of_timestep, through the C ABI.

Tolerance: the event list (a, b, type) in resolution order, exists[] and every
body field are bit-identical to the oracle, except the radius of merged bodies,
which may differ by 1 ulp: the device computes pow(x, 1.0/3.0) correctly
rounded, glibc's pow is not correctly rounded for about 5e-4 of arguments.
"""
from decimal import Decimal, getcontext

import numpy as np
import pytest

import oracle
from conftest import golden, make_params

pytestmark = pytest.mark.gpu


def ulps(a, b):
    a = np.ascontiguousarray(a, np.float64).view(np.int64)
    b = np.ascontiguousarray(b, np.float64).view(np.int64)
    return np.abs(a - b)


def assert_state_equal(b, ex, b_ref, ex_ref):
    assert b.shape == b_ref.shape
    assert np.array_equal(ex, ex_ref)
    live = ex_ref == 1
    assert np.array_equal(b[live][:, :7], b_ref[live][:, :7])
    assert ulps(b[live][:, 7], b_ref[live][:, 7]).max() <= 1


@pytest.fixture()
def gpu(lib):
    from ncorpion_b200 import api

    def _init(n_max, **kw):
        api.init(n_max, make_params(**kw))
        return api

    yield _init
    api.finalize()


def test_pow_one_third_correctly_rounded(lib):
    from ncorpion_b200 import api
    rng = np.random.default_rng(0)
    x = (10.0 ** rng.uniform(-16.5, -4.5, 4000)) * rng.uniform(0.5, 2.0, 4000)
    out = np.zeros_like(x)
    api.check(lib.ncgpu_probe_pow_third(api.ptr(x), api.ptr(out), len(x)), "pow")
    getcontext().prec = 60
    y = Decimal(1.0 / 3.0)
    exact = np.array([float((Decimal(v).ln() * y).exp()) for v in x])
    assert np.array_equal(out, exact)


@pytest.mark.parametrize("name,ctype", [("bf_sweep_merge", 2), ("bf_sweep_elastic", 0), ("bf_sweep_inelastic", 1)])
def test_brute_force_sweep(gpu, name, ctype):
    g = golden(name)
    api = gpu(4096, collision_bool=1, collision_type=ctype, collision_parameter=1.5)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    n = api.collide_brute()
    assert n == len(g["events"])
    assert np.array_equal(api.events(), g["events"])
    b, ex, cm = api.download(4096)
    w = oracle.PortWorld(4096, make_params(collision_bool=1, collision_type=ctype, collision_parameter=1.5))
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]))
    w.lib.orc_w_brute_force()
    b_ref, ex_ref, _ = w.get_state()
    assert_state_equal(b, ex, b_ref, ex_ref)


def test_brute_force_run_40_steps(gpu):
    """kick, collisions, drift, end_of_timestep x 40 on the device state."""
    g = golden("bf_run_merge")
    api = gpu(4096, collision_bool=1, collision_type=2)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    evs = []
    for _ in range(int(g["nsteps"])):
        api.step_brute_force()
        evs.append(api.events())
    assert np.array_equal(np.concatenate(evs), g["events"])
    b, ex, cm = api.download(4096)
    w = oracle.PortWorld(4096, make_params(collision_bool=1, collision_type=2))
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]))
    for _ in range(int(g["nsteps"])):
        w.lib.orc_w_step_brute_force()
    b_ref, ex_ref, cm_ref = w.get_state()
    assert_state_equal(b, ex, b_ref, ex_ref)
    assert np.array_equal(cm, cm_ref)


def test_dense_cluster_many_events(gpu):
    """A tight cluster where most bodies overlap: long chains of mergers in
    which merged bodies collide again within the same sweep."""
    rng = np.random.default_rng(4)
    n = 300
    b = np.zeros((n, 8))
    b[:, 0] = 1.0 + rng.normal(0, 5e-3, n)
    b[:, 1] = rng.normal(0, 5e-3, n)
    b[:, 2] = rng.normal(0, 1e-3, n)
    b[:, 3:6] = rng.normal(0, 1e-2, (n, 3))
    b[:, 4] += 1.0
    b[:, 6] = 10.0 ** rng.uniform(-9, -7, n)
    b[:, 7] = rng.uniform(5e-4, 2e-3, n)
    ex = np.ones(n, np.int32)
    ex[::17] = 0
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    for ctype in (2, 0):
        api = gpu(512, collision_bool=1, collision_type=ctype)
        api.upload(b, ex, cm)
        api.set_timestep(1e-3)
        api.collide_brute()
        ev = api.events()
        bg, exg, _ = api.download(512)
        api.finalize()
        w = oracle.PortWorld(512, make_params(collision_bool=1, collision_type=ctype))
        w.set_state(b, ex, cm, dt=1e-3)
        w.lib.orc_w_brute_force()
        assert len(w.events()) > 20
        assert np.array_equal(ev, w.events())
        b_ref, ex_ref, _ = w.get_state()
        assert_state_equal(bg, exg, b_ref, ex_ref)


def test_end_of_timestep_dumping_and_tidy(gpu):
    """Bodies inside the disruption radius merge into the central mass, bodies
    beyond the outer threshold leave and trigger a barycentre reduction, and
    the array is compacted by tidy_up."""
    from ncorpion_b200 import disks
    b = disks.gravity_disk(1000, seed=9)
    b[10:40, :3] *= 0.05       # inside disruption_threshold 0.1
    b[100:250, :3] *= 200.0     # beyond high_dumping_threshold 100
    ex = np.ones(1000, np.int32)
    ex[500:510] = 0
    cm = np.array([1e-4, 0, 0, 0, 1e-5, 0, 1.0, 1.0])
    api = gpu(1024)
    api.upload(b, ex, cm)
    hm = api.end_of_timestep()
    bg, exg, cmg = api.download(1024)
    w = oracle.PortWorld(1024, make_params())
    w.set_state(b, ex, cm)
    w.lib.orc_w_end_of_timestep.restype = __import__("ctypes").c_int
    hm_ref = w.lib.orc_w_end_of_timestep()
    b_ref, ex_ref, cm_ref = w.get_state()
    assert hm == hm_ref == 1000 - 10 - 30 - 150
    assert np.array_equal(exg, ex_ref) and np.array_equal(bg, b_ref) and np.array_equal(cmg, cm_ref)
