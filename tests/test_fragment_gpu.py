"""GPU: the fragmentation model (collision type 3, src/physics.c:710-1040) in
the brute-force sweep and in the mesh pass, and mesh gravity over the pairs the
fragments add, through the C ABI, against the oracle port (pinned to the
reference by tests/golden/frag_*.npz).

Tolerance: the event list (a, b, type), the outcome counts, exists[],
largest_id and pairs[] (order included) are identical.  Bodies that no event
touched are bit-identical.  The fields of the bodies an event touched agree to
1e-11 relative: the device evaluates the model's general powers with CUDA's
pow (within 2 ulp) where the reference calls libm's pow.  Accelerations from
mesh gravity after such a pass agree to 1e-10 relative.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import golden, make_params

pytestmark = pytest.mark.gpu

RTOL = 1e-11


def _digest(a):
    import hashlib
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def _ulps(a, b):
    a = np.ascontiguousarray(a, np.float64).view(np.int64)
    b = np.ascontiguousarray(b, np.float64).view(np.int64)
    return np.abs(a - b)


def assert_close_state(b, ex, b_ref, ex_ref, events, lid0):
    assert b.shape == b_ref.shape
    assert np.array_equal(ex, ex_ref)
    live = ex_ref == 1
    touched = np.zeros(len(b_ref), bool)
    touched[events[:, :2].ravel()] = True
    touched[lid0 + 1:] = True
    same = live & ~touched
    assert np.array_equal(b[same][:, :7], b_ref[same][:, :7])
    assert _ulps(b[same][:, 7], b_ref[same][:, 7]).max(initial=0) <= 1
    t = live & touched
    np.testing.assert_allclose(b[t], b_ref[t], rtol=RTOL, atol=0)
    print("touched bodies:", int(t.sum()), "max ulps:", int(_ulps(b[t], b_ref[t]).max(initial=0)))


@pytest.fixture()
def gpu(lib):
    from ncorpion_b200 import api

    def _init(n_max, params):
        api.init(n_max, params)
        return api

    yield _init
    api.finalize()


def test_brute_force_fragmentation_sweep(gpu):
    """Every outcome in one brute_force() sweep: fragments reuse freed slots
    and take part in the rest of the sweep."""
    g = golden("frag_bf")
    p = make_params(collision_bool=1, collision_type=3)
    api = gpu(16384, p)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    n = api.collide_brute()
    ev = api.events()
    assert n == len(g["events"]) and np.array_equal(ev, g["events"])
    assert np.array_equal(api.fragment_counts(), g["counts"])
    b, ex, cm = api.download(16384)
    assert b.shape[0] - 1 == int(g["out_largest_id"])
    w = oracle.PortWorld(16384, p)
    w.set_fragmentation()
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]))
    w.lib.orc_w_brute_force()
    b_ref, ex_ref, cm_ref = w.get_state()
    assert np.array_equal(_digest(b_ref), g["out_digest"])
    assert_close_state(b, ex, b_ref, ex_ref, ev, len(g["bodies"]) - 1)
    np.testing.assert_allclose(cm, cm_ref, rtol=RTOL, atol=0)


def mesh_frag_params(name):
    g = golden(name)
    p = make_params(mesh_bool=1, brute_force_bool=0, collision_bool=1, collision_type=3, collision_cube_cells=256,
                    N_tilde=int(g["N_tilde"]), pq_min_max=[int(v) for v in g["pq"]])
    return g, p


def port_mesh(g, p):
    w = oracle.PortWorld(70000, p)
    w.set_fragmentation(int(g["N_tilde"]), tuple(int(v) for v in g["pq"]))
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    w.three_largest()
    w.lib.orc_w_mesh()
    return w


@pytest.mark.parametrize("name", ["frag_mesh15", "frag_mesh4"])
def test_mesh_fragmentation_pass(gpu, name):
    """mesh() with fragments appended past largest_id: events, counts and the
    ordered pairs[] with the tail pairs at their events' positions."""
    g, p = mesh_frag_params(name)
    api = gpu(70000, p)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    assert np.array_equal(api.three_largest(), g["three"])
    n_pairs, n_ev, tn = api.mesh(float(g["gam"]), True)
    ev = api.events()
    assert np.array_equal(ev, g["events"])
    assert np.array_equal(api.fragment_counts(), g["counts"])
    pairs = api.pairs()
    assert n_pairs == len(pairs) == int(g["n_pairs"])
    assert np.array_equal(_digest(pairs), g["pairs_digest"])
    b, ex, cm = api.download(70000)
    assert b.shape[0] - 1 == int(g["out_largest_id"])
    w = port_mesh(g, p)
    assert np.array_equal(w.pairs(), pairs)
    b_ref, ex_ref, cm_ref = w.get_state()
    assert_close_state(b, ex, b_ref, ex_ref, ev, len(g["bodies"]) - 1)
    np.testing.assert_allclose(cm, cm_ref, rtol=RTOL, atol=0)


@pytest.mark.parametrize("name", ["frag_mesh15", "frag_mesh4"])
def test_mesh_gravity_after_fragmentation(gpu, name):
    """The kick after the pass: mesh gravity over pairs[] (fragments' tail
    pairs included) and the three largest bodies."""
    g, p = mesh_frag_params(name)
    api = gpu(70000, p)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    api.three_largest()
    api.mesh(float(g["gam"]), True)
    b0, _, _ = api.download(70000)
    api.kick()
    b1, ex1, _ = api.download(70000)
    w = port_mesh(g, p)
    r0, _, _ = w.get_state()
    w.lib.orc_w_kick_mesh()
    r1, ex_ref, _ = w.get_state()
    live = ex_ref == 1
    dv = (b1[:, 3:6] - b0[:, 3:6])[live]
    dv_ref = (r1[:, 3:6] - r0[:, 3:6])[live]
    scale = np.abs(dv_ref).max(axis=1, keepdims=True)
    err = np.abs(dv - dv_ref) / scale
    print("kick max relative difference:", float(err.max()))
    assert err.max() <= 1e-10


def test_mesh_fragmentation_steps(gpu):
    """Three iterations of the mesh integrator loop with fragmentation (the
    crowded ring, N_tilde 4), gamma updated on the host as the reference does."""
    from ncorpion_b200 import api as A
    g, p = mesh_frag_params("frag_mesh4")
    api = gpu(70000, p)
    api.upload(g["bodies"], g["exists"], g["cm"])
    dt = 2e-3
    api.set_timestep(dt)
    w = oracle.PortWorld(70000, p)
    w.set_fragmentation(int(g["N_tilde"]), tuple(int(v) for v in g["pq"]))
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=dt, gam=0.01)
    gam_g = gam_w = 0.01
    gmin = 4.4 / 256
    for _ in range(3):
        hm, tn = api.step_mesh(gam_g)
        gam_g = A.update_gamma(gam_g, tn, hm, 16.0, gmin)
        w.lib.orc_w_set_gam(C.c_double(gam_w))
        tn_w = w.lib.orc_w_step_mesh()
        hm_w = int(w.get_state()[1].sum())
        gam_w = A.update_gamma(gam_w, tn_w, hm_w, 16.0, gmin)
        assert (hm, tn) == (hm_w, tn_w)
    assert np.array_equal(api.fragment_counts(), w.fragment_counts())
    bg, exg, cmg = api.download(70000)
    b_ref, ex_ref, cm_ref = w.get_state()
    assert bg.shape == b_ref.shape and np.array_equal(exg, ex_ref)
    live = ex_ref == 1
    np.testing.assert_allclose(bg[live], b_ref[live], rtol=1e-9, atol=0)
    np.testing.assert_allclose(cmg, cm_ref, rtol=1e-12, atol=0)
