"""GPU parity of the mesh search (mesh / get_neighbours_mesh), the three
largest bodies' reordering, mesh gravity and the mesh integrator loop, through
the C ABI, against the oracle port (itself pinned to the reference by the
golden fixtures).

Tolerance: pairs[] (order included), total_neighbours, the event list, exists[]
and all body fields bit-identical, except the radius of merged bodies (1 ulp,
see test_collide_gpu.py).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import golden, make_params

pytestmark = pytest.mark.gpu


def _digest(a):
    import hashlib
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


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


def mesh_params(ctype=2, cells=256, **kw):
    base = dict(mesh_bool=1, brute_force_bool=0, collision_bool=1, collision_type=ctype, collision_parameter=1.5,
                collision_cube_cells=cells)
    base.update(kw)
    return make_params(**base)


@pytest.fixture()
def gpu(lib):
    from ncorpion_b200 import api

    def _init(n_max, params):
        api.init(n_max, params)
        return api

    yield _init
    api.finalize()


def collisional_disk(n, seed, holes=True):
    from ncorpion_b200 import disks
    rng = np.random.default_rng(seed)
    b = disks.mesh_disk(n, seed=seed)
    b[:, 7] = rng.uniform(2e-3, 6e-3, n)
    b[:, 6] = 4.0 / 3.0 * np.pi * 3.0 * b[:, 7] ** 3
    ex = np.ones(n, np.int32)
    if holes:
        ex[rng.choice(n, n // 50, replace=False)] = 0
    return b, ex


@pytest.mark.parametrize("name,ctype", [("mesh_merge", 2), ("mesh_inelastic", 1)])
def test_mesh_pass_matches_golden(gpu, name, ctype):
    g = golden(name)
    p = mesh_params(ctype)
    api = gpu(8192, p)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    assert np.array_equal(api.three_largest(), g["three"])
    n_pairs, n_ev, tn = api.mesh(float(g["gam"]), True)
    pairs = api.pairs()
    assert n_pairs == int(g["n_pairs"]) == len(pairs)
    assert tn == int(g["total_neighbours"])
    assert np.array_equal(pairs[:256], g["pairs_head"])
    assert np.array_equal(_digest(pairs), g["pairs_digest"])
    assert np.array_equal(api.events(), g["events"])
    b, ex, cm = api.download(8192)
    w = oracle.PortWorld(8192, p)
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    w.three_largest()
    w.lib.orc_w_mesh()
    b_ref, ex_ref, _ = w.get_state()
    assert_state_equal(b, ex, b_ref, ex_ref)


@pytest.mark.parametrize("gam,ctype,one_only", [(0.01, 2, 0), (0.012, 0, 0), (0.02, 2, 1), (0.03, 1, 1)])
def test_mesh_pass_random(gpu, gam, ctype, one_only):
    """Small cubes (gam * 256 < disk size): bodies outside the cube are never
    searched, and cells at the cube's x/y edges alias into the next row."""
    b, ex = collisional_disk(5000, seed=int(gam * 1e4) + ctype)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    p = mesh_params(ctype, one_collision_only_bool=one_only)
    api = gpu(8192, p)
    api.upload(b, ex, cm)
    api.set_timestep(5e-4)
    idx = api.three_largest()
    n_pairs, n_ev, tn = api.mesh(gam, True)
    w = oracle.PortWorld(8192, p)
    w.set_state(b, ex, cm, dt=5e-4, gam=gam)
    assert np.array_equal(idx, w.three_largest())
    w.lib.orc_w_mesh()
    assert np.array_equal(api.pairs(), w.pairs())
    assert tn == w.lib.orc_w_total_neighbours()
    assert np.array_equal(api.events(), w.events())
    bg, exg, _ = api.download(8192)
    b_ref, ex_ref, _ = w.get_state()
    assert_state_equal(bg, exg, b_ref, ex_ref)


def test_get_neighbours_mesh_and_kick(gpu):
    """get_neighbours_mesh (every body, no predicate) then the mesh-gravity
    kick: velocities bit-identical to the reference's vector_field mesh branch."""
    b, ex = collisional_disk(6000, seed=77)
    b[:, 7] = 1e-4
    cm = np.array([1e-6, 0, 0, 0, 0, 0, 1.0, 1.0])
    for soft in (0.0, 0.5):
        p = mesh_params(2, collision_bool=0, softening_parameter=soft)
        api = gpu(8192, p)
        api.upload(b, ex, cm)
        api.set_timestep(5e-4)
        api.three_largest()
        n_pairs, _, tn = api.mesh(0.02, False)
        api.kick()
        bg, exg, cmg = api.download(8192)
        pg = api.pairs()
        api.finalize()
        w = oracle.PortWorld(8192, p)
        w.set_state(b, ex, cm, dt=5e-4, gam=0.02)
        w.three_largest()
        w.lib.orc_w_get_neighbours_mesh()
        assert np.array_equal(pg, w.pairs())
        w.lib.orc_w_kick_mesh()
        b_ref, ex_ref, cm_ref = w.get_state()
        assert np.array_equal(bg, b_ref) and np.array_equal(cmg, cm_ref)


def test_mesh_steps_with_gamma_updates(gpu):
    """Six iterations of the mesh integrator loop with collisions (mergers),
    the host updating gamma from total_neighbours as the reference does."""
    from ncorpion_b200 import api as A
    b, ex = collisional_disk(5000, seed=5)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    p = mesh_params(2)
    api = gpu(8192, p)
    api.upload(b, ex, cm)
    api.set_timestep(5e-4)
    w = oracle.PortWorld(8192, p)
    w.set_state(b, ex, cm, dt=5e-4, gam=0.03)
    gam_g = gam_w = 0.03
    gmin = 4.4 / 256
    for _ in range(6):
        hm, tn = api.step_mesh(gam_g)
        gam_g = A.update_gamma(gam_g, tn, hm, 16.0, gmin)
        w.lib.orc_w_set_gam(C.c_double(gam_w))
        tn_w = w.lib.orc_w_step_mesh()
        hm_w = int(w.get_state()[1].sum())
        gam_w = A.update_gamma(gam_w, tn_w, hm_w, 16.0, gmin)
        assert (hm, tn) == (hm_w, tn_w)
        assert gam_g == gam_w
    bg, exg, cmg = api.download(8192)
    b_ref, ex_ref, cm_ref = w.get_state()
    assert_state_equal(bg, exg, b_ref, ex_ref)
    assert np.array_equal(cmg, cm_ref)


@pytest.mark.parametrize("name,ctype", [("mesh_big_merge", 2), ("mesh_big_inelastic", 1), ("mesh_big_frag", 3)])
def test_mesh_pass_big_bodies(gpu, name, ctype):
    """Bodies larger than the mesh size (src/collision.c:380-410), three of
    them past slot 2: their visits list every smaller body and every later big
    one, collisions with them are resolved at their turn, and the bodies after
    a visit are queried from their state at their own turn.  The fixtures also
    hold bodies that collide twice in one pass (merged into, then merged away).
    Then the kick: mesh gravity over pairs[] with the big bodies' pairs."""
    g = golden(name)
    p = mesh_params(ctype)
    api = gpu(16384, p)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    assert np.array_equal(api.three_largest(), g["three"])
    n_pairs, n_ev, tn = api.mesh(float(g["gam"]), True)
    assert np.array_equal(api.events(), g["events"])
    pairs = api.pairs()
    assert n_pairs == int(g["n_pairs"]) == len(pairs)
    assert np.array_equal(_digest(pairs), g["pairs_digest"])
    assert tn == int(g["total_neighbours"])
    b, ex, cm = api.download(16384)
    assert b.shape[0] - 1 == int(g["out_largest_id"])
    w = oracle.PortWorld(16384, p)
    if ctype == 3:
        w.set_fragmentation()
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    w.three_largest()
    w.lib.orc_w_mesh()
    b_ref, ex_ref, _ = w.get_state()
    assert np.array_equal(_digest(b_ref), g["out_digest"])
    live = ex_ref == 1
    if ctype == 3:
        assert np.array_equal(ex, ex_ref)
        np.testing.assert_allclose(b[live], b_ref[live], rtol=1e-11, atol=0)
    else:
        assert_state_equal(b, ex, b_ref, ex_ref)
    api.kick()
    w.lib.orc_w_kick_mesh()
    b1, _, _ = api.download(16384)
    r1, _, _ = w.get_state()
    if ctype == 3:
        np.testing.assert_allclose(b1[live][:, 3:6], r1[live][:, 3:6], rtol=1e-10, atol=0)
    else:
        assert np.array_equal(b1[live][:, 3:6], r1[live][:, 3:6])


def test_mesh_steps_big_bodies(gpu):
    """Four iterations of the mesh loop (mergers) with bodies larger than the
    mesh size, gamma updated on the host."""
    from ncorpion_b200 import api as A
    g = golden("mesh_big_merge")
    p = mesh_params(2)
    api = gpu(16384, p)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(5e-4)
    w = oracle.PortWorld(16384, p)
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=5e-4, gam=0.01)
    gam_g = gam_w = 0.01
    gmin = 4.4 / 256
    for _ in range(4):
        hm, tn = api.step_mesh(gam_g)
        gam_g = A.update_gamma(gam_g, tn, hm, 16.0, gmin)
        w.lib.orc_w_set_gam(C.c_double(gam_w))
        tn_w = w.lib.orc_w_step_mesh()
        hm_w = int(w.get_state()[1].sum())
        gam_w = A.update_gamma(gam_w, tn_w, hm_w, 16.0, gmin)
        assert (hm, tn) == (hm_w, tn_w)
    bg, exg, cmg = api.download(16384)
    b_ref, ex_ref, cm_ref = w.get_state()
    assert_state_equal(bg, exg, b_ref, ex_ref)
    assert np.array_equal(cmg, cm_ref)


@pytest.mark.parametrize("case", ["small_bodies", "big_bodies"])
def test_mesh_steps_fast_mode_match_exact(gpu, case):
    """The fast gravity modes' mesh steps against the exact mode's: the same
    pass (pairs[] and events), positions bit-identical after the first step,
    velocities within 1e-12 relative over three steps.  Without bodies larger
    than the mesh size the fast modes take the order-free pair sums
    (k_mesh_grav_fast); with them, the exact kernel's walk with parallel sums
    for CM_acc and bodies 0..2."""
    from ncorpion_b200 import api as A
    if case == "small_bodies":
        b, ex = collisional_disk(5000, seed=8)
        cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
        gam = 0.03
    else:
        g = golden("mesh_big_merge")
        b, ex, cm = g["bodies"], g["exists"], g["cm"]
        gam = 0.01
    out = {}
    for mode in (A.GRAVITY_EXACT, A.GRAVITY_MIXED, A.GRAVITY_FP64):
        api = gpu(16384, mesh_params(2, gravity_mode=mode))
        api.upload(b, ex, cm)
        api.set_timestep(5e-4)
        g_ = gam
        steps = []
        for s in range(3):
            hm, tn = api.step_mesh(g_)
            ev = api.events()
            st = api.download(16384)
            steps.append((hm, tn, ev, st))
            g_ = A.update_gamma(g_, tn, hm, 16.0, 4.4 / 256)
        out[mode] = steps
        api.finalize()
    ref = out[A.GRAVITY_EXACT]
    assert sum(len(s[2]) for s in ref) > 0
    for mode in (A.GRAVITY_MIXED, A.GRAVITY_FP64):
        for s, (hm, tn, ev, (bf, exf, cmf)) in enumerate(out[mode]):
            hm_r, tn_r, ev_r, (br, exr, cmr) = ref[s]
            assert (hm, tn) == (hm_r, tn_r) and np.array_equal(ev, ev_r)
            assert np.array_equal(exf, exr)
            live = exr == 1
            if s == 0:
                assert np.array_equal(bf[live][:, :3], br[live][:, :3])
            np.testing.assert_allclose(bf[live], br[live], rtol=1e-12, atol=0)
            np.testing.assert_allclose(cmf, cmr, rtol=1e-12, atol=1e-18)
