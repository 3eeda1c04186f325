"""GPU: the brute-force-gravity + mesh-collision mode (``par_mesh_brute_gravity``,
the fragmenting-disk workload's mode).  The reference has no such mode, so the
oracle is the composition of its pieces in the order of the mesh driver's loop
(src/rk4.c:760-790): mesh() (src/collision.c:324-417) after the three-largest
reordering, drift (src/rk4.c:109-127), kick (src/rk4.c:68-106) with the
brute-force vector_field (src/physics.c:174-202) instead of mesh gravity, then
end_of_timestep (src/rk4.c:130-404).  The oracle port runs each piece; its
pieces are pinned to the reference by the golden fixtures.

Tolerances:
  exact gravity, mergers        events, pairs[], total_neighbours and state
                                bit-identical over two steps (merged radii 1 ulp);
  exact gravity, fragmentation  events, outcome counts and exists[] identical;
                                fields 1e-9 relative over two steps (CUDA's pow in
                                the model against libm's);
  mixed gravity                 one step: events, pairs[] and positions as in
                                the exact case; each body's velocity change
                                within 1e-6 of dt times its mutual acceleration
                                (central mass off), the mixed kernel's bar.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import make_params

pytestmark = pytest.mark.gpu

N_MAX = 70000
CELLS = 256
DT = 2e-3


def _ulps(a, b):
    a = np.ascontiguousarray(a, np.float64).view(np.int64)
    b = np.ascontiguousarray(b, np.float64).view(np.int64)
    return np.abs(a - b)


def hybrid_params(ctype, mode, **kw):
    from ncorpion_b200 import api as A
    base = dict(mesh_bool=1, brute_force_bool=0, collision_bool=1, collision_type=ctype, collision_cube_cells=CELLS,
                mesh_brute_gravity=1, gravity_mode=mode, softening_parameter=0.5)
    if ctype == A.COLLISION_FRAGMENTATION:
        base.update(N_tilde=4, pq_min_max=[0, 1, 0, 1])
    base.update(kw)
    return make_params(**base)


def port_world(p, b, ex, cm, gam):
    w = oracle.PortWorld(N_MAX, p)
    if p.collision_type == 3:
        w.set_fragmentation(4, (0, 1, 0, 1))
    w.set_state(b, ex, cm, dt=DT, gam=gam)
    return w


def port_step(w, gam, mid=None):
    """One iteration of the loop with brute-force gravity; returns
    (how_many_moonlets, total_neighbours, state after the drift)."""
    w.lib.orc_w_set_gam(C.c_double(gam))
    w.lib.orc_w_events_reset()
    w.lib.orc_w_mesh_reset()
    w.three_largest()
    w.lib.orc_w_mesh()
    w.lib.orc_w_drift()
    drifted = w.get_state() if mid is not None else None
    w.lib.orc_w_kick()
    tn = w.lib.orc_w_total_neighbours()
    hm = w.lib.orc_w_end_of_timestep()
    w.lib.orc_w_mesh_reset()
    return hm, tn, drifted


@pytest.fixture()
def gpu(lib):
    from ncorpion_b200 import api

    def _init(params):
        api.init(N_MAX, params)
        return api

    yield _init
    api.finalize()


def crowded_ring(seed):
    from ncorpion_b200 import disks
    b = disks.frag_test_disk(4000, seed=seed)
    ex = np.ones(len(b), np.int32)
    return b, ex, np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])


@pytest.mark.parametrize("ctype", [2, 3], ids=["merger", "fragmentation"])
def test_hybrid_steps_exact(gpu, ctype):
    from ncorpion_b200 import api as A
    b, ex, cm = crowded_ring(seed=3)
    p = hybrid_params(ctype, A.GRAVITY_EXACT)
    api = gpu(p)
    api.upload(b, ex, cm)
    api.set_timestep(DT)
    w = port_world(p, b, ex, cm, 0.01)
    gam_g = gam_w = 0.01
    gmin = 4.4 / CELLS
    n_events = 0
    for _ in range(2):
        hm, tn = api.step_mesh(gam_g)
        hm_w, tn_w, _ = port_step(w, gam_w)
        ev = api.events()
        assert np.array_equal(ev, w.events())
        n_events += len(ev)
        assert (hm, tn) == (hm_w, tn_w)
        gam_g = A.update_gamma(gam_g, tn, hm, 16.0, gmin)
        gam_w = A.update_gamma(gam_w, tn_w, hm_w, 16.0, gmin)
    assert n_events > 0
    bg, exg, cmg = api.download(N_MAX)
    b_ref, ex_ref, cm_ref = w.get_state()
    assert bg.shape == b_ref.shape and np.array_equal(exg, ex_ref)
    live = ex_ref == 1
    if ctype == 3:
        assert np.array_equal(api.fragment_counts(), w.fragment_counts())
        np.testing.assert_allclose(bg[live], b_ref[live], rtol=1e-9, atol=0)
        np.testing.assert_allclose(cmg, cm_ref, rtol=1e-12, atol=0)
    else:
        assert np.array_equal(bg[live][:, :7], b_ref[live][:, :7])
        assert _ulps(bg[live][:, 7], b_ref[live][:, 7]).max(initial=0) <= 1
        assert np.array_equal(cmg, cm_ref)


def test_hybrid_pairs_match_the_mesh_pass(gpu):
    """The hybrid step's collision search is the reference's mesh(): ordered
    pairs[] and total_neighbours of the pass equal the port's."""
    from ncorpion_b200 import api as A
    b, ex, cm = crowded_ring(seed=4)
    p = hybrid_params(2, A.GRAVITY_EXACT)
    api = gpu(p)
    api.upload(b, ex, cm)
    api.set_timestep(DT)
    api.three_largest()
    n_pairs, _, tn = api.mesh(0.01, True)
    w = port_world(p, b, ex, cm, 0.01)
    w.three_largest()
    w.lib.orc_w_mesh()
    assert np.array_equal(api.pairs(), w.pairs())
    assert tn == w.lib.orc_w_total_neighbours()
    assert np.array_equal(api.events(), w.events())


@pytest.mark.parametrize("ctype", [2, 3], ids=["merger", "fragmentation"])
def test_hybrid_step_mixed(gpu, port, ctype):
    from ncorpion_b200 import api as A
    b, ex, cm = crowded_ring(seed=5)
    p = hybrid_params(ctype, A.GRAVITY_MIXED, reduce_to_COM_bool=0)
    api = gpu(p)
    api.upload(b, ex, cm)
    api.set_timestep(DT)
    hm, tn = api.step_mesh(0.01)
    ev = api.events()
    pe = hybrid_params(ctype, A.GRAVITY_EXACT, reduce_to_COM_bool=0)
    w = port_world(pe, b, ex, cm, 0.01)
    hm_w, tn_w, (bd, exd, cmd) = port_step(w, 0.01, mid=True)
    assert np.array_equal(ev, w.events()) and len(ev) > 0
    assert (hm, tn) == (hm_w, tn_w)
    bg, exg, cmg = api.download(N_MAX)
    b_ref, ex_ref, cm_ref = w.get_state()
    assert np.array_equal(exg, ex_ref)
    live = ex_ref == 1
    touched = np.zeros(len(b_ref), bool)
    touched[ev[:, :2].ravel()] = True
    touched[len(b):] = True
    if ctype == 3:
        np.testing.assert_allclose(bg[live][:, :3], b_ref[live][:, :3], rtol=1e-11, atol=0)
    else:
        assert np.array_equal(bg[live][:, :3], b_ref[live][:, :3])
    # mutual acceleration of the drifted state, exact FP64 (central mass off)
    a_mut, _ = port.vector_field(bd, exd, cmd, make_params(softening_parameter=0.5, central_mass_bool=0))
    dv_err = np.linalg.norm(bg[:, 3:6] - b_ref[:, 3:6], axis=1)
    scale = DT * np.linalg.norm(a_mut, axis=1)
    ok = live & (~touched if ctype == 3 else live)
    rel = dv_err[ok] / scale[ok]
    print(f"velocity change vs dt * mutual acceleration: max {rel.max():.3e}, median {np.median(rel):.3e}")
    assert rel.max() < 1e-6
