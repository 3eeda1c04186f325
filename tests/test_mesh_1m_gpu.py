"""GPU: the mesh workload at full size, N = 1,048,576, against the reference's
own mesh() and integrator loop compiled from its sources (oracle profile
``mesh_merge_1m``: 1024 cells per side, collision_cube_min 4.4, instant
mergers, 8.6 GB host hash table).

* One mesh() pass (src/collision.c:324-417) after the three-largest reordering
  (src/structure.c:914-1063): the ordered pairs[] (16.4M entries at the initial mesh size, compared
  whole and as a SHA-256 digest), total_neighbours, the ordered event list and
  the state are identical.
* The rest of that integrator iteration (drift, kick with mesh gravity,
  end_of_timestep) and two more whole iterations (src/rk4.c:760-790) in the
  exact gravity mode, gamma updated on the host as src/rk4.c:367-372 does:
  (how_many_moonlets, total_neighbours), gamma and the state identical at each
  step.

Tolerance: bit-identical, except merged radii (1 ulp: the correctly rounded
cube root against glibc's pow).
"""
import ctypes as C
import hashlib

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

N = 1 << 20
CELLS = 1024
DT = 5e-4
PROFILE = "mesh_merge_1m"


def _ulps(a, b):
    a = np.ascontiguousarray(a, np.float64).view(np.int64)
    b = np.ascontiguousarray(b, np.float64).view(np.int64)
    return np.abs(a - b)


def _assert_state(b, ex, cm, b_ref, ex_ref, cm_ref):
    assert b.shape == b_ref.shape
    assert np.array_equal(ex, ex_ref)
    live = ex_ref == 1
    assert np.array_equal(b[live][:, :7], b_ref[live][:, :7])
    assert _ulps(b[live][:, 7], b_ref[live][:, 7]).max(initial=0) <= 1
    assert np.array_equal(cm, cm_ref)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def ref():
    if not oracle.ref_available(PROFILE):
        pytest.skip(f"reference profile {PROFILE} not built (oracle/ref_build.py)")
    return oracle.Ref(PROFILE)


def test_mesh_pass_and_steps_at_one_million(lib, ref):
    from ncorpion_b200 import api, disks
    b0 = disks.mesh_disk(N, seed=0)
    ex0 = np.ones(N, np.int32)
    cm0 = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    gmin = 4.4 / CELLS
    gam = api.initial_gamma(N, CELLS, 0.5, 2.0, 0.015, 16.0, 4.4)
    p = api.default_params(G=1.0, softening_parameter=0.0, collision_bool=1, brute_force_bool=0, mesh_bool=1,
                           collision_type=api.COLLISION_MERGER, collision_cube_cells=CELLS,
                           how_many_neighbours=16.0, collision_cube_min=4.4, gravity_mode=api.GRAVITY_EXACT,
                           disruption_threshold=0.1, high_dumping_threshold=100.0)
    n_max = ref.n_max
    api.init(n_max, p)
    try:
        api.upload(b0, ex0, cm0)
        api.set_timestep(DT)
        ref.lib.orc_mesh_reset()
        ref.lib.orc_events_reset()
        ref.set_state(b0, ex0, cm0, dt=DT, gam=gam)

        # one mesh() pass
        three = api.three_largest()
        three_ref = np.zeros(3, np.int32)
        ref.lib.orc_three_largest(three_ref.ctypes.data_as(C.c_void_p))
        assert np.array_equal(three, three_ref)
        n_pairs, n_ev, tn = api.mesh(gam, True)
        ref.lib.orc_mesh()
        pairs, pairs_ref = api.pairs(), ref.pairs()
        print(f"pairs {len(pairs_ref)}, events {len(ref.events())}, total_neighbours {tn}")
        assert n_pairs == len(pairs) == len(pairs_ref) > 1_000_000
        assert _sha(pairs) == _sha(pairs_ref)
        assert np.array_equal(pairs, pairs_ref)
        assert tn == ref.lib.orc_total_neighbours()
        ev, ev_ref = api.events(), ref.events()
        assert len(ev_ref) > 0
        assert np.array_equal(ev, ev_ref)
        b, ex, cm = api.download(n_max)
        b_ref, ex_ref, cm_ref, _ = ref.get_state()
        _assert_state(b, ex, cm, b_ref, ex_ref, cm_ref)

        # the rest of the iteration: drift, kick (mesh gravity over pairs[]), end_of_timestep
        api.drift()
        api.kick()
        hm = api.end_of_timestep()
        ref.lib.orc_drift()
        ref.lib.orc_kick()
        ref.lib.orc_end_of_timestep()
        b, ex, cm = api.download(n_max)
        b_ref, ex_ref, cm_ref, sc = ref.get_state()
        assert hm == int(sc[2])
        _assert_state(b, ex, cm, b_ref, ex_ref, cm_ref)
        gam = api.update_gamma(gam, tn, hm, 16.0, gmin)
        assert gam == sc[1]

        # two more iterations of the loop
        for _ in range(2):
            ref.lib.orc_events_reset()
            hm, tn = api.step_mesh(gam)
            gam = api.update_gamma(gam, tn, hm, 16.0, gmin)
            ref.lib.orc_step_mesh()
            b, ex, cm = api.download(n_max)
            b_ref, ex_ref, cm_ref, sc = ref.get_state()
            assert hm == int(sc[2])
            assert gam == sc[1]
            assert np.array_equal(api.events(), ref.events())
            _assert_state(b, ex, cm, b_ref, ex_ref, cm_ref)
    finally:
        api.finalize()
