"""GPU parity of the central body's J2 term (src/physics.c:149-160) in every
gravity path, through the C ABI, against the reference's golden vectors and
the oracle port.

- exact brute-force gravity: accelerations and CM_acc bit-identical (CM_acc
  adds each body's central term, then its J2 term, in slot order);
- fp64 / mixed tiled gravity: total acceleration within 1e-12 / 1e-8
  relative, CM_acc within 1e-10 of its norm (the J2 term itself is FP64);
- mesh gravity: four mesh-loop steps with the fluid-body J2 (J2_value 0)
  whose central mass grows on the way, the state bit-identical to the
  reference run;
- the brute-force loop: kick / drift / end_of_timestep bit-identical to the
  port, with a constant J2;
- parameter checks: J2 without the central mass is refused (src/structure.c:1407).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import golden, make_params

pytestmark = pytest.mark.gpu

J2F = dict(J2_bool=1, J2=0.0, sideral_omega=2.0 * np.pi / 25.0)  # the fluid-body J2 profiles' Tearth = 25


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


GOLDEN = [("grav_j2_n512", dict(softening_parameter=0.5, J2_bool=1, J2=0.0125)), ("grav_j2f_n300", J2F)]


@pytest.mark.parametrize("name,kw", GOLDEN)
def test_exact_j2_matches_reference_golden(gpu, name, kw):
    g = golden(name)
    api = gpu(1024, **kw)
    acc, cma = api.vector_field(g["bodies"], g["exists"], g["cm"], mode="exact")
    assert np.array_equal(acc, g["acc"])
    assert np.array_equal(cma, g["cm_acc"])


@pytest.mark.parametrize("n", [1, 129, 2000])
@pytest.mark.parametrize("soft", [0.0, 0.5])
def test_exact_j2_matches_oracle(gpu, port, n, soft):
    from ncorpion_b200 import disks
    rng = np.random.default_rng(100 + n)
    b = disks.gravity_disk(n, seed=n + 7)
    ex = (rng.random(n) > 0.05).astype(np.int32)
    cm = np.array([2e-6, -1e-6, 3e-7, 0, 0, 0, float(rng.uniform(0.8, 1.4)), 1.0])
    api = gpu(4096, softening_parameter=soft, **J2F)
    acc, cma = api.vector_field(b, ex, cm, mode="exact")
    a_ref, c_ref = port.vector_field(b, ex, cm, make_params(softening_parameter=soft, **J2F))
    assert np.array_equal(acc, a_ref)
    assert np.array_equal(cma, c_ref)


@pytest.mark.parametrize("mode,tol", [("fp64", 1e-12), ("mixed", 1e-8)])
def test_tiled_j2_accuracy(gpu, port, mode, tol):
    from ncorpion_b200 import disks
    n = 6000
    b = disks.gravity_disk(n, seed=9)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.2, 1.0])
    kw = dict(softening_parameter=0.5, J2_bool=1, J2=0.0125)
    api = gpu(8192, **kw)
    acc, cma = api.vector_field(b, ex, cm, mode=mode)
    a_ref, c_ref = port.vector_field(b, ex, cm, make_params(**kw))
    rel = np.linalg.norm(acc - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
    assert rel.max() <= tol
    assert np.linalg.norm(cma - c_ref) <= 1e-10 * np.linalg.norm(c_ref)


def test_brute_force_loop_j2_bit_exact(gpu):
    """Eight iterations of the brute-force loop (kick, drift, end_of_timestep)
    with a constant J2, against the port."""
    from ncorpion_b200 import disks
    n = 700
    b = disks.gravity_disk(n, seed=21)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    kw = dict(softening_parameter=0.5, J2_bool=1, J2=0.0125)
    api = gpu(1024, **kw)
    api.upload(b, ex, cm)
    api.set_timestep(1e-3)
    w = oracle.PortWorld(1024, make_params(**kw))
    w.set_state(b, ex, cm, dt=1e-3)
    for _ in range(8):
        api.step_brute_force()
        w.lib.orc_w_step_brute_force()
    b2, ex2, cm2 = api.download(1024)
    b_ref, ex_ref, cm_ref = w.get_state()
    assert np.array_equal(b2, b_ref) and np.array_equal(ex2, ex_ref)
    assert np.array_equal(cm2, cm_ref)


def test_mesh_steps_j2_match_reference_golden(gpu):
    """The mesh loop without collisions (mesh gravity with the fluid-body J2):
    four steps, bodies dumped into the central mass on the way, the host
    updating gamma as the reference does; gamma after every step and the final
    state equal the reference run's."""
    from ncorpion_b200 import api as A
    g = golden("mesh_j2f_steps")
    api = gpu(16384, mesh_bool=1, brute_force_bool=0, collision_bool=0, collision_cube_cells=256, **J2F)
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    gam = float(g["gam"])
    for s in range(int(g["nsteps"])):
        hm, tn = api.step_mesh(gam)
        gam = A.update_gamma(gam, tn, hm, 16.0, 4.4 / 256)
        assert gam == g["gams"][s]
    b2, ex2, cm2 = api.download(16384)
    lid = int(g["out_largest_id"])
    assert np.array_equal(_digest(b2[:lid + 1]), g["out_digest"])
    assert np.array_equal(_digest(ex2[:lid + 1]), g["out_exists_digest"])
    assert np.array_equal(cm2, g["out_cm"])


def test_j2_needs_central_mass(lib):
    from ncorpion_b200 import api as A
    with pytest.raises(A.NcgpuError) as e:
        A.init(64, make_params(central_mass_bool=0, J2_bool=1, J2=0.01))
    assert e.value.status == A.E_ARG
    A.finalize()
