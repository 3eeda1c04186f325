"""CPU: the C restatement of the hot path (oracle/ncorpion_oracle.c) against
golden vectors produced by the reference's own code, and, where the
reference was compiled here (oracle/_ref), against it directly."""
import numpy as np
import pytest

import oracle
from conftest import golden, make_params

GRAV_CASES = [("grav_s05_n512", 0.5), ("grav_s0_n64", 0.0), ("grav_s0_n2", 0.0), ("grav_s05_n3", 0.5)]


@pytest.mark.parametrize("name,soft", GRAV_CASES)
def test_port_vector_field_matches_golden(port, name, soft):
    g = golden(name)
    p = make_params(softening_parameter=soft)
    acc, cma = port.vector_field(g["bodies"], g["exists"], g["cm"], p)
    assert np.array_equal(acc, g["acc"]), "port accelerations differ from the reference's bits"
    assert np.array_equal(cma, g["cm_acc"])


def test_port_steps_match_golden(port):
    """kick / drift loop of the brute-force driver (no collisions), 5 steps."""
    g = golden("steps_s0_n256")
    p = make_params()
    b, cm, ex = g["bodies"].copy(), g["cm"].copy(), g["exists"]
    dt = float(g["dt"])
    for _ in range(int(g["nsteps"])):
        b, cm = port.kick(b, ex, cm, dt, p)
        b, cm = port.drift(b, ex, cm, dt, p)
    assert np.array_equal(b, g["out_bodies"])
    assert np.array_equal(cm, g["out_cm"])


@pytest.mark.skipif(not oracle.ref_available("bf_grav_s05"), reason="reference not compiled here")
def test_port_vs_reference_random_holes(port):
    from ncorpion_b200 import disks
    rng = np.random.default_rng(7)
    for n in (5, 130, 1000):
        b = disks.gravity_disk(n, seed=int(rng.integers(1 << 30)))
        ex = (rng.random(n) > 0.1).astype(np.int32)
        cm = np.array([1e-5, -1e-5, 0, 0, 0, 0, 1.0, 1.0])
        ref = oracle.Ref("bf_grav_s05")
        ref.set_state(b, ex, cm)
        a_ref, c_ref = ref.vector_field()
        a, c = port.vector_field(b, ex, cm, make_params(softening_parameter=0.5))
        assert np.array_equal(a, a_ref) and np.array_equal(c, c_ref)


def _digest(a):
    import hashlib
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


@pytest.mark.parametrize("name,ctype", [("bf_sweep_merge", 2), ("bf_sweep_elastic", 0), ("bf_sweep_inelastic", 1)])
def test_port_brute_force_sweep_matches_golden(name, ctype):
    g = golden(name)
    w = oracle.PortWorld(4096, make_params(collision_bool=1, collision_type=ctype, collision_parameter=1.5))
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]))
    w.lib.orc_w_brute_force()
    b, ex, cm = w.get_state()
    assert np.array_equal(w.events(), g["events"])
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])


def test_port_brute_force_run_matches_golden():
    g = golden("bf_run_merge")
    w = oracle.PortWorld(4096, make_params(collision_bool=1, collision_type=2))
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]))
    for _ in range(int(g["nsteps"])):
        w.lib.orc_w_step_brute_force()
    b, ex, cm = w.get_state()
    assert np.array_equal(w.events(), g["events"])
    assert np.array_equal(_digest(b), g["out_digest"])
    assert np.array_equal(cm, g["out_cm"])


@pytest.mark.parametrize("name,ctype", [("mesh_merge", 2), ("mesh_inelastic", 1)])
def test_port_mesh_matches_golden(name, ctype):
    g = golden(name)
    p = make_params(mesh_bool=1, brute_force_bool=0, collision_bool=1, collision_type=ctype,
                    collision_parameter=1.5, collision_cube_cells=256)
    w = oracle.PortWorld(70000, p)
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    assert np.array_equal(w.three_largest(), g["three"])
    w.lib.orc_w_mesh()
    pairs = w.pairs()
    assert len(pairs) == int(g["n_pairs"])
    assert np.array_equal(pairs[:256], g["pairs_head"])
    assert np.array_equal(_digest(pairs), g["pairs_digest"])
    assert w.lib.orc_w_total_neighbours() == int(g["total_neighbours"])
    assert np.array_equal(w.events(), g["events"])
    b, ex, cm = w.get_state()
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])


@pytest.mark.skipif(not oracle.ref_available("bf_grav_s0"), reason="reference not compiled here")
def test_port_end_of_timestep_vs_reference():
    """Dumping into the central mass, removal beyond the outer threshold with
    the barycentre reduction, and tidy_up, against the reference's own
    end_of_timestep (thresholds 0.1 and 100 in that profile)."""
    import ctypes
    from ncorpion_b200 import disks
    b = disks.gravity_disk(1000, seed=9)
    b[10:40, :3] *= 0.05
    b[100:250, :3] *= 200.0
    ex = np.ones(1000, np.int32)
    ex[500:510] = 0
    cm = np.array([1e-4, 0, 0, 0, 1e-5, 0, 1.0, 1.0])
    ref = oracle.Ref("bf_grav_s0")
    ref.set_state(b, ex, cm)
    ref.lib.orc_end_of_timestep()
    rb, rex, rcm, sc = ref.get_state()
    w = oracle.PortWorld(2048, make_params())
    w.set_state(b, ex, cm)
    w.lib.orc_w_end_of_timestep.restype = ctypes.c_int
    hm = w.lib.orc_w_end_of_timestep()
    pb, pex, pcm = w.get_state()
    assert hm == int(sc[2]) == 810
    assert np.array_equal(rb, pb) and np.array_equal(rex, pex) and np.array_equal(rcm, pcm)


def test_port_fragmentation_sweep_matches_golden():
    """brute_force() with the fragmentation model (src/physics.c:710-1040):
    merger, super-catastrophic, partial and full outcomes in one sweep."""
    g = golden("frag_bf")
    w = oracle.PortWorld(16384, make_params(collision_bool=1, collision_type=3))
    w.set_fragmentation()
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]))
    w.lib.orc_w_brute_force()
    b, ex, cm = w.get_state()
    assert w.lib.orc_w_fragment_error() == 0
    assert np.array_equal(w.fragment_counts(), g["counts"]) and np.all(g["counts"] > 0)
    assert np.array_equal(w.events(), g["events"])
    assert b.shape[0] - 1 == int(g["out_largest_id"])
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])
    assert np.array_equal(cm, g["out_cm"])


@pytest.mark.parametrize("name", ["frag_mesh15", "frag_mesh4"])
def test_port_fragmentation_mesh_matches_golden(name):
    """mesh() with the fragmentation model: fragments appended past the sweep's
    largest_id, their mutual pairs in pairs[] (N_tilde 15 and the 2 x 2 lattice)."""
    g = golden(name)
    p = make_params(mesh_bool=1, brute_force_bool=0, collision_bool=1, collision_type=3, collision_cube_cells=256)
    w = oracle.PortWorld(70000, p)
    w.set_fragmentation(int(g["N_tilde"]), tuple(int(v) for v in g["pq"]))
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    assert np.array_equal(w.three_largest(), g["three"])
    w.lib.orc_w_mesh()
    pairs = w.pairs()
    assert w.lib.orc_w_fragment_error() == 0
    assert np.array_equal(w.fragment_counts(), g["counts"])
    assert np.array_equal(w.events(), g["events"])
    assert len(pairs) == int(g["n_pairs"]) and np.array_equal(_digest(pairs), g["pairs_digest"])
    b, ex, cm = w.get_state()
    assert b.shape[0] - 1 == int(g["out_largest_id"])
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])
    assert np.array_equal(cm, g["out_cm"])
    w.lib.orc_w_mesh_reset()


@pytest.mark.parametrize("name,ctype", [("mesh_big_merge", 2), ("mesh_big_inelastic", 1), ("mesh_big_frag", 3)])
def test_port_mesh_big_bodies_matches_golden(name, ctype):
    """The big-body branch of mesh() (src/collision.c:380-410)."""
    g = golden(name)
    p = make_params(mesh_bool=1, brute_force_bool=0, collision_bool=1, collision_type=ctype,
                    collision_parameter=1.5, collision_cube_cells=256)
    w = oracle.PortWorld(16384, p)
    if ctype == 3:
        w.set_fragmentation()
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    assert np.array_equal(w.three_largest(), g["three"])
    w.lib.orc_w_mesh()
    pairs = w.pairs()
    assert len(pairs) == int(g["n_pairs"]) and np.array_equal(_digest(pairs), g["pairs_digest"])
    assert w.lib.orc_w_total_neighbours() == int(g["total_neighbours"])
    assert np.array_equal(w.events(), g["events"])
    b, ex, cm = w.get_state()
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])
    w.lib.orc_w_mesh_reset()


# ---- the central body's J2 (src/physics.c:149-160) --------------------------

TEARTH_J2F = 25.0  # the sideral period of the fluid-body J2 profiles


def j2_params(name, **kw):
    """Port parameters of the J2 fixtures: a constant J2 (softening 0.5), or
    the fluid-body J2 (J2_value 0) of a central body with Tearth = 25."""
    if name == "grav_j2_n512":
        return make_params(softening_parameter=0.5, J2_bool=1, J2=0.0125, **kw)
    return make_params(J2_bool=1, J2=0.0, sideral_omega=2.0 * np.pi / TEARTH_J2F, **kw)


@pytest.mark.parametrize("name", ["grav_j2_n512", "grav_j2f_n300"])
def test_port_vector_field_j2_matches_golden(port, name):
    """Brute-force vector_field with the J2 term: accelerations and CM_acc,
    whose two terms per body (central, then J2) are added in that order."""
    g = golden(name)
    acc, cma = port.vector_field(g["bodies"], g["exists"], g["cm"], j2_params(name))
    assert np.array_equal(acc, g["acc"])
    assert np.array_equal(cma, g["cm_acc"])
    # the term is there: without it the accelerations differ
    acc0, _ = port.vector_field(g["bodies"], g["exists"], g["cm"], make_params(softening_parameter=0.5))
    assert not np.array_equal(acc0, g["acc"])


def test_port_mesh_steps_j2_matches_golden():
    """Four iterations of the mesh loop (mesh gravity, no collisions) with the
    fluid-body J2, bodies falling into the central mass on the way, so that J2
    follows the new mass (src/rk4.c:459-463)."""
    from ncorpion_b200 import api as A
    import ctypes as C
    g = golden("mesh_j2f_steps")
    p = j2_params("mesh_j2f_steps", mesh_bool=1, brute_force_bool=0, collision_cube_cells=256)
    w = oracle.PortWorld(16384, p)
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    gam = float(g["gam"])
    for s in range(int(g["nsteps"])):
        w.lib.orc_w_set_gam(C.c_double(gam))
        tn = w.lib.orc_w_step_mesh()
        gam = A.update_gamma(gam, tn, int(w.get_state()[1].sum()), 16.0, 4.4 / 256)
        assert gam == g["gams"][s]
    b, ex, cm = w.get_state()
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])
    assert np.array_equal(cm, g["out_cm"])
    assert cm[6] > g["cm"][6], "no body fell into the central mass"


@pytest.mark.skipif(not oracle.ref_available("bf_grav_j2f"), reason="reference not compiled here")
def test_port_vs_reference_j2_random_holes(port):
    from ncorpion_b200 import disks
    rng = np.random.default_rng(8)
    for n in (4, 129, 700):
        b = disks.gravity_disk(n, seed=int(rng.integers(1 << 30)))
        ex = (rng.random(n) > 0.1).astype(np.int32)
        cm = np.array([1e-5, -1e-5, 2e-6, 0, 0, 0, float(rng.uniform(0.8, 1.5)), 1.0])
        ref = oracle.Ref("bf_grav_j2f")
        ref.set_state(b, ex, cm)
        a_ref, c_ref = ref.vector_field()
        a, c = port.vector_field(b, ex, cm, j2_params("bf_grav_j2f"))
        assert np.array_equal(a, a_ref) and np.array_equal(c, c_ref)


# ---- tides raised on the central body (src/physics.c:496-542) --------------

TIDES = dict(central_tides_bool=1, Delta_t=1.0)


@pytest.mark.parametrize("name", ["tides_bf_steps", "tides_j2f_bf_steps"])
def test_port_tides_bf_steps_match_golden(name):
    """Six iterations of the brute-force loop with tides (and, in the second
    fixture, the fluid-body J2 that follows the changing rotation):
    SideralOmega after every step and the final state."""
    g = golden(name)
    if name == "tides_bf_steps":
        p = make_params(softening_parameter=0.5, **TIDES)
    else:
        p = make_params(J2_bool=1, J2=0.0, sideral_omega=2.0 * np.pi / TEARTH_J2F, **TIDES)
    w = oracle.PortWorld(4096, p)
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]))
    assert w.lib.orc_w_get_sideral_omega() == g["omegas"][0]
    for s in range(int(g["nsteps"])):
        w.lib.orc_w_step_brute_force()
        assert w.lib.orc_w_get_sideral_omega() == g["omegas"][s + 1]
    b, ex, cm = w.get_state()
    assert np.array_equal(b, g["out_bodies"]) and np.array_equal(ex, g["out_exists"])
    assert np.array_equal(cm, g["out_cm"])
    assert len(set(g["omegas"].tolist())) == len(g["omegas"]), "the rotation did not change"


def test_port_tides_mesh_steps_match_golden():
    from ncorpion_b200 import api as A
    import ctypes as C
    g = golden("tides_mesh_steps")
    p = make_params(J2_bool=1, J2=0.0, sideral_omega=2.0 * np.pi / TEARTH_J2F, mesh_bool=1, brute_force_bool=0,
                    collision_cube_cells=256, **TIDES)
    w = oracle.PortWorld(16384, p)
    w.set_state(g["bodies"], g["exists"], g["cm"], dt=float(g["dt"]), gam=float(g["gam"]))
    gam = float(g["gam"])
    for s in range(int(g["nsteps"])):
        w.lib.orc_w_set_gam(C.c_double(gam))
        tn = w.lib.orc_w_step_mesh()
        gam = A.update_gamma(gam, tn, int(w.get_state()[1].sum()), 16.0, 4.4 / 256)
        assert gam == g["gams"][s]
        assert w.lib.orc_w_get_sideral_omega() == g["omegas"][s + 1]
    b, ex, cm = w.get_state()
    assert np.array_equal(_digest(b), g["out_digest"]) and np.array_equal(_digest(ex), g["out_exists_digest"])
    assert np.array_equal(cm, g["out_cm"])


# ---- elliptic elements (cart2ell, src/structure.c:172-284) -----------------

@pytest.mark.parametrize("profile,at_rest", [("bf_grav_s05", False), ("bf_grav_s05", True), ("bf_grav_j2", False)])
def test_port_cart2ell_vs_reference(port, capfd, profile, at_rest):
    """The port's cart2ell against the reference's on every branch
    (conftest.elliptic_cases): the six elements bit for bit (NaNs with their
    signs: printf shows them), and the (k, h) warnings printed alike.  The J2
    profile holds a constant J2 of 0.0125, which corrects a on elliptic orbits."""
    if not oracle.ref_available(profile):
        pytest.skip("reference not compiled here")
    from conftest import elliptic_cases
    b, ex, cm = elliptic_cases(1500, seed=4, cm_at_rest=at_rest)
    j2 = 0.0125 if profile == "bf_grav_j2" else 0.0
    p = make_params(J2_bool=1, J2=j2) if j2 else make_params()
    ref = oracle.Ref(profile)
    mu = 1.0 * cm[6]
    live = np.flatnonzero(ex)
    capfd.readouterr()
    got = np.array([port.cart2ell(b[i], cm, mu + 1.0 * b[i, 6], p, j2)[0] for i in live])
    out_port = capfd.readouterr().out
    want = np.array([ref.cart2ell(b[i], cm, mu + 1.0 * b[i, 6], j2) for i in live])
    out_ref = capfd.readouterr().out
    assert np.array_equal(got.view(np.int64), want.view(np.int64))
    assert out_port == out_ref
    assert out_ref.count("Warning : Bad computation of (k,h)") >= 3
    assert got[0, 1] == 0.0 and got[1, 1] == 0.0      # R = 0, V2 = 0: lambda = 0
    assert np.isnan(got[2]).any() and np.isnan(got[4]).any()  # radial, planar retrograde
    assert got[3, 0] == np.inf                         # parabolic
    assert (got[:, 0] < 0).sum() >= 10                 # hyperbolic branch
