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
