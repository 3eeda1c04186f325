"""Regenerates the golden fixtures in tests/golden/ from the reference's own
code, compiled from source by oracle/ref_build.py (run that first, in a
checkout where the reference tree exists).

    python tests/golden/make_golden.py

Every fixture stores its inputs next to the reference's outputs, so the tests
never depend on regenerating the random disks bit for bit.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ncorpion_b200 import disks  # noqa: E402


def cm_state(seed):
    rng = np.random.default_rng(seed)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    cm[:6] = rng.normal(0, 1e-5, 6)
    return cm


def gravity_case(profile, n, seed, holes=()):
    b = disks.gravity_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    ex[list(holes)] = 0
    cm = cm_state(seed)
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm)
    acc, cma = ref.vector_field()
    return dict(bodies=b, exists=ex, cm=cm, acc=acc, cm_acc=cma)


def step_case(profile, n, seed, nsteps, dt, maker):
    b = maker(n, seed)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt)
    ref.lib.orc_events_reset()
    for _ in range(nsteps):
        ref.lib.orc_step_brute_force()
    b2, ex2, cm2, sc = ref.get_state()
    return dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), nsteps=np.int64(nsteps),
                out_bodies=b2, out_exists=ex2, out_cm=cm2, events=ref.events())


def main():
    out = {}
    out["grav_s05_n512"] = gravity_case("bf_grav_s05", 512, 11, holes=(3, 100, 511))
    out["grav_s0_n64"] = gravity_case("bf_grav_s0", 64, 12, holes=(0,))
    out["grav_s0_n2"] = gravity_case("bf_grav_s0", 2, 13)
    out["grav_s05_n3"] = gravity_case("bf_grav_s05", 3, 14)
    out["steps_s0_n256"] = step_case("bf_grav_s0", 256, 15, 5, 1e-3, lambda n, s: disks.gravity_disk(n, s))
    for k, v in out.items():
        np.savez_compressed(os.path.join(HERE, k + ".npz"), **v)
        print("wrote", k)


if __name__ == "__main__":
    main()
