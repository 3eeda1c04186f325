import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="session")
def port():
    import oracle
    return oracle.Port()


@pytest.fixture(scope="session")
def lib():
    from ncorpion_b200 import api, build
    build.build()
    return api.load()


def make_params(**kw):
    from ncorpion_b200 import api
    p = api.Params()
    # reference defaults for the path, as ncgpu_default_params sets them
    p.G = 1.0
    p.softening_parameter = 0.0
    p.central_mass_bool = 1
    p.mutual_bool = 1
    p.collision_bool = 0
    p.brute_force_bool = 1
    p.mesh_bool = 0
    p.collision_type = 2
    p.collision_parameter = 2.0
    p.one_collision_only_bool = 0
    p.collision_cube_cells = 1024
    p.how_many_neighbours = 16.0
    p.collision_cube_min = 80.0
    p.switch_to_brute_force = 110
    p.gravity_mode = 0
    p.near_theta = 0.15
    p.disruption_threshold = 0.1
    p.high_dumping_threshold = 100.0
    p.reduce_to_COM_bool = 1
    p.N_tilde = 15
    p.pq_min_max[:] = [-1, 3, -1, 1]
    p.mu_parameter = 0.55
    p.nu_parameter = 0.4
    p.C1_parameter = 1.5
    p.k_parameter = 0.2
    p.merging_threshold = 0.0002
    p.fragment_threshold = 1.5e-8
    p.mesh_brute_gravity = 0
    p.J2_bool = 0
    p.J2 = 0.0
    p.R_unit = 1.0
    p.sideral_omega = 2.0 * math.pi / 3.556721809
    p.central_tides_bool = 0
    p.k2 = 1.5
    p.Delta_t = 0.0015807
    p.dimensionless_moi = 0.3307
    for k, v in kw.items():
        if k == "pq_min_max":
            p.pq_min_max[:] = list(v)
            continue
        setattr(p, k, v)
    return p


def elliptic_cases(n=3000, seed=0, cm_at_rest=False):
    """Bodies for cart2ell (src/structure.c:172-284) with every branch of it:
    a disk of elliptic orbits (retrograde ones at small inclinations from 180
    degrees, where its two estimates of (k, h) part and it prints its warning),
    hyperbolic orbits (the atanh / sinh branch), a body on the central body
    (R = 0), one at rest relative to it (V2 = 0), a radial orbit (zero angular
    momentum: NaN elements), a parabolic orbit (2 mu = R V2: a = inf) and an
    exactly retrograde planar one (0 / 0).  The special bodies sit at dyadic
    offsets from the central body, so that cart2ell's subtractions are exact.
    Returns (bodies, exists, cm): G = 1, central mass 1, body masses 1e-9 (0
    for the parabolic and the planar retrograde bodies); the central body moves
    off the origin unless cm_at_rest."""
    from ncorpion_b200 import disks
    rng = np.random.default_rng(seed)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]) if cm_at_rest else \
        np.array([2.0 ** -10, -2.0 ** -11, 2.0 ** -12, 2.0 ** -9, 2.0 ** -10, -2.0 ** -11, 1.0, 1.0])
    b = disks.gravity_disk(n, seed=seed)
    b[:, :6] += cm[:6]
    b[:, 6] = 1e-9
    k = n // 50
    hyp = rng.choice(np.arange(40, n), k, replace=False)
    b[hyp, 3:6] = cm[3:6] + (b[hyp, 3:6] - cm[3:6]) * rng.uniform(1.5, 3.0, (k, 1))
    special = [
        ([0.0, 0.0, 0.0], [0.0, 0.0, 0.0], 1e-9),            # on the central body
        ([0.5, -0.25, 0.0], [0.0, 0.0, 0.0], 1e-9),          # at rest relative to it
        ([0.5, 0.25, 0.125], [0.25, 0.125, 0.0625], 1e-9),   # radial
        ([2.0, 0.0, 0.0], [0.0, 1.0, 0.0], 0.0),             # parabolic (mu = 1)
        ([1.0, 0.0, 0.0], [0.0, -1.0, 0.0], 0.0),            # retrograde, planar
    ]
    # retrograde at inclinations 1e-2 .. 1e-7 from 180 degrees, eccentric
    for q, dz in enumerate(10.0 ** -np.arange(2, 8)):
        for e in (0.0, 0.25, 0.5):
            special.append(([1.0 + 0.125 * q, 0.0, 0.0], [0.0, -(1.0 + e) ** 0.5, dz], 1e-9))
    for s_, (r, v, m) in enumerate(special):
        b[s_, :3] = cm[:3] + np.array(r)
        b[s_, 3:6] = cm[3:6] + np.array(v)
        b[s_, 6] = m
    ex = np.ones(n, np.int32)
    ex[rng.choice(np.arange(40, n), n // 40, replace=False)] = 0
    return b, ex, cm
