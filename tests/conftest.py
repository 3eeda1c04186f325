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
