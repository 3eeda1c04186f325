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


def digest(a):
    import hashlib
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def bf_sweep_case(profile, n, seed):
    """One brute_force() call from a disk whose close pairs collide at once."""
    b = disks.bf_collide_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=1e-3)
    ref.lib.orc_events_reset()
    ref.lib.orc_brute_force()
    b2, ex2, cm2, sc = ref.get_state()
    return dict(bodies=b, exists=ex, cm=cm, dt=np.float64(1e-3), events=ref.events(),
                out_digest=digest(b2), out_exists_digest=digest(ex2), out_cm=cm2)


def bf_run_case(profile, n, seed, nsteps):
    """nsteps iterations of the brute-force integrator loop with collisions."""
    b = disks.bf_collide_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=1e-3)
    ref.lib.orc_events_reset()
    for _ in range(nsteps):
        ref.lib.orc_step_brute_force()
    b2, ex2, cm2, sc = ref.get_state()
    return dict(bodies=b, exists=ex, cm=cm, dt=np.float64(1e-3), nsteps=np.int64(nsteps), events=ref.events(),
                out_digest=digest(b2), out_exists_digest=digest(ex2), out_cm=cm2,
                out_largest_id=np.int64(b2.shape[0] - 1))


def mesh_case(profile, n, seed, gam, dt):
    """three_largest + one mesh() call: ordered pairs[], events and state."""
    rng = np.random.default_rng(seed)
    b = disks.mesh_disk(n, seed=seed)
    b[:, 7] = rng.uniform(2e-3, 6e-3, n)
    b[:, 6] = 4.0 / 3.0 * np.pi * 3.0 * b[:, 7] ** 3
    ex = np.ones(n, np.int32)
    ex[rng.choice(n, n // 50, replace=False)] = 0
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt, gam=gam)
    ref.lib.orc_events_reset()
    idx = np.zeros(3, np.int32)
    ref.lib.orc_three_largest(idx.ctypes.data_as(oracle.P))
    ref.lib.orc_mesh()
    pairs = ref.pairs()
    b2, ex2, cm2, sc = ref.get_state()
    out = dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), gam=np.float64(gam), three=idx,
               events=ref.events(), n_pairs=np.int64(len(pairs)), pairs_digest=digest(pairs),
               pairs_head=pairs[:256].copy(), total_neighbours=np.int64(ref.lib.orc_total_neighbours()),
               out_digest=digest(b2), out_exists_digest=digest(ex2))
    ref.lib.orc_mesh_reset()
    return out


def frag_bf_case(profile, n, seed, dt):
    """One brute_force() sweep with the fragmentation model: events, outcome
    counts, state (appended fragments included) and central mass."""
    b = disks.frag_test_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt)
    ref.lib.orc_events_reset()
    ref.lib.orc_frag_counts_reset()
    ref.lib.orc_brute_force()
    b2, ex2, cm2, sc = ref.get_state()
    return dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), events=ref.events(),
                counts=ref.fragment_counts(), out_digest=digest(b2), out_exists_digest=digest(ex2), out_cm=cm2,
                out_largest_id=np.int64(b2.shape[0] - 1))


def frag_mesh_case(profile, n, seed, gam, dt, N_tilde, pq):
    """three_largest + one mesh() call with the fragmentation model."""
    b = disks.frag_test_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt, gam=gam)
    ref.lib.orc_events_reset()
    ref.lib.orc_frag_counts_reset()
    idx = np.zeros(3, np.int32)
    ref.lib.orc_three_largest(idx.ctypes.data_as(oracle.P))
    ref.lib.orc_mesh()
    pairs = ref.pairs()
    b2, ex2, cm2, sc = ref.get_state()
    out = dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), gam=np.float64(gam), three=idx,
               N_tilde=np.int64(N_tilde), pq=np.array(pq, np.int32), events=ref.events(),
               counts=ref.fragment_counts(), n_pairs=np.int64(len(pairs)), pairs_digest=digest(pairs),
               out_digest=digest(b2), out_exists_digest=digest(ex2), out_cm=cm2,
               out_largest_id=np.int64(b2.shape[0] - 1))
    ref.lib.orc_mesh_reset()
    return out


def big_disk(n, seed):
    """Mesh disk with six bodies larger than the mesh size (two at slots 1, 2,
    the others anywhere) among radii U[2e-3, 6e-3], 2% holes."""
    rng = np.random.default_rng(seed)
    b = disks.mesh_disk(n, seed=seed)
    b[:, 7] = rng.uniform(2e-3, 6e-3, n)
    big = rng.choice(n, 6, replace=False)
    big[:2] = [1, 2]
    b[big, 7] = rng.uniform(0.012, 0.03, len(big))
    b[:, 6] = 4.0 / 3.0 * np.pi * 3.0 * b[:, 7] ** 3
    ex = np.ones(n, np.int32)
    ex[rng.choice(n, n // 50, replace=False)] = 0
    ex[big] = 1
    return b, ex


def mesh_big_case(profile, n, seed, gam, dt):
    """three_largest + one mesh() call with bodies larger than the mesh size
    (the big-body branch, src/collision.c:380-410)."""
    b, ex = big_disk(n, seed)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt, gam=gam)
    ref.lib.orc_events_reset()
    ref.lib.orc_frag_counts_reset()
    idx = np.zeros(3, np.int32)
    ref.lib.orc_three_largest(idx.ctypes.data_as(oracle.P))
    ref.lib.orc_mesh()
    pairs = ref.pairs()
    b2, ex2, cm2, sc = ref.get_state()
    out = dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), gam=np.float64(gam), three=idx,
               events=ref.events(), counts=ref.fragment_counts(), n_pairs=np.int64(len(pairs)),
               pairs_digest=digest(pairs), total_neighbours=np.int64(ref.lib.orc_total_neighbours()),
               out_digest=digest(b2), out_exists_digest=digest(ex2), out_largest_id=np.int64(b2.shape[0] - 1))
    ref.lib.orc_mesh_reset()
    return out


def j2_gravity_case(profile, n, seed, mass, holes):
    """One vector_field with the J2 term; the central mass `mass` sets the
    fluid-body J2 when the profile's J2_value is 0."""
    b = disks.gravity_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    ex[list(holes)] = 0
    cm = cm_state(seed)
    cm[6] = mass
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm)
    acc, cma = ref.vector_field()
    return dict(bodies=b, exists=ex, cm=cm, acc=acc, cm_acc=cma)


def j2_mesh_steps_case(profile, n, seed, nsteps, gam, dt):
    """nsteps of the mesh integrator loop without collisions (mesh gravity
    with the fluid-body J2), four bodies placed inside the disruption
    threshold so that the central mass, and with it J2, changes.  The gamma
    the reference reaches after each step is stored for the replay."""
    rng = np.random.default_rng(seed)
    b = disks.mesh_disk(n, seed=seed)
    b[:, 7] = rng.uniform(2e-3, 6e-3, n)
    b[:, 6] = 4.0 / 3.0 * np.pi * 3.0 * b[:, 7] ** 3
    idx = rng.choice(n, 4, replace=False)
    ang = rng.uniform(0, 2 * np.pi, 4)
    b[idx, 0] = 0.05 * np.cos(ang)
    b[idx, 1] = 0.05 * np.sin(ang)
    b[idx, 2] = 0.001
    ex = np.ones(n, np.int32)
    ex[rng.choice(n, n // 50, replace=False)] = 0
    ex[idx] = 1
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt, gam=gam)
    gams = []
    for _ in range(nsteps):
        ref.lib.orc_step_mesh()
        gams.append(ref.get_state()[3][1])
    b2, ex2, cm2, sc = ref.get_state()
    return dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), gam=np.float64(gam), nsteps=np.int64(nsteps),
                gams=np.array(gams), out_digest=digest(b2), out_exists_digest=digest(ex2), out_cm=cm2,
                out_largest_id=np.int64(b2.shape[0] - 1))


def tides_bf_case(profile, n, seed, nsteps, dt):
    """nsteps of the brute-force loop (no collisions) with tides raised on the
    central body: the final state and SideralOmega after every step."""
    b = disks.gravity_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    ex[[3, n // 2]] = 0
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt)
    omegas = [ref.lib.orc_get_sideral_omega()]
    for _ in range(nsteps):
        ref.lib.orc_step_brute_force()
        omegas.append(ref.lib.orc_get_sideral_omega())
    b2, ex2, cm2, sc = ref.get_state()
    return dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), nsteps=np.int64(nsteps), omegas=np.array(omegas),
                out_bodies=b2, out_exists=ex2, out_cm=cm2)


def tides_mesh_case(profile, n, seed, nsteps, gam, dt):
    """nsteps of the mesh loop (no collisions) with tides and the fluid-body
    J2: gamma and SideralOmega after every step, the final state."""
    rng = np.random.default_rng(seed)
    b = disks.mesh_disk(n, seed=seed)
    b[:, 7] = rng.uniform(2e-3, 6e-3, n)
    b[:, 6] = 4.0 / 3.0 * np.pi * 3.0 * b[:, 7] ** 3
    ex = np.ones(n, np.int32)
    ex[rng.choice(n, n // 50, replace=False)] = 0
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm, dt=dt, gam=gam)
    gams, omegas = [], [ref.lib.orc_get_sideral_omega()]
    for _ in range(nsteps):
        ref.lib.orc_step_mesh()
        gams.append(ref.get_state()[3][1])
        omegas.append(ref.lib.orc_get_sideral_omega())
    b2, ex2, cm2, sc = ref.get_state()
    return dict(bodies=b, exists=ex, cm=cm, dt=np.float64(dt), gam=np.float64(gam), nsteps=np.int64(nsteps),
                gams=np.array(gams), omegas=np.array(omegas), out_digest=digest(b2), out_exists_digest=digest(ex2),
                out_cm=cm2, out_largest_id=np.int64(b2.shape[0] - 1))


OUTPUT_FILES = ["stat.txt", "collision.txt", "mass.txt", "radius.txt", "x.txt", "y.txt", "z.txt", "vx.txt",
                "vy.txt", "vz.txt", "readme.txt"]
ELLIPTIC_FILES = ["a.txt", "lambda.txt", "k.txt", "h.txt", "q.txt", "p.txt"]


def tree_case(profile, n, seed, holes=()):
    """falcON's field (src/ffm.c; the tree as the tree driver builds it before a
    kick, then vector_field) of one disk, with the exact brute-force field of
    the same state beside it."""
    b = disks.gravity_disk(n, seed=seed)
    ex = np.ones(n, np.int32)
    ex[list(holes)] = 0
    cm = cm_state(seed)
    ref = oracle.Ref(profile)
    ref.set_state(b, ex, cm)
    acc, cma, cells = ref.tree_field()
    exact = oracle.Ref("bf_grav_s0")
    exact.set_state(b, ex, cm)
    acc_x, cma_x = exact.vector_field()
    return dict(bodies=b, exists=ex, cm=cm, acc=acc, cm_acc=cma, cells=np.int64(cells), acc_exact=acc_x,
                cm_acc_exact=cma_x)


def filtered_stdout(text):
    """The program's console output without its wall-clock timing line."""
    return "\n".join(l for l in text.splitlines() if "integration took" not in l)


def program_run_case(profile, bodies, bodies_from=None, disk=None):
    """The whole reference program (oracle/_ref/<profile>/ncorpion) run on
    init.txt: digests of every output file and of the console output.  With
    bodies_from, the fixture names the fixture that holds the same bodies
    instead of storing them again; with disk = (generator, n, seed), a large
    input is stored as the recipe of ncorpion_b200.disks plus the digest of
    its init.txt (the test regenerates it and checks the digest first)."""
    import subprocess
    import tempfile
    d = tempfile.mkdtemp(prefix="ncref_run_")
    disks.write_init_txt(os.path.join(d, "init.txt"), bodies)
    exe = os.path.join(ROOT, "oracle", "_ref", profile, "ncorpion")
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, check=True)
    if disk is not None:
        out = dict(disk_generator=np.array(disk[0]), disk_n=np.int64(disk[1]), disk_seed=np.int64(disk[2]),
                   digest_init=digest(np.frombuffer(open(os.path.join(d, "init.txt"), "rb").read(), np.uint8)))
    elif bodies_from is not None:
        out = dict(bodies_from=np.array(bodies_from))
    else:
        out = dict(bodies=bodies)
    files = [f for f in OUTPUT_FILES + ELLIPTIC_FILES if os.path.exists(os.path.join(d, f))]
    if files != OUTPUT_FILES:
        out["files"] = np.array(files)
    for f in files:
        data = open(os.path.join(d, f), "rb").read()
        out["digest_" + f] = digest(np.frombuffer(data, np.uint8))
    out["digest_stdout"] = digest(np.frombuffer(filtered_stdout(r.stdout).encode(), np.uint8))
    out["collision_txt"] = np.frombuffer(open(os.path.join(d, "collision.txt"), "rb").read(), np.uint8)
    out["stat_txt"] = np.frombuffer(open(os.path.join(d, "stat.txt"), "rb").read(), np.uint8)
    return out


RESUME_FILES = ["init.txt", "resume.txt"]


def program_resume_case(profile, bodies, bodies_from):
    """The whole reference program run without output files and with
    resume_simulation_bool: digests of the files it writes at the end (the
    final state in init.txt, resume.txt) and of the console output."""
    import subprocess
    import tempfile
    d = tempfile.mkdtemp(prefix="ncref_run_")
    disks.write_init_txt(os.path.join(d, "init.txt"), bodies)
    exe = os.path.join(ROOT, "oracle", "_ref", profile, "ncorpion")
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, check=True)
    out = dict(bodies_from=np.array(bodies_from))
    for f in RESUME_FILES:
        data = open(os.path.join(d, f), "rb").read()
        out["digest_" + f] = digest(np.frombuffer(data, np.uint8))
    cols, radii = split_radius_column(open(os.path.join(d, "init.txt")).read())
    out["digest_init_without_radius"] = digest(np.frombuffer(cols.encode(), np.uint8))
    out["init_radius"] = radii
    out["digest_stdout"] = digest(np.frombuffer(filtered_stdout(r.stdout).encode(), np.uint8))
    return out


def split_radius_column(text):
    """init.txt as written by resume(): the text of its first seven columns and
    the eighth (the radius) parsed as doubles."""
    lines = text.splitlines()
    cols = "\n".join(" ".join(l.split()[:7]) for l in lines)
    radii = np.array([float(l.split()[7]) for l in lines])
    return cols, radii


def main(names=None):
    out = {}
    out["grav_s05_n512"] = lambda: gravity_case("bf_grav_s05", 512, 11, holes=(3, 100, 511))
    out["grav_s0_n64"] = lambda: gravity_case("bf_grav_s0", 64, 12, holes=(0,))
    out["grav_s0_n2"] = lambda: gravity_case("bf_grav_s0", 2, 13)
    out["grav_s05_n3"] = lambda: gravity_case("bf_grav_s05", 3, 14)
    out["steps_s0_n256"] = lambda: step_case("bf_grav_s0", 256, 15, 5, 1e-3, lambda n, s: disks.gravity_disk(n, s))
    out["bf_sweep_merge"] = lambda: bf_sweep_case("bf_merge", 2000, 0)
    out["bf_sweep_elastic"] = lambda: bf_sweep_case("bf_elastic", 2000, 0)
    out["bf_sweep_inelastic"] = lambda: bf_sweep_case("bf_inelastic", 2000, 0)
    out["bf_run_merge"] = lambda: bf_run_case("bf_merge", 2000, 0, 40)
    out["mesh_merge"] = lambda: mesh_case("mesh_merge_s", 6000, 21, 0.03, 5e-4)
    out["mesh_inelastic"] = lambda: mesh_case("mesh_inelastic_s", 6000, 22, 0.03, 5e-4)
    # the N = 2,000 collisional disk, 200 steps, output every 50 steps
    out["program_bf_merge"] = lambda: program_run_case("bf_merge", disks.bf_collide_disk(2000, seed=0))
    # the mesh driver: 20,000 bodies with four larger than the mesh size, 100 steps
    out["program_mesh_merge"] = lambda: program_run_case("mesh_prog", big_disk(20000, 7)[0])
    # fragmentation: every outcome in one sweep (dt = 0.02 on the crowded ring)
    out["frag_bf"] = lambda: frag_bf_case("bf_frag", 4000, 0, 0.02)
    out["frag_mesh15"] = lambda: frag_mesh_case("mesh_frag_s", 4000, 0, 0.01, 0.02, 15, (-1, 3, -1, 1))
    out["frag_mesh4"] = lambda: frag_mesh_case("mesh_frag4_s", 4000, 1, 0.01, 0.02, 4, (0, 1, 0, 1))
    # bodies larger than the mesh size, three of them past slot 2
    out["mesh_big_merge"] = lambda: mesh_big_case("mesh_merge_s", 10000, 100, 0.01, 5e-3)
    out["mesh_big_inelastic"] = lambda: mesh_big_case("mesh_inelastic_s", 10000, 101, 0.01, 5e-3)
    out["mesh_big_frag"] = lambda: mesh_big_case("mesh_frag_s", 10000, 102, 0.01, 5e-3)
    # the central body's J2: constant (softening 0.5) and fluid-body (M = 1.3)
    out["grav_j2_n512"] = lambda: j2_gravity_case("bf_grav_j2", 512, 31, 1.0, (3, 100, 511))
    out["grav_j2f_n300"] = lambda: j2_gravity_case("bf_grav_j2f", 300, 32, 1.3, (0, 7))
    out["mesh_j2f_steps"] = lambda: j2_mesh_steps_case("mesh_grav_j2f", 6000, 33, 4, 0.03, 5e-4)
    # whole-program runs of both drivers with the fluid-body J2
    out["program_bf_merge_j2"] = lambda: program_run_case("bf_merge_j2", disks.bf_collide_disk(2000, seed=0),
                                                          bodies_from="program_bf_merge")
    out["program_mesh_merge_j2"] = lambda: program_run_case("mesh_prog_j2", big_disk(20000, 7)[0],
                                                                bodies_from="program_mesh_merge")
    # tides raised on the central body (Delta_t = 1): alone, with the fluid-body
    # J2, in the mesh loop, and whole-program runs of both drivers
    out["tides_bf_steps"] = lambda: tides_bf_case("bf_tides", 512, 41, 6, 1e-3)
    out["tides_j2f_bf_steps"] = lambda: tides_bf_case("bf_tides_j2f", 512, 42, 6, 1e-3)
    out["tides_mesh_steps"] = lambda: tides_mesh_case("mesh_tides_j2f", 6000, 43, 4, 0.03, 5e-4)
    out["program_bf_merge_tides"] = lambda: program_run_case("bf_merge_tides", disks.bf_collide_disk(2000, seed=0),
                                                             bodies_from="program_bf_merge")
    out["program_mesh_merge_tides"] = lambda: program_run_case("mesh_prog_tides", big_disk(20000, 7)[0],
                                                               bodies_from="program_mesh_merge")
    # the mesh driver on 200,000 bodies of the mesh workload's disk, 20 steps
    out["program_mesh_merge_200k"] = lambda: program_run_case("mesh_prog_200k", disks.mesh_disk(200000, seed=0),
                                                              disk=("mesh_disk", 200000, 0))
    # both drivers with the elliptic files (brute force: with the cartesian ones
    # and the fluid-body J2; mesh: elliptic only)
    out["program_bf_merge_ell"] = lambda: program_run_case("bf_merge_ell", disks.bf_collide_disk(2000, seed=0),
                                                           bodies_from="program_bf_merge")
    out["program_mesh_merge_ell"] = lambda: program_run_case("mesh_prog_ell", big_disk(20000, 7)[0],
                                                             bodies_from="program_mesh_merge")
    # both drivers without output files, with the resuming files at the end; the
    # mesh driver also in its brute-force regime (below switch_to_brute_force)
    out["program_bf_merge_resume"] = lambda: program_resume_case("bf_merge_resume", disks.bf_collide_disk(2000, seed=0),
                                                                 "program_bf_merge")
    out["program_mesh_merge_resume"] = lambda: program_resume_case("mesh_prog_resume", big_disk(20000, 7)[0],
                                                                   "program_mesh_merge")
    out["program_mesh_naive_resume"] = lambda: program_resume_case("mesh_naive_resume",
                                                                   disks.bf_collide_disk(2000, seed=0),
                                                                   "program_bf_merge")
    # falcON (expansion order 3, theta_min 0.45), the reference's default gravity module
    out["tree_n4096"] = lambda: tree_case("tree_grav", 4096, 51, holes=(5, 77, 4000))
    for k, make in out.items():
        if names and k not in names:
            continue
        np.savez_compressed(os.path.join(HERE, k + ".npz"), **make())
        print("wrote", k)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
