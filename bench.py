"""Benchmark of the B200 mutual-interaction engine (one JSON line on rank 0).

Workload (one "step"): one gravity evaluation (vector_field, brute-force
branch + central mass) of the 65,536-body disk: masses log-uniform over
[1e-9, 1e-6], all radii 1e-5, softening_parameter 0.5 (epsilon = 1e-5), G = 1.
``value`` is pair-interactions/s (N(N-1) ordered interactions per step) of the
mixed-precision kernel with inputs resident in HBM; ``e2e`` is the same metric
through ncgpu_vector_field with pinned host buffers (copies inside the timed
region).  The all-FP64 kernels (exact reference order, and tiled) are timed on
the same input for the mixed-vs-FP64 ratio, and the mixed kernel's error is
measured against the exact FP64 result.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun the gravity headline is split over the ranks (strong scaling):
each rank evaluates the field of its part of the targets
(ncgpu_vector_field_part) and one NCCL all-reduce per step assembles the
whole field on every rank (ncorpion_b200/shard.py); ``value`` is the job's
pair-interactions/s.  The secondary sections (mesh, fragmenting disk,
collisional disk, adjoint) run as one replica per rank.  Times are the max
over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BODIES = 65536
SOFTENING = 0.5
FLOP_PER_INTERACTION = 20  # 3 sub, 3 FMA (r^2+eps^2), rsqrt (2), 3 mul, 3 FMA accumulate
# DRAM bytes (read + write) of one k_grav_tiled<mixed> launch at N=65,536, from one ncu capture of
# this script's gravity workload (profiles/k_grav_tiled_mixed_n65536.txt): 3.77 MB read + 105.56 MB written
# (the written bytes are the per-chunk partial sums: 103 source chunks x 3 x 65,536 doubles).
MIXED_DRAM_BYTES = 109.33e6
# DRAM bytes of one mesh step's two main kernels (k_mesh_write + k_mesh_grav_fast) captured at N=262,144
# (profiles/mesh_step_kernels_n262144.txt, current version: 40.3 MB + 36.0 MB), scaled by the bodies to
# N=1,048,576.
MESH_DRAM_BYTES_262K = 76.3e6
METRIC = "Pair-interactions/s mixed vs FP64 (rel err<1e-6); mesh collision steps/s at N=1M"
WORKLOAD = ("gravity-only single-step accelerations, N=65,536 disk (a~U[0.8,1.2], e~Rayleigh 0.01, "
            "i~Rayleigh 0.005), masses log-uniform [1e-9,1e-6], R=1e-5, softening 0.5*(R_k+R_p)")
REF_SAMPLE = 16384  # bodies per reference-arm step (bounded CPU sample)


def max_over_ranks(values, ws, device="cpu"):
    """Element-wise maximum of `values` over all ranks (the slowest rank's
    time); identity on a single rank."""
    if ws <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t]


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms.  start()
    returns once the first sample has arrived and stop() waits for one more,
    so that samples bracket a timed region shorter than nvidia-smi's start-up
    (each wait bounded)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
            return
        self._wait_for(1, 5.0)

    def _wait_for(self, n, limit_s):
        t0 = time.monotonic()
        while len(self.lines) < n and self.proc.poll() is None and time.monotonic() - t0 < limit_s:
            time.sleep(0.005)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self._wait_for(len(self.lines) + 1, 1.0)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload():
    from ncorpion_b200 import disks
    b = disks.gravity_disk(N_BODIES, seed=0)
    ex = np.ones(N_BODIES, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    return b, ex, cm


def params(mode, central=1):
    from ncorpion_b200 import api
    return api.default_params(G=1.0, softening_parameter=SOFTENING, central_mass_bool=central,
                              collision_bool=0, brute_force_bool=1, gravity_mode=mode)


def cpu_reference_rate(b, ex, cm, nsample):
    """The reference's own vector_field (compiled from its sources into
    oracle/_ref) on the first `nsample` bodies; falls back to the C port of
    it when the reference build is absent.  Returns (rate, seconds, kind)."""
    import oracle
    sub, exs = b[:nsample], ex[:nsample]
    if oracle.ref_available("bf_grav_s05"):
        ref = oracle.Ref("bf_grav_s05")
        ref.set_state(sub, exs, cm)
        t0 = time.perf_counter()
        ref.vector_field()
        dt = time.perf_counter() - t0
        kind = "reference"
    else:
        from ncorpion_b200.api import Params
        p = Params()
        p.G, p.softening_parameter, p.central_mass_bool, p.mutual_bool = 1.0, SOFTENING, 1, 1
        port = oracle.Port()
        t0 = time.perf_counter()
        port.vector_field(sub, exs, cm, p)
        dt = time.perf_counter() - t0
        kind = "port"
    return nsample * (nsample - 1) / dt, dt, kind


def run_reference_arm(a, ws, rank):
    if rank != 0:
        return 0
    b, ex, cm = make_workload()
    times = []
    for i in range(a.warmup + a.steps):
        rate, dt, kind = cpu_reference_rate(b, ex, cm, REF_SAMPLE)
        if i >= a.warmup:
            times.append(dt)
    t = float(np.mean(times))
    v = REF_SAMPLE * (REF_SAMPLE - 1) / t
    out = {"metric": METRIC, "value": v, "unit": "pair-interactions/s", "n_gpus": a.gpus, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": {"workload": WORKLOAD, "n": N_BODIES, "sample_bodies": REF_SAMPLE,
                      "parallelism": "single thread (the reference has no threading)"},
           "cpu_baseline": {"value": v, "unit": "pair-interactions/s", "cores": 1, "kind": kind,
                            "sample": f"reference vector_field (gcc -O2, oracle/_ref/bf_grav_s05) on the first "
                                      f"{REF_SAMPLE} of the {N_BODIES} bodies per step"},
           "e2e": {"value": v, "unit": "pair-interactions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


MESH_N = 1 << 20
MESH_STEPS = 100
MESH_DT = 5e-4
MESH_WORKLOAD = ("mesh collision search + mesh gravity, N=1,048,576 disk (a~U[0.5,2.0], e~Rayleigh 0.01, "
                 "i~Rayleigh 0.005), radii dN/dR~R^-3.5 over [1e-5,1e-3], 1024 cells per side, "
                 "collision_cube_min 4.4 (mesh size >= 2 x max radius), instant mergers, dt=5e-4")


def mesh_params(mode, cells=1024, **extra):
    from ncorpion_b200 import api
    return api.default_params(G=1.0, softening_parameter=0.0, collision_bool=1, brute_force_bool=0, mesh_bool=1,
                              collision_type=api.COLLISION_MERGER, collision_cube_cells=cells,
                              how_many_neighbours=16.0, collision_cube_min=4.4, gravity_mode=mode,
                              disruption_threshold=0.1, high_dumping_threshold=100.0, **extra)


def mesh_gamma0(n, cells=1024):
    """The initial mesh size of variable_initialization (src/structure.c:515-523)
    with sma 0.5 .. 2.0, inclination_max 0.015, how_many_neighbours 16."""
    from ncorpion_b200 import api
    return api.initial_gamma(n, cells, 0.5, 2.0, 0.015, 16.0, 4.4)


def bench_mesh(lib, api, torch, mode, steps, warmup, n_bodies=None, cells=1024, **extra):
    """Steps/s of the mesh integrator loop on the device state, CUDA events on
    the library stream; the half kick of integration_mesh first.  `extra`:
    further parameters (the central body's J2 and tides)."""
    from ncorpion_b200 import disks
    n_bodies = n_bodies or MESH_N
    b = disks.mesh_disk(n_bodies, seed=0)
    ex = np.ones(n_bodies, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    api.init(n_bodies + n_bodies // 20, mesh_params(mode, cells, **extra))
    api.upload(b, ex, cm)
    gmin = 4.4 / cells
    gam = mesh_gamma0(n_bodies, cells)
    api.set_timestep(MESH_DT / 2)
    api.three_largest()
    _, _, tn = api.mesh(gam, False)
    api.kick()
    api.mesh_reset()
    api.set_timestep(MESH_DT)
    gam = api.update_gamma(gam, tn, n_bodies, 16.0, gmin)
    st = torch.cuda.ExternalStream(lib.ncgpu_stream())
    for _ in range(warmup):
        hm, tn = api.step_mesh(gam)
        gam = api.update_gamma(gam, tn, hm, 16.0, gmin)
    ms, events, pairs, launches = [], 0, 0, 0
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        hm, tn = api.step_mesh(gam)
        e1.record(st)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        launches += lib.ncgpu_last_launch_count()
        events += len(api.events())
        pairs += tn
        gam = api.update_gamma(gam, tn, hm, 16.0, gmin)
    api.finalize()
    t = float(np.sum(ms)) / 1e3
    return {"steps_per_s": steps / t, "ms_per_step": 1e3 * t / steps, "steps": steps, "events": events,
            "pairs_per_step": pairs / steps, "bodies_end": hm, "gpu_launches": launches}


def bench_output(lib, api, torch, reps=5, cpu=True):
    """An output step of the mesh driver at N=1,048,576, as the drop-in runs it:
    snapshot, half backward kick of the copy (three largest, neighbours, mesh
    gravity), the cartesian files' text formatted on the device and copied to
    the host, display()'s statistics, snapshot end.  Host wall clock (every call
    synchronises).  Beside it, the reference's own formatting: fprintf of
    "%.14lf " for the same number of values on one host core."""
    import time
    from ncorpion_b200 import disks
    n = MESH_N
    b = disks.mesh_disk(n, seed=0)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    api.init(n + n // 20, mesh_params(api.GRAVITY_MIXED))
    api.upload(b, ex, cm)
    gmin = 4.4 / 1024
    gam = mesh_gamma0(n)
    api.set_timestep(MESH_DT)
    for _ in range(3):
        hm, tn = api.step_mesh(gam)
        gam = api.update_gamma(gam, tn, hm, 16.0, gmin)

    cap = lib.ncgpu_format_cartesian_cap()
    text = np.empty(cap, np.uint8)  # the caller's persistent host buffer, as the drop-in keeps one (pinned)
    api.check(lib.ncgpu_host_register(api.ptr(text), text.nbytes), "register")
    lens = (C.c_ulong * 8)()
    stats, idx, cmo, two = np.zeros(3), np.zeros(2, np.int32), np.zeros(8), np.zeros((2, 8))

    def one():
        api.snapshot_begin()
        api.set_timestep(MESH_DT / -2.0)
        api.three_largest()
        api.mesh(gam, False)
        api.kick()
        api.check(lib.ncgpu_format_cartesian(api.ptr(text), cap, lens), "ncgpu_format_cartesian")
        api.check(lib.ncgpu_output_stats(api.ptr(stats), api.ptr(idx), api.ptr(cmo), api.ptr(two)), "stats")
        api.snapshot_end()
        api.mesh_reset()
        api.set_timestep(MESH_DT)

    one()
    times = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
    text_bytes = int(sum(lens))
    nvals = int(np.count_nonzero(text[:text_bytes] == ord(" ")))

    # the elliptic files (write_elliptic_bool, mass and radius with them): the
    # device's cart2ell, the C library's atan2 on host threads, the device's text
    nb_cap = n + n // 20 + 1
    yx, F = np.empty(2 * nb_cap), np.empty(nb_cap)
    for a_ in (yx, F):
        api.check(lib.ncgpu_host_register(api.ptr(a_), a_.nbytes), "register")
    hidx, hrec, alk = np.empty(nb_cap, np.int32), np.empty((nb_cap, 8)), np.zeros((nb_cap, 6))
    nbod, nhost = C.c_int(0), C.c_int(0)
    t_atan2 = []

    def one_ell():
        api.snapshot_begin()
        api.set_timestep(MESH_DT / -2.0)
        api.three_largest()
        api.mesh(gam, False)
        api.kick()
        api.check(lib.ncgpu_output_stats(api.ptr(stats), api.ptr(idx), api.ptr(cmo), api.ptr(two)), "stats")
        api.check(lib.ncgpu_elliptic_begin(C.c_double(1.0 * cmo[6]), api.ptr(yx), yx.size, C.byref(nbod),
                                           api.ptr(hidx), api.ptr(hrec), nb_cap, C.byref(nhost)), "elliptic begin")
        t0 = time.perf_counter()
        api.check(lib.ncgpu_host_atan2(api.ptr(yx), api.ptr(F), nbod.value), "atan2")
        t_atan2.append(time.perf_counter() - t0)
        # listed bodies (hyperbolic, cart2ell's warning, NaNs) would go through the
        # caller's cart2ell here; this disk has none (checked below)
        api.check(lib.ncgpu_format_elliptic(api.ptr(F), api.ptr(alk), nhost.value, 1, api.ptr(text), cap, lens),
                  "elliptic text")
        api.snapshot_end()
        api.mesh_reset()
        api.set_timestep(MESH_DT)

    one_ell()
    times_ell = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        one_ell()
        times_ell.append(time.perf_counter() - t0)
    ell_bytes = int(sum(lens))
    for a_ in (text, yx, F):
        lib.ncgpu_host_unregister(api.ptr(a_))
    api.finalize()
    ms = 1e3 * float(np.median(times))
    ms_ell = 1e3 * float(np.median(times_ell))
    out = {"metric": "output step of the mesh driver at N=1,048,576 (cartesian files)", "ms": ms, "values": nvals,
           "text_bytes": text_bytes, "values_per_s": nvals / (ms * 1e-3),
           "note": "snapshot, half backward kick (three largest, neighbours, mesh gravity), device formatting, "
                   "statistics, the text copied into a host buffer through the C ABI; host wall clock, median of "
                   "%d" % reps,
           "elliptic": {"ms": ms_ell, "bodies": nbod.value, "listed_bodies": nhost.value, "text_bytes": ell_bytes,
                        "host_atan2_ms": 1e3 * float(np.median(t_atan2)),
                        "note": "the same output step with the elliptic files (a, lambda, k, h, q, p, mass, "
                                "radius): cart2ell on the device, atan2 by the C library on host threads, "
                                "device formatting; host wall clock, median of %d" % reps}}
    if nhost.value:
        out["elliptic"]["ms"] = None
        out["elliptic"]["note"] += "; not timed: bodies listed for the caller's cart2ell"
    if cpu:
        try:
            import tempfile
            import oracle
            import ctypes as Cc
            port = Cc.CDLL(oracle.build_port())
            port.orc_fprintf_values.restype = Cc.c_long
            port.orc_fprintf_values.argtypes = [Cc.c_void_p, Cc.c_long, Cc.c_char_p]
            vals = np.ascontiguousarray(b[:, :8].T.reshape(-1)[: nvals], dtype=np.float64)
            d = tempfile.mkdtemp(prefix="ncgpu_out_")
            t0 = time.perf_counter()
            port.orc_fprintf_values(vals.ctypes.data, len(vals), os.path.join(d, "values.txt").encode())
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": dt * 1e3, "unit": "ms", "cores": 1, "kind": "port",
                                   "sample": f'fprintf "%.14lf " of {len(vals)} values (display()\'s formatting '
                                             "alone, without the host copy's backward kick), one core"}
            # the elliptic files: cart2ell of every body, then the same formatting
            port.orc_cart2ell_all.restype = Cc.c_long
            port.orc_cart2ell_all.argtypes = [Cc.c_int, Cc.c_void_p, Cc.c_void_p, Cc.c_void_p, Cc.c_double,
                                              Cc.c_void_p, Cc.c_double, Cc.c_void_p, Cc.c_long]
            pe = mesh_params(api.GRAVITY_MIXED)
            ell = np.empty((8, n))
            t0 = time.perf_counter()
            port.orc_cart2ell_all(n - 1, b.ctypes.data, ex.ctypes.data, cm.ctypes.data, 1.0, Cc.byref(pe), 0.0,
                                  ell.ctypes.data, 6 * n)
            t_c2e = time.perf_counter() - t0
            ell[6], ell[7] = b[:, 6], b[:, 7]
            t0 = time.perf_counter()
            port.orc_fprintf_values(ell.ctypes.data, ell.size, os.path.join(d, "ell.txt").encode())
            t_pr = time.perf_counter() - t0
            out["elliptic"]["cpu_baseline"] = {
                "value": (t_c2e + t_pr) * 1e3, "unit": "ms", "cores": 1, "kind": "port",
                "cart2ell_ms": t_c2e * 1e3,
                "sample": f'cart2ell of {n} bodies and fprintf "%.14lf " of their {ell.size} values, one core'}
        except Exception as e:  # noqa: BLE001
            out["cpu_baseline"] = {"value": None, "unit": "ms", "cores": 1, "kind": "port", "sample": f"unavailable: {e}"}
    return out


def bench_programs():
    """The whole reference program and its drop-in build on the same init.txt,
    host wall clock: the brute-force driver on the N=2,000 collisional disk
    (200 steps, outputs every 50), the mesh driver on a 20,000-body disk with
    bodies larger than the mesh size (100 steps, outputs every 25) and on
    200,000 bodies of the mesh workload's disk (20 steps, outputs every 10).
    Output files and console output of the two are byte-identical (tests).
    Needs the programs built from the reference sources (oracle/_ref)."""
    import shutil
    import tempfile
    import time
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from ncorpion_b200 import disks
    out = {"metric": "whole-program wall time, reference program vs drop-in build"}
    cases = [("bf_merge", "collisional disk N=2,000, brute-force driver, 200 steps",
              lambda: disks.bf_collide_disk(2000, seed=0)),
             ("mesh_prog", "20,000-body disk (four bodies larger than the mesh size), mesh driver, 100 steps",
              None),
             ("mesh_prog_200k", "200,000-body disk of the mesh workload (radii dN/dR~R^-3.5 over [1e-5,1e-3]), "
              "mesh driver, 20 steps, outputs every 10", lambda: disks.mesh_disk(200000, seed=0))]
    for prof, what, make in cases:
        ref = os.path.join(ROOT, "oracle", "_ref", prof, "ncorpion")
        gpu = os.path.join(ROOT, "oracle", "_ref", prof, "ncorpion_gpu")
        if not (os.path.exists(ref) and os.path.exists(gpu)):
            out[prof] = {"unavailable": "programs not built (oracle/ref_build.py needs the reference sources)"}
            continue
        if make is None:
            from make_golden import big_disk
            bodies = big_disk(20000, 7)[0]
        else:
            bodies = make()
        res = {"workload": what}
        for name, exe in (("reference", ref), ("dropin", gpu)):
            walls, integ = [], []
            for _ in range(2):  # the better of two runs
                d = tempfile.mkdtemp(prefix="ncgpu_prog_")
                disks.write_init_txt(os.path.join(d, "init.txt"), bodies)
                t0 = time.perf_counter()
                r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=900)
                walls.append(time.perf_counter() - t0)
                res[name + "_rc"] = r.returncode
                # main()'s own timing of the integration (src/main.c): "The integration took X seconds"
                for line in r.stdout.splitlines():
                    if "integration took" in line:
                        integ.append(float(line.split("took")[1].split()[0]))
                shutil.rmtree(d, ignore_errors=True)
            res[name + "_s"] = min(walls)
            res[name + "_integration_s"] = min(integ) if integ else None
        res["speedup"] = res["reference_s"] / res["dropin_s"]
        if res["reference_integration_s"] and res["dropin_integration_s"]:
            res["speedup_integration"] = res["reference_integration_s"] / res["dropin_integration_s"]
        out[prof] = res
    return out


CENTRAL_N = 262144
CENTRAL_WORKLOAD = ("mesh steps (fast mode) of the N=262,144 mesh disk, 512 cells per side, alone, with the "
                    "fluid-body J2 (J2_value 0, Tearth 25), and with tides raised on the central body besides "
                    "(k2 1.5, Delta_t 1e-3, dimensionless_moi 0.3307)")


def bench_central(lib, api, torch, steps=20):
    """The central body's J2 and tides in the mesh loop: their cost per step,
    and the sequential SideralOmega recurrence of the tides per body."""
    j2 = dict(J2_bool=1, J2=0.0, sideral_omega=2.0 * np.pi / 25.0)
    tides = dict(central_tides_bool=1, k2=1.5, Delta_t=1e-3, dimensionless_moi=0.3307)
    runs = {"plain": bench_mesh(lib, api, torch, api.GRAVITY_MIXED, steps, 3, CENTRAL_N, 512),
            "j2": bench_mesh(lib, api, torch, api.GRAVITY_MIXED, steps, 3, CENTRAL_N, 512, **j2),
            "j2_tides": bench_mesh(lib, api, torch, api.GRAVITY_MIXED, steps, 3, CENTRAL_N, 512, **j2, **tides)}
    out = {"metric": "mesh steps/s with the central body's J2 and tides", "workload": CENTRAL_WORKLOAD}
    for k, v in runs.items():
        out[k] = {"steps_per_s": v["steps_per_s"], "ms_per_step": v["ms_per_step"]}
    tides_ms = runs["j2_tides"]["ms_per_step"] - runs["j2"]["ms_per_step"]
    out["tides_ms_per_kick"] = tides_ms
    out["tides_ns_per_body"] = tides_ms * 1e6 / CENTRAL_N
    out["note"] = ("the tides' SideralOmega recurrence is sequential (one warp: 11 dependent FP64 operations and "
                   "a division per body); J2 adds O(N) work to the kick")
    return out


FRAG_N = 262144
FRAG_DT = 2e-4
FRAG_STEPS = 100
FRAG_WORKLOAD = ("collisional fragmenting disk, N_0=262,144 (a~U[0.9,1.1], e,i~Rayleigh 0.02, R~U[2e-4,5e-4], "
                 "density 3), mesh collision search (1024 cells, collision_cube_min 4.4) with the fragmentation "
                 "model (N_tilde 4 on the lattice {0,1,0,1}, fragments appended on the device, N_max 1,048,576), "
                 "brute-force gravity of the stated mode over every body, dt=2e-4; a shortened run of 100 steps "
                 "of the 10,000-step workload")


def frag_params(mode):
    from ncorpion_b200 import api
    return api.default_params(G=1.0, softening_parameter=0.0, collision_bool=1, brute_force_bool=0, mesh_bool=1,
                              collision_type=api.COLLISION_FRAGMENTATION, collision_cube_cells=1024,
                              how_many_neighbours=16.0, collision_cube_min=4.4, gravity_mode=mode,
                              disruption_threshold=0.1, high_dumping_threshold=100.0, N_tilde=4,
                              pq_min_max=(C.c_int * 4)(0, 1, 0, 1), mesh_brute_gravity=1)


def bench_fragment(lib, api, torch, mode, steps):
    """Steps/s and energy drift of the fragmenting disk: mesh collisions with
    fragmentation, brute-force gravity of `mode`; CUDA events on the library
    stream around each step, energy (FP64, O(N^2)) before and after."""
    from ncorpion_b200 import disks
    b = disks.fragment_disk(FRAG_N, seed=0)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    b, cm = disks.reduce_to_com(b, cm)
    api.init(1 << 20, frag_params(mode))
    api.upload(b, np.ones(FRAG_N, np.int32), cm)
    gmin = 4.4 / 1024
    gam = gmin
    api.set_timestep(FRAG_DT)
    e0 = api.energy()
    st = torch.cuda.ExternalStream(lib.ncgpu_stream())
    ms, launches, hm = [], 0, FRAG_N
    for _ in range(steps):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(st)
        hm, tn = api.step_mesh(gam)
        ev1.record(st)
        ev1.synchronize()
        ms.append(ev0.elapsed_time(ev1))
        launches += lib.ncgpu_last_launch_count()
        gam = api.update_gamma(gam, tn, hm, 16.0, gmin)
    e1 = api.energy()
    counts = api.fragment_counts()
    api.finalize()
    t = float(np.sum(ms)) / 1e3
    return {"steps_per_s": steps / t, "ms_per_step": 1e3 * t / steps, "steps": steps, "bodies_end": int(hm),
            "outcomes": {"merger": int(counts[0]), "super_catastrophic": int(counts[1]), "partial": int(counts[2]),
                         "full": int(counts[3])},
            "energy_start": float(e0[0]), "energy_end": float(e1[0]),
            "energy_drift_rel": float((e1[0] - e0[0]) / abs(e0[0])), "gpu_launches": launches}


BF_N, BF_STEPS, BF_DT = 2000, 200, 1e-3
ADJ_N, ADJ_STEPS = 16384, 1000


def bench_bf_collide(lib, api, torch, cpu_ref):
    """C1: brute-force gravity (exact FP64) + brute-force collision search with
    instant mergers on the N=2,000 disk, 200 integrator steps on the device;
    beside it the reference's own loop (oracle/_ref/bf_merge) for the same steps."""
    from ncorpion_b200 import disks
    b = disks.bf_collide_disk(BF_N, seed=0)
    ex = np.ones(BF_N, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    p = api.default_params(G=1.0, softening_parameter=0.0, collision_bool=1, brute_force_bool=1, mesh_bool=0,
                           collision_type=api.COLLISION_MERGER, gravity_mode=api.GRAVITY_EXACT,
                           disruption_threshold=0.1, high_dumping_threshold=100.0)
    api.init(4096, p)
    api.upload(b, ex, cm)
    api.set_timestep(BF_DT)
    for _ in range(3):
        api.step_brute_force()
    api.upload(b, ex, cm)
    st = torch.cuda.ExternalStream(lib.ncgpu_stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(BF_STEPS):
        hm = api.step_brute_force()
    e1.record(st)
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    api.finalize()
    out = {"metric": "brute-force collisional steps/s at N=2,000", "steps_per_s": BF_STEPS / t,
           "ms_per_step": 1e3 * t / BF_STEPS, "bodies_end": int(hm),
           "workload": "N=2,000 disk (a~U[0.8,1.2], e~Rayleigh 0.01, i~Rayleigh 0.005), equal masses (1e-3 in "
                       "all), R=2e-3, instant mergers, exact FP64 gravity, dt=1e-3, 200 steps", "cpu_baseline": None}
    if cpu_ref:
        import oracle
        if oracle.ref_available("bf_merge"):
            ref = oracle.Ref("bf_merge")
            ref.set_state(b, ex, cm, dt=BF_DT)
            t0 = time.perf_counter()
            for _ in range(BF_STEPS):
                ref.lib.orc_step_brute_force()
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": BF_STEPS / dt, "unit": "steps/s", "cores": 1, "kind": "reference",
                                   "sample": f"the same 200 steps, reference loop (gcc -O2), {dt:.1f} s, 1 thread"}
    return out


def bench_adjoint(lib, api, torch, nsteps=ADJ_STEPS):
    """C4: forward + adjoint of the differentiable leapfrog (ncgpu_leapfrog_vjp:
    forward with checkpoints every 32 steps, then the reverse sweep with
    recomputation) at N=16,384 for the workload's 1,000 steps, in the MIXED
    mode (FP32 pair terms for far tile pairs) and the FP64 mode; CUDA events on
    the library stream."""
    from ncorpion_b200 import disks
    b, cm = disks.reduce_to_com(disks.adjoint_disk(ADJ_N, 0), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]))
    adj = np.random.default_rng(0).normal(size=(ADJ_N, 3))
    args = (b[:, :3], b[:, 3:6], b[:, 6], b[:, 7], cm, 1e-3, nsteps, adj)
    out = {"metric": "forward+adjoint leapfrog steps/s at N=16,384", "checkpoint": 32, "steps": nsteps,
           "workload": "gravity-only disk, N=16,384, log-uniform masses, R=1e-2, softening 0.5 (R_k+R_p), dt=1e-3, "
                       f"{nsteps} steps: forward with checkpoints, reverse sweep with recomputation"}
    for name, mode in (("mixed", api.GRAVITY_MIXED), ("fp64", api.GRAVITY_EXACT)):
        api.init(ADJ_N, api.default_params(G=1.0, softening_parameter=0.5, collision_bool=0, gravity_mode=mode))
        api.leapfrog_vjp(*args)  # warm-up: the same call (the library keeps its buffers for the next one)
        st = torch.cuda.ExternalStream(lib.ncgpu_stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        api.leapfrog_vjp(*args)
        e1.record(st)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        api.finalize()
        out[name] = {"steps_per_s": nsteps / t, "ms_per_step": 1e3 * t / nsteps}
    out["steps_per_s"] = out["mixed"]["steps_per_s"]
    out["ms_per_step"] = out["mixed"]["ms_per_step"]
    return out


# Algorithmic bytes per body of the mesh step's O(N) kernels (reads + writes of the arrays each one must touch):
# kick / drift: exists 4 + acceleration or position 24 + velocity 24 read, 24 written; the records: the cell
# order 4 + the fields gathered (7 doubles + exists + did; 5 doubles + exists) read, a 64-byte record written;
# end of step: exists + position read; cell keys: exists + radius + position read, key + value + cell written;
# a radix pass: key + value read and written (histogram: the key read).
MESH_KERNEL_BYTES = {"k_kick": 76, "k_drift": 76, "k_mesh_records": 132, "k_grav_records": 112, "k_eot_flag": 28,
                     "k_mesh_keys": 48, "k_radix_scatter": 16, "k_radix_hist": 4}


def mesh_kernel_times(prof, n, calls):
    """Per-kernel device time of a profiled mesh run, per call (the steps, the warm-up and the half kick),
    with the algorithmic bytes per second of the O(N) kernels at n bodies."""
    tot = {}
    for e in prof.events():
        if e.device_type.name != "CUDA":
            continue
        k = e.name.replace("(anonymous namespace)::", "").replace("ncg::", "").replace("void ", "").split("(")[0]
        k = k.split("<")[0]  # template arguments apart
        c = tot.setdefault(k, [0, 0.0])
        c[0] += 1
        c[1] += e.device_time_total
    out = {}
    for k, (cnt, us) in sorted(tot.items(), key=lambda kv: -kv[1][1]):
        d = {"launches": cnt, "us_per_launch": us / cnt}
        if k in MESH_KERNEL_BYTES:
            d["alg_gb_per_s"] = MESH_KERNEL_BYTES[k] * n / (us / cnt * 1e-6) / 1e9
        out[k] = d
    return out


def mesh_cpu_reference(nsteps=3):
    """The reference's mesh() + mesh gravity loop (oracle/_ref/mesh_merge_1m,
    1 thread, 8.6 GB hash table) for a few steps of the same disk."""
    import oracle
    from ncorpion_b200 import disks
    if not oracle.ref_available("mesh_merge_1m"):
        return None
    b = disks.mesh_disk(MESH_N, seed=0)
    ref = oracle.Ref("mesh_merge_1m")
    ref.set_state(b, np.ones(MESH_N, np.int32), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]), dt=MESH_DT,
                  gam=mesh_gamma0(MESH_N))
    t0 = time.perf_counter()
    for _ in range(nsteps):
        ref.lib.orc_step_mesh()
    dt = time.perf_counter() - t0
    return {"value": nsteps / dt, "unit": "mesh steps/s", "cores": 1, "kind": "reference",
            "sample": f"{nsteps} iterations of the reference's mesh loop (mesh, drift, kick, end_of_timestep) on "
                      f"the same 1,048,576-body disk ({dt:.1f} s, 1 thread)"}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mesh", action="store_true")
    ap.add_argument("--no-frag", action="store_true")
    ap.add_argument("--no-bf", action="store_true", help="skip the N=2,000 brute-force collisional section")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the forward+adjoint section")
    ap.add_argument("--no-central", action="store_true", help="skip the J2 / tides section")
    ap.add_argument("--no-output", action="store_true", help="skip the output-step section")
    ap.add_argument("--no-programs", action="store_true", help="skip the whole-program section")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="collectives between the ranks (gloo: several ranks may share one GPU, e.g. to test the "
                         "multi-rank path on a one-GPU machine)")
    ap.add_argument("--mesh-n", type=int, default=MESH_N, help="mesh workload bodies (smaller cases for profiling)")
    ap.add_argument("--mesh-cells", type=int, default=1024)
    ap.add_argument("--mesh-steps", type=int, default=MESH_STEPS)
    ap.add_argument("--adj-steps", type=int, default=ADJ_STEPS,
                    help="steps of the forward+adjoint section (the workload's 1,000; fewer for profiling)")
    ap.add_argument("--mesh-only", action="store_true",
                    help="profiling aid: only the mesh section (fast mode), its own JSON line")
    ap.add_argument("--kernel-times", action="store_true",
                    help="with --mesh-only: per-kernel device times of the timed steps (CUPTI tracing through "
                         "torch.profiler) and each one's algorithmic bytes per second")
    a = ap.parse_args(argv)
    a.warmup = max(a.warmup, 3)
    ws, rank, local = dist_info()
    if a.impl == "reference":
        return run_reference_arm(a, ws, rank)

    import torch
    if a.dist_backend == "gloo" and local >= torch.cuda.device_count():
        local = local % torch.cuda.device_count()  # ranks sharing a GPU (gloo only)
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group(a.dist_backend, timeout=timedelta(seconds=120))
    from ncorpion_b200 import api, build
    if not os.path.exists(api.LIB_PATH):
        build.build()
    lib = api.load()

    if a.mesh_only:
        if a.kernel_times:
            from torch.profiler import profile, ProfilerActivity
            with profile(activities=[ProfilerActivity.CUDA]) as prof:
                r = bench_mesh(lib, api, torch, api.GRAVITY_MIXED, a.mesh_steps, a.warmup, a.mesh_n, a.mesh_cells)
            r["kernel_times"] = mesh_kernel_times(prof, a.mesh_n, a.mesh_steps + a.warmup + 1)
        else:
            r = bench_mesh(lib, api, torch, api.GRAVITY_MIXED, a.mesh_steps, a.warmup, a.mesh_n, a.mesh_cells)
        if rank == 0:
            print(json.dumps({"metric": f"mesh collision steps/s at N={a.mesh_n} (fast mode)",
                              "value": r["steps_per_s"], "unit": "steps/s", "n_gpus": ws, "steps": a.mesh_steps,
                              "warmup": a.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                              "config": {"workload": MESH_WORKLOAD, "n": a.mesh_n, "cells": a.mesh_cells},
                              "mesh": r}))
        if ws > 1:
            torch.distributed.destroy_process_group()
        return 0

    b, ex, cm = make_workload()
    n = N_BODIES
    pairs = n * (n - 1)
    api.init(n, params(api.GRAVITY_MIXED))
    dev = torch.device("cuda", local)
    d_b = torch.from_numpy(b).to(dev)
    d_ex = torch.from_numpy(ex).to(dev)
    d_acc = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    d_cma = torch.zeros(3, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    cmh = np.ascontiguousarray(cm)
    sp = C.c_void_p(stream.cuda_stream)

    def step(mode):
        # this rank's part of the targets, then (N > 1) the all-reduce that
        # assembles the field on every rank, ordered on `stream`
        st = lib.ncgpu_vector_field_part(C.c_void_p(d_b.data_ptr()), C.c_void_p(d_ex.data_ptr()), n - 1,
                                         api.ptr(cmh), rank, ws, C.c_void_p(d_acc.data_ptr()),
                                         C.c_void_p(d_cma.data_ptr()), mode, sp)
        api.check(st, "ncgpu_vector_field_part")
        if ws > 1:
            torch.distributed.all_reduce(d_acc)

    def timed(mode, steps, warmup):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                step(mode)
            torch.cuda.synchronize()
            if ws > 1:
                torch.distributed.barrier()
            tot, kern, launches = 0.0, [], 0
            for _ in range(steps):
                flush.zero_()  # L2 flush between timed steps (outside the events)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step(mode)
                e1.record(stream)
                launches += lib.ncgpu_last_launch_count()
                e1.synchronize()
                tot += e0.elapsed_time(e1)
                kern.append(api.last_kernel_ms())
            torch.cuda.synchronize()
            if ws > 1:
                torch.distributed.barrier()
        ms, kms = max_over_ranks([tot / steps, float(np.mean(kern))], ws, dev)
        return ms, kms, launches

    clock = ClockSampler(local)
    clock.start()
    ms_mixed, kms_mixed, launches = timed(api.GRAVITY_MIXED, a.steps, a.warmup)
    clocks = clock.stop()
    ms_fp64t, kms_fp64t, _ = timed(api.GRAVITY_FP64, max(3, a.steps // 3), 3)
    ms_exact, kms_exact, _ = timed(api.GRAVITY_EXACT, 3, 3)

    # accuracy of the mixed kernel against the exact FP64 result
    def accel(mode, central):
        api.set_params(params(mode, central))
        with torch.cuda.stream(stream):
            step(mode)
        torch.cuda.synchronize()
        return d_acc.cpu().numpy().copy()

    a_ex_mut = accel(api.GRAVITY_EXACT, 0)
    a_mx_mut = accel(api.GRAVITY_MIXED, 0)
    a_ex_tot = accel(api.GRAVITY_EXACT, 1)
    a_mx_tot = accel(api.GRAVITY_MIXED, 1)
    rel_mut = np.linalg.norm(a_mx_mut - a_ex_mut, axis=1) / np.linalg.norm(a_ex_mut, axis=1)
    rel_tot = np.linalg.norm(a_mx_tot - a_ex_tot, axis=1) / np.linalg.norm(a_ex_tot, axis=1)
    api.set_params(params(api.GRAVITY_MIXED))

    # end to end with host buffers (pinned host memory): one GPU, the C ABI's
    # host-buffer call; N GPUs, the sharded field (copies in, this rank's part,
    # all-reduce, copies out)
    hb = b.copy()
    hex_ = ex.copy()
    api.check(lib.ncgpu_host_register(api.ptr(hb), hb.nbytes), "register")
    api.check(lib.ncgpu_host_register(api.ptr(hex_), hex_.nbytes), "register")
    cma = np.zeros(3)
    hacc = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    hb_t, hex_t = torch.from_numpy(hb), torch.from_numpy(hex_)

    def e2e_step():
        if ws == 1:
            api.check(lib.ncgpu_vector_field(api.ptr(hb), api.ptr(hex_), n - 1, api.ptr(cmh), api.ptr(cma),
                                             api.GRAVITY_MIXED), "e2e")
            return
        with torch.cuda.stream(stream):
            d_b.copy_(hb_t, non_blocking=True)
            d_ex.copy_(hex_t, non_blocking=True)
            step(api.GRAVITY_MIXED)
            hacc.copy_(d_acc, non_blocking=True)

    for _ in range(2):
        e2e_step()
        torch.cuda.synchronize()
        hb[:] = b
    e2e_t = []
    # the library stream carries the copies in, the kernels and the copies out (one GPU); `stream` (N GPUs)
    lst = torch.cuda.ExternalStream(lib.ncgpu_stream()) if ws == 1 else stream
    for _ in range(a.steps):
        hb[:] = b
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lst)
        e2e_step()
        e1.record(lst)
        e1.synchronize()
        e2e_t.append(e0.elapsed_time(e1) * 1e-3)
    torch.cuda.synchronize()
    lib.ncgpu_host_unregister(api.ptr(hb))
    lib.ncgpu_host_unregister(api.ptr(hex_))
    e2e_s = max_over_ranks([float(np.mean(e2e_t))], ws, dev)[0]

    rates = api.probe_fp32_rates()
    fp32_peak = max(rates["ffma_tflops"], rates["ffma2_tflops"])
    api.finalize()

    mesh = None
    if not a.no_mesh:
        mesh_fast = bench_mesh(lib, api, torch, api.GRAVITY_MIXED, a.mesh_steps, 3, a.mesh_n, a.mesh_cells)
        mesh_exact = bench_mesh(lib, api, torch, api.GRAVITY_EXACT, min(10, a.mesh_steps), 3, a.mesh_n,
                                a.mesh_cells)
        n_pairs = mesh_fast["pairs_per_step"]
        # algorithmic bytes per step: 56 B/body state read + 8 B key/index + 72 B drift + 72 B kick
        # per body; 8 B written + 16 B read per pair (search and gravity)
        alg = a.mesh_n * (56 + 8 + 72 + 72) + n_pairs * (8 + 16)
        hbm_peak = 6426.2
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                hbm_peak = json.load(f)["hbm_gbs"]
        except Exception:
            pass
        ach = alg / (mesh_fast["ms_per_step"] * 1e-3) / 1e9
        wl = MESH_WORKLOAD if (a.mesh_n, a.mesh_cells) == (MESH_N, 1024) else \
            f"{MESH_WORKLOAD} -- reduced to N={a.mesh_n}, {a.mesh_cells} cells per side"
        mesh = {"metric": f"mesh collision steps/s at N={a.mesh_n}", "workload": wl, "fast": mesh_fast,
                "exact": mesh_exact,
                "note": "fast: CM_acc and the three largest bodies' sums as two-level parallel sums; exact: "
                        "sequential FP64 chains (bit-identical state); the pass's pairs[], events and the exact "
                        "mode's state are checked against the reference at this size by tests/test_mesh_1m_gpu.py",
                "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                             "algorithmic_bytes_per_step": alg,
                             "traffic": MESH_DRAM_BYTES_262K * a.mesh_n / 262144,
                             "traffic_note": "k_mesh_write + k_mesh_grav_fast DRAM bytes from an ncu capture at N=262,144, "
                                             "scaled by the body count",
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)"},
                "cpu_baseline": mesh_cpu_reference() if (rank == 0 and ws == 1 and not a.no_cpu_baseline
                                                         and a.mesh_n == MESH_N) else None}
    bf = None if a.no_bf else bench_bf_collide(lib, api, torch, rank == 0 and ws == 1 and not a.no_cpu_baseline)
    adjoint = None if a.no_adjoint else bench_adjoint(lib, api, torch, a.adj_steps)
    central = None if a.no_central else bench_central(lib, api, torch)
    output = None if a.no_output else bench_output(lib, api, torch, cpu=(rank == 0 and ws == 1 and not a.no_cpu_baseline))
    programs = bench_programs() if (rank == 0 and ws == 1 and not a.no_programs and not a.no_cpu_baseline) else None
    frag = None
    if not a.no_frag:
        fm = bench_fragment(lib, api, torch, api.GRAVITY_MIXED, FRAG_STEPS)
        f64 = bench_fragment(lib, api, torch, api.GRAVITY_FP64, FRAG_STEPS)
        frag = {"metric": "fragmenting-disk steps/s and energy drift", "workload": FRAG_WORKLOAD, "mixed": fm,
                "fp64": f64,
                "note": "no reference mode couples mesh collisions with brute-force gravity; the energy includes "
                        "the collisions' own losses, so the mixed-minus-FP64 difference of the drift is the "
                        "gravity precision's share"}
    # one launch (one GPU) processes its part of the interactions
    achieved = FLOP_PER_INTERACTION * (pairs / ws) / (kms_mixed * 1e-3) / 1e12

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        try:
            rate, dt, kind = cpu_reference_rate(b, ex, cm, N_BODIES)
            cpu = {"value": rate, "unit": "pair-interactions/s", "cores": 1, "kind": kind,
                   "sample": f"one full vector_field call on all {N_BODIES} bodies ({dt:.1f} s, 1 thread, "
                             "reference sources gcc -O2)"}
        except Exception as e:  # reference build absent on this machine
            cpu = {"value": None, "unit": "pair-interactions/s", "cores": 1, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        value = pairs / (ms_mixed * 1e-3)  # the whole job's field, split over the ranks
        # the metric's second half, compact and early in the line (the full mesh record is further down)
        mesh_headline = None
        if mesh is not None:
            mcpu = mesh.get("cpu_baseline") or {}
            mesh_headline = {"n": a.mesh_n, "cells": a.mesh_cells,
                             "fast_steps_per_s": mesh["fast"]["steps_per_s"],
                             "fast_ms_per_step": mesh["fast"]["ms_per_step"],
                             "exact_steps_per_s": mesh["exact"]["steps_per_s"],
                             "exact_ms_per_step": mesh["exact"]["ms_per_step"],
                             "hbm_frac_fast": mesh["roofline"]["frac"],
                             "reference_cpu_steps_per_s": mcpu.get("value"),
                             "pairs_bit_exact_vs_reference": "tests/test_mesh_1m_gpu.py"}
        out = {
            "metric": METRIC, "value": value, "unit": "pair-interactions/s", "mesh_headline": mesh_headline,
            "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32 pair terms, f64 state/accumulation", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N_BODIES, "gravity_mode": "mixed",
                       "l2": "flushed between timed steps (256 MiB write outside the events)",
                       "parallelism": (f"targets split over {ws} GPUs, one NCCL all-reduce of the field per step; "
                                       "secondary sections one replica per GPU") if ws > 1 else "single GPU"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak, "traffic": MIXED_DRAM_BYTES,
                         "traffic_note": "bytes per launch from ncu (dram__bytes_read.sum + dram__bytes_write.sum); "
                                         "algorithmic input 2.6 MB, the rest is the per-chunk partial sums",
                         "kernel": "k_grav_tiled<mixed>", "kernel_ms": kms_mixed,
                         "flop_per_interaction": FLOP_PER_INTERACTION,
                         "peak_source": "measured in this run: best of the scalar FFMA and packed f32x2 FMA "
                                        "dependency-chain probes (ncgpu_probe_fp32_rates)",
                         "probes": rates,
                         "rsqrt_bound_frac": (pairs / ws) / (kms_mixed * 1e-3) / (rates["rsqrt_gops"] * 1e9)},
            "cpu_baseline": cpu,
            "e2e": {"value": pairs / e2e_s, "unit": "pair-interactions/s",
                    "h2d_bytes_per_step": int(hb.nbytes + hex_.nbytes),
                    # one GPU: the records come back whole (64 B each) + CM_acc; N GPUs: the field (24 B each)
                    "d2h_bytes_per_step": int(n * 64 + 24) if ws == 1 else int(n * 24),
                    "ms_per_step": e2e_s * 1e3},
            "gpu_launches": launches,
            "clocks": clocks,
            "fp64_exact": {"value": pairs / (ms_exact * 1e-3), "ms_per_step": ms_exact,
                           "kernel_ms": kms_exact},
            "fp64_tiled": {"value": pairs / (ms_fp64t * 1e-3), "ms_per_step": ms_fp64t,
                           "kernel_ms": kms_fp64t},
            "speedup_mixed_vs_fp64_exact": ms_exact / ms_mixed,
            "speedup_mixed_vs_fp64_tiled": ms_fp64t / ms_mixed,
            "mesh": mesh,
            "fragment": frag,
            "brute_force_collisional": bf,
            "adjoint": adjoint,
            "central_body": central,
            "output_step": output,
            "programs": programs,
            "accuracy": {"mutual_rel_err_max": float(rel_mut.max()),
                         "mutual_rel_err_median": float(np.median(rel_mut)),
                         "total_rel_err_max": float(rel_tot.max()),
                         "total_rel_err_median": float(np.median(rel_tot)),
                         "reference": "exact FP64 kernel (bit-identical to the reference's vector_field)"},
        }
        print(json.dumps(out))
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
