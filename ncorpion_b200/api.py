"""ctypes binding of the C ABI declared in ``include/ncgpu.h``.

This is the Python face of the same library a C host links against.  It loads
``ncorpion_b200/libncgpu.so`` and raises if it is missing: there is no CPU or
PyTorch fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import LIB_PATH

OK = 0
E_ARG, E_CUDA, E_CAPACITY, E_NMAX, E_STATE, E_TIMEOUT, E_UNSUPPORTED, E_FRAGMENT = -1, -2, -3, -4, -5, -6, -7, -8

GRAVITY_EXACT, GRAVITY_FP64, GRAVITY_MIXED = 0, 1, 2
GRAVITY_MODES = {"exact": GRAVITY_EXACT, "fp64": GRAVITY_FP64, "mixed": GRAVITY_MIXED}
COLLISION_ELASTIC, COLLISION_INELASTIC, COLLISION_MERGER, COLLISION_FRAGMENTATION = 0, 1, 2, 3


class Params(C.Structure):
    """Mirror of ``struct ncgpu_params`` (the parameters.h macros on the path)."""

    _fields_ = [
        ("G", C.c_double),
        ("softening_parameter", C.c_double),
        ("central_mass_bool", C.c_int),
        ("mutual_bool", C.c_int),
        ("collision_bool", C.c_int),
        ("brute_force_bool", C.c_int),
        ("mesh_bool", C.c_int),
        ("collision_type", C.c_int),
        ("collision_parameter", C.c_double),
        ("one_collision_only_bool", C.c_int),
        ("collision_cube_cells", C.c_int),
        ("how_many_neighbours", C.c_double),
        ("collision_cube_min", C.c_double),
        ("switch_to_brute_force", C.c_int),
        ("gravity_mode", C.c_int),
        ("near_theta", C.c_double),
        ("disruption_threshold", C.c_double),
        ("high_dumping_threshold", C.c_double),
        ("reduce_to_COM_bool", C.c_int),
        ("N_tilde", C.c_int),
        ("pq_min_max", C.c_int * 4),
        ("mu_parameter", C.c_double),
        ("nu_parameter", C.c_double),
        ("C1_parameter", C.c_double),
        ("k_parameter", C.c_double),
        ("merging_threshold", C.c_double),
        ("fragment_threshold", C.c_double),
        ("mesh_brute_gravity", C.c_int),
        ("J2_bool", C.c_int),
        ("J2", C.c_double),
        ("R_unit", C.c_double),
        ("sideral_omega", C.c_double),
        ("central_tides_bool", C.c_int),
        ("k2", C.c_double),
        ("Delta_t", C.c_double),
        ("dimensionless_moi", C.c_double),
    ]


class LeapfrogArgs(C.Structure):
    """Mirror of ``struct ncgpu_leapfrog_args``."""

    _fields_ = [
        ("n", C.c_int),
        ("x0", C.c_void_p), ("v0", C.c_void_p), ("m", C.c_void_p), ("R", C.c_void_p), ("cm", C.c_void_p),
        ("dt", C.c_double), ("nsteps", C.c_int), ("checkpoint", C.c_int),
        ("x_final", C.c_void_p), ("v_final", C.c_void_p), ("adj_x_final", C.c_void_p),
        ("grad_x0", C.c_void_p), ("grad_v0", C.c_void_p), ("grad_m", C.c_void_p),
        ("tan_x0", C.c_void_p), ("tan_v0", C.c_void_p), ("tan_m", C.c_void_p), ("tan_x_final", C.c_void_p),
    ]


class NcgpuError(RuntimeError):
    def __init__(self, status, where, lib=None):
        msg = f"{where}: status {status}"
        if lib is not None:
            msg += f" ({lib.ncgpu_strerror(status).decode()})"
            if status == E_CUDA:
                msg += f": {lib.ncgpu_last_error().decode()}"
        super().__init__(msg)
        self.status = status


_lib = None

P = C.c_void_p
EXPORTS = {
    # name: (restype, argtypes)
    "ncgpu_default_params": (None, [P]),
    "ncgpu_init": (C.c_int, [C.c_int, P]),
    "ncgpu_finalize": (None, []),
    "ncgpu_strerror": (C.c_char_p, [C.c_int]),
    "ncgpu_last_error": (C.c_char_p, []),
    "ncgpu_vector_field": (C.c_int, [P, P, C.c_int, P, P, C.c_int]),
    "ncgpu_vector_field_dev": (C.c_int, [P, P, C.c_int, P, P, P, C.c_int, P]),
    "ncgpu_vector_field_part": (C.c_int, [P, P, C.c_int, P, C.c_int, C.c_int, P, P, C.c_int, P]),
    "ncgpu_last_launch_count": (C.c_int, []),
    "ncgpu_stream": (C.c_void_p, []),
    "ncgpu_vector_field_static": (C.c_int, [P, P, C.c_int, P, P, P, P, P]),
    "ncgpu_check_error": (C.c_int, [P]),
    "ncgpu_noalloc_scratch_bytes": (C.c_ulong, []),
    "ncgpu_upload": (C.c_int, [P, P, C.c_int, P]),
    "ncgpu_download": (C.c_int, [P, P, P, P]),
    "ncgpu_set_timestep": (C.c_int, [C.c_double]),
    "ncgpu_kick": (C.c_int, []),
    "ncgpu_set_params": (C.c_int, [P]),
    "ncgpu_host_register": (C.c_int, [P, C.c_ulong]),
    "ncgpu_host_unregister": (C.c_int, [P]),
    "ncgpu_probe_fp32_peak": (C.c_int, [P]),
    "ncgpu_probe_fp32_rates": (C.c_int, [P, P, P]),
    "ncgpu_probe_wait_timeout": (C.c_int, [C.c_int, P]),
    "ncgpu_last_kernel_ms": (C.c_int, [P]),
    "ncgpu_collide_brute": (C.c_int, [P]),
    "ncgpu_fragment_counts": (C.c_int, [P]),
    "ncgpu_energy": (C.c_int, [P]),
    "ncgpu_get_sideral_omega": (C.c_int, [P]),
    "ncgpu_get_j2": (C.c_int, [P, P]),
    "ncgpu_total_momentum": (C.c_int, [P]),
    "ncgpu_get_largest_id": (C.c_int, [P, P]),
    "ncgpu_snapshot_begin": (C.c_int, []),
    "ncgpu_snapshot_end": (C.c_int, []),
    "ncgpu_format_cartesian": (C.c_int, [P, C.c_ulong, P]),
    "ncgpu_format_cartesian_cap": (C.c_ulong, []),
    "ncgpu_output_stats": (C.c_int, [P, P, P, P]),
    "ncgpu_elliptic_begin": (C.c_int, [C.c_double, P, C.c_ulong, P, P, P, C.c_int, P]),
    "ncgpu_format_elliptic": (C.c_int, [P, P, C.c_int, C.c_int, P, C.c_ulong, P]),
    "ncgpu_elliptic_values": (C.c_int, [P, C.c_ulong]),
    "ncgpu_host_atan2": (C.c_int, [P, P, C.c_long]),
    "ncgpu_set_sideral_omega": (C.c_int, [C.c_double]),
    "ncgpu_probe_pow_third": (C.c_int, [P, P, C.c_int]),
    "ncgpu_probe_div": (C.c_int, [P, P, P, C.c_int]),
    "ncgpu_probe_seq_sum": (C.c_int, [P, C.c_long, P, P, C.c_int, C.c_int]),
    "ncgpu_get_events": (C.c_int, [P, P, C.c_int, P]),
    "ncgpu_end_of_timestep": (C.c_int, [P]),
    "ncgpu_step_brute_force": (C.c_int, [P]),
    "ncgpu_three_largest": (C.c_int, [P]),
    "ncgpu_mesh": (C.c_int, [C.c_double, C.c_int, P, P, P]),
    "ncgpu_get_pairs": (C.c_int, [P, C.c_int, P]),
    "ncgpu_mesh_reset": (C.c_int, []),
    "ncgpu_set_force_naive": (C.c_int, [C.c_int]),
    "ncgpu_step_mesh": (C.c_int, [C.c_double, P, P]),
    "ncgpu_leapfrog": (C.c_int, [P]),
    "ncgpu_leapfrog_vjp": (C.c_int, [P]),
    "ncgpu_leapfrog_jvp": (C.c_int, [P]),
    "ncgpu_drift": (C.c_int, []),
}


def load(path: str | None = None):
    """Load libncgpu.so (once) and declare the exported signatures."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m ncorpion_b200.build` "
            "(the GPU path has no fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def check(status: int, where: str):
    if status != OK:
        raise NcgpuError(status, where, _lib)


def default_params(**kw) -> Params:
    lib = load()
    p = Params()
    lib.ncgpu_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def init(n_max: int, params: Params):
    lib = load()
    check(lib.ncgpu_init(int(n_max), C.byref(params)), "ncgpu_init")


def set_params(params: Params):
    check(load().ncgpu_set_params(C.byref(params)), "ncgpu_set_params")


def probe_fp32_peak() -> float:
    v = C.c_double(0.0)
    check(load().ncgpu_probe_fp32_peak(C.byref(v)), "ncgpu_probe_fp32_peak")
    return v.value


def probe_fp32_rates() -> dict:
    """Measured FP32 rates: scalar FFMA and packed f32x2 FMA (TFLOP/s) and
    rsqrt.approx (Gop/s)."""
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    check(load().ncgpu_probe_fp32_rates(C.byref(a), C.byref(b), C.byref(c)), "ncgpu_probe_fp32_rates")
    return {"ffma_tflops": a.value, "ffma2_tflops": b.value, "rsqrt_gops": c.value}


def last_kernel_ms() -> float:
    v = C.c_double(0.0)
    check(load().ncgpu_last_kernel_ms(C.byref(v)), "ncgpu_last_kernel_ms")
    return v.value


def finalize():
    load().ncgpu_finalize()


def _bodies(b):
    b = np.ascontiguousarray(b, dtype=np.float64)
    assert b.ndim == 2 and b.shape[1] == 8
    return b


def vector_field(bodies, exists=None, cm=None, mode="exact"):
    """Accelerations of all existing bodies (copy of ``bodies``' layout with
    vx, vy, vz replaced by the acceleration) and the central-mass CM_acc."""
    lib = load()
    b = _bodies(bodies).copy()
    n = b.shape[0]
    ex = np.ones(n, np.int32) if exists is None else np.ascontiguousarray(exists, dtype=np.int32)
    cmv = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]) if cm is None else np.ascontiguousarray(cm, np.float64)
    cma = np.zeros(3)
    st = lib.ncgpu_vector_field(ptr(b), ptr(ex), n - 1, ptr(cmv), ptr(cma), GRAVITY_MODES.get(mode, mode))
    check(st, "ncgpu_vector_field")
    acc = b[:, 3:6].copy()
    acc[ex == 0] = 0.0
    return acc, cma


def upload(bodies, exists, cm):
    lib = load()
    b = _bodies(bodies)
    ex = np.ascontiguousarray(exists, dtype=np.int32)
    cmv = np.ascontiguousarray(cm, np.float64)
    check(lib.ncgpu_upload(ptr(b), ptr(ex), b.shape[0] - 1, ptr(cmv)), "ncgpu_upload")


def download(n_max: int):
    lib = load()
    b = np.zeros((n_max, 8))
    ex = np.zeros(n_max, np.int32)
    lid = C.c_int(0)
    cm = np.zeros(8)
    check(lib.ncgpu_download(ptr(b), ptr(ex), C.byref(lid), ptr(cm)), "ncgpu_download")
    k = lid.value + 1
    return b[:k].copy(), ex[:k].copy(), cm


def set_timestep(dt: float):
    check(load().ncgpu_set_timestep(float(dt)), "ncgpu_set_timestep")


def kick():
    check(load().ncgpu_kick(), "ncgpu_kick")


def drift():
    check(load().ncgpu_drift(), "ncgpu_drift")


def end_of_timestep() -> int:
    n = C.c_int(0)
    check(load().ncgpu_end_of_timestep(C.byref(n)), "ncgpu_end_of_timestep")
    return n.value


def step_brute_force() -> int:
    n = C.c_int(0)
    check(load().ncgpu_step_brute_force(C.byref(n)), "ncgpu_step_brute_force")
    return n.value


def collide_brute() -> int:
    n = C.c_int(0)
    check(load().ncgpu_collide_brute(C.byref(n)), "ncgpu_collide_brute")
    return n.value


def events(with_records=False):
    """(n, 3) int array of (a, b, type) of the last sweep, plus the (n, 8)
    records when asked."""
    lib = load()
    n = C.c_int(0)
    check(lib.ncgpu_get_events(None, None, 0, C.byref(n)), "ncgpu_get_events")
    k = n.value
    ev = np.zeros((max(k, 1), 3), np.int32)
    rec = np.zeros((max(k, 1), 8))
    check(lib.ncgpu_get_events(ptr(ev), ptr(rec), k, C.byref(n)), "ncgpu_get_events")
    return (ev[:k], rec[:k]) if with_records else ev[:k]


def three_largest():
    idx = np.zeros(3, np.int32)
    check(load().ncgpu_three_largest(ptr(idx)), "ncgpu_three_largest")
    return idx


def mesh(gam: float, with_collisions: bool = True):
    """(n_pairs, n_events, total_neighbours) of one mesh pass."""
    np_, ne, tn = C.c_int(0), C.c_int(0), C.c_long(0)
    check(load().ncgpu_mesh(float(gam), int(with_collisions), C.byref(np_), C.byref(ne), C.byref(tn)), "ncgpu_mesh")
    return np_.value, ne.value, tn.value


def pairs():
    lib = load()
    n = C.c_int(0)
    check(lib.ncgpu_get_pairs(None, 0, C.byref(n)), "ncgpu_get_pairs")
    out = np.zeros((max(n.value, 1), 2), np.int32)
    check(lib.ncgpu_get_pairs(ptr(out), n.value, C.byref(n)), "ncgpu_get_pairs")
    return out[:n.value]


def mesh_reset():
    check(load().ncgpu_mesh_reset(), "ncgpu_mesh_reset")


def step_mesh(gam: float):
    hm, tn = C.c_int(0), C.c_long(0)
    check(load().ncgpu_step_mesh(float(gam), C.byref(hm), C.byref(tn)), "ncgpu_step_mesh")
    return hm.value, tn.value


def initial_gamma(n_0, cells, sma_min, sma_max, inclination_max, how_many_neighbours, cube_min):
    """Initial mesh size of variable_initialization (src/structure.c:515-523,
    host side, libm pow), clamped below at cube_min / cells."""
    gam = (sma_max ** 3 - sma_min ** 3) ** (1.0 / 3.0) * \
        (4.0 * np.pi * how_many_neighbours * np.sin(inclination_max) / (float(n_0) * 81.0)) ** (1.0 / 3.0)
    gam_min = cube_min / float(cells)
    return gam_min if gam < gam_min else gam


def update_gamma(gam, total_neighbours, how_many_moonlets, how_many_neighbours, gam_min):
    """Mesh-size update of src/rk4.c:367-372 (host side, libm pow)."""
    average = 2.0 * float(total_neighbours) / float(how_many_moonlets)
    gam = gam * (how_many_neighbours / average) ** (1.0 / 3.0)
    return gam_min if gam < gam_min else gam


def _c3(a):
    return np.ascontiguousarray(a, np.float64).reshape(-1, 3)


def leapfrog(x0, v0, m, R, cm, dt, nsteps, checkpoint=32):
    """Final positions and velocities of the collisionless brute-force
    integrator (half drift, nsteps x (kick, drift), half back-drift)."""
    x0, v0 = _c3(x0), _c3(v0)
    n = x0.shape[0]
    m = np.ascontiguousarray(m, np.float64)
    R = np.ascontiguousarray(R, np.float64)
    cm = np.ascontiguousarray(cm, np.float64)
    xf, vf = np.zeros((n, 3)), np.zeros((n, 3))
    a = LeapfrogArgs(n, x0.ctypes.data, v0.ctypes.data, m.ctypes.data, R.ctypes.data, cm.ctypes.data, float(dt),
                     int(nsteps), int(checkpoint), xf.ctypes.data, vf.ctypes.data, None, None, None, None)
    check(load().ncgpu_leapfrog(C.byref(a)), "ncgpu_leapfrog")
    return xf, vf


def leapfrog_vjp(x0, v0, m, R, cm, dt, nsteps, adj_x_final, checkpoint=32):
    """(dL/dx0, dL/dv0, dL/dm) for a given dL/dx_final."""
    x0, v0, adj = _c3(x0), _c3(v0), _c3(adj_x_final)
    n = x0.shape[0]
    m = np.ascontiguousarray(m, np.float64)
    R = np.ascontiguousarray(R, np.float64)
    cm = np.ascontiguousarray(cm, np.float64)
    gx, gv, gm = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    a = LeapfrogArgs(n, x0.ctypes.data, v0.ctypes.data, m.ctypes.data, R.ctypes.data, cm.ctypes.data, float(dt),
                     int(nsteps), int(checkpoint), None, None, adj.ctypes.data, gx.ctypes.data, gv.ctypes.data,
                     gm.ctypes.data)
    check(load().ncgpu_leapfrog_vjp(C.byref(a)), "ncgpu_leapfrog_vjp")
    return gx, gv, gm


def leapfrog_jvp(x0, v0, m, R, cm, dt, nsteps, tan_x0, tan_v0, tan_m):
    """Directional derivative of x_final along (tan_x0, tan_v0, tan_m)."""
    x0, v0, tx, tv = _c3(x0), _c3(v0), _c3(tan_x0), _c3(tan_v0)
    n = x0.shape[0]
    m = np.ascontiguousarray(m, np.float64)
    R = np.ascontiguousarray(R, np.float64)
    cm = np.ascontiguousarray(cm, np.float64)
    tm = np.ascontiguousarray(tan_m, np.float64)
    out = np.zeros((n, 3))
    a = LeapfrogArgs(n, x0.ctypes.data, v0.ctypes.data, m.ctypes.data, R.ctypes.data, cm.ctypes.data, float(dt),
                     int(nsteps), 32, None, None, None, None, None, None, tx.ctypes.data, tv.ctypes.data,
                     tm.ctypes.data, out.ctypes.data)
    check(load().ncgpu_leapfrog_jvp(C.byref(a)), "ncgpu_leapfrog_jvp")
    return out


def fragment_counts() -> np.ndarray:
    """(merger, super-catastrophic, partial, full) outcomes since the upload."""
    out = np.zeros(4, np.int32)
    check(load().ncgpu_fragment_counts(ptr(out)), "ncgpu_fragment_counts")
    return out


def snapshot_begin():
    check(load().ncgpu_snapshot_begin(), "ncgpu_snapshot_begin")


def snapshot_end():
    check(load().ncgpu_snapshot_end(), "ncgpu_snapshot_end")


def format_cartesian() -> list:
    """The 8 cartesian files' texts (x y z vx vy vz mass radius) of the state,
    as display() writes them, without the newlines."""
    lib = load()
    cap = lib.ncgpu_format_cartesian_cap()
    buf = C.create_string_buffer(cap)
    lens = (C.c_ulong * 8)()
    check(lib.ncgpu_format_cartesian(buf, cap, lens), "ncgpu_format_cartesian")
    raw = buf.raw
    out, pos = [], 0
    for f in range(8):
        out.append(raw[pos:pos + lens[f]].decode())
        pos += lens[f]
    return out


def elliptic_begin(mu: float):
    """cart2ell on the device up to the mean longitude's atan2: returns
    (yx (n, 2): the atan2 arguments of the existing bodies in slot order,
    host_idx: the slots of the bodies the caller converts itself, host_rec
    (k, 8): their records)."""
    lib = load()
    lid = C.c_int(0)
    check(lib.ncgpu_get_largest_id(C.byref(lid), None), "ncgpu_get_largest_id")
    n_slots = max(1, lid.value + 1)
    yx = np.zeros((n_slots, 2))
    n_b, n_h = C.c_int(0), C.c_int(0)
    idx = np.zeros(n_slots, np.int32)
    rec = np.zeros((n_slots, 8))
    check(lib.ncgpu_elliptic_begin(C.c_double(mu), ptr(yx), 2 * n_slots, C.byref(n_b), ptr(idx), ptr(rec), n_slots,
                                   C.byref(n_h)), "ncgpu_elliptic_begin")
    return yx[:n_b.value].copy(), idx[:n_h.value].copy(), rec[:n_h.value].copy()


def host_atan2(yx: np.ndarray) -> np.ndarray:
    """atan2(y, x) of each row with the C library's atan2 (ncgpu_host_atan2)."""
    yx = np.ascontiguousarray(yx, np.float64)
    F = np.zeros(len(yx))
    check(load().ncgpu_host_atan2(ptr(yx), ptr(F), len(yx)), "ncgpu_host_atan2")
    return F


def format_elliptic(F, host_alkhqp, mass_radius: bool = False) -> list:
    """The texts of a, lambda, k, h, q, p (then mass and radius) after
    elliptic_begin, from F = atan2 of its arguments and the caller's elements
    of the listed bodies ((k, 6))."""
    lib = load()
    F = np.ascontiguousarray(F, np.float64)
    alk = np.ascontiguousarray(np.asarray(host_alkhqp, np.float64).reshape(-1, 6))
    cap = lib.ncgpu_format_cartesian_cap()
    buf = C.create_string_buffer(cap)
    nf = 8 if mass_radius else 6
    lens = (C.c_ulong * 8)()
    check(lib.ncgpu_format_elliptic(ptr(F), ptr(alk), len(alk), int(mass_radius), buf, cap, lens),
          "ncgpu_format_elliptic")
    raw = buf.raw
    out, pos = [], 0
    for f in range(nf):
        out.append(raw[pos:pos + lens[f]].decode())
        pos += lens[f]
    return out


def elliptic_values(n: int) -> np.ndarray:
    """(8, n): a, lambda, k, h, q, p, mass, radius of the last elliptic output."""
    v = np.zeros((8, max(n, 1)))
    check(load().ncgpu_elliptic_values(ptr(v), v.size), "ncgpu_elliptic_values")
    return v.reshape(-1)[:8 * n].reshape(8, n)


def output_stats():
    """(stats (total_mass, M1, M2), (i1, i2), cm (8), two bodies (2 x 8)) as display() computes them."""
    lib = load()
    stats = np.zeros(3)
    idx = np.zeros(2, np.int32)
    cm = np.zeros(8)
    two = np.zeros((2, 8))
    check(lib.ncgpu_output_stats(ptr(stats), ptr(idx), ptr(cm), ptr(two)), "ncgpu_output_stats")
    return stats, idx, cm, two


def get_j2() -> float:
    """The J2 in force of the device state (0 without J2)."""
    j = C.c_double(0.0)
    check(load().ncgpu_get_j2(C.byref(j), None), "ncgpu_get_j2")
    return j.value


def get_sideral_omega() -> float:
    """The central body's sideral rotation of the device state."""
    w = C.c_double(0.0)
    check(load().ncgpu_get_sideral_omega(C.byref(w)), "ncgpu_get_sideral_omega")
    return w.value


def set_sideral_omega(omega: float):
    check(load().ncgpu_set_sideral_omega(float(omega)), "ncgpu_set_sideral_omega")


def energy() -> np.ndarray:
    """(E, kinetic, central potential, mutual potential) of the device state."""
    out = np.zeros(4)
    check(load().ncgpu_energy(ptr(out)), "ncgpu_energy")
    return out
