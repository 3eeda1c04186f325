"""TEST INFRASTRUCTURE ONLY: CPU oracles for the parity tests and the CPU
baseline.  Never imported by the product package ``ncorpion_b200``.

* ``Port``   the plain-C restatement ``oracle/ncorpion_oracle.c`` (runtime
             parameters), built with gcc into ``oracle/_build/liboracle.so``.
* ``Ref``    the reference's own sources compiled per profile by
             ``oracle/ref_build.py`` into ``oracle/_ref/<profile>/libref.so``
             (available where the reference tree was present at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SRC = os.path.join(HERE, "ncorpion_oracle.c")
PORT_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
P = C.c_void_p


def build_port(force: bool = False) -> str:
    os.makedirs(os.path.dirname(PORT_LIB), exist_ok=True)
    if force or not os.path.exists(PORT_LIB) or os.path.getmtime(PORT_LIB) < os.path.getmtime(PORT_SRC):
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", PORT_SRC, "-o", PORT_LIB, "-lm"],
                       check=True)
    return PORT_LIB


def _p(a):
    return C.c_void_p(a.ctypes.data)


class Port:
    """ctypes face of the C restatement."""

    def __init__(self):
        self.lib = C.CDLL(build_port())
        L = self.lib
        L.orc_vector_field.argtypes = [C.c_int, P, P, P, P, P, P]
        L.orc_kick.argtypes = [C.c_int, P, P, P, C.c_double, P]
        L.orc_drift.argtypes = [C.c_int, P, P, P, C.c_double, P]
        L.orc_cart2ell.argtypes = [P, P, C.c_double, P, C.c_double, P]
        L.orc_cart2ell.restype = C.c_int
        L.orc_cart2ell_all.argtypes = [C.c_int, P, P, P, C.c_double, P, C.c_double, P, C.c_long]
        L.orc_cart2ell_all.restype = C.c_long

    def vector_field(self, bodies, exists, cm, params):
        b = np.ascontiguousarray(bodies, np.float64)
        ex = np.ascontiguousarray(exists, np.int32)
        cmv = np.ascontiguousarray(cm, np.float64)
        acc = np.zeros((b.shape[0], 3))
        cma = np.zeros(3)
        self.lib.orc_vector_field(b.shape[0] - 1, _p(b), _p(ex), _p(cmv), C.byref(params), _p(acc), _p(cma))
        return acc, cma

    def kick(self, bodies, exists, cm, dt, params):
        """One kick; with tides, params.sideral_omega is updated in place."""
        b = np.ascontiguousarray(bodies, np.float64).copy()
        cmv = np.ascontiguousarray(cm, np.float64).copy()
        ex = np.ascontiguousarray(exists, np.int32)
        self.lib.orc_kick(b.shape[0] - 1, _p(b), _p(ex), _p(cmv), C.c_double(dt), C.byref(params))
        return b, cmv

    def cart2ell(self, rec, cm, mu, params, j2=0.0):
        """cart2ell of one record: (alkhqp (6), whether it printed the (k, h) warning)."""
        r = np.ascontiguousarray(rec, np.float64)
        cmv = np.ascontiguousarray(cm, np.float64)
        out = np.zeros(6)
        w = self.lib.orc_cart2ell(_p(r), _p(cmv), C.c_double(mu), C.byref(params), C.c_double(j2), _p(out))
        return out, bool(w)

    def cart2ell_all(self, bodies, exists, cm, mu, params, j2=0.0):
        """display()'s elliptic values of the existing bodies: (6, n)."""
        b = np.ascontiguousarray(bodies, np.float64)
        ex = np.ascontiguousarray(exists, np.int32)
        cmv = np.ascontiguousarray(cm, np.float64)
        n = int(np.count_nonzero(ex))
        out = np.zeros((6, max(n, 1)))
        got = self.lib.orc_cart2ell_all(b.shape[0] - 1, _p(b), _p(ex), _p(cmv), C.c_double(mu), C.byref(params),
                                        C.c_double(j2), _p(out), out.size)
        assert got == n
        return out[:, :n].copy()

    def drift(self, bodies, exists, cm, dt, params):
        b = np.ascontiguousarray(bodies, np.float64).copy()
        cmv = np.ascontiguousarray(cm, np.float64).copy()
        ex = np.ascontiguousarray(exists, np.int32)
        self.lib.orc_drift(b.shape[0] - 1, _p(b), _p(ex), _p(cmv), C.c_double(dt), C.byref(params))
        return b, cmv


def ref_available(profile: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, profile, "libref.so"))


class Ref:
    """One profile of the reference compiled from source (global state: one
    instance per process and profile)."""

    _cache: dict = {}

    def __new__(cls, profile: str):
        if profile in cls._cache:
            return cls._cache[profile]
        self = super().__new__(cls)
        path = os.path.join(REF_DIR, profile, "libref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        self.lib = L
        self.profile = profile
        L.orc_init.restype = C.c_int
        L.orc_set_state.argtypes = [C.c_int, P, P, P, C.c_double, C.c_double]
        L.orc_get_state.argtypes = [P, P, P, P]
        L.orc_get_state.restype = C.c_int
        L.orc_vector_field.argtypes = [P, P]
        L.orc_set_timestep.argtypes = [C.c_double]
        L.orc_get_sideral_omega.restype = C.c_double
        L.orc_set_sideral_omega.argtypes = [C.c_double]
        L.orc_events.argtypes = [P, C.c_int]
        L.orc_events.restype = C.c_int
        L.orc_n_max.restype = C.c_int
        if hasattr(L, "orc_pairs"):
            L.orc_pairs.argtypes = [P, C.c_int]
            L.orc_pairs.restype = C.c_int
            L.orc_total_neighbours.restype = C.c_long
            L.orc_three_largest.argtypes = [P]
            L.orc_mesh_counts.argtypes = [P]
        L.orc_set_free.argtypes = [C.c_int, P]
        if hasattr(L, "orc_frag_counts"):
            L.orc_frag_counts.argtypes = [P]
        if hasattr(L, "orc_cart2ell"):
            L.orc_cart2ell.argtypes = [P, P, C.c_double, C.c_double, P]
        if hasattr(L, "orc_tree_build"):
            L.orc_tree_build.restype = C.c_int
        if L.orc_init() != 0:
            raise MemoryError("reference init failed")
        self.n_max = L.orc_n_max()
        cls._cache[profile] = self
        return self

    def set_state(self, bodies, exists, cm, dt=1e-3, gam=0.0):
        b = np.ascontiguousarray(bodies, np.float64)
        ex = np.ascontiguousarray(exists, np.int32)
        cmv = np.ascontiguousarray(cm, np.float64)
        assert b.shape[0] <= self.n_max
        self.lib.orc_set_state(b.shape[0] - 1, _p(b), _p(ex), _p(cmv), C.c_double(dt), C.c_double(gam))

    def get_state(self):
        b = np.zeros((self.n_max, 8))
        ex = np.zeros(self.n_max, np.int32)
        cm = np.zeros(8)
        sc = np.zeros(8)
        lid = self.lib.orc_get_state(_p(b), _p(ex), _p(cm), _p(sc))
        return b[:lid + 1].copy(), ex[:lid + 1].copy(), cm, sc

    def vector_field(self):
        b, ex, cm, sc = self.get_state()
        acc = np.zeros((b.shape[0], 3))
        cma = np.zeros(3)
        self.lib.orc_vector_field(_p(acc), _p(cma))
        return acc, cma

    def tree_field(self, slot_order=True):
        """falcON's field of the current state (a falcON profile): the tree
        built as the tree driver builds it before a kick (src/rk4.c:576-586),
        vector_field on it, the tree released (src/rk4.c:337-346).  With
        slot_order the bodies enter the tree in slot order, as in a run's first
        tree; otherwise in the previous tree's Peano-Hilbert order, as in every
        later one.  Returns (acc, cm_acc, cells)."""
        if not getattr(self, "_tree_tables", False):
            self.lib.orc_tree_tables()
            self._tree_tables = True
        if slot_order:
            self.lib.orc_tree_slot_order()
        cells = self.lib.orc_tree_build()
        try:
            acc, cma = self.vector_field()
        finally:
            self.lib.orc_tree_free()
        return acc, cma, cells

    def cart2ell(self, rec, cm, mu, j2=0.0):
        """The reference's cart2ell of one record (its globals CM_buffer = cm,
        J2 = j2): alkhqp (6)."""
        r = np.ascontiguousarray(rec, np.float64)
        cmv = np.ascontiguousarray(cm, np.float64)
        out = np.zeros(6)
        self.lib.orc_cart2ell(_p(r), _p(cmv), C.c_double(j2), C.c_double(mu), _p(out))
        return out

    def fragment_counts(self):
        """(merger, super-catastrophic, partial, full) since the last reset."""
        out = np.zeros(4, np.int32)
        self.lib.orc_frag_counts(_p(out))
        return out

    def events(self):
        n = self.lib.orc_events(None, 0)
        out = np.zeros((max(n, 1), 3), np.int32)
        self.lib.orc_events(_p(out), n)
        return out[:n]

    def pairs(self):
        n = self.lib.orc_pairs(None, 0)
        out = np.zeros((max(n, 1), 2), np.int32)
        self.lib.orc_pairs(_p(out), n)
        return out[:n]


class PortWorld:
    """The port's stateful world: collisions, brute-force sweep and mesh."""

    def __init__(self, n_max, params):
        self.lib = C.CDLL(build_port())
        L = self.lib
        L.orc_w_init.argtypes = [C.c_int, P]
        L.orc_w_set.argtypes = [C.c_int, P, P, P, C.c_double, C.c_double]
        L.orc_w_get.argtypes = [P, P, P]
        L.orc_w_get.restype = C.c_int
        L.orc_w_events.argtypes = [P, C.c_int]
        L.orc_w_events.restype = C.c_int
        L.orc_w_pairs.argtypes = [P, C.c_long]
        L.orc_w_pairs.restype = C.c_long
        L.orc_w_total_neighbours.restype = C.c_long
        L.orc_w_set_timestep.argtypes = [C.c_double]
        L.orc_w_set_gam.argtypes = [C.c_double]
        L.orc_w_three_largest.argtypes = [P]
        L.orc_cell_index.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
        L.orc_cell_index.restype = C.c_long
        L.orc_w_step_mesh.restype = C.c_long
        L.orc_w_end_of_timestep.restype = C.c_int
        L.orc_w_step_brute_force.restype = C.c_int
        L.orc_w_set_fragmentation.argtypes = [C.c_int, P, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.c_double]
        L.orc_w_fragment_counts.argtypes = [P]
        L.orc_w_set_force_naive.argtypes = [C.c_int]
        L.orc_w_get_sideral_omega.restype = C.c_double
        L.orc_w_set_sideral_omega.argtypes = [C.c_double]
        self.n_max = n_max
        self.params = params
        if L.orc_w_init(n_max, C.byref(params)) != 0:
            raise MemoryError("port world init failed")

    def set_state(self, bodies, exists, cm, dt=1e-3, gam=0.0):
        b = np.ascontiguousarray(bodies, np.float64)
        ex = np.ascontiguousarray(exists, np.int32)
        cmv = np.ascontiguousarray(cm, np.float64)
        self.lib.orc_w_set(b.shape[0] - 1, _p(b), _p(ex), _p(cmv), C.c_double(dt), C.c_double(gam))

    def get_state(self):
        b = np.zeros((self.n_max, 8))
        ex = np.zeros(self.n_max, np.int32)
        cm = np.zeros(8)
        lid = self.lib.orc_w_get(_p(b), _p(ex), _p(cm))
        return b[:lid + 1].copy(), ex[:lid + 1].copy(), cm

    def events(self):
        n = self.lib.orc_w_events(None, 0)
        out = np.zeros((max(n, 1), 3), np.int32)
        self.lib.orc_w_events(_p(out), n)
        return out[:n]

    def pairs(self):
        n = self.lib.orc_w_pairs(None, 0)
        out = np.zeros((max(n, 1), 2), np.int32)
        self.lib.orc_w_pairs(_p(out), n)
        return out[:n]

    def three_largest(self):
        idx = np.zeros(3, np.int32)
        self.lib.orc_w_three_largest(_p(idx))
        return idx

    def set_fragmentation(self, N_tilde=15, pq=(-1, 3, -1, 1), mu=0.55, nu=0.4, C1=1.5, k=0.2,
                          merging_threshold=0.0002, fragment_threshold=1.5e-8):
        """The fragmentation constants (src/parameters.h:297-307); resets the
        outcome counters."""
        pqa = np.ascontiguousarray(pq, np.int32)
        self.lib.orc_w_set_fragmentation(N_tilde, _p(pqa), mu, nu, C1, k, merging_threshold, fragment_threshold)

    def fragment_counts(self):
        """(merger, super-catastrophic, partial, full) fragmentation outcomes."""
        out = np.zeros(4, np.int32)
        self.lib.orc_w_fragment_counts(_p(out))
        return out
