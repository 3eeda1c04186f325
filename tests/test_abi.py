"""CPU: the C-ABI library builds for sm_100a, loads without a GPU and exports
every entry point that include/*.h declares; the Python binding declares the
same set; calls without a GPU fail with a status, not a crash."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT, make_params


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(ncgpu_\w+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"ncgpu_init", "ncgpu_vector_field", "ncgpu_kick", "ncgpu_drift"} <= names


def test_library_exports_declared_symbols(lib):
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), f"libncgpu.so does not export {name}"


def test_binding_covers_header(lib):
    from ncorpion_b200 import api
    assert declared_symbols() <= set(api.EXPORTS), declared_symbols() - set(api.EXPORTS)


def test_strerror_and_state_errors(lib):
    from ncorpion_b200 import api
    assert lib.ncgpu_strerror(api.E_NMAX).decode().startswith("Cannot add a body")
    # nothing initialised: every state call reports E_STATE
    lib.ncgpu_finalize()
    assert lib.ncgpu_kick() == api.E_STATE
    assert lib.ncgpu_drift() == api.E_STATE
    assert lib.ncgpu_set_timestep(ctypes.c_double(1e-3)) == api.E_STATE


def test_init_rejects_bad_arguments(lib):
    from ncorpion_b200 import api
    assert lib.ncgpu_init(0, ctypes.byref(make_params())) == api.E_ARG
    assert lib.ncgpu_init(10, None) == api.E_ARG
    assert lib.ncgpu_init(10, ctypes.byref(make_params(gravity_mode=7))) == api.E_ARG
