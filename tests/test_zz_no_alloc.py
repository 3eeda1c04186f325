"""GPU: ncgpu_vector_field_static, the force evaluation for callers that
cannot allocate device memory when they need forces (a host whose device
memory belongs to its own pool allocator, an integration loop that forbids
allocation once it runs).  It needs no ncgpu_init and keeps its scratch in a
fixed device array inside libncgpu.so.

Checked through the C ABI against the allocating entry point
ncgpu_vector_field_dev in the exact mode, with that mode's tolerance
(bit-identical accelerations and CM_acc):

* in this process, on calls in a row with a shrinking input after init /
  finalize cycles, so that the shared scratch still holds the previous call's
  larger contents;
* in a fresh process, where the first static call is the first call of the
  library on the device (the set-up that loads the device code and the array):
  a second call leaves the device's free memory unchanged, and after a stand-in
  pool allocator has taken all but 32 MB of the device a third call still
  succeeds with the same result.

This file is collected last.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, make_params

pytestmark = pytest.mark.gpu


def _dev(t):
    return C.c_void_p(t.data_ptr())


def test_static_scratch_matches_allocating_entry_point(lib):
    import torch
    from ncorpion_b200 import api, disks

    assert 0 < lib.ncgpu_noalloc_scratch_bytes() < 64 << 20
    # the third case carries the fluid-body J2 (two CM_acc terms per body)
    cases = [(3000, 1, 0.5, 0.05, {}), (1200, 2, 0.0, 0.1, {}),
             (2000, 3, 0.5, 0.05, dict(J2_bool=1, J2=0.0, sideral_omega=2.0 * np.pi / 25.0))]
    for n, seed, soft, hole_frac, extra in cases:
        b = disks.gravity_disk(n, seed=seed)
        rng = np.random.default_rng(seed)
        ex = (rng.random(n) > hole_frac).astype(np.int32)
        cm = np.array([1e-6, -2e-6, 0.0, 0, 0, 0, 1.0, 1.0])
        params = make_params(softening_parameter=soft, **extra)
        d_b = torch.from_numpy(b).cuda()
        d_ex = torch.from_numpy(ex).cuda()
        acc_s = torch.full((n, 3), np.nan, dtype=torch.float64, device="cuda")
        cma_s = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
        st = lib.ncgpu_vector_field_static(_dev(d_b), _dev(d_ex), n - 1, api.ptr(cm), C.byref(params), _dev(acc_s),
                                           _dev(cma_s), None)
        api.check(st, "ncgpu_vector_field_static")
        torch.cuda.synchronize()

        api.init(n, params)
        acc_d = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        cma_d = torch.zeros(3, dtype=torch.float64, device="cuda")
        st = lib.ncgpu_vector_field_dev(_dev(d_b), _dev(d_ex), n - 1, api.ptr(cm), _dev(acc_d), _dev(cma_d),
                                        api.GRAVITY_EXACT, None)
        api.check(st, "ncgpu_vector_field_dev")
        api.check(lib.ncgpu_check_error(None), "ncgpu_check_error")
        torch.cuda.synchronize()
        api.finalize()

        assert np.array_equal(acc_s.cpu().numpy(), acc_d.cpu().numpy())
        assert np.array_equal(cma_s.cpu().numpy(), cma_d.cpu().numpy())


def test_static_scratch_rejects_oversize(lib):
    from ncorpion_b200 import api
    import torch
    n = 70000  # more slots than the fixed scratch holds
    d = torch.zeros((n, 8), dtype=torch.float64, device="cuda")
    e = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    cma = torch.zeros(3, dtype=torch.float64, device="cuda")
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    st = lib.ncgpu_vector_field_static(_dev(d), _dev(e), n - 1, api.ptr(cm), C.byref(make_params()), _dev(out),
                                       _dev(cma), None)
    assert st == api.E_CAPACITY


FRESH_PROCESS = r'''
import ctypes as C
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from conftest import make_params
from ncorpion_b200 import api, disks

lib = api.load()
n = 4000
b = disks.gravity_disk(n, seed=11)
ex = np.ones(n, np.int32)
ex[::37] = 0
cm = np.array([3e-7, 1e-7, 0.0, 0, 0, 0, 1.0, 1.0])
params = make_params(softening_parameter=0.5)
dev = lambda t: C.c_void_p(t.data_ptr())
d_b = torch.from_numpy(b).cuda()
d_ex = torch.from_numpy(ex).cuda()
outs = [(torch.full((n, 3), np.nan, dtype=torch.float64, device="cuda"),
         torch.full((3,), np.nan, dtype=torch.float64, device="cuda")) for _ in range(3)]
torch.cuda.synchronize()

def static(k):
    st = lib.ncgpu_vector_field_static(dev(d_b), dev(d_ex), n - 1, api.ptr(cm), C.byref(params),
                                       dev(outs[k][0]), dev(outs[k][1]), None)
    api.check(st, "ncgpu_vector_field_static")
    torch.cuda.synchronize()

static(0)                                   # set-up: the library's first call on this device
free_a = torch.cuda.mem_get_info()[0]
static(1)
free_b = torch.cuda.mem_get_info()[0]
assert free_a == free_b, (free_a, free_b)

api.init(n, params)                         # the allocating entry point, for the comparison
acc_d = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
cma_d = torch.zeros(3, dtype=torch.float64, device="cuda")
api.check(lib.ncgpu_vector_field_dev(dev(d_b), dev(d_ex), n - 1, api.ptr(cm), dev(acc_d), dev(cma_d),
                                     api.GRAVITY_EXACT, None), "ncgpu_vector_field_dev")
api.check(lib.ncgpu_check_error(None), "ncgpu_check_error")
api.finalize()
torch.cuda.synchronize()

# a pool allocator takes the device: all but 32 MB of what is free
free = torch.cuda.mem_get_info()[0]
hog = None
for margin in (32, 64, 128, 256):
    try:
        hog = torch.empty(free - (margin << 20), dtype=torch.uint8, device="cuda")
        break
    except RuntimeError:
        torch.cuda.empty_cache()
assert hog is not None
print("left free (MB):", torch.cuda.mem_get_info()[0] >> 20)
static(2)
for k in range(3):
    assert torch.equal(outs[k][0], acc_d) and torch.equal(outs[k][1], cma_d), k
print("fresh-process static calls ok")
'''


def test_static_first_call_in_a_fresh_process(lib):
    env = dict(os.environ)
    env.pop("CUDA_MODULE_LOADING", None)  # CUDA's default: lazy loading
    r = subprocess.run([sys.executable, "-c", FRESH_PROCESS, ROOT], capture_output=True, text=True, timeout=600,
                       env=env)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process static calls ok" in r.stdout
