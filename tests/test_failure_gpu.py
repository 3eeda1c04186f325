"""GPU: failure paths that end in a status, never in a fault or a hang.

- A device wait that runs out (a barrier nothing completes, bounded like
  every wait in the library) returns NCGPU_E_TIMEOUT, and the next call works.
  One failed probe costs about 7,800 cycles on a B200 (measured), so the
  library's limit of 2^20 probes ends a stuck wait after about four seconds.
- Fragments that would be appended past N_max return NCGPU_E_NMAX (the
  reference prints its N_max message and aborts, src/structure.c:860-863).
- A body count beyond N_max at upload is refused (NCGPU_E_ARG).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden, make_params

pytestmark = pytest.mark.gpu


@pytest.fixture()
def api(lib):
    from ncorpion_b200 import api as A
    yield A
    A.finalize()


def test_bounded_wait_times_out_and_library_stays_usable(api):
    from ncorpion_b200 import disks
    api.init(1024, make_params(softening_parameter=0.5))
    cyc = C.c_double(0.0)
    st = api.load().ncgpu_probe_wait_timeout(4096, C.byref(cyc))
    assert st == api.E_TIMEOUT
    print("cycles per failed barrier probe:", cyc.value)
    assert cyc.value > 0
    b = disks.gravity_disk(512, seed=3)
    acc, cma = api.vector_field(b, np.ones(512, np.int32), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]), mode="exact")
    assert np.all(np.isfinite(acc))


def test_fragments_past_nmax_return_nmax(api):
    g = golden("frag_bf")
    n = len(g["bodies"])
    api.init(n + 2, make_params(collision_bool=1, collision_type=3))
    api.upload(g["bodies"], g["exists"], g["cm"])
    api.set_timestep(float(g["dt"]))
    with pytest.raises(api.NcgpuError) as e:
        api.collide_brute()
    assert e.value.status == api.E_NMAX


def test_upload_beyond_nmax_is_refused(api):
    from ncorpion_b200 import disks
    api.init(100, make_params())
    b = disks.gravity_disk(200, seed=1)
    with pytest.raises(api.NcgpuError) as e:
        api.upload(b, np.ones(200, np.int32), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]))
    assert e.value.status == api.E_ARG
