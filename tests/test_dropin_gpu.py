"""GPU: the drop-in build.  The reference program with its integration
drivers taken from ncorpion_b200/host/rk4_gpu.c on libncgpu.so
(oracle/_ref/<profile>/ncorpion_gpu, see oracle/ref_build.py):

- brute force (bf_merge): the N = 2,000 collisional disk for 200 steps
  (instant mergers, outputs every 50 steps);
- mesh (mesh_prog): a 20,000-body disk with bodies larger than the mesh size,
  100 steps (mesh search with mergers, mesh gravity, adaptive mesh size,
  outputs every 25 steps);
- the mesh driver on 200,000 bodies of the mesh workload's disk, 20 steps
  (mesh_prog_200k; the input is regenerated from its recipe and checked
  against its digest);
- both again with the central body's fluid-body J2 (bf_merge_j2,
  mesh_prog_j2: J2_value 0, Tearth 25), and with tides raised on the central
  body besides (bf_merge_tides, mesh_prog_tides: Delta_t 1), whose rotation
  the output files print.

Every output file (positions, velocities, masses, radii, stat.txt,
collision.txt, readme.txt) and the console output must be byte-identical to
the reference program's own run (golden digests).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu

PROGRAMS = [("bf_merge", "program_bf_merge"), ("mesh_prog", "program_mesh_merge"),
            ("bf_merge_j2", "program_bf_merge_j2"), ("mesh_prog_j2", "program_mesh_merge_j2"),
            ("bf_merge_tides", "program_bf_merge_tides"), ("mesh_prog_tides", "program_mesh_merge_tides"),
            ("mesh_prog_200k", "program_mesh_merge_200k"), ("bf_merge_ell", "program_bf_merge_ell"),
            ("mesh_prog_ell", "program_mesh_merge_ell")]


def _digest(b):
    import hashlib
    return np.frombuffer(hashlib.sha256(b).digest(), np.uint8)


@pytest.mark.parametrize("profile,fixture", PROGRAMS)
def test_dropin_program_matches_reference_outputs(lib, profile, fixture):
    exe = os.path.join(ROOT, "oracle", "_ref", profile, "ncorpion_gpu")
    if not os.path.exists(exe):
        pytest.skip("drop-in build not present (needs the reference sources)")
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import OUTPUT_FILES, filtered_stdout
    from ncorpion_b200 import disks
    g = golden(fixture)
    d = tempfile.mkdtemp(prefix="ncgpu_dropin_")
    if "disk_generator" in g:  # a large input stored as its recipe
        bodies = getattr(disks, str(g["disk_generator"]))(int(g["disk_n"]), seed=int(g["disk_seed"]))
    else:
        bodies = golden(str(g["bodies_from"]))["bodies"] if "bodies_from" in g else g["bodies"]
    disks.write_init_txt(os.path.join(d, "init.txt"), bodies)
    if "digest_init" in g:
        init = open(os.path.join(d, "init.txt"), "rb").read()
        assert np.array_equal(_digest(init), g["digest_init"]), "the regenerated input differs from the fixture's"
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    bad = []
    for f in ([str(x) for x in g["files"]] if "files" in g else OUTPUT_FILES):
        data = open(os.path.join(d, f), "rb").read()
        if not np.array_equal(_digest(data), g["digest_" + f]):
            bad.append(f)
    assert not bad, f"output files differ from the reference run: {bad}"
    assert np.array_equal(_digest(filtered_stdout(r.stdout).encode()), g["digest_stdout"])


RESUMING = [("bf_merge_resume", "program_bf_merge_resume"), ("mesh_prog_resume", "program_mesh_merge_resume"),
            ("mesh_naive_resume", "program_mesh_naive_resume")]


@pytest.mark.parametrize("profile,fixture", RESUMING)
def test_dropin_program_without_outputs_resumes_like_reference(lib, profile, fixture):
    """Both drivers with write_to_files_bool 0 and resume_simulation_bool 1:
    the final half backward drift (brute force) or kick (mesh; in the third
    case below switch_to_brute_force, so brute-force gravity and collisions)
    runs on a device copy of the state, and the resuming files the program
    writes at the end (the final state in init.txt, resume.txt) and the console
    output are byte-identical to the reference program's.  The one exception is
    the radius of a body made by a merger, which resume() prints with 20
    decimals: it may differ in its last bit (the device's correctly rounded
    cube root against glibc's pow), so init.txt's radius column is compared
    within 2 ulp and the rest of the file byte for byte."""
    exe = os.path.join(ROOT, "oracle", "_ref", profile, "ncorpion_gpu")
    if not os.path.exists(exe):
        pytest.skip("drop-in build not present (needs the reference sources)")
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import filtered_stdout, split_radius_column
    from ncorpion_b200 import disks
    g = golden(fixture)
    d = tempfile.mkdtemp(prefix="ncgpu_dropin_")
    disks.write_init_txt(os.path.join(d, "init.txt"), golden(str(g["bodies_from"]))["bodies"])
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    data = open(os.path.join(d, "resume.txt"), "rb").read()
    assert np.array_equal(_digest(data), g["digest_resume.txt"])
    cols, radii = split_radius_column(open(os.path.join(d, "init.txt")).read())
    assert np.array_equal(_digest(cols.encode()), g["digest_init_without_radius"])
    ref = g["init_radius"]
    assert radii.shape == ref.shape
    ulp = np.abs(radii.view(np.int64) - ref.view(np.int64))
    print("init.txt: radii differing from the reference's:", int((ulp > 0).sum()), "max ulp:", int(ulp.max()))
    assert ulp.max() <= 2
    if ulp.max() == 0:
        assert np.array_equal(_digest(open(os.path.join(d, "init.txt"), "rb").read()), g["digest_init.txt"])
    assert np.array_equal(_digest(filtered_stdout(r.stdout).encode()), g["digest_stdout"])
