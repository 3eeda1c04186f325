"""GPU: the drop-in build.  The reference program with its brute-force
integration taken from ncorpion_b200/host/rk4_gpu.c on libncgpu.so
(oracle/_ref/bf_merge/ncorpion_gpu, see oracle/ref_build.py) runs the
N = 2,000 collisional disk for 200 steps (instant mergers, outputs every 50
steps); every output file (positions, velocities, masses, radii, stat.txt,
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

EXE = os.path.join(ROOT, "oracle", "_ref", "bf_merge", "ncorpion_gpu")


def _digest(b):
    import hashlib
    return np.frombuffer(hashlib.sha256(b).digest(), np.uint8)


@pytest.mark.skipif(not os.path.exists(EXE), reason="drop-in build not present (needs the reference sources)")
def test_dropin_program_matches_reference_outputs(lib):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import OUTPUT_FILES, filtered_stdout
    from ncorpion_b200 import disks
    g = golden("program_bf_merge")
    d = tempfile.mkdtemp(prefix="ncgpu_dropin_")
    disks.write_init_txt(os.path.join(d, "init.txt"), g["bodies"])
    r = subprocess.run([EXE], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    bad = []
    for f in OUTPUT_FILES:
        data = open(os.path.join(d, f), "rb").read()
        if not np.array_equal(_digest(data), g["digest_" + f]):
            bad.append(f)
    assert not bad, f"output files differ from the reference run: {bad}"
    assert np.array_equal(_digest(filtered_stdout(r.stdout).encode()), g["digest_stdout"])
