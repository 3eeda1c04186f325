"""bench.py's clock sampler (host logic, no GPU): a stand-in nvidia-smi on
PATH prints samples after a start-up delay longer than a short timed region.
The sampler must hold one sample from before the region and one from after
it, report the median SM clock and the throttle reasons that were active,
and say so when nvidia-smi is missing."""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

FAKE = """#!{py}
import sys, time
time.sleep(0.3)
i = 0
while True:
    cap = "Active" if i == 1 else "Not Active"
    print("0, %d, 1965, 700.00, 0x4, Not Active, Not Active, Not Active, %s" % (1965 - 10 * (i % 2), cap), flush=True)
    i += 1
    time.sleep(0.05)
"""


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_samples_bracket_a_short_region(tmp_path, monkeypatch):
    fake = tmp_path / "nvidia-smi"
    fake.write_text(FAKE.format(py=sys.executable))
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ.get("PATH", ""))
    bench = _bench()
    cs = bench.ClockSampler(0)
    cs.start()
    n_before = len(cs.lines)
    time.sleep(0.01)  # a timed region far shorter than nvidia-smi's start-up
    out = cs.stop()
    assert n_before >= 1
    assert out["samples"] >= 2
    assert out["sm_max_mhz"] == 1965.0
    assert 1955.0 <= out["sm_mhz"] <= 1965.0
    assert set(out["reasons"]) <= {"sw_power_cap"}


def test_missing_nvidia_smi_is_reported(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    bench = _bench()
    cs = bench.ClockSampler(0)
    cs.start()
    out = cs.stop()
    assert out["sm_mhz"] is None and out["reasons"] == ["nvidia-smi unavailable"]
