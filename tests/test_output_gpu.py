"""GPU: output staging (ncgpu_snapshot_begin/end, ncgpu_format_cartesian,
ncgpu_output_stats) against the reference's display() semantics.

- every value's text is "%.14lf " as glibc prints it: the exact decimal of the
  double rounded to 14 digits, ties to even (Python's %-formatting is the same
  correctly rounded conversion), for random values, exact ties, signed zeros,
  subnormals, large values and infinities;
- the central body comes first in the x..vz files, mass and radius list the
  bodies only, holes are skipped;
- the statistics follow display()'s loop (total mass summed in slot order, the
  first most massive body, then the first most massive of the others);
- a snapshot leaves the bodies untouched and carries SideralOmega over.
The whole-program tests (test_dropin_gpu.py) check the files byte for byte.
"""
import numpy as np
import pytest

from conftest import make_params

pytestmark = pytest.mark.gpu


def _fmt(v):
    return "%.14f " % v


@pytest.fixture()
def gpu(lib):
    from ncorpion_b200 import api

    def _init(n_max, **kw):
        api.init(n_max, make_params(**kw))
        return api

    yield _init
    api.finalize()


def test_format_cartesian_matches_printf(gpu):
    rng = np.random.default_rng(3)
    n = 20000
    b = np.empty((n, 8))
    b[:, :6] = rng.standard_normal((n, 6)) * np.exp2(rng.integers(-40, 20, (n, 6)).astype(np.float64))
    b[:, 6] = np.exp(rng.uniform(np.log(1e-12), 0.0, n))
    b[:, 7] = rng.uniform(1e-6, 1e-2, n)
    special = [0.0, -0.0, 5e-324, -5e-324, 1.0 / 32768, 3.0 / 32768, -5.0 / 32768, 0.5e-14, 1e-14, 123456.789,
               -98765.4321, 2.0 ** 60, -(2.0 ** 70), 1.7e24, np.inf, -np.inf, 0.999999999999995, 9.999999999999995]
    b[:len(special), 0] = special
    b[:len(special), 3] = special[::-1]
    ex = (rng.random(n) > 0.02).astype(np.int32)
    ex[:len(special)] = 1
    cm = np.array([1e-6, -2e-7, 3e-9, 4e-8, -5e-8, 6e-8, 1.25, 1.0])
    api = gpu(n + 10)
    api.upload(b, ex, cm)
    files = api.format_cartesian()
    live = np.flatnonzero(ex)
    for f in range(6):
        want = _fmt(cm[f]) + "".join(_fmt(v) for v in b[live, f])
        assert files[f] == want, f"file {f}"
    assert files[6] == "".join(_fmt(v) for v in b[live, 6])
    assert files[7] == "".join(_fmt(v) for v in b[live, 7])


def test_format_rejects_out_of_range(gpu):
    from ncorpion_b200 import api as A
    b = np.zeros((3, 8))
    b[:, 6] = 1e-9
    b[1, 0] = 1e30  # beyond the formatter's 128-bit range
    api = gpu(8)
    api.upload(b, np.ones(3, np.int32), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]))
    with pytest.raises(A.NcgpuError) as e:
        api.format_cartesian()
    assert e.value.status == A.E_UNSUPPORTED
    b[1, 0] = 1.0
    api.upload(b, np.ones(3, np.int32), np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]))
    assert len(api.format_cartesian()) == 8  # and the library goes on


def _display_stats(b, ex):
    """display()'s loop (src/display.c:321-371) in Python floats."""
    total, M1, M2, i1, i2 = 0.0, 0.0, 0.0, 0, 0
    for p in range(b.shape[0]):
        if not ex[p]:
            continue
        m = float(b[p, 6])
        total += m
        if m > M1:
            M2, i2, M1, i1 = M1, i1, m, p
        elif m > M2:
            M2, i2 = m, p
    return total, M1, M2, i1, i2


@pytest.mark.parametrize("case", ["random", "ties", "one", "none"])
def test_output_stats_follow_display(gpu, case):
    rng = np.random.default_rng(7)
    n = 5000
    b = rng.standard_normal((n, 8))
    b[:, 6] = rng.uniform(1e-9, 1e-6, n)
    ex = (rng.random(n) > 0.1).astype(np.int32)
    if case == "ties":
        b[:, 6] = np.round(b[:, 6] * 1e7) * 1e-7  # many equal masses
        b[[17, 3000, 4500], 6] = 5e-6
    elif case == "one":
        ex[:] = 0
        ex[1234] = 1
    elif case == "none":
        ex[:] = 0
    api = gpu(n + 10)
    api.upload(b, ex, np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0]))
    stats, idx, cm, two = api.output_stats()
    total, M1, M2, i1, i2 = _display_stats(b, ex)
    assert stats[0] == total and stats[1] == M1 and stats[2] == M2
    assert (idx[0], idx[1]) == (i1, i2)
    assert np.array_equal(two[0], b[i1]) and np.array_equal(two[1], b[i2])


def test_snapshot_leaves_the_bodies(gpu):
    from ncorpion_b200 import disks
    n = 3000
    b = disks.gravity_disk(n, seed=2)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    api = gpu(n + 10, softening_parameter=0.5, central_tides_bool=1, Delta_t=1.0)
    api.upload(b, ex, cm)
    api.set_timestep(1e-3)
    api.kick()
    before = api.download(n + 10)
    w0 = api.get_sideral_omega()
    api.snapshot_begin()
    api.set_timestep(-5e-4)
    api.kick()  # the copy's tides change the rotation
    api.drift()
    copy = api.download(n + 10)
    w1 = api.get_sideral_omega()
    api.snapshot_end()
    after = api.download(n + 10)
    assert not np.array_equal(copy[0], before[0])
    assert np.array_equal(after[0], before[0]) and np.array_equal(after[2], before[2])
    assert w1 != w0 and api.get_sideral_omega() == w1


# ---- elliptic files (cart2ell, src/structure.c:172-284) ---------------------

def _fmt_c(v):
    """glibc's "%.14lf " of v, NaNs with their signs."""
    if np.isnan(v):
        return "-nan " if np.signbit(v) else "nan "
    return _fmt(v)


def _elliptic_on_device(api, port, b, ex, cm, params, j2, mass_radius):
    """Both halves of the device's elliptic output, the caller's part done as
    the drop-in does it: atan2 by the C library (ncgpu_host_atan2), the listed
    bodies through cart2ell (the oracle's, pinned to the reference's)."""
    mu = 1.0 * cm[6]
    yx, hidx, hrec = api.elliptic_begin(mu)
    F = api.host_atan2(yx)
    alk = np.array([port.cart2ell(r, cm, mu + 1.0 * r[6], params, j2)[0] for r in hrec]).reshape(-1, 6)
    return yx, hidx, hrec, F, alk


@pytest.mark.parametrize("at_rest,j2", [(False, 0.0), (True, 0.0), (False, 0.0125)])
def test_format_elliptic_matches_cart2ell_and_printf(gpu, port, capfd, at_rest, j2):
    """The six elliptic files (and mass, radius) against the oracle's cart2ell
    of every existing body, text for text; the bodies the device lists are
    exactly those cart2ell takes out of the elliptic branch (hyperbolic, its
    (k, h) warning, NaNs), in slot order, and converting them prints the
    reference's warnings as display()'s loop would."""
    from conftest import elliptic_cases
    b, ex, cm = elliptic_cases(3000, seed=6, cm_at_rest=at_rest)
    params = dict(J2_bool=1, J2=j2) if j2 else {}
    api = gpu(4000, **params)
    p = make_params(**params)
    api.upload(b, ex, cm)
    assert api.get_j2() == j2
    capfd.readouterr()
    yx, hidx, hrec, F, alk = _elliptic_on_device(api, port, b, ex, cm, p, j2, True)
    printed = capfd.readouterr().out
    files = api.format_elliptic(F, alk, mass_radius=True)
    live = np.flatnonzero(ex)
    want = port.cart2ell_all(b, ex, cm, 1.0 * cm[6], p, j2)
    want_printed = capfd.readouterr().out
    assert printed == want_printed and printed.count("Warning") >= 3
    for f in range(6):
        assert files[f] == "".join(_fmt_c(v) for v in want[f]), f"file {f}"
    assert files[6] == "".join(_fmt(v) for v in b[live, 6])
    assert files[7] == "".join(_fmt(v) for v in b[live, 7])
    # the listed bodies: slots ascending, records as uploaded
    assert np.all(np.diff(hidx) > 0) and np.array_equal(hrec, b[hidx])
    expect = []
    for i in live:
        a, warned = port.cart2ell(b[i], cm, 1.0 * cm[6] + 1.0 * b[i, 6], p, j2)
        if warned or np.isnan(a).any() or a[0] < 0:
            expect.append(i)
    capfd.readouterr()
    hyp_or_nan = set(expect)
    assert hyp_or_nan <= set(hidx.tolist())
    assert len(hidx) >= 30 and len(hidx) < len(live) // 10
    # a second format call gives the same texts; values agree with the texts' numbers
    assert api.format_elliptic(F, alk, mass_radius=False) == files[:6]
    v = api.elliptic_values(len(live))
    assert np.array_equal(v[:6].view(np.int64), want.view(np.int64))
    assert np.array_equal(v[6], b[live, 6]) and np.array_equal(v[7], b[live, 7])


def test_format_elliptic_out_of_range_values(gpu, port):
    """A value beyond the formatter's range (a = R / 2 = 5e29 for a far body at
    rest): NCGPU_E_UNSUPPORTED, and the values are there for the caller to
    print, equal to cart2ell's."""
    from ncorpion_b200 import api as A
    from conftest import elliptic_cases
    b, ex, cm = elliptic_cases(200, seed=7)
    b[6, :3] = cm[:3] + np.array([1e30, 0.0, 0.0])
    b[6, 3:6] = cm[3:6]
    api = gpu(256)
    p = make_params()
    api.upload(b, ex, cm)
    yx, hidx, hrec, F, alk = _elliptic_on_device(api, port, b, ex, cm, p, 0.0, False)
    with pytest.raises(A.NcgpuError) as e:
        api.format_elliptic(F, alk)
    assert e.value.status == A.E_UNSUPPORTED
    live = np.flatnonzero(ex)
    v = api.elliptic_values(len(live))
    want = port.cart2ell_all(b, ex, cm, 1.0, p, 0.0)
    assert np.array_equal(v[:6].view(np.int64), want.view(np.int64))
    assert v[0, 6] == 5e29


def test_elliptic_state_rules(gpu):
    """format_elliptic needs a begin first and the same listed-body count."""
    from ncorpion_b200 import api as A
    from conftest import elliptic_cases
    b, ex, cm = elliptic_cases(100, seed=8)
    api = gpu(128)
    api.upload(b, ex, cm)
    with pytest.raises(A.NcgpuError) as e:
        api.format_elliptic(np.zeros(int(ex.sum())), np.zeros((0, 6)))
    assert e.value.status == A.E_STATE
    yx, hidx, hrec = api.elliptic_begin(1.0)
    assert len(hidx) > 0
    with pytest.raises(A.NcgpuError) as e:
        api.format_elliptic(np.zeros(len(yx)), np.zeros((0, 6)))
    assert e.value.status == A.E_ARG
