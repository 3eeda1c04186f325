"""The device's sequential FP64 sums against the plain loop, through the C ABI:
the staged one-add-at-a-time loop (total_momentum, src/structure.c:1193-1227;
the central body's acceleration, src/physics.c:137-139; the mesh's chains) and
the routine that takes whole runs of terms at once while the running sum stays
in one binade (display()'s total mass, src/display.c:352).

For the second, the cases aim at the places where that could go wrong: binade
changes up and down, ties (terms that are odd multiples of half the sum's
spacing), a sum that is an exact power of two, sign changes, zeros, subnormal
and huge values, infinities and NaNs, and sizes that end inside a window.
Tolerance: bit-identical to numpy's add.accumulate (a strictly sequential
loop), NaN payloads aside.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plain(x, s0):
    return np.add.accumulate(np.concatenate([[s0], x]))[-1] if len(x) else np.float64(s0)


def _device(lib, api, chains, s0, runs=1):
    n = len(chains[0])
    x = np.ascontiguousarray(np.concatenate(chains)) if n else np.zeros(1)
    s = np.ascontiguousarray(s0, dtype=np.float64)
    out = np.empty(len(chains))
    api.check(lib.ncgpu_probe_seq_sum(api.ptr(x), n, api.ptr(s), api.ptr(out), len(chains), runs),
              "ncgpu_probe_seq_sum")
    return out


def _same(a, b):
    return a.view(np.int64) == b.view(np.int64) or (np.isnan(a) and np.isnan(b))


def _cases(rng, n):
    U = lambda: rng.uniform(0.0, 1.0, n)
    N = lambda: rng.standard_normal(n)
    k = np.arange(n)
    return [
        ("masses", 1e-9 * (0.5 + U()), 0.0),
        ("masses from a body", 1e-9 * U(), 1.0),
        ("signed walk", N(), 0.0),
        ("signed walk, offset", N(), 100.0 * rng.standard_normal()),
        ("cauchy", rng.standard_cauchy(n), 0.0),
        ("drift", 1e-3 * N() + 1e-5, 0.3),
        ("dyadic", np.ldexp(rng.integers(0, 64, n).astype(float), -rng.integers(0, 60, n)), 1.0),
        ("dyadic signed", np.ldexp(rng.integers(-32, 32, n).astype(float), -rng.integers(0, 60, n)), 8.0),
        ("ties near 1", np.ldexp(rng.integers(-4, 4, n).astype(float), -52 + rng.integers(0, 4, n)), 1.0),
        ("ties near -1", np.ldexp(rng.integers(-4, 4, n).astype(float), -53), -1.0),
        ("tiny on a power of two", np.where(k % 3 == 0, 0.0, np.ldexp(U(), -70)), 1.0),
        ("tiny below a power of two", -np.ldexp(U(), -70), 1.0),
        ("tiny on minus a power of two", np.ldexp(U(), -70), -1.0),
        ("half spacings below", np.full(n, -2.0 ** -54), 1.0),
        ("equal", np.full(n, 1.0 / 3.0), 0.0),
        ("alternating", np.where(k % 2 == 1, -1.0, 1.0) * (1.0 + k * 1e-3), 0.0),
        ("wide", N() * np.ldexp(1.0, rng.integers(-100, 100, n)), 0.0),
        ("signed zeros", np.where(k % 2 == 1, -0.0, 0.0), -0.0),
        ("subnormal", np.ldexp(N(), -1060), 0.0),
        ("low range", np.ldexp(N(), -960), 2.0 ** -955),
        ("huge", np.ldexp(U(), 1000), 0.0),
        ("overflow", np.ldexp(U(), 1015), 2.0 ** 1020),
    ]


@pytest.mark.parametrize("runs", [1, 0])
@pytest.mark.parametrize("n", [0, 1, 31, 1000, 1024, 1025, 5000, 33_000])
def test_seq_sum_matches_the_plain_loop(lib, n, runs):
    from ncorpion_b200 import api
    rng = np.random.default_rng(n + 11)
    cases = _cases(rng, n)
    if n >= 4:
        x = rng.standard_normal(n)
        x[rng.integers(0, n)] = np.inf
        cases.append(("inf", x.copy(), 0.0))
        x[rng.integers(0, n)] = -np.inf
        cases.append(("inf and -inf", x.copy(), 0.0))
        x = rng.standard_normal(n)
        x[rng.integers(0, n)] = np.nan
        cases.append(("nan", x, 0.0))
    with np.errstate(over="ignore", invalid="ignore"):
        want = [_plain(x, s0) for _, x, s0 in cases]
        got = _device(lib, api, [x for _, x, _ in cases], [s0 for _, _, s0 in cases], runs)
    bad = [name for (name, _, _), w, g in zip(cases, want, got) if not _same(w, g)]
    assert not bad, bad


@pytest.mark.parametrize("runs", [1, 0])
def test_seq_sum_long_chains(lib, runs):
    """Chains of 2^20 terms, the mesh workload's size, in the shapes its sums
    take: positive masses, a zero-mean walk (the central body's acceleration
    from a symmetric disk), heavy-tailed terms (a moonlet's acceleration)."""
    from ncorpion_b200 import api
    rng = np.random.default_rng(5)
    n = 1 << 20
    chains = [1e-9 * (0.5 + rng.uniform(0, 1, n)), 1e-3 * rng.standard_normal(n),
              1e-3 * rng.standard_cauchy(n), 1e-3 * rng.standard_normal(n) + 1e-6]
    s0 = [0.0, 0.0, 0.0, 0.25]
    want = [_plain(x, s) for x, s in zip(chains, s0)]
    got = _device(lib, api, chains, s0, runs)
    assert all(_same(w, g) for w, g in zip(want, got))
