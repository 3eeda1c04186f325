"""The falcON oracle (the reference's default gravity module, src/ffm.c; Dehnen
2002), pinned on CPU: the reference's tree code compiled from source
(oracle/_ref/tree_grav, expansion order 3, theta_min 0.45) and the golden
fixture it wrote (tests/golden/tree_n4096.npz).

falcON's field is an approximation of the exact one, so the checks are its
accuracy against the exact brute-force field of the same state (bit-pinned to
the reference's vector_field elsewhere) and the properties the method keeps:
each cell-cell interaction is symmetric, so the total momentum change equals
the exact field's to rounding; bodies that do not exist get nothing; the same
state, with the bodies entering the tree in slot order (a run's first tree),
gives the same bits.  Tolerances (measured: median 2.2e-3, 99th
percentile 3.7e-2, worst error 1.9e-3 of the RMS mutual acceleration): median
relative error of the mutual part below 5e-3, 99th percentile below 0.08,
worst absolute error below 5e-3 of the RMS mutual acceleration.
"""
import numpy as np
import pytest

import oracle
from conftest import golden


def _mutual(bodies, exists):
    """The exact mutual part by numpy (G = 1), for the error scale."""
    x, m = bodies[:, :3], np.where(exists.astype(bool), bodies[:, 6], 0.0)
    out = np.zeros_like(x)
    for lo in range(0, len(x), 512):
        d = x[None, :, :] - x[lo:lo + 512, None, :]
        r2 = (d * d).sum(-1)
        np.fill_diagonal(r2[:, lo:lo + 512], np.inf)
        out[lo:lo + 512] = (m[None, :, None] * d / r2[..., None] ** 1.5).sum(1)
    return out


def test_falcon_fixture_accuracy():
    g = golden("tree_n4096")
    ex = g["exists"].astype(bool)
    mut = _mutual(g["bodies"], g["exists"])[ex]
    err = np.linalg.norm((g["acc"] - g["acc_exact"])[ex], axis=1)
    rel = err / np.linalg.norm(mut, axis=1)
    rms = np.sqrt((mut * mut).sum(1).mean())
    assert np.median(rel) < 5e-3
    assert np.percentile(rel, 99) < 0.08
    assert err.max() < 5e-3 * rms
    assert int(g["cells"]) > 1


def test_falcon_fixture_momentum_and_holes():
    g = golden("tree_n4096")
    ex = g["exists"].astype(bool)
    m = g["bodies"][ex, 6][:, None]
    diff = (m * (g["acc"] - g["acc_exact"])[ex]).sum(0)
    scale = np.abs(m * _mutual(g["bodies"], g["exists"])[ex]).sum(0)
    assert np.all(np.abs(diff) < 1e-12 * scale)
    assert np.all(g["acc"][~ex] == 0.0)
    np.testing.assert_array_equal(g["cm_acc"], g["cm_acc_exact"])


@pytest.mark.skipif(not oracle.ref_available("tree_grav"), reason="reference not built here")
def test_falcon_reference_reproduces_fixture():
    g = golden("tree_n4096")
    ref = oracle.Ref("tree_grav")
    ref.set_state(g["bodies"], g["exists"], g["cm"])
    acc, cma, cells = ref.tree_field()
    assert cells == int(g["cells"])
    assert np.array_equal(acc.view(np.int64), g["acc"].view(np.int64))
    acc2, _, _ = ref.tree_field()
    assert np.array_equal(acc2.view(np.int64), acc.view(np.int64))
    # a later tree of a run inserts the bodies in the previous tree's
    # Peano-Hilbert order: the leaves' sums change order, the field by ulps
    acc3, _, _ = ref.tree_field(slot_order=False)
    ex = g["exists"].astype(bool)
    scale = np.abs(g["acc"][ex]).max()
    assert np.abs(acc3 - acc)[ex].max() < 1e-14 * scale
