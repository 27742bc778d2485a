"""GPU tests of the tile shapes of the mixed particle-output kernel and of
the autotuner that picks among them.

Every shape must give the same potentials: with the default 1024-source
tile, bit for bit whatever the targets per thread and the dispatch (each
target's operations and their order do not depend on them); with other tile
lengths the FP32 partial sums close at other points, so the results agree
to FP32 rounding and keep the mixed path's accuracy against the FP64 direct
sum.  The autotuner must time all 18 shapes, return the fastest and install
it for later calls and sessions.
"""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs

pytestmark = pytest.mark.gpu

SHAPES = [(tpt, tile, d) for d in (B.DISPATCH_GRID, B.DISPATCH_QUEUE) for tpt in (1, 2, 4)
          for tile in (512, 1024, 2048)]


@pytest.fixture(autouse=True)
def clean_table():
    yield
    for k in (B.Kernel.COULOMB, B.Kernel.YUKAWA, B.Kernel.REGULARIZED_COULOMB):
        for a in (B.Approximation.LAGRANGE, B.Approximation.HERMITE):
            B.tuning_set(None, k, a)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("kernel,kp,approx,degree,sc", [(1, 0.0, 1, 8, 1.0), (2, 0.5, 1, 6, 1.0),
                                                        (3, 1e-3, 1, 7, 1.0), (1, 0.0, 2, 5, 4.0)])
def test_every_shape_gives_the_same_potentials(kernel, kp, approx, degree, sc):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(3, 60000, targets="other")
    kw = dict(kernel=kernel, kernel_param=kp, approximation=approx, theta=0.7, degree=degree,
              max_source_leaf=400, max_target_leaf=400, size_check=sc, precision=B.PRECISION_MIXED)
    ref = B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw)
    idx = np.arange(0, len(tx), 60)
    exact = B.direct(tx[idx], ty[idx], tz[idx], sx, sy, sz, sq, kernel=kernel, kernel_param=kp)
    err_ref = _rel(ref[idx], exact)
    for tpt, tile, disp in SHAPES:
        B.tuning_set({"targets_per_thread": tpt, "source_tile": tile, "dispatch": disp}, kernel, approx)
        out = B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw)
        if tile == 1024:
            assert np.array_equal(out, ref), (tpt, tile, disp)
        else:
            assert _rel(out, ref) < 1e-7, (tpt, tile, disp)
            assert _rel(out[idx], exact) < max(2 * err_ref, 1e-6), (tpt, tile, disp)


def test_autotune_times_every_shape_and_installs_the_fastest():
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(4, 150000)
    kw = dict(kernel=B.Kernel.COULOMB, kernel_param=0.0, approximation=B.Approximation.LAGRANGE, theta=0.7,
              degree=8, max_source_leaf=1000, max_target_leaf=1000, size_check=1.0)
    best, trials = B.autotune([(tx, ty, tz, sx, sy, sz, sq)], **kw)
    assert len(trials) == 18
    assert {(t["targets_per_thread"], t["source_tile"], t["dispatch"]) for t in trials} == set(SHAPES)
    assert all(t["ms"] > 0 for t in trials)
    assert best["ms"] == min(t["ms"] for t in trials)
    shape, installed = B.tuning_get(B.Kernel.COULOMB, B.Approximation.LAGRANGE)
    assert installed and shape == best
    # later calls and sessions use it and stay accurate
    out = B.treecode(tx, ty, tz, sx, sy, sz, sq, precision=B.PRECISION_MIXED, **kw)
    sess = B.Session([(tx, ty, tz, sx, sy, sz, sq)], precision=B.PRECISION_MIXED, **kw)
    (s_out,) = sess.evaluate(sq)
    sess.close()
    assert np.array_equal(out, s_out)
    idx = np.arange(0, len(tx), 150)
    exact = B.direct(tx[idx], ty[idx], tz[idx], sx, sy, sz, sq)
    assert _rel(out[idx], exact) < 1e-6


def test_autotune_on_a_batch_of_systems():
    rng = np.random.default_rng(9)
    systems = []
    for n in (3000, 20000, 70000):
        x, y, z, q = (rng.uniform(0, 1, n) for _ in range(4))
        systems.append((x, y, z, x.copy(), y.copy(), z.copy(), q))
    kw = dict(kernel=B.Kernel.REGULARIZED_COULOMB, kernel_param=1e-3, theta=0.7, degree=7, max_source_leaf=500,
              max_target_leaf=500, size_check=1.0)
    best, trials = B.autotune(systems, **kw)
    assert len(trials) == 18 and best["ms"] > 0
    pots = B.treecode_batch(systems, precision=B.PRECISION_MIXED, **kw)
    for (x, y, z, sx, sy, sz, q), p in zip(systems, pots):
        exact = B.direct(x, y, z, sx, sy, sz, q, kernel=B.Kernel.REGULARIZED_COULOMB, kernel_param=1e-3)
        assert _rel(p, exact) < 1e-6
