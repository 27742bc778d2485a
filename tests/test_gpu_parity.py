"""GPU parity of the FP64 path against the oracle and the reference.

Bar (FP64 plain path): norm-wise relative L2 difference <= 1e-12 and
per-target |difference| <= 1e-12 * max|phi| against the CPU FP64 oracle and
against the reference's own outputs (golden fixtures).  The known-answer cases
of the reference's tests run through the product with the reference's
tolerances.  All calls go through the C ABI (libbarytree_b200.so).
"""
import numpy as np
import pytest

import barytree_b200 as B
import refcases as R
from conftest import golden_files, uniform_inputs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-12
TOL_MAX = 1e-12


def _product(tx, ty, tz, sx, sy, sz, sq, kernel, kp, approx, ctype, theta, degree, ls, lt, sc, beta=-1.0):
    return B.callTreedriver(len(tx), len(sx), tx, ty, tz, None, sx, sy, sz, sq, None, kernel, 1, np.array([kp]),
                            B.Singularity.SKIPPING, approx, ctype, True, 0, beta=beta if beta >= 0 else None,
                            theta=theta, degree=degree, sourceLeafSize=ls, targetLeafSize=lt, sizeCheck=sc)


def _oracle(tx, ty, tz, sx, sy, sz, sq, kernel, kp, approx, ctype, theta, degree, ls, lt, sc, beta=-1.0):
    return O.treecode(tx, ty, tz, None, sx, sy, sz, sq, None, kernel, [kp], 1, approx, ctype, theta, degree,
                      ls, lt, sc, beta, 0)


def _close(a, b):
    scale = np.max(np.abs(b)) if len(b) else 1.0
    l2 = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
    assert l2 <= TOL_L2, f"rel-L2 {l2:.3e}"
    assert np.max(np.abs(a - b)) <= TOL_MAX * scale, f"max {np.max(np.abs(a - b)) / scale:.3e}"


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("/")[-1][:-4])
def test_matches_reference_golden(path):
    g = np.load(path)
    k, kp, ap, ct, th, deg, ls, lt, sc = g["params"]
    launches = B.kernel_launch_count()
    pot = _product(g["tx"], g["ty"], g["tz"], g["sx"], g["sy"], g["sz"], g["sq"], int(k), kp, int(ap), int(ct),
                   th, int(deg), int(ls), int(lt), sc)
    assert B.kernel_launch_count() > launches          # the CUDA path ran
    _close(pot, g["potential"])


@pytest.mark.parametrize("ctype,approx", [(1, 1), (1, 2), (2, 1), (2, 2), (3, 1)])
@pytest.mark.parametrize("kernel,kp", [(1, 0.0), (2, 0.5), (3, 1e-3)])
@pytest.mark.parametrize("degree", [2, 7])
def test_matches_oracle_random(ctype, approx, kernel, kp, degree):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(degree * 10 + kernel, 6000, targets="other")
    sc = 4.0 if approx == 2 else 1.0
    args = (tx, ty, tz, sx, sy, sz, sq, kernel, kp, approx, ctype, 0.7, degree, 160, 110, sc)
    _close(_product(*args), _oracle(*args))


@pytest.mark.parametrize("ctype", [1, 2, 3])
def test_degree_12_and_targets_equal_sources(ctype):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(21, 12000, targets="same")
    args = (tx, ty, tz, sx, sy, sz, sq, 1, 0.0, 1, ctype, 0.8, 12, 800, 800, 1.0)
    _close(_product(*args), _oracle(*args))


@pytest.mark.parametrize("ctype,approx", [(1, 1), (1, 2), (2, 1), (2, 2), (3, 1)])
def test_lattice_exact_node_coincidence(ctype, approx):
    """Particles on a lattice coincide with Chebyshev nodes (the |d| < DBL_MIN rule)."""
    g = np.arange(12, dtype=float)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x, y, z = X.ravel().copy(), Y.ravel().copy(), Z.ravel().copy()
    q = np.cos(np.arange(len(x)) * 0.37)
    args = (x.copy(), y.copy(), z.copy(), x, y, z, q, 1, 0.0, approx, ctype, 0.7, 2, 20, 20,
            4.0 if approx == 2 else 1.0)
    _close(_product(*args), _oracle(*args))


def test_beta_path():
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(3, 3000)
    for ctype in (1, 2, 3):
        args = (tx, ty, tz, sx, sy, sz, sq, 2, 0.5, 1, ctype, -1.0, -1, 1, 1, 1.0, 0.3)
        _close(_product(*args), _oracle(*args))


@pytest.mark.parametrize("n_t,n_s", [(1, 5000), (5000, 1), (3, 3), (1, 1)])
def test_tiny_and_ragged(n_t, n_s):
    rng = np.random.default_rng(n_t * 7 + n_s)
    tx, ty, tz = (rng.uniform(-1, 1, n_t) for _ in range(3))
    sx, sy, sz, sq = (rng.uniform(-1, 1, n_s) for _ in range(4))
    for ctype in (1, 2, 3):
        args = (tx, ty, tz, sx, sy, sz, sq, 1, 0.0, 1, ctype, 0.7, 3, 50, 50, 1.0)
        _close(_product(*args), _oracle(*args))


def test_empty_inputs():
    t = np.zeros(0)
    s = np.ones(10)
    out = _product(t, t, t, s, s, s, s, 1, 0.0, 1, 1, 0.7, 3, 5, 5, 1.0)
    assert len(out) == 0
    tx = np.ones(4)
    out = _product(tx, tx, tx, t, t, t, t, 1, 0.0, 1, 1, 0.7, 3, 5, 5, 1.0)
    assert np.all(out == 0.0)


@pytest.mark.parametrize("kernel,approx,tol", R.LATTICE100_CASES)
def test_reference_lattice100(kernel, approx, tol):
    x, y, z, q = R.lattice(100)
    pot = _product(x.copy(), y.copy(), z.copy(), x, y, z, q, kernel, 0.5, approx, 1, 0.7, 2, 3, 3, 1.0)
    true = R.lattice_closed_form(100, kernel)
    assert np.all(np.abs(pot - true) / np.abs(true) < tol)


@pytest.mark.parametrize("kernel,approx,tol", R.ONE_TARGET_CASES)
def test_reference_one_target(kernel, approx, tol):
    tx, ty, tz, sx, sy, sz, sq = R.one_target_sources()
    pot = _product(tx, ty, tz, sx, sy, sz, sq, kernel, 0.5, approx, 1, 0.8, 4, 100, 100, 0.0)
    d = O.direct(tx, ty, tz, sx, sy, sz, sq, kernel, 0.5)
    assert abs(pot[0] - d[0]) / abs(d[0]) < tol


def test_reference_bldtt():
    tx, ty, tz, sx, sy, sz, sq = R.bldtt_inputs()
    pot = _product(tx, ty, tz, sx, sy, sz, sq, 1, 0.5, 1, 3, 0.9, 3, 20, 20, 1.0)
    d = O.direct(tx, ty, tz, sx, sy, sz, sq, 1, 0.5)
    assert abs(pot.sum() - d.sum()) / abs(d.sum()) < 6e-3


@pytest.mark.parametrize("kernel,kp", [(1, 0.0), (2, 0.5), (3, 1e-3)])
def test_gpu_direct_matches_oracle(kernel, kp):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(5, 3000, targets="same")
    a = B.direct(tx, ty, tz, sx, sy, sz, sq, kernel, kp)
    b = O.direct(tx, ty, tz, sx, sy, sz, sq, kernel, kp)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13


def test_deterministic():
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(8, 20000)
    for ctype in (1, 3):
        args = (tx, ty, tz, sx, sy, sz, sq, 1, 0.0, 1, ctype, 0.7, 6, 500, 500, 1.0)
        a = _product(*args)
        b = _product(*args)
        assert np.array_equal(a, b)


def test_inputs_not_modified():
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(12, 2000, targets="other")
    keep = [a.copy() for a in (tx, ty, tz, sx, sy, sz, sq)]
    _product(tx, ty, tz, sx, sy, sz, sq, 1, 0.0, 1, 3, 0.7, 4, 50, 50, 1.0)
    for a, b in zip((tx, ty, tz, sx, sy, sz, sq), keep):
        assert np.array_equal(a, b)


def test_accuracy_vs_direct_config1_shape():
    """Config-1 shape at 1/5 size: PC Coulomb Lagrange n=8, theta 0.7, leaf 2000."""
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(0, 20000)
    pot = _product(tx, ty, tz, sx, sy, sz, sq, 1, 0.0, 1, 1, 0.7, 8, 2000, 2000, 1.0)
    d = B.direct(tx, ty, tz, sx, sy, sz, sq, 1, 0.0)
    assert np.linalg.norm(pot - d) / np.linalg.norm(d) < 1e-6
