"""GPU accuracy of the mixed-precision path.

Mixed precision evaluates PP/PC/CP/M2L in FP32 on centre-relative
coordinates with FP64 reductions.  Bar: relative L2 difference from the FP64
treecode <= 5e-7 (FP32 rounding of leaf-centre-relative displacements, about
6e-8 of the leaf half-width, and of the proxy charges; measured 2.9e-7 for
Coulomb PC at N=30,000), and relative L2 error against the FP64 direct sum
within the 1e-6 tolerance at degree 8.
"""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs

pytestmark = pytest.mark.gpu

TOL_VS_FP64_TREE = 5e-7
TOL_VS_FP64_TREE_YUKAWA = 1e-6   # ex2.approx and the FP32 exponent argument add ~3e-7 (measured 6.9e-7)
TOL_VS_DIRECT = 1e-6


def _run(args, precision):
    tx, ty, tz, sx, sy, sz, sq, kernel, kp, ctype, degree, leaf = args
    return B.treecode(tx, ty, tz, sx, sy, sz, sq, kernel=kernel, kernel_param=kp, compute_type=ctype, theta=0.7,
                      degree=degree, max_source_leaf=leaf, max_target_leaf=leaf, precision=precision)


@pytest.mark.parametrize("ctype", [1, 2, 3])
@pytest.mark.parametrize("kernel,kp", [(1, 0.0), (2, 0.5), (3, 1e-3)])
def test_mixed_matches_fp64_tree(ctype, kernel, kp):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(31 + kernel, 30000, targets="other")
    args = (tx, ty, tz, sx, sy, sz, sq, kernel, kp, ctype, 6, 400)
    a = _run(args, B.PRECISION_MIXED)
    b = _run(args, B.PRECISION_FP64)
    err = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert err <= (TOL_VS_FP64_TREE_YUKAWA if kernel == 2 else TOL_VS_FP64_TREE), err


@pytest.mark.parametrize("ctype", [1, 3])
def test_mixed_vs_direct_degree8(ctype):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(2, 60000)
    pot = _run((tx, ty, tz, sx, sy, sz, sq, 1, 0.0, ctype, 8, 1000), B.PRECISION_MIXED)
    idx = np.arange(0, len(tx), 7)
    d = B.direct(tx[idx], ty[idx], tz[idx], sx, sy, sz, sq)
    assert np.linalg.norm(pot[idx] - d) / np.linalg.norm(d) <= TOL_VS_DIRECT


@pytest.mark.parametrize("kernel,kp", [(1, 0.0), (2, 0.5), (3, 1e-3)])
def test_mixed_hermite_particle_cluster(kernel, kp):
    """Hermite PC in mixed precision (FP32 over the 8 moments, FP64 upward
    pass) against the FP64 Hermite treecode, and against the direct sum."""
    rng = np.random.default_rng(40 + kernel)
    n = 40000
    x, y, z = (np.clip(rng.normal(0, 0.25, n), -1, 1) for _ in range(3))
    q = rng.choice([-1.0, 1.0], n)
    kw = dict(kernel=kernel, kernel_param=kp, approximation=2, degree=6, max_source_leaf=1000, max_target_leaf=1000,
              size_check=4.0)
    a = B.treecode(x, y, z, x, y, z, q, precision=B.PRECISION_MIXED, **kw)
    b = B.treecode(x, y, z, x, y, z, q, precision=B.PRECISION_FP64, **kw)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= (TOL_VS_FP64_TREE_YUKAWA if kernel == 2 else TOL_VS_FP64_TREE)
    idx = np.arange(0, n, 13)
    d = B.direct(x[idx], y[idx], z[idx], x, y, z, q, kernel, kp)
    assert np.linalg.norm(a[idx] - d) / np.linalg.norm(d) <= TOL_VS_DIRECT


def test_mixed_hermite_grid_outputs_run_in_fp64():
    """Hermite cluster-particle has no FP32 kernels: the mixed option
    evaluates it with the FP64 kernels, bit for bit."""
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(4, 8000)
    a = B.treecode(tx, ty, tz, sx, sy, sz, sq, approximation=2, compute_type=2, degree=4, max_source_leaf=200,
                   max_target_leaf=200, size_check=4.0, precision=B.PRECISION_MIXED)
    b = B.treecode(tx, ty, tz, sx, sy, sz, sq, approximation=2, compute_type=2, degree=4, max_source_leaf=200,
                   max_target_leaf=200, size_check=4.0, precision=B.PRECISION_FP64)
    assert np.array_equal(a, b)


def test_mixed_close_pairs():
    """Pairs far closer than the leaf size (1e-6 .. 1e-9 apart) dominate their
    targets' potentials; the near field recomputes such displacements from the
    FP64 coordinates, so the mixed result stays within the FP64 treecode's
    bar for these targets too."""
    rng = np.random.default_rng(13)
    n = 40000
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    k = 200
    sep = 10.0 ** rng.uniform(-9, -6, k)
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    x[1:2 * k:2] = x[0:2 * k:2] + sep * d[:, 0]
    y[1:2 * k:2] = y[0:2 * k:2] + sep * d[:, 1]
    z[1:2 * k:2] = z[0:2 * k:2] + sep * d[:, 2]
    q = rng.uniform(-1, 1, n)
    a = B.treecode(x, y, z, x, y, z, q, degree=8, max_source_leaf=500, max_target_leaf=500,
                   precision=B.PRECISION_MIXED)
    b = B.treecode(x, y, z, x, y, z, q, degree=8, max_source_leaf=500, max_target_leaf=500,
                   precision=B.PRECISION_FP64)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= TOL_VS_FP64_TREE
    pair = np.arange(2 * k)                 # these targets' potentials are dominated by the close pair
    assert np.max(np.abs(a[pair] - b[pair]) / np.abs(b[pair])) <= 1e-6


def test_mixed_coincident_points():
    """Targets equal to sources, and every source duplicated: coincident
    pairs must be skipped (r^2 == 0), as in the FP64 path."""
    rng = np.random.default_rng(9)
    x, y, z = (np.repeat(rng.uniform(-1, 1, 10000), 2) for _ in range(3))
    q = rng.uniform(-1, 1, 20000)
    a = B.treecode(x, y, z, x, y, z, q, degree=6, max_source_leaf=300, max_target_leaf=300,
                   precision=B.PRECISION_MIXED)
    b = B.treecode(x, y, z, x, y, z, q, degree=6, max_source_leaf=300, max_target_leaf=300,
                   precision=B.PRECISION_FP64)
    assert np.all(np.isfinite(a))
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-6


@pytest.mark.parametrize("kernel", [1, 2])
def test_mixed_single_particle_leaves(kernel):
    """Leaves of one particle (radius 0) evaluated against themselves: the
    coincident self pair must be skipped, as in FP64."""
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(17, 3000)
    kw = dict(kernel=kernel, kernel_param=0.5 if kernel == 2 else 0.0, degree=3, max_source_leaf=1,
              max_target_leaf=1)
    a = B.treecode(tx, ty, tz, sx, sy, sz, sq, precision=B.PRECISION_MIXED, **kw)
    b = B.treecode(tx, ty, tz, sx, sy, sz, sq, precision=B.PRECISION_FP64, **kw)
    assert np.all(np.isfinite(a))
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= TOL_VS_FP64_TREE_YUKAWA
