"""The reference's other kernels (FP64): regularized Yukawa, sin-over-r,
RBS u / v, the user kernel (exp(-k r)/r), and the 1-D periodic atan and MQ
kernels, in every approximation and compute type the reference provides
them in (src/interaction_compute/interaction_compute_{pc,cp,cc}.c), against
the reference build (oracle/_ref).  Bar: the FP64 parity bar, relative L2
<= 1e-12 and per-target |diff| <= 1e-12 max|phi|."""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    # kernel, kernel parameters, approximation, compute type
    (4, [0.5, 0.02], 1, 1), (4, [0.5, 0.02], 1, 2), (4, [0.5, 0.02], 1, 3),
    (8, [2.0], 1, 1), (8, [2.0], 1, 2), (8, [2.0], 1, 3), (8, [2.0], 2, 1), (8, [2.0], 2, 2),
    (10, [0.05], 1, 1), (10, [0.05], 1, 2), (10, [0.05], 1, 3),
    (11, [0.05], 1, 1), (11, [0.05], 1, 3),
    (12, [0.5], 1, 1), (12, [0.5], 1, 2), (12, [0.5], 1, 3),
    (5, [2.0, 0.1], 1, 1), (9, [2.0, 0.1], 1, 1),
]


@pytest.mark.parametrize("kernel,kp,approx,ctype", CASES)
def test_kernel_matches_reference_build(kernel, kp, approx, ctype):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(50 + kernel + 7 * ctype, 6000,
                                                targets="other" if ctype != 1 else "same")
    deg, sc = (5, 4.0) if approx == 2 else (6, 1.0)
    ref = O.ref_treecode(tx, ty, tz, None, sx, sy, sz, sq, None, kernel, kp, 1, approx, ctype, 0.7, deg, 200, 200,
                         sc, -1.0, 0)
    got = B.callTreedriver(len(tx), len(sx), tx, ty, tz, None, sx, sy, sz, sq, None, kernel, len(kp), np.array(kp),
                           B.Singularity.SKIPPING, approx, ctype, True, 0, theta=0.7, degree=deg,
                           sourceLeafSize=200, targetLeafSize=200, sizeCheck=sc)
    assert np.all(np.isfinite(got))
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_regularized_yukawa_subtraction_matches_reference_build():
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    rng = np.random.default_rng(61)
    n = 6000
    x, y, z = (rng.uniform(0, 1, n) for _ in range(3))
    q, w, tq = rng.uniform(-1, 1, n), rng.uniform(0.5, 1.5, n), rng.uniform(-1, 1, n)
    kp = [0.5, 0.02]
    ref = O.ref_treecode(x, y, z, tq, x.copy(), y.copy(), z.copy(), q, w, 4, kp, 2, 1, 1, 0.7, 6, 200, 200, 1.0,
                         -1.0, 0)
    got = B.callTreedriver(n, n, x, y, z, tq, x.copy(), y.copy(), z.copy(), q, w, 4, 2, np.array(kp),
                           B.Singularity.SUBTRACTION, 1, 1, True, 0, theta=0.7, degree=6, sourceLeafSize=200,
                           targetLeafSize=200, sizeCheck=1.0)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12


@pytest.mark.parametrize("kernel,kp,tol", [(8, [2.0], 1e-4), (4, [0.5, 0.02], 1e-4), (10, [0.05], 1e-4),
                                           (5, [2.0, 0.1], 1e-3)])
def test_treecode_vs_gpu_direct_sum(kernel, kp, tol):
    """The new kernels' treecode against the FP64 direct sum (bt_direct_ex).
    The periodic atan kernel has a kink where the separation wraps, which
    the polynomial interpolation resolves slowly (measured 3.5e-4 at degree
    8; the treecode itself matches the reference build to 1e-12)."""
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(70 + kernel, 20000)
    got = B.callTreedriver(len(tx), len(sx), tx, ty, tz, None, sx, sy, sz, sq, None, kernel, len(kp), np.array(kp),
                           B.Singularity.SKIPPING, 1, 1, True, 0, theta=0.7, degree=8, sourceLeafSize=500,
                           targetLeafSize=500, sizeCheck=1.0)
    idx = np.arange(0, len(tx), 7)
    d = B.direct(tx[idx], ty[idx], tz[idx], sx, sy, sz, sq, kernel, kp)
    assert np.linalg.norm(got[idx] - d) / np.linalg.norm(d) <= tol


def test_mixed_request_runs_new_kernels_in_fp64():
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(80, 8000)
    kw = dict(kernel=8, kernel_param=2.0, degree=6, max_source_leaf=300, max_target_leaf=300)
    a = B.treecode(tx, ty, tz, sx, sy, sz, sq, precision=B.PRECISION_MIXED, **kw)
    b = B.treecode(tx, ty, tz, sx, sy, sz, sq, precision=B.PRECISION_FP64, **kw)
    assert np.array_equal(a, b)
