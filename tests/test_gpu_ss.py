"""Singularity subtraction (SS) through BaryTreeInterface on the GPU.

Checked against the reference's own Python golden values
(interfaces/python/testBaryTreeInterface.py:48,69: Yukawa + SS, N=5000,
explicit theta/degree and the beta path) and against the reference build
(oracle/_ref, compiled from the reference's sources) for every kernel /
approximation / compute type the reference provides SS for.  Bar: the FP64
parity bar, relative L2 <= 1e-12 and per-target |diff| <= 1e-12 max|phi|
(the golden values to 1e-12 relative)."""
import numpy as np
import pytest

import barytree_b200 as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN_EXPLICIT = 588.7432483318685     # testBaryTreeInterface.py:48
GOLDEN_BETA = 588.7445889051367         # testBaryTreeInterface.py:69


def _golden_inputs():
    rs = np.random.RandomState(1)       # the golden test's np.random.seed(1) stream
    n = 5000
    rho = rs.rand(n)
    x, y, z = rs.rand(n), rs.rand(n), rs.rand(n)
    return x, y, z, rho, np.ones(n)


def test_python_golden_yukawa_subtraction():
    x, y, z, rho, w = _golden_inputs()
    n = len(x)
    out = B.callTreedriver(n, n, x, y, z, rho, x.copy(), y.copy(), z.copy(), rho.copy(), w.copy(),
                           B.Kernel.YUKAWA, 1, np.array([0.5]), B.Singularity.SUBTRACTION,
                           B.Approximation.LAGRANGE, B.ComputeType.PARTICLE_CLUSTER, True, 0,
                           theta=0.8, degree=4, sourceLeafSize=50, targetLeafSize=10, sizeCheck=1.0)
    assert abs(out[0] - GOLDEN_EXPLICIT) <= 1e-12 * abs(GOLDEN_EXPLICIT)
    out = B.callTreedriver(n, n, x, y, z, rho, x.copy(), y.copy(), z.copy(), rho.copy(), w.copy(),
                           B.Kernel.YUKAWA, 1, np.array([0.5]), B.Singularity.SUBTRACTION,
                           B.Approximation.LAGRANGE, B.ComputeType.PARTICLE_CLUSTER, True, 0, beta=0.1,
                           sizeCheck=1.0)
    assert abs(out[0] - GOLDEN_BETA) <= 1e-12 * abs(GOLDEN_BETA)


def _inputs(seed, n, other):
    rng = np.random.default_rng(seed)
    sx, sy, sz = (rng.uniform(0, 1, n) for _ in range(3))
    sq = rng.uniform(-1, 1, n)
    sw = rng.uniform(0.5, 1.5, n)                # quadrature-like weights
    if other:
        tx, ty, tz = (rng.uniform(0, 1, n) for _ in range(3))
    else:
        tx, ty, tz = sx.copy(), sy.copy(), sz.copy()
    tq = rng.uniform(-1, 1, n)
    return tx, ty, tz, tq, sx, sy, sz, sq, sw


CASES = [
    # (kernel, kernel parameters, approximation, compute type)
    (1, [0.7], 1, 1), (1, [0.7], 2, 1), (2, [0.5], 1, 1), (2, [0.5], 2, 1), (3, [0.7, 1e-2], 1, 1),
    (3, [0.7, 1e-2], 2, 1), (1, [0.7], 1, 2), (2, [0.5], 1, 2), (1, [0.7], 1, 3), (2, [0.5], 1, 3),
]


@pytest.mark.parametrize("kernel,kp,approx,ctype", CASES)
def test_subtraction_matches_reference_build(kernel, kp, approx, ctype):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    tx, ty, tz, tq, sx, sy, sz, sq, sw = _inputs(3 + kernel + 10 * ctype, 6000, other=ctype != 1)
    deg, sc = (5, 4.0) if approx == 2 else (6, 1.0)
    ref = O.ref_treecode(tx, ty, tz, tq, sx, sy, sz, sq, sw, kernel, kp, 2, approx, ctype, 0.7, deg, 200, 200, sc,
                         -1.0, 0)
    got = B.callTreedriver(len(tx), len(sx), tx, ty, tz, tq, sx, sy, sz, sq, sw, kernel, len(kp), np.array(kp),
                           B.Singularity.SUBTRACTION, approx, ctype, True, 0, theta=0.7, degree=deg,
                           sourceLeafSize=200, targetLeafSize=200, sizeCheck=sc)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_subtraction_with_unit_weights_and_zero_target_charges_equals_skipping():
    """With w = 1 and target charges 0, subtraction adds nothing to skipping
    (Yukawa: the kernels coincide term by term)."""
    tx, ty, tz, tq, sx, sy, sz, sq, sw = _inputs(5, 8000, other=True)
    kw = dict(theta=0.7, degree=6, sourceLeafSize=300, targetLeafSize=300, sizeCheck=1.0)
    args = (len(tx), len(sx), tx, ty, tz, np.zeros(len(tx)), sx, sy, sz, sq, np.ones(len(sx)), B.Kernel.YUKAWA, 1,
            np.array([0.5]))
    ss = B.callTreedriver(*args, B.Singularity.SUBTRACTION, 1, 1, True, 0, **kw)
    sk = B.callTreedriver(*args, B.Singularity.SKIPPING, 1, 1, True, 0, **kw)
    assert np.linalg.norm(ss - sk) / np.linalg.norm(sk) <= 1e-13
