"""GPU tests of the tensor-core leaf P2M (tcgen05, 3xTF32) of the mixed
Lagrange path, against the FP64 SIMT P2M (option BT_UPWARD_FP64) and the
FP64 direct sum.

The two upward passes must agree to within a few FP32 roundings at every
degree (the tensor-core kernel covers n + 1 <= 16: (n+1)^2 rows in one or
two 128-row tiles): 5e-7 relative in the potentials, where the proxy charges
carry about 1.4e-7 (3xTF32 products, short FP32 sums on the tensor core,
FP64 across 32-particle chunks); the potentials must keep the mixed path's
accuracy against the direct sum.  They must not be bit-identical (proof that
the tensor-core kernel ran).  Every leaf exercises the
exact-node rule: its extreme particles sit on the end nodes of its grid.
"""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("degree", list(range(1, 13)))
def test_tensor_core_p2m_against_fp64_p2m(degree):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(21, 80000)
    kw = dict(theta=0.7, degree=degree, max_source_leaf=500, max_target_leaf=500, size_check=1.0,
              precision=B.PRECISION_MIXED)
    tc, rep = B.treecode(tx, ty, tz, sx, sy, sz, sq, return_report=True, **kw)
    f64 = B.treecode(tx, ty, tz, sx, sy, sz, sq, upward=B.UPWARD_FP64, **kw)
    assert rep["pc_ptwise"] > 0
    assert not np.array_equal(tc, f64)
    assert _rel(tc, f64) < 5e-7
    idx = np.arange(0, len(tx), 80)
    exact = B.direct(tx[idx], ty[idx], tz[idx], sx, sy, sz, sq)
    assert _rel(tc[idx], exact) <= 1.05 * _rel(f64[idx], exact) + 3e-7


@pytest.mark.parametrize("kernel,kp", [(B.Kernel.YUKAWA, 0.5), (B.Kernel.REGULARIZED_COULOMB, 1e-3)])
def test_tensor_core_p2m_other_kernels(kernel, kp):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(22, 60000, targets="other")
    kw = dict(kernel=kernel, kernel_param=kp, theta=0.7, degree=7, max_source_leaf=400, max_target_leaf=400,
              size_check=1.0, precision=B.PRECISION_MIXED)
    tc = B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw)
    f64 = B.treecode(tx, ty, tz, sx, sy, sz, sq, upward=B.UPWARD_FP64, **kw)
    assert _rel(tc, f64) < 5e-7


def test_tensor_core_p2m_with_learned_degrees_and_sessions():
    from barytree_b200 import selector
    selector.install_default()
    rng = np.random.default_rng(23)
    n = 400000
    c = rng.uniform(-0.6, 0.6, (4, 3))
    pts = np.concatenate([rng.normal(c[k], 0.1, (n // 5, 3)) for k in range(4)] + [rng.uniform(-1, 1, (n // 5, 3))])
    pts = np.clip(pts, -1, 1)
    x, y, z = pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy()
    q = rng.uniform(-1, 1, len(x))
    kw = dict(theta=0.7, degree=10, max_source_leaf=2000, max_target_leaf=2000, size_check=1.0,
              precision=B.PRECISION_MIXED, degree_policy=B.DEGREE_LEARNED, tolerance=1e-6)
    tc = B.treecode(x, y, z, x, y, z, q, **kw)
    f64 = B.treecode(x, y, z, x, y, z, q, upward=B.UPWARD_FP64, **kw)
    assert _rel(tc, f64) < 5e-7
    idx = np.arange(0, len(x), 400)
    exact = B.direct(x[idx], y[idx], z[idx], x, y, z, q)
    assert _rel(tc[idx], exact) < 1e-6
    sess = B.Session([(x, y, z, x, y, z, q)], **kw)
    (s_out,) = sess.evaluate(q)
    sess.close()
    assert np.array_equal(s_out, tc)


def test_expired_tensor_core_wait_is_reported_and_the_context_survives(monkeypatch):
    """Failure path without a fault: with BARYTREE_B200_TEST_EXPIRE_TC_WAIT
    set, every block of the tensor-core P2M waits (bounded) on an mbarrier
    phase that nothing completes, before issuing any MMA; the call must
    return BT_ERR_TIMEOUT, and the next call must work."""
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(24, 20000)
    kw = dict(theta=0.7, degree=6, max_source_leaf=400, max_target_leaf=400, precision=B.PRECISION_MIXED)
    good = B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw)
    monkeypatch.setenv("BARYTREE_B200_TEST_EXPIRE_TC_WAIT", "1")
    with pytest.raises(B.BaryTreeError) as e:
        B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw)
    assert e.value.code == B.BT_ERR_TIMEOUT and "tensor-core wait expired" in B.last_error()
    monkeypatch.delenv("BARYTREE_B200_TEST_EXPIRE_TC_WAIT")
    assert np.array_equal(B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw), good)


@pytest.mark.parametrize("degree,leaf,clustered", [(6, 1000, True), (4, 300, False), (7, 2500, True), (2, 200, False)])
def test_tensor_core_hermite_p2m_against_fp64(degree, leaf, clustered):
    """Hermite particle-cluster in mixed precision: the 8 moments per node on
    the tensor cores (degrees with n + 1 <= 8; leaves above 2048 particles
    exercise the chunked nodes and their reduction) against the FP64 Hermite
    P2M (BT_UPWARD_FP64), and both against the direct sum."""
    rng = np.random.default_rng(40 + degree)
    n = 120000
    if clustered:
        x, y, z = (np.clip(rng.normal(0, 0.25, n), -1, 1) for _ in range(3))
    else:
        x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    q = rng.choice([-1.0, 1.0], n)
    kw = dict(approximation=B.Approximation.HERMITE, theta=0.7, degree=degree, max_source_leaf=leaf,
              max_target_leaf=leaf, size_check=4.0, precision=B.PRECISION_MIXED)
    tc, rep = B.treecode(x, y, z, x, y, z, q, return_report=True, **kw)
    f64 = B.treecode(x, y, z, x, y, z, q, upward=B.UPWARD_FP64, **kw)
    assert rep["pc_ptwise"] > 0
    assert not np.array_equal(tc, f64)
    assert _rel(tc, f64) < 5e-7
    idx = np.arange(0, n, 60)
    exact = B.direct(x[idx], y[idx], z[idx], x, y, z, q)
    assert _rel(tc[idx], exact) <= 1.05 * _rel(f64[idx], exact) + 3e-7
