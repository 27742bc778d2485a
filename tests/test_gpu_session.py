"""Sessions (bt_session_*): the device sequence captured once as a CUDA
graph and replayed for new charges gives exactly what a fresh call gives;
the two dispatch modes of the mixed kernels give identical results."""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ctype", [1, 2, 3])
@pytest.mark.parametrize("precision", [B.PRECISION_FP64, B.PRECISION_MIXED])
def test_session_replay_equals_fresh_calls(ctype, precision):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(7, 20000, targets="other" if ctype != 1 else "same")
    kw = dict(kernel=2, kernel_param=0.5, compute_type=ctype, degree=6, max_source_leaf=400, max_target_leaf=300,
              precision=precision)
    s = B.Session([(tx, ty, tz, sx, sy, sz, sq)], **kw)
    rng = np.random.default_rng(3)
    for q in (sq, rng.uniform(-1, 1, len(sx)), sq):
        (got,), rep = s.evaluate(q, return_report=True)
        assert np.array_equal(got, B.treecode(tx, ty, tz, sx, sy, sz, q, **kw))
        assert rep["kernel_launches"] > 0 and rep["ms_eval_kernel"] > 0
    s.close()


def test_session_batch_and_learned():
    rng = np.random.default_rng(5)
    systems = []
    for n in (3000, 17000, 800):
        x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
        systems.append((x, y, z, x.copy(), y.copy(), z.copy(), rng.uniform(-1, 1, n)))
    kw = dict(degree=8, max_source_leaf=500, max_target_leaf=500, precision=B.PRECISION_MIXED)
    s = B.Session(systems, **kw)
    q2 = [rng.uniform(-1, 1, len(t[6])) for t in systems]
    for got, ref in zip(s.evaluate(q2), B.treecode_batch([t[:6] + (q,) for t, q in zip(systems, q2)], **kw)):
        assert np.array_equal(got, ref)
    from barytree_b200 import selector
    selector.install_default()
    x, y, z, q = selector.blobs(60000, 2)
    kwl = dict(degree=10, max_source_leaf=1000, max_target_leaf=1000, precision=B.PRECISION_MIXED,
               degree_policy=B.DEGREE_LEARNED, tolerance=1e-6)
    sl = B.Session([(x, y, z, x, y, z, q)], **kwl)
    assert np.array_equal(sl.evaluate(q)[0], B.treecode(x, y, z, x, y, z, q, **kwl))


@pytest.mark.parametrize("ctype", [1, 3])
def test_dispatch_modes_agree(ctype):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(8, 30000, targets="other")
    kw = dict(compute_type=ctype, degree=7, max_source_leaf=500, max_target_leaf=500, precision=B.PRECISION_MIXED)
    a = B.treecode(tx, ty, tz, sx, sy, sz, sq, dispatch=B.DISPATCH_QUEUE, **kw)
    b = B.treecode(tx, ty, tz, sx, sy, sz, sq, dispatch=B.DISPATCH_GRID, **kw)
    assert np.array_equal(a, b)


def test_session_rejects_wrong_charge_count():
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(9, 1000)
    s = B.Session([(tx, ty, tz, sx, sy, sz, sq)], degree=4, max_source_leaf=100, max_target_leaf=100)
    with pytest.raises(B.BaryTreeError):
        s.evaluate(sq[:-1])


def test_session_writes_into_a_reused_output_array():
    rng = np.random.default_rng(9)
    systems = []
    for n in (5000, 12000):
        x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
        systems.append((x, y, z, x.copy(), y.copy(), z.copy(), rng.uniform(-1, 1, n)))
    kw = dict(degree=6, max_source_leaf=400, max_target_leaf=400, precision=B.PRECISION_MIXED)
    s = B.Session(systems, **kw)
    out = np.full(17000, np.nan)
    for _ in range(2):
        q2 = [rng.uniform(-1, 1, len(t[6])) for t in systems]
        got = s.evaluate(q2, out=out)
        fresh = s.evaluate(q2)
        for g, f in zip(got, fresh):
            assert np.array_equal(g, f)
            assert np.shares_memory(g, out)
        assert np.array_equal(np.concatenate(got), out)
    with pytest.raises(B.BaryTreeError):
        s.evaluate(q2, out=np.empty(16999))
    with pytest.raises(B.BaryTreeError):
        s.evaluate(q2, out=np.empty(17000, dtype=np.float32))
    s.close()
