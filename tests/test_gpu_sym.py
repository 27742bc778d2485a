"""GPU tests of the symmetric near-field pairs of the mixed path (targets =
sources, Coulomb, Yukawa and regularized Coulomb): leaf pairs that list each other
with no possible close pair are evaluated once for both sides
(bt_sym.cu).  Against the same call with BT_SYMMETRY_OFF the potentials
agree to FP32 rounding (the sums close in another order) and keep the mixed
path's accuracy against the FP64 direct sum; they are the same bit for bit
on every run, in a session and in a batch; calls the pass does not apply
to are bit-identical to BT_SYMMETRY_OFF."""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _clustered(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.6, 0.6, (4, 3))
    pts = np.concatenate([rng.normal(c[k], 0.1, (n // 5, 3)) for k in range(4)] + [rng.uniform(-1, 1, (n // 5, 3))])
    pts = np.clip(pts, -1, 1)
    return pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy(), rng.uniform(-1, 1, len(pts))


@pytest.mark.parametrize("kernel,kp,approx,sc,ctype", [(B.Kernel.COULOMB, 0.0, 1, 1.0, 1),
                                                       (B.Kernel.REGULARIZED_COULOMB, 1e-3, 1, 1.0, 1),
                                                       (B.Kernel.COULOMB, 0.0, 2, 4.0, 1),
                                                       (B.Kernel.YUKAWA, 0.5, 1, 1.0, 1),
                                                       (B.Kernel.YUKAWA, 0.5, 1, 1.0, 3),
                                                       (B.Kernel.COULOMB, 0.0, 1, 1.0, 2)])
def test_symmetric_pairs_against_both_directions(kernel, kp, approx, sc, ctype):
    x, y, z, q = _clustered(200000, 41)
    kw = dict(kernel=kernel, kernel_param=kp, approximation=approx, theta=0.7, degree=6, max_source_leaf=500,
              max_target_leaf=500, size_check=sc, precision=B.PRECISION_MIXED, compute_type=ctype)
    sym = B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, **kw)
    off = B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, symmetry=B.SYMMETRY_OFF, **kw)
    assert not np.array_equal(sym, off)                  # the pass ran
    assert _rel(sym, off) < 5e-7
    assert np.array_equal(B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, **kw), sym)   # deterministic
    idx = np.arange(0, len(x), 200)
    exact = B.direct(x[idx], y[idx], z[idx], x, y, z, q, kernel=kernel, kernel_param=kp)
    assert _rel(sym[idx], exact) <= 1.05 * _rel(off[idx], exact) + 2e-7


def test_symmetric_pairs_with_learned_degrees_sessions_and_batches():
    from barytree_b200 import selector
    selector.install_default()
    x, y, z, q = _clustered(300000, 42)
    kw = dict(theta=0.7, degree=10, max_source_leaf=2000, max_target_leaf=2000, size_check=1.0,
              precision=B.PRECISION_MIXED, degree_policy=B.DEGREE_LEARNED, tolerance=1e-6)
    sym = B.treecode(x, y, z, x, y, z, q, **kw)
    off = B.treecode(x, y, z, x, y, z, q, symmetry=B.SYMMETRY_OFF, **kw)
    assert _rel(sym, off) < 5e-7
    idx = np.arange(0, len(x), 300)
    assert _rel(sym[idx], B.direct(x[idx], y[idx], z[idx], x, y, z, q)) < 1e-6
    s = B.Session([(x, y, z, x, y, z, q)], **kw)
    assert np.array_equal(s.evaluate(q)[0], sym)
    s.close()
    # a batch of two systems equals the separate calls
    x2, y2, z2, q2 = _clustered(100000, 43)
    kb = dict(kw)
    kb.pop("degree_policy"); kb.pop("tolerance")
    pots = B.treecode_batch([(x, y, z, x, y, z, q), (x2, y2, z2, x2, y2, z2, q2)], **kb)
    assert np.array_equal(pots[0], B.treecode(x, y, z, x, y, z, q, **kb))
    assert np.array_equal(pots[1], B.treecode(x2, y2, z2, x2, y2, z2, q2, **kb))


@pytest.mark.parametrize("case", ["targets_differ", "big_leaves", "fp64"])
def test_symmetry_does_not_apply(case):
    n = 20000 if case == "big_leaves" else 80000
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(44, n, targets="other" if case == "targets_differ" else "same")
    leaf = 2500 if case == "big_leaves" else 400          # big: octants of ~2500 particles stay leaves
    kw = dict(theta=0.7, degree=5, max_source_leaf=leaf, max_target_leaf=leaf,
              precision=B.PRECISION_FP64 if case == "fp64" else B.PRECISION_MIXED)
    assert np.array_equal(B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw),
                          B.treecode(tx, ty, tz, sx, sy, sz, sq, symmetry=B.SYMMETRY_OFF, **kw))


@pytest.mark.parametrize("kernel,kp", [(B.Kernel.COULOMB, 0.0), (B.Kernel.YUKAWA, 0.5),
                                       (B.Kernel.REGULARIZED_COULOMB, 1e-9)])
def test_close_pairs_across_touching_leaves(kernel, kp):
    """Pairs 1e-7 apart straddling the root's split planes sit in touching
    leaves, which the symmetric pass takes with FP32 distances clamped at the
    close-pair distance and FP64 terms for the clamped pairs: those targets,
    dominated by their partner, keep the FP64 accuracy of the mixed path."""
    rng = np.random.default_rng(45)
    n = 60000
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    mid = [(a.min() + a.max()) / 2 for a in (x, y, z)]
    k = 64
    py, pz = rng.uniform(-0.9, 0.9, k), rng.uniform(-0.9, 0.9, k)
    # pairs across the x plane, and across the y plane
    cx = np.concatenate([np.full(k, mid[0] - 5e-8), np.full(k, mid[0] + 5e-8), py, py + 1e-8])
    cy = np.concatenate([py, py + 1e-8, np.full(k, mid[1] - 5e-8), np.full(k, mid[1] + 5e-8)])
    cz = np.concatenate([pz, pz, pz, pz])
    x, y, z = np.concatenate([x, cx]), np.concatenate([y, cy]), np.concatenate([z, cz])
    q = rng.uniform(-1, 1, len(x))
    kw = dict(kernel=kernel, kernel_param=kp, theta=0.7, degree=6, max_source_leaf=400, max_target_leaf=400,
              size_check=1.0, precision=B.PRECISION_MIXED)
    sym = B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, **kw)
    off = B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, symmetry=B.SYMMETRY_OFF, **kw)
    assert not np.array_equal(sym, off)
    idx = np.arange(n, len(x))                            # the planted targets
    exact = B.direct(x[idx], y[idx], z[idx], x, y, z, q, kernel=kernel, kernel_param=kp)
    err_sym = np.abs(sym[idx] - exact) / np.abs(exact)
    err_off = np.abs(off[idx] - exact) / np.abs(exact)
    assert err_sym.max() < 1e-6 and err_off.max() < 1e-6, (err_sym.max(), err_off.max())
    assert _rel(sym, off) < 5e-7
    assert np.array_equal(B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, **kw), sym)


_THREADS_SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[2])
import barytree_b200 as B
rng = np.random.default_rng(43)
c = rng.uniform(-0.6, 0.6, (4, 3))
pts = np.clip(np.concatenate([rng.normal(c[k], 0.1, (40000, 3)) for k in range(4)] +
                             [rng.uniform(-1, 1, (40000, 3))]), -1, 1)
x, y, z = pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy()
q = rng.uniform(-1, 1, len(x))
pot, rep = B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, theta=0.7, degree=6, max_source_leaf=500,
                      max_target_leaf=500, precision=B.PRECISION_MIXED, return_report=True)
np.savez(sys.argv[1], pot=pot, sym=rep["sym_ptwise"], pp=rep["pp_ptwise"])
"""


@pytest.mark.parametrize("threads", [[1, 16], [3, 8]])
def test_symmetric_pass_independent_of_host_threads(tmp_path, threads):
    """The host builds the symmetric pairs in parallel (OpenMP) and numbers
    them per head unit and partner node, so the pair list, the slices and
    therefore the potentials do not depend on the number of host threads:
    the same evaluation in fresh processes with different OMP_NUM_THREADS
    gives the same bits and the same count of symmetric evaluations."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    res = []
    for t in threads:
        path = str(tmp_path / f"pot_{t}.npz")
        env = dict(os.environ, OMP_NUM_THREADS=str(t))
        subprocess.run([sys.executable, "-c", _THREADS_SCRIPT, path, ROOT], env=env, check=True, timeout=600)
        res.append(np.load(path))
    assert res[0]["sym"] > 0
    assert res[0]["sym"] == res[1]["sym"] and res[0]["pp"] == res[1]["pp"]
    assert np.array_equal(res[0]["pot"], res[1]["pot"])
