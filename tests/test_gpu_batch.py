"""Batched evaluation (bt_eval_batch): every system gets the trees, lists and
potentials a separate call gives it, bit for bit, while all systems share one
upward pass, one evaluation kernel and one downward pass."""
import numpy as np
import pytest

import barytree_b200 as B

pytestmark = pytest.mark.gpu


def _systems(seed, sizes, same=True):
    rng = np.random.default_rng(seed)
    out = []
    for nt, ns in sizes:
        sx, sy, sz = (rng.uniform(0, 1, ns) for _ in range(3))
        sq = rng.uniform(-1, 1, ns)
        if same and nt == ns:
            tx, ty, tz = sx.copy(), sy.copy(), sz.copy()
        else:
            tx, ty, tz = (rng.uniform(0, 1, nt) for _ in range(3))
        out.append((tx, ty, tz, sx, sy, sz, sq))
    return out


SIZES = [(3000, 3000), (1, 1), (0, 500), (700, 0), (12000, 12000), (257, 257), (5000, 2000), (2, 9000)]


@pytest.mark.parametrize("ctype", [1, 2, 3])
@pytest.mark.parametrize("precision", [B.PRECISION_FP64, B.PRECISION_MIXED])
def test_batch_equals_separate_calls(ctype, precision):
    # some systems' targets are their sources and some are not: the symmetric
    # near-field pass applies to whole calls whose targets are all the
    # sources, so it is switched off here (test_gpu_sym.py covers batches
    # where it applies)
    systems = _systems(1, SIZES, same=(ctype == 1))
    kw = dict(kernel=3, kernel_param=1e-3, compute_type=ctype, degree=7, theta=0.7, max_source_leaf=300,
              max_target_leaf=300, precision=precision, symmetry=B.SYMMETRY_OFF)
    pots = B.treecode_batch(systems, **kw)
    for s, p in zip(systems, pots):
        ref = B.treecode(*s, **kw) if len(s[0]) else np.zeros(0)
        assert np.array_equal(p, ref)


def test_batch_host_and_gpu_tree_builds_agree():
    systems = _systems(2, SIZES)
    kw = dict(kernel=1, degree=6, max_source_leaf=200, max_target_leaf=200, precision=B.PRECISION_MIXED)
    a = B.treecode_batch(systems, tree_build=B.TREE_GPU, **kw)
    b = B.treecode_batch(systems, tree_build=B.TREE_HOST, **kw)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_batch_of_uneven_systems_vs_direct():
    """Config-4 style: regularized Coulomb (eps 1e-3, the self term q/eps
    included as the reference includes it), degree 7, theta 0.7, mixed
    precision, log-uniform sizes; per-system relative L2 error against the
    FP64 direct sum within the treecode's own FP64 error plus 5e-7."""
    rng = np.random.default_rng(4)
    sizes = np.round(np.exp(rng.uniform(np.log(1e3), np.log(3e4), 24))).astype(int)
    systems = _systems(5, [(n, n) for n in sizes])
    kw = dict(kernel=3, kernel_param=1e-3, degree=7, theta=0.7, max_source_leaf=2000, max_target_leaf=2000)
    mixed = B.treecode_batch(systems, precision=B.PRECISION_MIXED, **kw)
    fp64 = B.treecode_batch(systems, precision=B.PRECISION_FP64, **kw)
    for s, m, f in zip(systems, mixed, fp64):
        d = B.direct(*s, kernel=3, kernel_param=1e-3)
        e64 = np.linalg.norm(f - d) / np.linalg.norm(d)
        em = np.linalg.norm(m - d) / np.linalg.norm(d)
        assert em <= e64 + 5e-7, (len(d), em, e64)


def test_batch_rejects_bad_offsets():
    x = np.zeros(4)
    with pytest.raises(B.BaryTreeError):
        B.treecode_batch_ptr(2, np.array([0, 3, 2]), np.array([0, 2, 4]), *(x.ctypes.data,) * 8)


def test_learned_batch_equals_separate_calls_and_host_tree():
    """The learned selection's error share is computed per system, so a
    batch of systems selects the same degrees as separate calls (bit for bit),
    each system keeps its own accuracy, and the host-built trees give the
    same selection as the GPU-built ones."""
    from barytree_b200 import selector
    selector.install_default()
    systems = []
    for k, n in enumerate((150_000, 60_000, 220_000)):
        x, y, z, q = selector.blobs(n, 300 + k)
        if k == 1:
            q = q * 1e-3                         # a system with a much smaller potential scale
        systems.append((x, y, z, x.copy(), y.copy(), z.copy(), q))
    kw = dict(kernel=1, degree=10, theta=0.7, max_source_leaf=2000, max_target_leaf=2000,
              precision=B.PRECISION_MIXED, degree_policy=B.DEGREE_LEARNED, tolerance=1e-6)
    pots = B.treecode_batch(systems, **kw)
    host = B.treecode_batch(systems, tree_build=B.TREE_HOST, **kw)
    for s, p, h in zip(systems, pots, host):
        ref = B.treecode(*s, **kw)
        assert np.array_equal(p, ref)
        assert np.array_equal(p, h)
        idx = np.arange(0, len(s[0]), 37)
        d = B.direct(s[0][idx], s[1][idx], s[2][idx], s[3], s[4], s[5], s[6])
        assert np.linalg.norm(p[idx] - d) / np.linalg.norm(d) <= 1e-6
