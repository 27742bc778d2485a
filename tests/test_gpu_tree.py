"""GPU tree build: the same nodes, boxes, radii and particle order as the
host build, and the same nodes, boxes, radii and per-node particle sets as
the reference's own build (src/tree/tree.c:19-59,
src/tree/tree_linked_list.c:16-293, src/tree/partition.c:14-392).
Bit-exact: integer node data and permutations compare equal; boxes and
radii compare bitwise except for the sign of a zero bound."""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import same_members, uniform_inputs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _clustered(seed, n):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.7, 0.7, (4, 3))
    pts = np.concatenate([np.clip(rng.normal(c[i], 0.05, (n // 4, 3)), -1, 1) for i in range(4)])
    return pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy()


def _duplicates(seed, n):
    """Every point twice, and points on a lattice of quarter steps (exact
    ties with the midpoints)."""
    rng = np.random.default_rng(seed)
    base = rng.uniform(-1, 1, (n // 3, 3))
    pts = np.concatenate([base, base, np.round(rng.uniform(-1, 1, (n - 2 * (n // 3), 3)) * 4) / 4])
    return pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy()


def _compare(x, y, z, maxpar):
    gi, gd, go = B.tree_summary(x, y, z, maxpar, tree_build=B.TREE_GPU, return_order=True)
    hi, hd, ho = B.tree_summary(x, y, z, maxpar, tree_build=B.TREE_HOST, return_order=True)
    assert np.array_equal(gi, hi)
    # equal values; only the sign of a zero bound may differ (min/max over
    # {-0.0, +0.0} keeps the first one met, and the GPU meets them in another
    # order), which no later arithmetic can observe
    assert np.array_equal(gd, hd)
    assert np.array_equal(gd.view(np.int64)[gd != 0], hd.view(np.int64)[hd != 0])
    assert np.array_equal(go, ho)
    return gi, gd, go


@pytest.mark.parametrize("maxpar", [1, 7, 100, 5000])
def test_gpu_tree_matches_oracle(maxpar):
    _, _, _, x, y, z, _ = uniform_inputs(9, 3000)
    gi, gd, _ = _compare(x, y, z, maxpar)
    oi, od = O.tree(x, y, z, maxpar)
    assert np.array_equal(gi, oi)
    assert np.array_equal(gd, od)


@pytest.mark.parametrize("make,n,maxpar", [(_clustered, 12000, 50), (_duplicates, 9000, 40),
                                           (_clustered, 40001, 333)])
def test_gpu_tree_matches_reference_build(make, n, maxpar):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    x, y, z = make(3, n)
    gi, gd, go = _compare(x, y, z, maxpar)
    ri, rd = O.ref_tree(x, y, z, maxpar)
    assert np.array_equal(gi[:, :3], ri[:, :3])
    assert np.array_equal(gd, rd)
    # same particles per node; the order inside a node is the input order here
    # and the reference's swap order there
    assert same_members(gi, go, O.ref_tree_order(x, y, z, maxpar))


def test_gpu_tree_coincident_block():
    """More coincident points than a leaf holds: the node stays a leaf in
    both builds (the reference would recurse without end, so it is not run)."""
    x, y, z = _duplicates(5, 6000)
    x = np.concatenate([x, np.full(700, 0.25)])
    y = np.concatenate([y, np.full(700, -0.5)])
    z = np.concatenate([z, np.full(700, 0.0)])
    gi, _, _ = _compare(x, y, z, 40)
    leaf = gi[gi[:, 2] == 0]
    assert (leaf[:, 1] - leaf[:, 0] + 1).max() >= 700


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4097])
def test_gpu_tree_small_and_ragged(n):
    rng = np.random.default_rng(n)
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    _compare(x, y, z, 1)
    _compare(x, y, z, 2)


def test_gpu_tree_large():
    """2M clustered points, 2000 per leaf (multi-chunk nodes at every level)."""
    x, y, z = _clustered(11, 2_000_000)
    gi, _, go = _compare(x, y, z, 2000)
    assert np.array_equal(np.sort(go), np.arange(len(x)))
    assert gi[0, 0] == 1 and gi[0, 1] == len(x)


def test_gpu_tree_eval_matches_host_tree():
    """The whole evaluation through either build gives bit-identical results."""
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(21, 20000, targets="other")
    for ctype in (1, 2, 3):
        kw = dict(compute_type=ctype, degree=6, max_source_leaf=300, max_target_leaf=200)
        a = B.treecode(tx, ty, tz, sx, sy, sz, sq, tree_build=B.TREE_GPU, **kw)
        b = B.treecode(tx, ty, tz, sx, sy, sz, sq, tree_build=B.TREE_HOST, **kw)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("ctype,theta,degree,leaf,sc", [(1, 0.7, 8, 50, 1.0), (2, 0.5, 3, 20, 4.0),
                                                        (1, 0.9, 2, 7, 1.0), (2, 0.8, 6, 300, 1.0)])
def test_gpu_traversal_lists_match_host_traversal(ctype, theta, degree, leaf, sc):
    """Particle-cluster and cluster-particle lists traversed on the GPU
    (bt_gpulists.cu) equal the host traversal's on the same GPU-built trees
    (BARYTREE_B200_HOST_LISTS selects the host traversal) and the host-built
    plan's, entry for entry and in order: clustered and duplicate points,
    deep trees (small leaves), distinct targets."""
    import os
    x, y, z = _clustered(4, 12000)
    tx, ty, tz = _duplicates(5, 9000)
    args = (tx, ty, tz, x, y, z, ctype, 1, theta, degree, leaf, leaf, sc)
    gpu = B.interaction_lists(*args, tree_build=B.TREE_GPU)
    os.environ["BARYTREE_B200_HOST_LISTS"] = "1"
    try:
        host = B.interaction_lists(*args, tree_build=B.TREE_GPU)
    finally:
        del os.environ["BARYTREE_B200_HOST_LISTS"]
    ref = B.interaction_lists(*args)
    assert gpu[0] == host[0] == ref[0] and gpu[1] == host[1] == ref[1]
    assert len(gpu[2]) > 0
    assert np.array_equal(gpu[2], host[2]) and np.array_equal(gpu[2], ref[2])
