"""GPU tests of target sharding (bt_options.shard_index / shard_count), the
multi-GPU decomposition of one system: every shard builds the trees, lists
and proxies, evaluates a contiguous run of target leaves of about equal cost
(with target grids, the grids of those leaves and their ancestors) and
leaves the other potentials 0, so one all-reduce (sum) over the shards gives
the result.  Here the shards run one after another on one GPU: their sum
must equal the unsharded potentials bit for bit, every target must come from
exactly one shard, and the shards' costs must be balanced.  With the
symmetric near-field pass (targets = sources) a leaf pair's partner side can
land on targets another shard owns; those sums agree with the unsharded
result to FP64 rounding."""
import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs

pytestmark = pytest.mark.gpu


def _clustered(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.6, 0.6, (4, 3))
    pts = np.concatenate([rng.normal(c[k], 0.12, (n // 5, 3)) for k in range(4)] + [rng.uniform(-1, 1, (n // 5, 3))])
    pts = np.clip(pts, -1, 1)
    return pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy(), rng.uniform(-1, 1, len(pts))


@pytest.mark.parametrize("precision,nshards", [(B.PRECISION_FP64, 2), (B.PRECISION_MIXED, 3), (B.PRECISION_MIXED, 4)])
def test_sum_of_shards_is_the_unsharded_result(precision, nshards):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(31, 120000, targets="other")
    kw = dict(theta=0.7, degree=6, max_source_leaf=500, max_target_leaf=500, size_check=1.0, precision=precision)
    full = B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw)
    parts = [B.treecode(tx, ty, tz, sx, sy, sz, sq, shard=(k, nshards), **kw) for k in range(nshards)]
    assert np.array_equal(np.sum(parts, axis=0), full)
    nonzero = np.array([p != 0 for p in parts])
    assert np.all(nonzero.sum(axis=0) == 1)          # every target from exactly one shard
    counts = nonzero.sum(axis=1)
    assert counts.min() > 0.5 * len(tx) / nshards    # balanced (uniform inputs: cost ~ targets)


def test_sharded_learned_degrees_and_sessions():
    from barytree_b200 import selector
    selector.install_default()
    x, y, z, q = _clustered(300000, 32)
    kw = dict(theta=0.7, degree=10, max_source_leaf=2000, max_target_leaf=2000, size_check=1.0,
              precision=B.PRECISION_MIXED, degree_policy=B.DEGREE_LEARNED, tolerance=1e-6)
    # without the symmetric pass every shard evaluates its own targets only:
    # the sum is the unsharded result bit for bit
    off = dict(kw, symmetry=B.SYMMETRY_OFF)
    full_off = B.treecode(x, y, z, x, y, z, q, **off)
    parts = [B.treecode(x, y, z, x, y, z, q, shard=(k, 2), **off) for k in range(2)]
    assert np.array_equal(parts[0] + parts[1], full_off)
    # with it, a leaf pair belongs to the shard owning its head leaf, which
    # adds the partner's side into targets the other shard owns: the pair
    # values are the unsharded ones, and the sum differs from the unsharded
    # result only by the grouping of the FP64 sums of a leaf's slices
    full = B.treecode(x, y, z, x, y, z, q, **kw)
    parts, reps = zip(*[B.treecode(x, y, z, x, y, z, q, shard=(k, 2), return_report=True, **kw) for k in range(2)])
    _, rfull = B.treecode(x, y, z, x, y, z, q, return_report=True, **kw)
    assert rfull["sym_ptwise"] > 0 and all(r["sym_ptwise"] > 0 for r in reps)
    assert reps[0]["sym_ptwise"] + reps[1]["sym_ptwise"] == rfull["sym_ptwise"]
    total = parts[0] + parts[1]
    assert np.max(np.abs(total - full)) <= 1e-13 * np.max(np.abs(full))
    assert np.linalg.norm(total - full_off) <= 5e-7 * np.linalg.norm(full_off)
    sparts = []
    for k in range(2):
        s = B.Session([(x, y, z, x, y, z, q)], shard=(k, 2), **kw)
        sparts.append(s.evaluate(q)[0])
        s.close()
    assert np.array_equal(sparts[0], parts[0]) and np.array_equal(sparts[1], parts[1])


def test_one_shard_is_the_unsharded_call():
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(33, 50000)
    kw = dict(theta=0.7, degree=5, max_source_leaf=400, max_target_leaf=400, precision=B.PRECISION_MIXED)
    assert np.array_equal(B.treecode(tx, ty, tz, sx, sy, sz, sq, shard=(0, 1), **kw),
                          B.treecode(tx, ty, tz, sx, sy, sz, sq, **kw))
    # one shard of one is no sharding: the symmetric pass stays on
    x, y, z, q = _clustered(40000, 34)
    assert np.array_equal(B.treecode(x, y, z, x, y, z, q, shard=(0, 1), **kw),
                          B.treecode(x, y, z, x, y, z, q, **kw))


# cluster-particle and cluster-cluster: target grids split by subtree; with
# singularity subtraction the correction term belongs to the shard's targets
GRID_CASES = [
    dict(compute_type=B.ComputeType.CLUSTER_CLUSTER, kernel=B.Kernel.YUKAWA, kernel_param=[0.5],
         precision=B.PRECISION_FP64, nshards=2),
    dict(compute_type=B.ComputeType.CLUSTER_CLUSTER, kernel=B.Kernel.COULOMB, kernel_param=[],
         precision=B.PRECISION_MIXED, nshards=3),
    dict(compute_type=B.ComputeType.CLUSTER_PARTICLE, kernel=B.Kernel.COULOMB, kernel_param=[],
         approximation=B.Approximation.HERMITE, precision=B.PRECISION_FP64, nshards=2),
    dict(compute_type=B.ComputeType.CLUSTER_PARTICLE, kernel=B.Kernel.YUKAWA, kernel_param=[0.5],
         precision=B.PRECISION_MIXED, nshards=4),
    dict(compute_type=B.ComputeType.CLUSTER_CLUSTER, kernel=B.Kernel.COULOMB, kernel_param=[0.5],
         singularity=B.Singularity.SUBTRACTION, precision=B.PRECISION_FP64, nshards=2),
    dict(compute_type=B.ComputeType.PARTICLE_CLUSTER, kernel=B.Kernel.YUKAWA, kernel_param=[0.5],
         singularity=B.Singularity.SUBTRACTION, precision=B.PRECISION_FP64, nshards=3),
]


@pytest.mark.parametrize("case", GRID_CASES, ids=["cc-yukawa-fp64", "cc-coulomb-mixed", "cp-hermite-fp64",
                                                  "cp-yukawa-mixed", "cc-subtraction-fp64",
                                                  "pc-subtraction-fp64"])
def test_sum_of_grid_and_subtraction_shards_is_the_unsharded_result(case):
    case = dict(case)
    nshards = case.pop("nshards")
    x, y, z, q = _clustered(150000, 35)
    rng = np.random.default_rng(36)
    kw = dict(theta=0.8, degree=6, max_source_leaf=600, max_target_leaf=600, size_check=1.0, **case)
    if case.get("singularity") == B.Singularity.SUBTRACTION:
        kw.update(target_q=q.copy(), source_w=rng.uniform(0.5, 1.5, len(q)))
    tx, ty, tz = x + 1e-3, y.copy(), z.copy()          # targets apart from the sources
    full = B.treecode(tx, ty, tz, x, y, z, q, **kw)
    parts = [B.treecode(tx, ty, tz, x, y, z, q, shard=(k, nshards), **kw) for k in range(nshards)]
    assert np.array_equal(np.sum(parts, axis=0), full)
    nonzero = np.array([p != 0 for p in parts])
    assert np.all(nonzero.sum(axis=0) == 1)
    counts = nonzero.sum(axis=1)
    assert counts.min() > 0.3 * len(tx) / nshards
