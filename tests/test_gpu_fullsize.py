"""Parity at the full sizes of the benchmark configurations (the seed-0
inputs of bench.py), where the small parity cases cannot reach: deep, uneven
trees, millions of particles, degree 10.

* FP64 plain path against the reference itself (its own routines, built from
  its sources): configuration 1 (100,000 particles) on every target, and
  configurations 3 (4M Gaussian, Hermite n=6, size check 4, leaf 1000) and 5
  (16M clustered, Lagrange n=10, leaf 2000) on a strided sample of the target
  batches.  A sampled batch holds exactly the values a full reference call
  gives it (tests/refjobs.py, oracle/ref_sampled.c).  Bar, as for the small
  cases: rel-L2 <= 1e-12 and per target |diff| <= 1e-12 max|phi|.
* Interaction lists of the evaluation path (trees built on the GPU) against
  the reference's InteractionLists_Make at configurations 1, 2 (1M
  cluster-cluster, theta 0.8), 3 and 5: bit for bit, membership and order.
* Mixed precision at full size against the FP64 direct sum on 10,000
  strided targets: <= 1e-6 rel-L2 (configurations 1, 2, 3 and 5, the last
  with the learned degree selection).

The reference runs in spawned worker processes while the GPU side runs.
"""
import os

import numpy as np
import pytest

import barytree_b200 as B
import refjobs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12
MIXED_TOL = 1e-6

# reference potentials: (config, sampled batches or None for all, threads)
POT_JOBS = {1: ("pot", 1, None, 4), 3: ("pot", 3, 48, 4), 5: ("pot", 5, 24, 6)}
LIST_JOBS = {c: ("lists", c) for c in (1, 2, 3, 5)}


@pytest.fixture(scope="module")
def ref():
    if not O.ref_available() or not os.path.exists(os.path.join(O.REF_DIR, "libBaryTree_refsample.so")):
        pytest.skip("reference build oracle/_ref not present")
    jobs = refjobs.Jobs(list(POT_JOBS.values()) + list(LIST_JOBS.values()), processes=4)
    yield jobs
    jobs.close()


def _fp64(cid):
    cfg, x, y, z, q = refjobs.inputs(cid)
    pot = B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, kernel=cfg["kernel"], kernel_param=cfg["kp"],
                     approximation=cfg["approx"], compute_type=cfg["ctype"], theta=cfg["theta"],
                     degree=cfg["degree"], max_source_leaf=cfg["leaf"], max_target_leaf=cfg["leaf"],
                     size_check=cfg["sc"], precision=B.PRECISION_FP64)
    return pot


@pytest.mark.parametrize("cid", [1, 2, 3, 5])
def test_lists_match_reference_full_size(ref, cid):
    cfg, x, y, z, q = refjobs.inputs(cid)
    a = B.interaction_lists(x, y, z, x.copy(), y.copy(), z.copy(), cfg["ctype"], cfg["approx"], cfg["theta"],
                            cfg["degree"], cfg["leaf"], cfg["leaf"], cfg["sc"], tree_build=B.TREE_GPU)
    b = ref.get(LIST_JOBS[cid])
    assert a[0] == b[0] and a[1] == b[1]
    assert a[2].shape == b[2].shape and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("cid", [1, 2, 3, 5])
def test_mixed_full_size_vs_direct(cid):
    cfg, x, y, z, q = refjobs.inputs(cid)
    learned = cid == 5
    if learned:
        from barytree_b200 import selector
        selector.install_default()
    pot = B.treecode(x, y, z, x.copy(), y.copy(), z.copy(), q, kernel=cfg["kernel"], kernel_param=cfg["kp"],
                     approximation=cfg["approx"], compute_type=cfg["ctype"], theta=cfg["theta"],
                     degree=cfg["degree"], max_source_leaf=cfg["leaf"], max_target_leaf=cfg["leaf"],
                     size_check=cfg["sc"], precision=B.PRECISION_MIXED,
                     degree_policy=B.DEGREE_LEARNED if learned else B.DEGREE_FIXED, tolerance=MIXED_TOL)
    n = len(x)
    idx = np.arange(0, n, max(1, n // 10000))
    d = B.direct(x[idx], y[idx], z[idx], x, y, z, q, cfg["kernel"], cfg["kp"])
    err = np.linalg.norm(pot[idx] - d) / np.linalg.norm(d)
    assert err <= MIXED_TOL, f"config {cid}: rel-L2 {err:.3e}"


@pytest.mark.parametrize("cid", [1, 3, 5])
def test_fp64_matches_reference_full_size(ref, cid):
    pot = _fp64(cid)
    idx, want, nsel, nb = ref.get(POT_JOBS[cid])
    assert len(idx) > 0 and (cid != 1 or (nsel == nb and len(idx) == len(pot)))
    got = pot[idx]
    l2 = np.linalg.norm(got - want) / np.linalg.norm(want)
    mx = np.max(np.abs(got - want)) / np.max(np.abs(want))
    assert l2 <= TOL, f"config {cid}: rel-L2 {l2:.3e} over {len(idx)} targets in {nsel} of {nb} batches"
    assert mx <= TOL, f"config {cid}: max {mx:.3e} over {len(idx)} targets in {nsel} of {nb} batches"
