"""CPU tests of the tile-shape table behind the autotuner (no device needed):
installing, reading back, removing, saving and loading shapes, rejecting
shapes the particle-output kernel does not provide, and refusing to tune
anything but the mixed-precision kernel."""
import numpy as np
import pytest

import barytree_b200 as B


@pytest.fixture(autouse=True)
def clean_table():
    yield
    for k in (B.Kernel.COULOMB, B.Kernel.YUKAWA):
        for a in (B.Approximation.LAGRANGE, B.Approximation.HERMITE):
            B.tuning_set(None, k, a)


def test_defaults_when_nothing_installed():
    shape, installed = B.tuning_get(B.Kernel.COULOMB, B.Approximation.LAGRANGE)
    assert not installed
    assert (shape["targets_per_thread"], shape["source_tile"], shape["dispatch"]) == (2, 1024, B.DISPATCH_GRID)


def test_set_get_remove_save_load(tmp_path):
    s1 = {"targets_per_thread": 4, "source_tile": 512, "dispatch": B.DISPATCH_QUEUE, "ms": 1.5}
    s2 = {"targets_per_thread": 1, "source_tile": 2048, "dispatch": B.DISPATCH_GRID, "ms": 2.0}
    B.tuning_set(s1, B.Kernel.COULOMB, B.Approximation.LAGRANGE)
    B.tuning_set(s2, B.Kernel.YUKAWA, B.Approximation.HERMITE)
    got, inst = B.tuning_get(B.Kernel.COULOMB, B.Approximation.LAGRANGE)
    assert inst and got == s1
    assert not B.tuning_get(B.Kernel.COULOMB, B.Approximation.HERMITE)[1]
    path = str(tmp_path / "tuning.json")
    assert B.save_tuning(path) == 2
    B.tuning_set(None, B.Kernel.COULOMB, B.Approximation.LAGRANGE)
    B.tuning_set(None, B.Kernel.YUKAWA, B.Approximation.HERMITE)
    assert not B.tuning_get(B.Kernel.COULOMB, B.Approximation.LAGRANGE)[1]
    assert B.load_tuning(path) == 2
    assert B.tuning_get(B.Kernel.YUKAWA, B.Approximation.HERMITE) == (s2, True)


@pytest.mark.parametrize("tpt,tile,disp", [(3, 1024, 2), (2, 1000, 2), (2, 1024, 0), (8, 512, 1)])
def test_invalid_shapes_rejected(tpt, tile, disp):
    with pytest.raises(B.BaryTreeError) as e:
        B.tuning_set({"targets_per_thread": tpt, "source_tile": tile, "dispatch": disp})
    assert e.value.code == B.BT_ERR_PARAM
    assert not B.tuning_get()[1]


def test_autotune_needs_mixed_precision():
    rng = np.random.default_rng(0)
    x, y, z, q = (rng.uniform(-1, 1, 100) for _ in range(4))
    best = B.Tuning()
    opts = B.Options(B.PRECISION_FP64, 0, 1e-6, 0, 0, 0, 0)
    off = np.array([0, 100], dtype=np.int64)
    p = lambda a: a.ctypes.data_as(B._dp)  # noqa: E731
    rc = B.lib().bt_autotune(1, off.ctypes.data_as(B._llp), off.ctypes.data_as(B._llp), p(x), p(y), p(z), p(x),
                             p(y), p(z), p(q), 1, 0.0, 1, 1, 0.7, 8, 50, 50, 1.0, B.ctypes.byref(opts),
                             B.ctypes.byref(best), None, 0, None)
    assert rc == B.BT_ERR_UNSUPPORTED
    assert "BT_PRECISION_MIXED" in B.last_error()


def test_invalid_upward_option_is_a_parameter_error():
    rng = np.random.default_rng(1)
    x, y, z, q = (rng.uniform(-1, 1, 50) for _ in range(4))
    with pytest.raises(B.BaryTreeError) as e:
        B.treecode(x, y, z, x, y, z, q, precision=B.PRECISION_MIXED, upward=7)
    assert e.value.code == B.BT_ERR_PARAM and "upward" in B.last_error()


def test_shard_arguments_are_checked_before_any_device_use():
    rng = np.random.default_rng(2)
    x, y, z, q = (rng.uniform(-1, 1, 60) for _ in range(4))
    with pytest.raises(B.BaryTreeError) as e:
        B.treecode(x, y, z, x, y, z, q, precision=B.PRECISION_MIXED, shard=(3, 3))
    assert e.value.code == B.BT_ERR_PARAM
    with pytest.raises(B.BaryTreeError) as e:
        B.treecode(x, y, z, x, y, z, q, compute_type=B.ComputeType.CLUSTER_CLUSTER, shard=(-1, 2))
    assert e.value.code == B.BT_ERR_PARAM and "shard index" in B.last_error()
    with pytest.raises(B.BaryTreeError) as e:
        B.treecode(x, y, z, x, y, z, q, compute_type=B.ComputeType.CLUSTER_PARTICLE, shard=(0, -2))
    assert e.value.code == B.BT_ERR_PARAM and "shard count" in B.last_error()
