import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the oracle (gcc) and the product library (nvcc) if absent."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "libbt_oracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not os.path.exists(os.path.join(ROOT, "barytree_b200", "libbarytree_b200.so")):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "barytree_b200", "csrc")], check=True)
    yield


def uniform_inputs(seed, n, targets="same"):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    q = rng.uniform(-1, 1, n)
    if targets == "same":
        tx, ty, tz = x.copy(), y.copy(), z.copy()
    else:
        tx, ty, tz = (np.clip(rng.normal(0, 0.4, n), -1, 1) for _ in range(3))
    return tx, ty, tz, x, y, z, q


def golden_files():
    d = os.path.join(ROOT, "tests", "golden")
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(".npz"))


def same_members(ints, order_a, order_b):
    """Whether two particle permutations put the same particles in every
    leaf of the tree summary `ints` (1-based ibeg, iend, children, level)."""
    for b, e, nch, _ in ints:
        if nch == 0 and not np.array_equal(np.sort(order_a[b - 1:e]), np.sort(order_b[b - 1:e])):
            return False
    return True
