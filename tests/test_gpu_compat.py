"""GPU tests of the driver-level compatibility layer.

The strongest check is the reference's own test program (tests/serial_tests.c),
compiled against the reference's headers and linked against
libbarytree_b200.so instead of the reference sources (oracle/_ref/tests_b200,
built by `make -C oracle ref`): all six of its tests -- closed-form lattice
direct sums, lattice treecodes in Lagrange/Hermite x Coulomb/Yukawa x
skipping/subtraction, single-target accuracy, parameter monotonicity, wrapper
equivalence and the cluster-cluster sum -- must pass through this library's
treedriver, directdriver and BaryTreeInterface.

Also: treedriver adds into the potential and equals BaryTreeInterface bit for
bit, and the direct sum with singularity subtraction equals a numpy
restatement of the reference's subtraction pair terms and correction.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import barytree_b200 as B
from compat_structs import RunParams, declare, particles
from conftest import ROOT

pytestmark = pytest.mark.gpu

TESTS_B200 = os.path.join(ROOT, "oracle", "_ref", "tests_b200")
NAMES = ["direct_sum_on_10_particles", "treecode_on_100_particles", "treecode_on_1_target_10000_sources",
         "treecode_parameters_on_1_target_5000_sources", "treecode_wrapper", "BLDTT"]


@pytest.mark.parametrize("idx", range(6), ids=NAMES)
def test_reference_test_program_against_this_library(idx):
    if not os.path.exists(TESTS_B200):
        pytest.skip("oracle/_ref/tests_b200 not built (make -C oracle ref)")
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.dirname(B.LIB_PATH))
    r = subprocess.run([TESTS_B200, str(idx)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    assert "TEST FAILED" not in r.stdout
    assert f"Completed test_{NAMES[idx]}()" in r.stdout


_dp = ctypes.POINTER(ctypes.c_double)


def _setup(lib, kernel, kp, approx, sing, ctype, theta, degree, leaf, sc):
    rp = ctypes.POINTER(RunParams)()
    kp = np.asarray(kp, dtype=np.float64)
    lib.RunParams_Setup(ctypes.byref(rp), kernel, len(kp), kp.ctypes.data_as(_dp), approx, sing, ctype, theta,
                        degree, leaf, leaf, sc, -1.0, 0)
    return rp


@pytest.mark.parametrize("kernel,kp,approx,sing,ctype", [(1, [0.5], 1, 1, 1), (2, [0.5], 2, 2, 1),
                                                         (1, [0.5], 1, 2, 3), (3, [0.4, 0.01], 1, 2, 1)])
def test_treedriver_adds_and_equals_interface(kernel, kp, approx, sing, ctype):
    lib = declare(ctypes.CDLL(B.LIB_PATH))
    rng = np.random.default_rng(11)
    n = 6000
    sx, sy, sz = (rng.uniform(-1, 1, n) for _ in range(3))
    sq, sw = rng.uniform(-1, 1, n), rng.uniform(0.5, 1.5, n)
    tx, ty, tz = sx.copy(), sy.copy(), sz.copy()
    tq = rng.uniform(-1, 1, n)
    rp = _setup(lib, kernel, kp, approx, sing, ctype, 0.7, 6, 300, 1.0)
    src, tgt = particles(sx, sy, sz, sq, sw), particles(tx, ty, tz, tq)
    pot = np.zeros(n)
    times = np.zeros(13)
    lib.treedriver(ctypes.byref(src), ctypes.byref(tgt), rp, pot.ctypes.data_as(_dp), times.ctypes.data_as(_dp))
    want = B.treecode(tx, ty, tz, sx, sy, sz, sq, kernel=kernel, kernel_param=kp, approximation=approx,
                      compute_type=ctype, theta=0.7, degree=6, max_source_leaf=300, max_target_leaf=300,
                      size_check=1.0, singularity=sing, target_q=tq, source_w=sw)
    assert np.array_equal(pot, want)
    assert times[0] > 0 and times[12] > 0
    lib.treedriver(ctypes.byref(src), ctypes.byref(tgt), rp, pot.ctypes.data_as(_dp), times.ctypes.data_as(_dp))
    assert np.array_equal(pot, want + want)          # accumulates like the reference
    lib.RunParams_Free(ctypes.byref(rp))


def _ss_direct_numpy(tx, ty, tz, tq, sx, sy, sz, sq, sw, kernel, kp):
    """Restatement of the reference's subtraction pair terms and correction
    (src/kernels/coulomb/coulomb_ss_pp.c, yukawa/yukawa_ss_pp.c,
    regularized-coulomb/regularized-coulomb_ss_pp.c:30-45,
    regularized-yukawa/regularized-yukawa_ss_pp.c,
    src/interaction_compute/interaction_compute_correction.c:22-45)."""
    dx, dy, dz = tx[:, None] - sx[None, :], ty[:, None] - sy[None, :], tz[:, None] - sz[None, :]
    r2 = dx * dx + dy * dy + dz * dz
    r = np.sqrt(r2)
    q, w, t = sq[None, :], sw[None, :], tq[:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        if kernel == 1:
            f = np.where(r > np.finfo(float).tiny, (q - t * np.exp(-r2 / kp[0] ** 2)) * w / r, 0.0)
            c = 2 * np.pi * kp[0] ** 2
        elif kernel == 2:
            f = np.where(r > np.finfo(float).tiny, (q - t) * w * np.exp(-kp[0] * r) / r, 0.0)
            c = 4 * np.pi / kp[0] ** 2
        elif kernel == 3:
            f = (q - t * np.exp(-r2 / kp[0] ** 2)) * w / np.sqrt(r2 + kp[1] ** 2)
            c = 2 * np.pi * kp[0] ** 2
        else:
            f = (q - t) * w * np.exp(-kp[0] * r) / np.sqrt(r2 + kp[1] ** 2)
            c = 4 * np.pi / kp[0] ** 2
    return f.sum(axis=1) + c * tq


@pytest.mark.parametrize("kernel,kp", [(1, [0.5]), (2, [0.5]), (3, [0.4, 0.01]), (4, [0.5, 0.01])])
def test_direct_sum_with_subtraction(kernel, kp):
    rng = np.random.default_rng(5)
    ns, nt = 3000, 1000
    sx, sy, sz = (rng.uniform(-1, 1, ns) for _ in range(3))
    sq, sw = rng.uniform(-1, 1, ns), rng.uniform(0.5, 1.5, ns)
    tx, ty, tz = sx[:nt].copy(), sy[:nt].copy(), sz[:nt].copy()    # coincident pairs included
    tq = rng.uniform(-1, 1, nt)
    got = B.direct(tx, ty, tz, sx, sy, sz, sq, kernel=kernel, kernel_param=kp,
                   singularity=B.Singularity.SUBTRACTION, target_q=tq, source_w=sw)
    want = _ss_direct_numpy(tx, ty, tz, tq, sx, sy, sz, sq, sw, kernel, np.asarray(kp))
    assert np.linalg.norm(got - want) <= 1e-13 * np.linalg.norm(want)
    # kernels without a subtraction term ignore the setting, as in the reference
    plain = B.direct(tx, ty, tz, sx, sy, sz, sq, kernel=B.Kernel.ATAN, kernel_param=[2.0, 0.1])
    ss = B.direct(tx, ty, tz, sx, sy, sz, sq, kernel=B.Kernel.ATAN, kernel_param=[2.0, 0.1],
                  singularity=B.Singularity.SUBTRACTION, target_q=tq, source_w=sw)
    assert np.array_equal(plain, ss)
