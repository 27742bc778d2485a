"""ctypes loaders for the oracle libraries (test infrastructure only).

* ``libbt_oracle.so`` -- the CPU FP64 restatement of the BaryTree treecode
  (``oracle/bt_oracle.c``), built by ``make -C oracle``.
* ``_ref/libBaryTree_ref.so`` and ``_ref/libBaryTree_reflists.so`` -- the
  reference's own C sources compiled here by ``make -C oracle ref`` (present
  only where the reference tree was available at build time; the built files
  travel with the repository checkout).

Only tests, the smoke check and the benchmark's CPU-baseline leg import this
module.  The barytree_b200 product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

_BTI_ARGS = (
    ctypes.c_int, ctypes.c_int,
    _dp, _dp, _dp, _dp,
    _dp, _dp, _dp, _dp, _dp,
    _dp, ctypes.c_int, ctypes.c_int, _dp,
    ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ctypes.c_double, ctypes.c_double, ctypes.c_int,
)

_LISTS_ARGS = (
    ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
    ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
    ctypes.c_int, ctypes.c_int, ctypes.c_double,
    _ip, _ip, _ip, ctypes.c_long,
)


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def build_oracle() -> None:
    """Compile the restatement (cheap; gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        path = os.path.join(HERE, "libbt_oracle.so")
        if not os.path.exists(path):
            build_oracle()
        lib = ctypes.CDLL(path)
        lib.bto_direct.argtypes = (ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _dp, _dp, _dp, _dp,
                                   ctypes.c_int, ctypes.c_double, _dp)
        lib.bto_direct.restype = ctypes.c_int
        lib.bto_treecode.argtypes = _BTI_ARGS
        lib.bto_treecode.restype = ctypes.c_int
        lib.bto_lists.argtypes = _LISTS_ARGS
        lib.bto_lists.restype = ctypes.c_long
        lib.bto_tree.argtypes = (ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _ip, _dp, ctypes.c_int)
        lib.bto_tree.restype = ctypes.c_int
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libBaryTree_ref.so")) and \
        os.path.exists(os.path.join(REF_DIR, "libBaryTree_reflists.so"))


_ref = None
_reflists = None


def ref_lib():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(os.path.join(REF_DIR, "libBaryTree_ref.so"))
        lib.BaryTreeInterface.argtypes = _BTI_ARGS
        lib.BaryTreeInterface.restype = None
        _ref = lib
    return _ref


def reflists_lib():
    global _reflists
    if _reflists is None:
        lib = ctypes.CDLL(os.path.join(REF_DIR, "libBaryTree_reflists.so"))
        lib.refl_lists.argtypes = _LISTS_ARGS
        lib.refl_lists.restype = ctypes.c_long
        lib.refl_tree.argtypes = (ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _ip, _dp, ctypes.c_int)
        lib.refl_tree.restype = ctypes.c_int
        _reflists = lib
    return _reflists


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def direct(tx, ty, tz, sx, sy, sz, sq, kernel=1, kernel_param=0.0):
    """FP64 direct sum on the CPU (OpenMP)."""
    tx, ty, tz, sx, sy, sz, sq = map(_c, (tx, ty, tz, sx, sy, sz, sq))
    out = np.zeros(len(tx))
    oracle_lib().bto_direct(len(tx), _p(tx), _p(ty), _p(tz), len(sx), _p(sx), _p(sy), _p(sz), _p(sq),
                            kernel, float(kernel_param), _p(out))
    return out


def _call_bti(fn, tx, ty, tz, tq, sx, sy, sz, sq, sw, kernel, kparams, singularity, approximation,
              compute_type, theta, degree, max_source_leaf, max_target_leaf, size_check, beta, verbosity):
    tx, ty, tz, sx, sy, sz, sq = map(_c, (tx, ty, tz, sx, sy, sz, sq))
    tq = _c(tq) if tq is not None else np.zeros(len(tx))
    sw = _c(sw) if sw is not None else np.ones(len(sx))
    kp = _c(np.atleast_1d(kparams if kparams is not None else [0.0]))
    out = np.zeros(len(tx))
    rc = fn(len(tx), len(sx), _p(tx), _p(ty), _p(tz), _p(tq), _p(sx), _p(sy), _p(sz), _p(sq), _p(sw),
            _p(out), int(kernel), len(kp), _p(kp), int(singularity), int(approximation), int(compute_type),
            float(theta), int(degree), int(max_source_leaf), int(max_target_leaf), float(size_check),
            float(beta), int(verbosity))
    return out, rc


def treecode(*args, **kw):
    """The restatement: same arguments as BaryTreeInterface; returns the potential."""
    out, rc = _call_bti(oracle_lib().bto_treecode, *args, **kw)
    if rc != 0:
        raise RuntimeError(f"bto_treecode returned {rc}")
    return out


def ref_treecode(*args, **kw):
    """The reference itself (built from its own sources), same arguments."""
    out, _ = _call_bti(ref_lib().BaryTreeInterface, *args, **kw)
    return out


def _lists(fn, tx, ty, tz, sx, sy, sz, compute_type, approximation, theta, degree, max_s, max_t, size_check):
    tx, ty, tz, sx, sy, sz = map(_c, (tx, ty, tz, sx, sy, sz))
    units = ctypes.c_int(0)
    nodes = ctypes.c_int(0)
    cap = 1 << 16
    while True:
        ent = np.zeros(3 * cap, dtype=np.int32)
        n = fn(len(tx), len(sx), _p(tx), _p(ty), _p(tz), _p(sx), _p(sy), _p(sz), int(compute_type),
               int(approximation), float(theta), int(degree), int(max_s), int(max_t), float(size_check),
               ctypes.byref(units), ctypes.byref(nodes), ent.ctypes.data_as(_ip), cap)
        if n >= 0:
            return units.value, nodes.value, ent[: 3 * n].reshape(-1, 3)
        cap *= 4


def lists(*args):
    return _lists(oracle_lib().bto_lists, *args)


def ref_lists(*args):
    return _lists(reflists_lib().refl_lists, *args)


def _tree(fn, x, y, z, maxpar):
    x, y, z = map(_c, (x, y, z))
    cap = max(64, 4 * len(x) // max(1, maxpar) + 64)
    ints = np.zeros(4 * cap, dtype=np.int32)
    dbl = np.zeros(7 * cap)
    n = fn(len(x), _p(x), _p(y), _p(z), int(maxpar), ints.ctypes.data_as(_ip), _p(dbl), cap)
    assert n >= 0
    return ints[: 4 * n].reshape(-1, 4), dbl[: 7 * n].reshape(-1, 7)


def tree(x, y, z, maxpar):
    return _tree(oracle_lib().bto_tree, x, y, z, maxpar)


def ref_tree(x, y, z, maxpar):
    return _tree(reflists_lib().refl_tree, x, y, z, maxpar)


def ref_tree_order(x, y, z, maxpar):
    """The reference's particle permutation (0-based input index per sorted slot)."""
    x, y, z = map(_c, (x, y, z))
    L = reflists_lib()
    L.refl_tree_order.argtypes = (ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _ip)
    L.refl_tree_order.restype = ctypes.c_int
    order = np.zeros(max(1, len(x)), dtype=np.int32)
    L.refl_tree_order(len(x), _p(x), _p(y), _p(z), int(maxpar), order.ctypes.data_as(_ip))
    return order[: len(x)]


_refsample = None


def refsample_lib():
    global _refsample
    if _refsample is None:
        lib = ctypes.CDLL(os.path.join(REF_DIR, "libBaryTree_refsample.so"))
        lib.refs_setup.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                   ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp)
        lib.refs_setup.restype = ctypes.c_void_p
        lib.refs_num_batches.argtypes = (ctypes.c_void_p,)
        lib.refs_num_batches.restype = ctypes.c_int
        lib.refs_batch_work.argtypes = (ctypes.c_void_p, ctypes.c_int)
        lib.refs_batch_work.restype = ctypes.c_longlong
        lib.refs_batch_size.argtypes = (ctypes.c_void_p, ctypes.c_int)
        lib.refs_batch_size.restype = ctypes.c_int
        lib.refs_eval.argtypes = (ctypes.c_void_p, ctypes.c_int, _ip, ctypes.c_int, _dp, _dp)
        lib.refs_eval.restype = ctypes.c_double
        lib.refs_free.argtypes = (ctypes.c_void_p,)
        lib.refs_free.restype = None
        _refsample = lib
    return _refsample


class RefSampled:
    """The reference's particle-cluster treecode (built from its own sources)
    with setup and per-batch evaluation split (oracle/ref_sampled.c): full-size
    systems are set up once, then any subset of the target batches is
    evaluated with exactly the values a full call gives those targets."""

    def __init__(self, tx, ty, tz, sx, sy, sz, sq, kernel, kparams, approximation, theta, degree, max_source_leaf,
                 max_target_leaf, size_check):
        tx, ty, tz, sx, sy, sz, sq = map(_c, (tx, ty, tz, sx, sy, sz, sq))
        kp = _c(np.atleast_1d(kparams if kparams is not None else [0.0]))
        self.lib = refsample_lib()
        self.nt = len(tx)
        phases = np.zeros(4)
        self.h = self.lib.refs_setup(len(tx), len(sx), _p(tx), _p(ty), _p(tz), _p(sx), _p(sy), _p(sz), _p(sq),
                                     int(kernel), len(kp), _p(kp), int(approximation), float(theta), int(degree),
                                     int(max_source_leaf), int(max_target_leaf), float(size_check), _p(phases))
        self.setup_seconds = dict(zip(("source_tree", "target_batches", "source_proxies", "lists"),
                                      map(float, phases)))
        self.nbatches = self.lib.refs_num_batches(self.h)
        self.work = np.array([self.lib.refs_batch_work(self.h, b) for b in range(self.nbatches)], dtype=np.int64)
        self.sizes = np.array([self.lib.refs_batch_size(self.h, b) for b in range(self.nbatches)], dtype=np.int64)

    def evaluate(self, batches, threads=1, out=None, batch_seconds=False):
        """Potentials of the given batches' targets, written into `out`
        (caller order; NaN elsewhere if `out` is None).  Returns (out, wall
        seconds), and with batch_seconds=True also each batch's own seconds."""
        sel = np.ascontiguousarray(batches, dtype=np.int32)
        if out is None:
            out = np.full(self.nt, np.nan)
        per = np.zeros(len(sel))
        secs = self.lib.refs_eval(self.h, len(sel), sel.ctypes.data_as(_ip), int(threads), _p(out), _p(per))
        return (out, secs, per) if batch_seconds else (out, secs)

    def close(self):
        if self.h:
            self.lib.refs_free(self.h)
            self.h = None

    def __del__(self):
        self.close()
