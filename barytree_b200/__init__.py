"""barytree_b200 -- B200-native barycentric treecode (BaryTree drop-in).

Python host side of the library.  It mirrors the reference's ctypes binding
(``interfaces/python/BaryTreeInterface.py``): the same enums and the same
``callTreedriver`` function, so existing scripts switch by changing the
import.  Everything computes in ``libbarytree_b200.so`` (hand-written sm_100a
CUDA kernels behind a C ABI); there is no CPU fallback, and loading fails
loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import os
from enum import IntEnum

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("BARYTREE_B200_LIB") or os.path.join(_HERE, "libbarytree_b200.so")


class CEnum(IntEnum):
    @classmethod
    def from_param(cls, obj):
        return int(obj)


class Kernel(CEnum):
    NO_KERNEL = 0
    COULOMB = 1
    YUKAWA = 2
    REGULARIZED_COULOMB = 3
    REGULARIZED_YUKAWA = 4
    ATAN = 5
    TCF = 6
    DCF = 7
    SIN_OVER_R = 8
    MQ = 9
    RBS_U = 10
    RBS_V = 11
    USER = 12


class Singularity(CEnum):
    NO_SINGULARITY = 0
    SKIPPING = 1
    SUBTRACTION = 2


class Approximation(CEnum):
    NO_APPROXIMATION = 0
    LAGRANGE = 1
    HERMITE = 2


class ComputeType(CEnum):
    NO_COMPUTE_TYPE = 0
    PARTICLE_CLUSTER = 1
    CLUSTER_PARTICLE = 2
    CLUSTER_CLUSTER = 3


# status codes (include/barytree_b200.h)
BT_OK, BT_ERR_PARAM, BT_ERR_UNSUPPORTED, BT_ERR_CUDA, BT_ERR_TIMEOUT, BT_ERR_NO_DEVICE = range(6)
PRECISION_FP64, PRECISION_MIXED = 0, 1
DEGREE_FIXED, DEGREE_LEARNED = 0, 1
TREE_GPU, TREE_HOST = 0, 1
DISPATCH_AUTO, DISPATCH_QUEUE, DISPATCH_GRID = 0, 1, 2
UPWARD_AUTO, UPWARD_FP64 = 0, 1
SYMMETRY_AUTO, SYMMETRY_OFF = 0, 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("degree_policy", ctypes.c_int), ("tolerance", ctypes.c_double),
                ("device", ctypes.c_int), ("inputs_on_device", ctypes.c_int), ("tree_build", ctypes.c_int),
                ("dispatch", ctypes.c_int), ("upward", ctypes.c_int), ("shard_index", ctypes.c_int),
                ("shard_count", ctypes.c_int), ("symmetry", ctypes.c_int)]


class Report(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_double), ("ms_setup", ctypes.c_double), ("ms_upward", ctypes.c_double),
                ("ms_compute", ctypes.c_double), ("ms_downward", ctypes.c_double), ("ms_transfer", ctypes.c_double),
                ("num_pp", ctypes.c_longlong), ("num_pc", ctypes.c_longlong), ("num_cp", ctypes.c_longlong),
                ("num_cc", ctypes.c_longlong), ("pp_ptwise", ctypes.c_longlong), ("pc_ptwise", ctypes.c_longlong),
                ("cp_ptwise", ctypes.c_longlong), ("cc_ptwise", ctypes.c_longlong),
                ("ms_eval_kernel", ctypes.c_double), ("eval_flops", ctypes.c_longlong),
                ("source_nodes", ctypes.c_int), ("target_nodes", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("selected", ctypes.c_longlong * 14), ("sym_ptwise", ctypes.c_longlong)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["selected"] = list(self.selected)
        return d


class Tuning(ctypes.Structure):
    """bt_tuning: tile shape of the mixed particle-output kernel."""
    _fields_ = [("targets_per_thread", ctypes.c_int), ("source_tile", ctypes.c_int), ("dispatch", ctypes.c_int),
                ("ms", ctypes.c_float)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BaryTreeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"barytree_b200 error {code}: {msg}")
        self.code = code


_BTI_ARGS = (
    ctypes.c_int, ctypes.c_int,
    _dp, _dp, _dp, _dp,
    _dp, _dp, _dp, _dp, _dp,
    _dp, ctypes.c_int, ctypes.c_int, _dp,
    ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ctypes.c_double, ctypes.c_double, ctypes.c_int,
)

# every exported symbol of include/barytree_b200.h
EXPORTED_SYMBOLS = ("BaryTreeInterface", "BaryTreeInterface_ex", "bt_eval", "bt_direct", "bt_lists", "bt_lists_ex",
                    "bt_tree_dump", "bt_tree_dump_ex", "bt_eval_batch", "bt_direct_ex", "bt_session_create", "bt_session_eval", "bt_session_destroy", "bt_measure_peaks", "bt_last_error", "bt_kernel_launch_count",
                    "bt_selector_nweights", "bt_selector_set", "bt_selector_training_data", "bt_selector_train",
                    "bt_mlp_loss_grad", "bt_mlp_predict", "bt_eval_ex", "bt_direct_full", "bt_eval_noalloc",
                    "treedriver", "directdriver", "RunParams_Setup", "RunParams_Validate", "RunParams_Free",
                    "RunParams_Print", "bt_autotune", "bt_tuning_set", "bt_tuning_get")

_lib = None


def lib():
    """Load libbarytree_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not found: build it with `make -C barytree_b200/csrc`")
    L = ctypes.CDLL(LIB_PATH)
    L.BaryTreeInterface.argtypes = _BTI_ARGS
    L.BaryTreeInterface.restype = None
    L.BaryTreeInterface_ex.argtypes = _BTI_ARGS
    L.BaryTreeInterface_ex.restype = ctypes.c_int
    L.bt_eval.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                          ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                          ctypes.POINTER(Options), ctypes.POINTER(Report))
    L.bt_eval.restype = ctypes.c_int
    L.bt_direct.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                            ctypes.c_int, ctypes.c_double, ctypes.c_int)
    L.bt_direct.restype = ctypes.c_int
    L.bt_lists.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
                           ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                           ctypes.c_int, ctypes.c_int, ctypes.c_double, _ip, _ip, _ip, ctypes.c_long)
    L.bt_lists.restype = ctypes.c_long
    L.bt_lists_ex.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
                              ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                              _ip, _ip, _ip, ctypes.c_long)
    L.bt_lists_ex.restype = ctypes.c_long
    L.bt_tree_dump.argtypes = (ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _ip, _dp, ctypes.c_int)
    L.bt_tree_dump.restype = ctypes.c_int
    L.bt_eval_batch.argtypes = (ctypes.c_int, _llp, _llp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                ctypes.POINTER(Options), ctypes.POINTER(Report))
    L.bt_eval_batch.restype = ctypes.c_int
    L.bt_direct_ex.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int,
                               ctypes.c_int, _dp, ctypes.c_int)
    L.bt_direct_ex.restype = ctypes.c_int
    L.bt_direct_full.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                 ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int)
    L.bt_direct_full.restype = ctypes.c_int
    L.bt_eval_ex.argtypes = (ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                             ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                             ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                             ctypes.c_double, ctypes.POINTER(Options), ctypes.POINTER(Report))
    L.bt_eval_ex.restype = ctypes.c_int
    L.bt_autotune.argtypes = (ctypes.c_int, _llp, _llp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int,
                              ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(Options),
                              ctypes.POINTER(Tuning), ctypes.POINTER(Tuning), ctypes.c_int,
                              ctypes.POINTER(ctypes.c_int))
    L.bt_autotune.restype = ctypes.c_int
    L.bt_tuning_set.argtypes = (ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Tuning))
    L.bt_tuning_set.restype = ctypes.c_int
    L.bt_tuning_get.argtypes = (ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Tuning),
                                ctypes.POINTER(ctypes.c_int))
    L.bt_tuning_get.restype = ctypes.c_int
    L.bt_session_create.argtypes = (ctypes.c_int, _llp, _llp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(Options),
                                    ctypes.POINTER(ctypes.c_void_p))
    L.bt_session_create.restype = ctypes.c_int
    L.bt_session_eval.argtypes = (ctypes.c_void_p, _dp, _dp, ctypes.POINTER(Report))
    L.bt_session_eval.restype = ctypes.c_int
    L.bt_session_destroy.argtypes = (ctypes.c_void_p,)
    L.bt_session_destroy.restype = ctypes.c_int
    L.bt_tree_dump_ex.argtypes = (ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _dp,
                                  _ip, ctypes.c_int)
    L.bt_tree_dump_ex.restype = ctypes.c_int
    L.bt_measure_peaks.argtypes = (ctypes.c_int, _dp, _dp, _dp)
    L.bt_measure_peaks.restype = ctypes.c_int
    _fp = ctypes.POINTER(ctypes.c_float)
    L.bt_selector_nweights.argtypes = ()
    L.bt_selector_nweights.restype = ctypes.c_long
    L.bt_selector_set.argtypes = (_fp, ctypes.c_long)
    L.bt_selector_set.restype = ctypes.c_int
    L.bt_selector_training_data.argtypes = (ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_uint, _fp, _fp, ctypes.c_int)
    L.bt_selector_training_data.restype = ctypes.c_long
    L.bt_selector_train.argtypes = (_fp, _fp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                    ctypes.c_uint, _fp, _fp, ctypes.c_int)
    L.bt_selector_train.restype = ctypes.c_int
    L.bt_mlp_loss_grad.argtypes = (_fp, _fp, _fp, ctypes.c_int, _fp, _fp, ctypes.c_int)
    L.bt_mlp_loss_grad.restype = ctypes.c_int
    L.bt_mlp_predict.argtypes = (_fp, _fp, ctypes.c_long, _fp, ctypes.c_int)
    L.bt_mlp_predict.restype = ctypes.c_int
    L.bt_last_error.argtypes = ()
    L.bt_last_error.restype = ctypes.c_char_p
    L.bt_kernel_launch_count.argtypes = ()
    L.bt_kernel_launch_count.restype = ctypes.c_longlong
    _lib = L
    return L


def last_error() -> str:
    return lib().bt_last_error().decode()


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _shard(shard):
    """(shard_index, shard_count) from None or a pair."""
    if shard is None:
        return 0, 0
    k, n = shard
    return int(k), int(n)


def _check(rc):
    if rc != BT_OK:
        raise BaryTreeError(rc, last_error())


def callTreedriver(numTargets, numSources,
                   targetX, targetY, targetZ, targetValue,
                   sourceX, sourceY, sourceZ, sourceValue, sourceWeight,
                   kernelName, numberOfKernelParameters, kernelParameters, singularityHandling,
                   approximationName, computeType, GPUpresent=True, verbosity=0,
                   beta=None, theta=None, degree=None, sourceLeafSize=None, targetLeafSize=None, sizeCheck=None):
    """Evaluate potentials at the targets; same arguments and defaults as the
    reference binding (interfaces/python/BaryTreeInterface.py:82-152).

    Either ``beta`` or all of theta/degree/sourceLeafSize/targetLeafSize must
    be given; sizeCheck defaults to 1.0 (Lagrange) or 4.0 (Hermite).  The
    computation always runs on the GPU; ``GPUpresent`` is accepted for
    signature compatibility.  Raises BaryTreeError instead of exiting.
    """
    if beta:
        theta, degree, sourceLeafSize, targetLeafSize = -1.0, -1, 1, 1
    else:
        assert theta is not None, "If beta isn't provided, theta must be."
        assert degree is not None, "If beta isn't provided, degree must be."
        assert sourceLeafSize is not None, "If beta isn't provided, sourceLeafSize must be."
        assert targetLeafSize is not None, "If beta isn't provided, targetLeafSize must be."
        beta = -1
    if not sizeCheck:
        sizeCheck = 4.0 if approximationName == Approximation.HERMITE else 1.0
    tx, ty, tz, sx, sy, sz, sq = map(_c, (targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue))
    tq = _c(targetValue) if targetValue is not None else None
    sw = _c(sourceWeight) if sourceWeight is not None else None
    kp = _c(np.atleast_1d(kernelParameters if kernelParameters is not None else [0.0]))
    out = np.zeros(numTargets)
    rc = lib().BaryTreeInterface_ex(int(numTargets), int(numSources), _p(tx), _p(ty), _p(tz), _p(tq),
                                    _p(sx), _p(sy), _p(sz), _p(sq), _p(sw), _p(out), int(kernelName),
                                    int(numberOfKernelParameters), _p(kp), int(singularityHandling),
                                    int(approximationName), int(computeType), float(theta), int(degree),
                                    int(sourceLeafSize), int(targetLeafSize), float(sizeCheck), float(beta),
                                    int(verbosity))
    _check(rc)
    return out


def treecode(tx, ty, tz, sx, sy, sz, sq, kernel=Kernel.COULOMB, kernel_param=0.0,
             approximation=Approximation.LAGRANGE, compute_type=ComputeType.PARTICLE_CLUSTER,
             theta=0.7, degree=8, max_source_leaf=2000, max_target_leaf=2000, size_check=1.0,
             precision=PRECISION_FP64, degree_policy=DEGREE_FIXED, tolerance=1e-6, device=0,
             tree_build=TREE_GPU, dispatch=DISPATCH_AUTO, return_report=False,
             singularity=Singularity.SKIPPING, target_q=None, source_w=None, beta=-1.0, upward=UPWARD_AUTO, shard=None, symmetry=SYMMETRY_AUTO):
    """Extended entry point (bt_eval_ex): options for precision / degree policy /
    tree build and a report.  kernel_param may be a sequence (two parameters
    for regularized Coulomb/Yukawa, atan, MQ); singularity subtraction takes
    the target charges and source weights."""
    tx, ty, tz, sx, sy, sz, sq = map(_c, (tx, ty, tz, sx, sy, sz, sq))
    tq = _c(target_q) if target_q is not None else None
    sw = _c(source_w) if source_w is not None else None
    kp = _c(np.atleast_1d(np.asarray(kernel_param, dtype=np.float64)))
    out = np.zeros(len(tx))
    opts = Options(int(precision), int(degree_policy), float(tolerance), int(device), 0, int(tree_build), int(dispatch), int(upward), *_shard(shard), int(symmetry))
    rep = Report()
    rc = lib().bt_eval_ex(len(tx), len(sx), _p(tx), _p(ty), _p(tz), _p(tq), _p(sx), _p(sy), _p(sz), _p(sq), _p(sw),
                          _p(out), int(kernel), len(kp), _p(kp), int(singularity), int(approximation),
                          int(compute_type), float(theta), int(degree), int(max_source_leaf), int(max_target_leaf),
                          float(size_check), float(beta), ctypes.byref(opts), ctypes.byref(rep))
    _check(rc)
    return (out, rep.as_dict()) if return_report else out


def treecode_batch(systems, kernel=Kernel.COULOMB, kernel_param=0.0, approximation=Approximation.LAGRANGE,
                   compute_type=ComputeType.PARTICLE_CLUSTER, theta=0.7, degree=8, max_source_leaf=2000,
                   max_target_leaf=2000, size_check=1.0, precision=PRECISION_FP64, degree_policy=DEGREE_FIXED,
                   tolerance=1e-6, device=0, tree_build=TREE_GPU, dispatch=DISPATCH_AUTO, return_report=False, upward=UPWARD_AUTO, shard=None, symmetry=SYMMETRY_AUTO):
    """bt_eval_batch over a list of systems (tx, ty, tz, sx, sy, sz, sq); returns one potential array per system."""
    systems = [tuple(map(_c, s)) for s in systems]
    toff = np.concatenate([[0], np.cumsum([len(s[0]) for s in systems])]).astype(np.int64)
    soff = np.concatenate([[0], np.cumsum([len(s[3]) for s in systems])]).astype(np.int64)
    cat = [_c(np.concatenate([s[i] for s in systems]) if systems else np.zeros(0)) for i in range(7)]
    out = np.zeros(int(toff[-1]))
    rep = treecode_batch_ptr(len(systems), toff, soff, *(a.ctypes.data for a in cat), out.ctypes.data,
                             kernel=kernel, kernel_param=kernel_param, approximation=approximation,
                             compute_type=compute_type, theta=theta, degree=degree, max_source_leaf=max_source_leaf,
                             max_target_leaf=max_target_leaf, size_check=size_check, precision=precision,
                             degree_policy=degree_policy, tolerance=tolerance, device=device, tree_build=tree_build,
                             dispatch=dispatch, upward=upward, shard=shard, symmetry=symmetry)
    pots = [out[toff[k]:toff[k + 1]].copy() for k in range(len(systems))]
    return (pots, rep) if return_report else pots


def treecode_batch_ptr(nsys, target_offsets, source_offsets, tx, ty, tz, sx, sy, sz, sq, out,
                       kernel=Kernel.COULOMB, kernel_param=0.0, approximation=Approximation.LAGRANGE,
                       compute_type=ComputeType.PARTICLE_CLUSTER, theta=0.7, degree=8, max_source_leaf=2000,
                       max_target_leaf=2000, size_check=1.0, precision=PRECISION_FP64, degree_policy=DEGREE_FIXED,
                       tolerance=1e-6, device=0, inputs_on_device=False, tree_build=TREE_GPU,
                       dispatch=DISPATCH_AUTO, upward=UPWARD_AUTO, shard=None, symmetry=SYMMETRY_AUTO):
    """bt_eval_batch on raw addresses; offsets are host int64 arrays of nsys+1 entries."""
    cast = lambda a: ctypes.cast(ctypes.c_void_p(int(a)), _dp)  # noqa: E731
    toff = np.ascontiguousarray(target_offsets, dtype=np.int64)
    soff = np.ascontiguousarray(source_offsets, dtype=np.int64)
    opts = Options(int(precision), int(degree_policy), float(tolerance), int(device), int(bool(inputs_on_device)),
                   int(tree_build), int(dispatch), int(upward), *_shard(shard), int(symmetry))
    rep = Report()
    rc = lib().bt_eval_batch(int(nsys), toff.ctypes.data_as(_llp), soff.ctypes.data_as(_llp), cast(tx), cast(ty),
                             cast(tz), cast(sx), cast(sy), cast(sz), cast(sq), cast(out), int(kernel),
                             float(kernel_param), int(approximation), int(compute_type), float(theta), int(degree),
                             int(max_source_leaf), int(max_target_leaf), float(size_check), ctypes.byref(opts),
                             ctypes.byref(rep))
    _check(rc)
    return rep.as_dict()


class Session:
    """bt_session_*: trees, lists and the device sequence built once for fixed
    particle positions; evaluate(charges) replays the captured CUDA graph.

    systems: a list of (tx, ty, tz, sx, sy, sz, sq); sq are the charges used
    for a learned degree selection (and need not be passed again)."""

    def __init__(self, systems, kernel=Kernel.COULOMB, kernel_param=0.0, approximation=Approximation.LAGRANGE,
                 compute_type=ComputeType.PARTICLE_CLUSTER, theta=0.7, degree=8, max_source_leaf=2000,
                 max_target_leaf=2000, size_check=1.0, precision=PRECISION_FP64, degree_policy=DEGREE_FIXED,
                 tolerance=1e-6, device=0, dispatch=DISPATCH_AUTO, upward=UPWARD_AUTO, shard=None, symmetry=SYMMETRY_AUTO):
        systems = [tuple(map(_c, s)) for s in systems]
        self.toff = np.concatenate([[0], np.cumsum([len(s[0]) for s in systems])]).astype(np.int64)
        self.soff = np.concatenate([[0], np.cumsum([len(s[3]) for s in systems])]).astype(np.int64)
        cat = [_c(np.concatenate([s[i] for s in systems])) for i in range(7)]
        opts = Options(int(precision), int(degree_policy), float(tolerance), int(device), 0, TREE_GPU, int(dispatch), int(upward), *_shard(shard), int(symmetry))
        h = ctypes.c_void_p()
        rc = lib().bt_session_create(len(systems), self.toff.ctypes.data_as(_llp), self.soff.ctypes.data_as(_llp),
                                     *(_p(a) for a in cat), int(kernel), float(kernel_param), int(approximation),
                                     int(compute_type), float(theta), int(degree), int(max_source_leaf),
                                     int(max_target_leaf), float(size_check), ctypes.byref(opts), ctypes.byref(h))
        _check(rc)
        self._h = h

    def evaluate(self, charges, return_report=False, out=None):
        """Potentials per system for new source charges (one array per system, or concatenated).

        out: optional float64 array of all systems' targets (concatenated),
        reused across calls by an iterative solver; the potentials are
        written there and the per-system results are views of it.  Without
        it each call returns fresh arrays."""
        q = _c(np.concatenate(charges) if isinstance(charges, (list, tuple)) else charges)
        if len(q) != self.soff[-1]:
            raise BaryTreeError(BT_ERR_PARAM, f"expected {self.soff[-1]} charges, got {len(q)}")
        nt = int(self.toff[-1])
        if out is not None and (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (nt,)
                                or not out.flags.c_contiguous):
            raise BaryTreeError(BT_ERR_PARAM, f"out must be a contiguous float64 array of {nt} values")
        buf = out if out is not None else np.empty(nt)
        rep = Report()
        _check(lib().bt_session_eval(self._h, _p(q), _p(buf), ctypes.byref(rep)))
        pots = [buf[self.toff[k]:self.toff[k + 1]] for k in range(len(self.toff) - 1)]
        return (pots, rep.as_dict()) if return_report else pots

    def close(self):
        if getattr(self, "_h", None):
            lib().bt_session_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def autotune(systems, kernel=Kernel.COULOMB, kernel_param=0.0, approximation=Approximation.LAGRANGE,
             compute_type=ComputeType.PARTICLE_CLUSTER, theta=0.7, degree=8, max_source_leaf=2000,
             max_target_leaf=2000, size_check=1.0, degree_policy=DEGREE_FIXED, tolerance=1e-6, device=0,
             upward=UPWARD_AUTO, shard=None, symmetry=SYMMETRY_AUTO):
    """bt_autotune: times the mixed particle-output kernel's 18 tile shapes on
    this workload (a list of systems (tx, ty, tz, sx, sy, sz, sq), as for
    Session; with shard, on that target shard's work) and installs the
    fastest for (device, kernel, approximation).  Returns (best, trials) as
    dicts."""
    systems = [tuple(map(_c, s)) for s in systems]
    toff = np.concatenate([[0], np.cumsum([len(s[0]) for s in systems])]).astype(np.int64)
    soff = np.concatenate([[0], np.cumsum([len(s[3]) for s in systems])]).astype(np.int64)
    cat = [_c(np.concatenate([s[i] for s in systems])) for i in range(7)]
    opts = Options(PRECISION_MIXED, int(degree_policy), float(tolerance), int(device), 0, TREE_GPU, DISPATCH_AUTO,
                   int(upward), *_shard(shard), int(symmetry))
    best = Tuning()
    trials = (Tuning * 32)()
    nt = ctypes.c_int(0)
    rc = lib().bt_autotune(len(systems), toff.ctypes.data_as(_llp), soff.ctypes.data_as(_llp),
                           *(_p(a) for a in cat), int(kernel), float(kernel_param), int(approximation),
                           int(compute_type), float(theta), int(degree), int(max_source_leaf), int(max_target_leaf),
                           float(size_check), ctypes.byref(opts), ctypes.byref(best), trials, 32, ctypes.byref(nt))
    _check(rc)
    return best.as_dict(), [trials[i].as_dict() for i in range(nt.value)]


def tuning_get(kernel=Kernel.COULOMB, approximation=Approximation.LAGRANGE, device=0):
    """(shape dict, installed) for (device, kernel, approximation)."""
    t = Tuning()
    inst = ctypes.c_int(0)
    _check(lib().bt_tuning_get(int(device), int(kernel), int(approximation), ctypes.byref(t), ctypes.byref(inst)))
    return t.as_dict(), bool(inst.value)


def tuning_set(shape, kernel=Kernel.COULOMB, approximation=Approximation.LAGRANGE, device=0):
    """Install a shape dict (as returned by autotune), or None to remove it."""
    if shape is None:
        _check(lib().bt_tuning_set(int(device), int(kernel), int(approximation), None))
        return
    t = Tuning(int(shape["targets_per_thread"]), int(shape["source_tile"]), int(shape["dispatch"]),
               float(shape.get("ms", 0.0)))
    _check(lib().bt_tuning_set(int(device), int(kernel), int(approximation), ctypes.byref(t)))


def save_tuning(path, device=0):
    """Write every installed shape of a device to a JSON file."""
    import json
    out = []
    for k in Kernel:
        for a in (Approximation.LAGRANGE, Approximation.HERMITE):
            shape, inst = tuning_get(k, a, device)
            if inst:
                out.append({"kernel": int(k), "approximation": int(a), **shape})
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    return len(out)


def load_tuning(path, device=0):
    """Install the shapes of a file written by save_tuning."""
    import json
    with open(path) as f:
        entries = json.load(f)
    for e in entries:
        tuning_set(e, e["kernel"], e["approximation"], device)
    return len(entries)


def treecode_ptr(nt, ns, tx, ty, tz, sx, sy, sz, sq, out, kernel=Kernel.COULOMB, kernel_param=0.0,
                 approximation=Approximation.LAGRANGE, compute_type=ComputeType.PARTICLE_CLUSTER, theta=0.7,
                 degree=8, max_source_leaf=2000, max_target_leaf=2000, size_check=1.0, precision=PRECISION_FP64,
                 degree_policy=DEGREE_FIXED, tolerance=1e-6, device=0, inputs_on_device=False,
                 tree_build=TREE_GPU, dispatch=DISPATCH_AUTO, upward=UPWARD_AUTO, shard=None, symmetry=SYMMETRY_AUTO):
    """bt_eval on raw addresses (ints): device pointers when inputs_on_device, else host pointers."""
    cast = lambda a: ctypes.cast(ctypes.c_void_p(int(a)), _dp)  # noqa: E731
    opts = Options(int(precision), int(degree_policy), float(tolerance), int(device), int(bool(inputs_on_device)),
                   int(tree_build), int(dispatch), int(upward), *_shard(shard), int(symmetry))
    rep = Report()
    rc = lib().bt_eval(int(nt), int(ns), cast(tx), cast(ty), cast(tz), cast(sx), cast(sy), cast(sz), cast(sq),
                       cast(out), int(kernel), float(kernel_param), int(approximation), int(compute_type),
                       float(theta), int(degree), int(max_source_leaf), int(max_target_leaf), float(size_check),
                       ctypes.byref(opts), ctypes.byref(rep))
    _check(rc)
    return rep.as_dict()


def measure_peaks(device=0):
    """(fp64 TFLOP/s, fp32 TFLOP/s, rsqrt Gop/s) measured by the library's probes."""
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    _check(lib().bt_measure_peaks(int(device), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return a.value, b.value, c.value


def direct(tx, ty, tz, sx, sy, sz, sq, kernel=Kernel.COULOMB, kernel_param=0.0, device=0,
           singularity=Singularity.SKIPPING, target_q=None, source_w=None):
    """FP64 direct sum on the GPU (error reference); kernel_param may be a
    sequence of kernel parameters (two for regularized Yukawa, atan, MQ).
    With singularity subtraction, target_q and source_w are required."""
    tx, ty, tz, sx, sy, sz, sq = map(_c, (tx, ty, tz, sx, sy, sz, sq))
    tq = _c(target_q) if target_q is not None else None
    sw = _c(source_w) if source_w is not None else None
    out = np.zeros(len(tx))
    kp = _c(np.atleast_1d(np.asarray(kernel_param, dtype=np.float64)))
    rc = lib().bt_direct_full(len(tx), len(sx), _p(tx), _p(ty), _p(tz), _p(tq), _p(sx), _p(sy), _p(sz), _p(sq),
                              _p(sw), _p(out), int(kernel), len(kp), _p(kp), int(singularity), int(device))
    _check(rc)
    return out


def interaction_lists(tx, ty, tz, sx, sy, sz, compute_type, approximation, theta, degree,
                      max_source_leaf, max_target_leaf, size_check, tree_build=None, device=0):
    """(units, nodes, entries[k,3]) in the canonical (unit, kind, node) form.
    tree_build=TREE_GPU plans as the evaluation path does (trees built on the
    GPU); the default builds the trees on the host."""
    tx, ty, tz, sx, sy, sz = map(_c, (tx, ty, tz, sx, sy, sz))
    units, nodes = ctypes.c_int(0), ctypes.c_int(0)
    cap = 1 << 16
    while True:
        ent = np.zeros(3 * cap, dtype=np.int32)
        args = (len(tx), len(sx), _p(tx), _p(ty), _p(tz), _p(sx), _p(sy), _p(sz), int(compute_type),
                int(approximation), float(theta), int(degree), int(max_source_leaf), int(max_target_leaf),
                float(size_check))
        if tree_build is None:
            n = lib().bt_lists(*args, ctypes.byref(units), ctypes.byref(nodes), ent.ctypes.data_as(_ip), cap)
        else:
            n = lib().bt_lists_ex(*args, int(tree_build), int(device), ctypes.byref(units), ctypes.byref(nodes),
                                  ent.ctypes.data_as(_ip), cap)
        if n == -2:
            _check(BT_ERR_CUDA)
        if n >= 0:
            return units.value, nodes.value, ent[: 3 * n].reshape(-1, 3)
        cap = max(cap * 4, 1 << 20)


def tree_summary(x, y, z, maxparnode, tree_build=TREE_HOST, device=0, return_order=False):
    """Per node (ibeg, iend, num_children, level) and (box..., radius); with
    return_order also the particle permutation (order[i] = input index of
    sorted particle i).  tree_build=TREE_GPU builds on the GPU."""
    x, y, z = map(_c, (x, y, z))
    cap = max(64, 4 * len(x) // max(1, maxparnode) + 64)
    ints = np.zeros(4 * cap, dtype=np.int32)
    dbl = np.zeros(7 * cap)
    order = np.zeros(max(1, len(x)), dtype=np.int32)
    n = lib().bt_tree_dump_ex(len(x), _p(x), _p(y), _p(z), int(maxparnode), int(tree_build), int(device),
                              ints.ctypes.data_as(_ip), _p(dbl), order.ctypes.data_as(_ip), cap)
    if n == -1:
        raise BaryTreeError(BT_ERR_PARAM, "tree capacity")
    if n < 0:
        raise BaryTreeError(BT_ERR_CUDA, last_error())
    res = (ints[: 4 * n].reshape(-1, 4), dbl[: 7 * n].reshape(-1, 7))
    return res + (order[: len(x)],) if return_order else res


def kernel_launch_count() -> int:
    return int(lib().bt_kernel_launch_count())


# Leaf size of the reference's GPU build on its beta path: with OpenACC on,
# RunParams_Setup sets 3000 particles per source and target leaf
# (src/run_params/run_params.c:101-103); its CPU build uses 50/5 and 5/50.
BETA_GPU_LEAF = 3000


class _RunParams(ctypes.Structure):
    """struct RunParams of include/barytree_compat.h (the reference's
    src/run_params/struct_run_params.h:7-31)."""
    _fields_ = [("kernel", ctypes.c_int), ("num_kernel_params", ctypes.c_int), ("kernel_params", _dp),
                ("approximation", ctypes.c_int), ("singularity", ctypes.c_int), ("compute_type", ctypes.c_int),
                ("theta", ctypes.c_double), ("size_check_factor", ctypes.c_double),
                ("interp_degree", ctypes.c_int), ("interp_pts_per_cluster", ctypes.c_int),
                ("interp_charges_per_cluster", ctypes.c_int), ("interp_weights_per_cluster", ctypes.c_int),
                ("max_per_source_leaf", ctypes.c_int), ("max_per_target_leaf", ctypes.c_int),
                ("beta", ctypes.c_double), ("verbosity", ctypes.c_int)]


def beta_parameters(beta, compute_type=ComputeType.PARTICLE_CLUSTER, approximation=Approximation.LAGRANGE):
    """theta, degree and size check that the reference's accuracy knob beta
    in [0, 1] stands for (run_params.c:51-95), from the library's
    RunParams_Setup; the leaf sizes returned are the reference GPU build's
    (BETA_GPU_LEAF).  Larger beta: smaller theta, higher degree."""
    L = lib()
    rp = ctypes.POINTER(_RunParams)
    L.RunParams_Setup.argtypes = (ctypes.POINTER(rp), ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int)
    L.RunParams_Setup.restype = None
    L.RunParams_Free.argtypes = (ctypes.POINTER(rp),)
    L.RunParams_Free.restype = None
    p = rp()
    kp = np.zeros(1)
    L.RunParams_Setup(ctypes.byref(p), int(Kernel.COULOMB), 1, _p(kp), int(approximation), int(Singularity.SKIPPING),
                      int(compute_type), 0.0, 0, 1, 1, 0.0, float(beta), 0)
    s = p.contents
    out = {"beta": float(beta), "theta": s.theta, "degree": s.interp_degree, "size_check": s.size_check_factor,
           "max_source_leaf": BETA_GPU_LEAF, "max_target_leaf": BETA_GPU_LEAF}
    L.RunParams_Free(ctypes.byref(p))
    return out
