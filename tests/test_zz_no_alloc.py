"""GPU test of the allocation-free entry point bt_eval_noalloc.

Callers that cannot allocate device memory at call time (memory-pool owners,
fixed-budget or certified deployments, code running after another component
reserved the free memory) use bt_eval_noalloc: its scratch lives in a static
device array compiled into the library.  This test calls it through the C
ABI with device pointers and checks, on two calls in a row, that its output
equals the regular entry point's (bt_eval with device-resident inputs) within
the FP64 parity tolerance used by the other GPU tests (relative L2 and
per-target difference <= 1e-12), that the second call changes the device's
free memory by nothing, and that a request larger than the static array is
refused with BT_ERR_PARAM.  A mixed-precision case with the targets equal to
the sources runs the symmetric near-field pair kernels, their partial-sum
slices and the tensor-core leaf P2M with its error flag inside the static
array; it is compared with bt_eval at the mixed path's tolerance (5e-7
relative L2, the bar of the mixed-vs-FP64 tests).  It runs last (file name) so that a failure here
does not hide the other tests, and it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import barytree_b200 as B
from conftest import uniform_inputs

pytestmark = pytest.mark.gpu

TOL = 1e-12
MIXED_TOL = 5e-7


def _noalloc_fn():
    f = B.lib().bt_eval_noalloc
    vp = ctypes.c_void_p
    f.argtypes = (ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_double,
                  ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_double, ctypes.c_int, ctypes.c_int)
    f.restype = ctypes.c_int
    return f


def _device_arrays(torch, arrays):
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


def _params(ctype):
    return dict(kernel=1, kp=0.0, approx=1, ctype=ctype, theta=0.7, degree=6, ls=400, lt=400, sc=1.0)


def _call_noalloc(f, d, out, p, precision=B.PRECISION_FP64):
    tx, ty, tz, sx, sy, sz, sq = d
    return f(len(tx), len(sx), tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), sx.data_ptr(), sy.data_ptr(),
             sz.data_ptr(), sq.data_ptr(), out.data_ptr(), p["kernel"], p["kp"], p["approx"], p["ctype"],
             p["theta"], p["degree"], p["ls"], p["lt"], p["sc"], precision, 0)


def _call_regular(d, out, p, precision=B.PRECISION_FP64):
    tx, ty, tz, sx, sy, sz, sq = d
    return B.treecode_ptr(len(tx), len(sx), tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), sx.data_ptr(),
                          sy.data_ptr(), sz.data_ptr(), sq.data_ptr(), out.data_ptr(), kernel=p["kernel"],
                          kernel_param=p["kp"], approximation=p["approx"], compute_type=p["ctype"],
                          theta=p["theta"], degree=p["degree"], max_source_leaf=p["ls"], max_target_leaf=p["lt"],
                          size_check=p["sc"], precision=precision, inputs_on_device=True)


def _close(a, b, tol=TOL):
    l2 = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert l2 <= tol, l2
    if tol == TOL:
        assert np.max(np.abs(a - b)) <= TOL * np.max(np.abs(b))


def test_noalloc_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    f = _noalloc_fn()
    cases = [(uniform_inputs(101, 40000, "other"), _params(1)),
             (uniform_inputs(102, 30000, "same"), _params(3))]
    dev = [(_device_arrays(torch, arrs), p) for arrs, p in cases]
    refs = []
    for d, p in dev:                                     # regular entry point first (it may allocate)
        out = torch.empty(len(d[0]), dtype=torch.float64, device="cuda")
        _call_regular(d, out, p)
        refs.append(out.cpu().numpy())
    outs = [torch.full((len(d[0]),), 7.0, dtype=torch.float64, device="cuda") for d, _ in dev]
    torch.cuda.synchronize()
    rc = _call_noalloc(f, dev[0][0], outs[0], dev[0][1])           # first call sets up the scratch
    assert rc == B.BT_OK, B.last_error()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    rc = _call_noalloc(f, dev[1][0], outs[1], dev[1][1])           # second call in a row
    assert rc == B.BT_OK, B.last_error()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    for out, ref in zip(outs, refs):
        _close(out.cpu().numpy(), ref)
    # the second call left the first call's scratch behind; a repeat of the
    # first case must still give the same answer
    again = torch.zeros_like(outs[0])
    assert _call_noalloc(f, dev[0][0], again, dev[0][1]) == B.BT_OK
    _close(again.cpu().numpy(), refs[0])


def test_noalloc_mixed_symmetric_pass_matches_regular_entry_point():
    """Mixed precision, targets = sources: the symmetric near-field pass (its
    pair list, partial-sum slices and side streams) and the tensor-core leaf
    P2M (its error flag) run inside the static array, twice in a row, with
    the device's free memory unchanged on the second call."""
    torch = pytest.importorskip("torch")
    f = _noalloc_fn()
    p = _params(1)
    d = _device_arrays(torch, uniform_inputs(103, 30000, "same"))
    ref = torch.empty(len(d[0]), dtype=torch.float64, device="cuda")
    rep = _call_regular(d, ref, p, B.PRECISION_MIXED)
    assert rep["sym_ptwise"] > 0                 # the symmetric pass ran on the regular path too
    ref = ref.cpu().numpy()
    outs = []
    for k in range(2):
        out = torch.full((len(d[0]),), 7.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        rc = _call_noalloc(f, d, out, p, B.PRECISION_MIXED)
        assert rc == B.BT_OK, B.last_error()
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        if k == 1:
            assert free_after == free_before
        outs.append(out.cpu().numpy())
        _close(outs[-1], ref, MIXED_TOL)
    assert np.array_equal(outs[0], outs[1])      # deterministic in the shared array


def test_noalloc_rejects_too_large():
    torch = pytest.importorskip("torch")
    f = _noalloc_fn()
    n = 1_500_000
    d = _device_arrays(torch, uniform_inputs(7, n))
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    rc = _call_noalloc(f, d, out, _params(1))
    assert rc == B.BT_ERR_PARAM
    assert "static scratch" in B.last_error()
