"""CPU tests of the product's host side (no GPU needed).

The tree build and the MAC interaction lists run on the host in C; they must
equal the reference's bit for bit (node sets, boxes, radii, numbering, list
membership and order).  Also: the C-ABI library loads and exports every
symbol the public header declares, and argument errors are reported with
status codes instead of exiting.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import barytree_b200 as B
from conftest import ROOT, golden_files, same_members, uniform_inputs
from oracle import oracle as O


def _header_functions():
    inc = os.path.join(ROOT, "include")
    src = "\n".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ \*]*?\b([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                                 src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    names = _header_functions()
    assert "BaryTreeInterface" in names and "bt_eval" in names and "treedriver" in names
    lib = ctypes.CDLL(B.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    assert set(B.EXPORTED_SYMBOLS) <= set(names)


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("/")[-1][:-4])
def test_lists_match_reference_golden(path):
    g = np.load(path)
    k, kp, ap, ct, th, deg, ls, lt, sc = g["params"]
    units, nodes, ent = B.interaction_lists(g["tx"], g["ty"], g["tz"], g["sx"], g["sy"], g["sz"], int(ct),
                                            int(ap), th, int(deg), int(ls), int(lt), sc)
    assert units == int(g["units"]) and nodes == int(g["nodes"])
    assert np.array_equal(ent, g["lists"])


def _clustered(seed, n):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.7, 0.7, (4, 3))
    pts = np.concatenate([np.clip(rng.normal(c[i], 0.05, (n // 4, 3)), -1, 1) for i in range(4)])
    q = rng.uniform(-1, 1, len(pts))
    return pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy(), q


@pytest.mark.parametrize("ctype", [1, 2, 3])
@pytest.mark.parametrize("case", ["uniform", "clustered", "lattice", "tiny", "single_leaf"])
def test_lists_match_oracle(ctype, case):
    if case == "uniform":
        tx, ty, tz, sx, sy, sz, _ = uniform_inputs(11, 8000, "other")
        ls, lt, deg = 200, 100, 4
    elif case == "clustered":
        sx, sy, sz, _ = _clustered(5, 8000)
        tx, ty, tz, _ = _clustered(6, 6000)
        ls, lt, deg = 150, 150, 3
    elif case == "lattice":
        i = np.arange(300, dtype=float)
        sx = sy = sz = i
        tx, ty, tz = i.copy(), i.copy(), i.copy()
        ls, lt, deg = 3, 3, 2
    elif case == "tiny":
        tx, ty, tz, sx, sy, sz, _ = uniform_inputs(2, 5, "same")
        ls, lt, deg = 1, 1, 1
    else:
        tx, ty, tz, sx, sy, sz, _ = uniform_inputs(4, 500, "same")
        ls, lt, deg = 1000, 1000, 5
    for ap, sc in ((1, 1.0), (2, 4.0), (1, 0.0)):
        a = B.interaction_lists(tx, ty, tz, sx, sy, sz, ctype, ap, 0.7, deg, ls, lt, sc)
        b = O.lists(tx, ty, tz, sx, sy, sz, ctype, ap, 0.7, deg, ls, lt, sc)
        assert a[0] == b[0] and a[1] == b[1]
        assert np.array_equal(a[2], b[2])


@pytest.mark.parametrize("maxpar", [1, 7, 100, 5000])
def test_tree_matches_oracle(maxpar):
    _, _, _, x, y, z, _ = uniform_inputs(9, 3000)
    a_int, a_dbl = B.tree_summary(x, y, z, maxpar)
    b_int, b_dbl = O.tree(x, y, z, maxpar)
    assert np.array_equal(a_int, b_int)
    assert np.array_equal(a_dbl, b_dbl)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_tree_matches_reference_build():
    sx, sy, sz, _ = _clustered(8, 12000)
    a_int, a_dbl = B.tree_summary(sx, sy, sz, 50)
    b_int, b_dbl = O.ref_tree(sx, sy, sz, 50)
    assert np.array_equal(a_int[:, :3], b_int[:, :3])    # ibeg, iend, children
    assert np.array_equal(a_dbl, b_dbl)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_tree_membership_matches_reference_build():
    """Every node holds the same particles as in the reference's build.  The
    order inside a node differs: the reference partitions in place by swaps
    (src/tree/partition.c:14-120), the builds here keep input order."""
    sx, sy, sz, _ = _clustered(8, 12000)
    ints, _, order = B.tree_summary(sx, sy, sz, 50, return_order=True)
    ref = O.ref_tree_order(sx, sy, sz, 50)
    assert same_members(ints, order, ref)
    leaf = ints[ints[:, 2] == 0]
    assert all(np.array_equal(order[b - 1:e], np.sort(order[b - 1:e])) for b, e, _, _ in leaf)


def _bti(**over):
    tx, ty, tz, sx, sy, sz, sq = uniform_inputs(1, 100)
    args = dict(nt=100, ns=100, tx=tx, ty=ty, tz=tz, tq=None, sx=sx, sy=sy, sz=sz, sq=sq, sw=None,
                kernel=1, kp=np.array([0.5]), sing=1, approx=1, ctype=1, theta=0.7, deg=4, ls=10, lt=10, sc=1.0,
                beta=-1.0)
    args.update(over)
    out = np.full(max(args["nt"], 1), 7.0)
    p = lambda a: None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    rc = B.lib().BaryTreeInterface_ex(args["nt"], args["ns"], p(args["tx"]), p(args["ty"]), p(args["tz"]),
                                      p(args["tq"]), p(args["sx"]), p(args["sy"]), p(args["sz"]), p(args["sq"]),
                                      p(args["sw"]), p(out), args["kernel"], len(args["kp"]), p(args["kp"]), args["sing"],
                                      args["approx"], args["ctype"], args["theta"], args["deg"], args["ls"],
                                      args["lt"], args["sc"], args["beta"], 0)
    return rc, out


def test_error_codes_without_exiting():
    assert _bti(sx=None)[0] == B.BT_ERR_PARAM                  # NULL source array
    assert _bti(tx=None)[0] == B.BT_ERR_PARAM
    assert _bti(nt=-1)[0] == B.BT_ERR_PARAM
    assert _bti(sing=2)[0] == B.BT_ERR_PARAM                    # subtraction without target charges / weights
    w = np.ones(100)
    # subtraction exists for CP / CC only with Coulomb and Yukawa, Lagrange
    # (src/interaction_compute/interaction_compute_cp.c:121-248)
    assert _bti(sing=2, tq=w, sw=w, ctype=2, approx=2)[0] == B.BT_ERR_UNSUPPORTED
    assert _bti(sing=2, tq=w, sw=w, ctype=3, kernel=3)[0] == B.BT_ERR_UNSUPPORTED
    assert _bti(sing=3)[0] == B.BT_ERR_PARAM
    assert _bti(kernel=6)[0] == B.BT_ERR_UNSUPPORTED            # TCF: no kernel in the reference
    assert _bti(kernel=5, ctype=2, kp=np.array([1.0, 0.1]))[0] == B.BT_ERR_UNSUPPORTED   # atan is PC only
    assert _bti(kernel=4, approx=2, kp=np.array([0.5, 0.1]))[0] == B.BT_ERR_UNSUPPORTED  # no Hermite reg. Yukawa
    assert _bti(kernel=4)[0] == B.BT_ERR_PARAM                  # regularized Yukawa needs (kappa, eps)
    assert _bti(ctype=3, approx=2)[0] == B.BT_ERR_UNSUPPORTED   # CC Hermite (interaction_compute_cc.c:146)
    assert _bti(approx=0)[0] == B.BT_ERR_PARAM
    assert _bti(ctype=0)[0] == B.BT_ERR_PARAM
    assert _bti(ls=0)[0] == B.BT_ERR_PARAM
    rc, out = _bti(deg=13)
    assert rc == B.BT_ERR_UNSUPPORTED
    assert B.last_error() != ""


def test_empty_inputs_zero_output():
    rc, out = _bti(ns=0)
    assert rc == B.BT_OK and np.all(out[:100] == 0.0)           # output zeroed (BaryTreeInterface.c:29)
    rc, _ = _bti(nt=0)
    assert rc == B.BT_OK


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device status on a machine without a GPU")
def test_no_device_status():
    rc, out = _bti()
    assert rc == B.BT_ERR_NO_DEVICE
    assert np.all(out[:100] == 0.0)


@pytest.mark.parametrize("cid", [1, 2, 3])
def test_lists_match_reference_benchmark_configs(cid):
    """The interaction lists of the benchmark configurations at their full
    sizes (100k particle-cluster; 1M cluster-cluster, theta 0.8; 4M Gaussian
    Hermite with size check 4 and leaf 1000), from the seed-0 inputs of
    bench.py, against the reference's own InteractionLists_Make: bit for bit."""
    if not O.ref_available():
        pytest.skip("reference build oracle/_ref not present")
    import refjobs
    cfg, x, y, z, _ = refjobs.inputs(cid)
    args = (x, y, z, x.copy(), y.copy(), z.copy(), cfg["ctype"], cfg["approx"], cfg["theta"], cfg["degree"],
            cfg["leaf"], cfg["leaf"], cfg["sc"])
    a = B.interaction_lists(*args)
    b = O.ref_lists(*args)
    assert a[0] == b[0] and a[1] == b[1]
    assert a[2].shape == b[2].shape and np.array_equal(a[2], b[2])
