"""CPU tests of the driver-level compatibility layer (RunParams_*, treedriver,
directdriver; include/barytree_compat.h).

The struct layouts are the ABI a program compiled against the reference's
headers relies on: they are checked three ways -- the C compiler's offsets
with this library's header, the ctypes mirror, and the behaviour of the
reference's own RunParams_Setup (built from its sources in oracle/_ref) read
through that mirror.  RunParams_Setup must fill every field as the
reference's does, including the beta path.  Argument errors return without
touching the potential (no device is needed to reach them).
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import barytree_b200 as B
from compat_structs import Particles, RunParams, declare, fields, particles
from conftest import ROOT
from oracle import oracle as O

# x86-64 LP64 offsets of the reference structs (struct_particles.h:5-27,
# struct_run_params.h:7-31)
PARTICLES_OFFSETS = {"num": 0, "x": 8, "y": 16, "z": 24, "q": 32, "w": 40, "ibeg": 48, "iend": 56, "order": 64,
                     "sources_w_dummy": 72, "targets_q_dummy": 76, "targets_x_duplicate": 80,
                     "targets_y_duplicate": 84, "targets_z_duplicate": 88, "targets_q_duplicate": 92}
RUNPARAMS_OFFSETS = {"kernel": 0, "num_kernel_params": 4, "kernel_params": 8, "approximation": 16,
                     "singularity": 20, "compute_type": 24, "theta": 32, "size_check_factor": 40,
                     "interp_degree": 48, "interp_pts_per_cluster": 52, "interp_charges_per_cluster": 56,
                     "interp_weights_per_cluster": 60, "max_per_source_leaf": 64, "max_per_target_leaf": 68,
                     "beta": 72, "verbosity": 80}


def _ours():
    return declare(ctypes.CDLL(B.LIB_PATH))


def test_struct_layouts_of_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "barytree_compat.h"', 'int main(void) {']
    for s, offs in (("Particles", PARTICLES_OFFSETS), ("RunParams", RUNPARAMS_OFFSETS)):
        for f in offs:
            lines.append(f'printf("{s} {f} %zu\\n", offsetof(struct {s}, {f}));')
        lines.append(f'printf("{s} sizeof %zu\\n", sizeof(struct {s}));')
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=gnu11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n"):
        if ln:
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for s, offs, cls in (("Particles", PARTICLES_OFFSETS, Particles), ("RunParams", RUNPARAMS_OFFSETS, RunParams)):
        for f, off in offs.items():
            assert got[(s, f)] == off == getattr(cls, f).offset, (s, f)
        assert got[(s, "sizeof")] == ctypes.sizeof(cls)
    assert ctypes.sizeof(Particles) == 96 and ctypes.sizeof(RunParams) == 88


SETUP_CASES = [(k, ct, ap, sg, beta) for k, ct, ap, sg in
               [(1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 1, 1), (1, 1, 2, 2), (4, 3, 1, 2), (5, 2, 1, 1)]
               for beta in (-1.0, 0.0, 0.3, 0.5, 0.77, 1.0, 1.5)]


@pytest.mark.parametrize("kernel,ctype,approx,sing,beta", SETUP_CASES)
def test_runparams_setup_matches_reference(kernel, ctype, approx, sing, beta):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    ref = declare(O.ref_lib())
    ours = _ours()
    kp = np.array([0.5, 0.02])
    out = []
    for lib in (ours, ref):
        rp = ctypes.POINTER(RunParams)()
        lib.RunParams_Setup(ctypes.byref(rp), kernel, 2, kp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            approx, sing, ctype, 0.7, 6, 300, 200, 2.5, beta, 0)
        out.append(fields(rp.contents))
        lib.RunParams_Free(ctypes.byref(rp))
    assert out[0] == out[1]


def test_runparams_validate_and_free():
    lib = _ours()
    rp = ctypes.POINTER(RunParams)()
    kp = np.array([1.0])
    lib.RunParams_Setup(ctypes.byref(rp), 1, 1, kp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1, 1, 1,
                        0.8, 4, 100, 100, 1.0, -1.0, 0)
    assert rp.contents.interp_pts_per_cluster == 125
    rp.contents.approximation = 2
    rp.contents.singularity = 2
    rp.contents.interp_degree = 6
    lib.RunParams_Validate(rp)
    r = rp.contents
    assert (r.interp_pts_per_cluster, r.interp_charges_per_cluster, r.interp_weights_per_cluster) == (343, 2744, 2744)
    lib.RunParams_Free(ctypes.byref(rp))
    assert not rp                      # the caller's pointer is cleared
    lib.RunParams_Free(ctypes.byref(rp))


def test_driver_argument_errors_leave_potential_untouched(capfd):
    lib = _ours()
    rp = ctypes.POINTER(RunParams)()
    kp = np.array([0.5])
    lib.RunParams_Setup(ctypes.byref(rp), 1, 1, kp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1, 2, 1,
                        0.8, 4, 100, 100, 1.0, -1.0, 0)
    n = 16
    x, y, z, q = (np.linspace(0, 1, n) + k for k in range(4))
    src = particles(x, y, z, q)                # no weights: subtraction must refuse
    tgt = particles(x.copy(), y.copy(), z.copy(), q.copy())
    pot = np.full(n, 7.0)
    times = np.zeros(13)
    dp = ctypes.POINTER(ctypes.c_double)
    for fn in (lib.treedriver, lib.directdriver):
        fn(ctypes.byref(src), ctypes.byref(tgt), rp, pot.ctypes.data_as(dp), times.ctypes.data_as(dp))
        assert np.all(pot == 7.0)
    tgt.x = None                               # a required array unset
    lib.treedriver(ctypes.byref(src), ctypes.byref(tgt), rp, pot.ctypes.data_as(dp), times.ctypes.data_as(dp))
    assert np.all(pot == 7.0)
    err = capfd.readouterr().err
    assert "requires source weights" in err and "required particle arrays" in err
    lib.RunParams_Free(ctypes.byref(rp))
