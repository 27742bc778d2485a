"""The reference's own known-answer cases (tests/serial_tests.c), restated.

Inputs are generated exactly as the reference tests do: diagonal lattices for
the closed-form cases, and glibc ``srand(1)``/``rand()`` (called through
ctypes) for the random ones, so the particles are bit-identical to the
reference tests'.  Each case returns inputs, parameters and a checker with the
reference's own tolerance.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

_libc = ctypes.CDLL("libc.so.6")
_libc.rand.restype = ctypes.c_int
RAND_MAX = 2147483647


def _rand_stream(count):
    return np.array([_libc.rand() for _ in range(count)], dtype=np.float64) / RAND_MAX


def lattice(n):
    """Particles at (i,i,i) with charge i (serial_tests.c:59-71, 231-243)."""
    i = np.arange(n, dtype=np.float64)
    return i.copy(), i.copy(), i.copy(), i.copy()


def lattice_closed_form(n, kernel, kappa=0.5):
    """Closed-form skipping potentials on the lattice (serial_tests.c:80-93, 135-147)."""
    out = np.zeros(n)
    for i in range(n):
        s = 0.0
        for j in range(n):
            if j == i:
                continue
            r = abs(j - i) * math.sqrt(3)
            s += j / r if kernel == 1 else j * math.exp(-kappa * r) / r
        out[i] = s
    return out


def one_target_sources():
    """1 target at the origin, 10 000 sources from srand(1) (serial_tests.c:560-588)."""
    _libc.srand(1)
    n = 10000
    r = _rand_stream(5 * n).reshape(n, 5)
    x, y, z = r[:, 0] * 2 - 1, r[:, 1] * 2 - 1, r[:, 2] * 2 - 1
    q = r[:, 3] * 2 - 1
    t = np.zeros(1)
    return t, t.copy(), t.copy(), x, y, z, q


def parameters_sources():
    """1 target at the origin, 5 000 sources from srand(1) (serial_tests.c:971-1017)."""
    _libc.srand(1)
    n = 5000
    r = _rand_stream(5 * n).reshape(n, 5)
    t = np.zeros(1)
    return t, t.copy(), t.copy(), r[:, 0] * 2 - 1, r[:, 1] * 2 - 1, r[:, 2] * 2 - 1, r[:, 3] * 2 - 1


def bldtt_inputs():
    """5 000 targets and sources interleaved from srand(1) (serial_tests.c:1440-1460)."""
    _libc.srand(1)
    n = 5000
    r = _rand_stream(9 * n).reshape(n, 9)
    tx, ty, tz = r[:, 0] * 2 - 1, r[:, 1] * 2 - 1, r[:, 2] * 2 - 1
    sx, sy, sz, sq = r[:, 4] * 2 - 1, r[:, 5] * 2 - 1, r[:, 6] * 2 - 1, r[:, 7] * 2 - 1
    return tx, ty, tz, sx, sy, sz, sq


# (kernel, approximation, tolerance) of test_treecode_on_100_particles, skipping forms
# (serial_tests.c:290, 353, 416, 478)
LATTICE100_CASES = [(1, 1, 3e-3), (2, 1, 8e-3), (1, 2, 3e-4), (2, 2, 5e-4)]

# (kernel, approximation, tolerance) of test_treecode_on_1_target_10000_sources, skipping forms
# (serial_tests.c:628, 682, 736, 790)
ONE_TARGET_CASES = [(1, 1, 2e-4), (2, 1, 2e-4), (1, 2, 2e-5), (2, 2, 2e-5)]
