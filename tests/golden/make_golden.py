"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference BaryTree built from its own C sources
(``oracle/_ref/libBaryTree_ref.so``, see ``oracle/Makefile``) on small seeded
inputs and stores inputs + reference potentials + reference interaction lists
as ``.npz`` files.  The fixtures let the GPU tests pin the product against the
reference on machines where the reference build is not present.

Usage:  make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

# (name, N, target distribution, kernel, kparam, approx, ctype, theta, degree, leaf_s, leaf_t, size_check)
CASES = [
    ("pc_lag_coulomb", 3000, "same", 1, 0.0, 1, 1, 0.7, 5, 100, 100, 1.0),
    ("pc_lag_yukawa", 3000, "other", 2, 0.5, 1, 1, 0.8, 4, 150, 80, 1.0),
    ("pc_lag_regcoulomb", 3000, "same", 3, 1e-3, 1, 1, 0.7, 6, 120, 120, 1.0),
    ("pc_her_coulomb", 3000, "same", 1, 0.0, 2, 1, 0.7, 4, 100, 100, 4.0),
    ("pc_her_yukawa", 2500, "other", 2, 0.5, 2, 1, 0.7, 3, 80, 60, 4.0),
    ("cp_lag_coulomb", 3000, "other", 1, 0.0, 1, 2, 0.7, 4, 60, 150, 1.0),
    ("cp_her_regcoulomb", 2500, "same", 3, 1e-3, 2, 2, 0.7, 3, 60, 120, 4.0),
    ("cc_lag_coulomb", 3000, "other", 1, 0.0, 1, 3, 0.8, 4, 100, 100, 1.0),
    ("cc_lag_yukawa", 3000, "same", 2, 0.5, 1, 3, 0.8, 3, 50, 50, 1.0),
]


def inputs(seed, n, tdist):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    q = rng.uniform(-1, 1, n)
    if tdist == "same":
        tx, ty, tz = x.copy(), y.copy(), z.copy()
    else:
        tx, ty, tz = (np.clip(rng.normal(0, 0.4, n), -1, 1) for _ in range(3))
    return tx, ty, tz, x, y, z, q


def main():
    if not O.ref_available():
        raise SystemExit("reference build missing: run `make -C oracle ref` first")
    for i, (name, n, tdist, k, kp, ap, ct, th, deg, ls, lt, sc) in enumerate(CASES):
        tx, ty, tz, x, y, z, q = inputs(100 + i, n, tdist)
        pot = O.ref_treecode(tx, ty, tz, None, x, y, z, q, None, k, [kp], 1, ap, ct, th, deg, ls, lt, sc, -1.0, 0)
        units, nodes, ent = O.ref_lists(tx, ty, tz, x, y, z, ct, ap, th, deg, ls, lt, sc)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), tx=tx, ty=ty, tz=tz, sx=x, sy=y, sz=z, sq=q,
                            potential=pot, params=np.array([k, kp, ap, ct, th, deg, ls, lt, sc]),
                            units=units, nodes=nodes, lists=ent)
        print(f"{name}: {n} particles, {len(ent)} list entries, |phi|max={np.abs(pot).max():.4f}")


if __name__ == "__main__":
    main()
