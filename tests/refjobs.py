"""Reference computations at the benchmark configurations' full sizes, run in
spawned worker processes (test infrastructure).

Each job rebuilds the seed-0 inputs of bench.py's configuration and calls the
reference's own CPU code (oracle/_ref, built from its sources):
  * ("lists", cid): the reference's InteractionLists_Make on the full system;
  * ("pot", cid, nbatches, threads): the reference's particle-cluster treecode
    with its setup on the full system and InteractionCompute_PC on every
    k-th target batch (all batches with nbatches=None) -- each sampled
    target holds exactly the value a full reference call gives it
    (oracle/ref_sampled.c).
Workers are started with the spawn method, so a parent that already holds a
CUDA context is never forked.
"""
from __future__ import annotations

import multiprocessing as mp

import numpy as np


def inputs(cid):
    import bench
    cfg = dict(bench.CONFIGS[cid])
    x, y, z, q, _ = bench.make_inputs(cfg, 0)
    return cfg, x, y, z, q


def run(job):
    from oracle import oracle as O
    kind, cid = job[0], job[1]
    cfg, x, y, z, q = inputs(cid)
    if kind == "lists":
        return O.ref_lists(x, y, z, x.copy(), y.copy(), z.copy(), cfg["ctype"], cfg["approx"], cfg["theta"],
                           cfg["degree"], cfg["leaf"], cfg["leaf"], cfg["sc"])
    nbatches, threads = job[2], job[3]
    R = O.RefSampled(x, y, z, x.copy(), y.copy(), z.copy(), q, cfg["kernel"], [cfg["kp"]], cfg["approx"],
                     cfg["theta"], cfg["degree"], cfg["leaf"], cfg["leaf"], cfg["sc"])
    nb = R.nbatches
    sel = np.arange(nb) if nbatches is None else np.unique(np.linspace(0, nb - 1, nbatches).astype(int))
    out, _ = R.evaluate(sel, threads)
    R.close()
    idx = np.flatnonzero(~np.isnan(out))
    return idx, out[idx], len(sel), nb


class Jobs:
    """Runs reference jobs in a spawned pool; get(job) waits for one."""

    def __init__(self, jobs, processes):
        self.pool = mp.get_context("spawn").Pool(processes)
        self.res = {j: self.pool.apply_async(run, (j,)) for j in jobs}

    def get(self, job, timeout=3600):
        return self.res[job].get(timeout)

    def close(self):
        self.pool.terminate()
        self.pool.join()
