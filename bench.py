"""Benchmark of the treecode evaluation on B200 (one JSON line on rank 0).

A step is one complete treecode evaluation (tree, lists, upward pass,
interaction kernels, downward pass, reorder) of one synthetic system of the
chosen configuration.

  value  -- targets/s with the inputs resident in HBM when the timed region
            starts (bt_eval with device pointers)
  e2e    -- targets/s through the C ABI with pinned host buffers, host->device
            copies of the inputs and the device->host read of the potentials
            inside the timed region
  roofline -- the dominant kernels (particle-output evaluation, PC + PP, and
            the symmetric near-field pairs): evaluations per second against
            the MUFU rsqrt rate measured on this GPU by the library's probe
            (mixed Lagrange), or FLOP/s against the measured FMA peak; DRAM
            traffic from the committed ncu summary of the same workload
  fp64_plain, baselines -- the plain FP64 treecode at the configuration's
            degree (the north_star denominator), and for the learned
            selection the lowest fixed degree meeting the tolerance (mixed and
            FP64) and the reference's beta knob, with the speed-up's factors
  cpu_baseline -- the reference BaryTree (built from its own sources) on the
            host cores: the full system for configurations 1, 3 and 5 (its
            setup timed, its evaluation sampled by target batch and
            extrapolated by the interaction count), smaller independent
            systems for 2 and 4

Multi-GPU (--gpus N under torchrun): every rank evaluates its own independent
system of the configuration (weak scaling, no data-path collective); the
timing is the max over ranks.

`--impl reference` times the reference's CPU implementation on this host's
cores instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))


def host_threads_per_rank():
    """torchrun starts every rank with OMP_NUM_THREADS=1.  The library plans
    each call on the host with OpenMP (interaction lists, the degree
    selection's list rewrite, the symmetric pairs), so each rank gets an
    equal share of the host's cores instead.  Runs at import, before the
    library and its OpenMP runtime are loaded; an explicit setting other
    than 1 is kept."""
    local = int(os.environ.get("LOCAL_WORLD_SIZE", "1") or 1)
    if local > 1 and os.environ.get("OMP_NUM_THREADS") == "1":
        os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or 1) // local))


host_threads_per_rank()
sys.path.insert(0, ROOT)

CONFIGS = {
    1: dict(workload="N=100,000 uniform [-1,1]^3, charges U[-1,1], Coulomb, particle-cluster Lagrange n=8, "
                     "theta 0.7, leaf 2000", N=100_000, dist="uniform", kernel=1, kp=0.0, approx=1, ctype=1,
            degree=8, theta=0.7, leaf=2000, sc=1.0, sample_n=60_000),
    2: dict(workload="N=1,000,000 uniform [-1,1]^3, charges U[-1,1], Yukawa kappa=0.5, cluster-cluster "
                     "Lagrange n=8, theta 0.8, leaf 2000", N=1_000_000, dist="uniform", kernel=2, kp=0.5, approx=1,
            ctype=3, degree=8, theta=0.8, leaf=2000, sc=1.0, sample_n=60_000),
    3: dict(workload="N=4,000,000 Gaussian sigma 0.25 clipped to [-1,1]^3, charges +-1, Coulomb, particle-cluster "
                     "Hermite n=6, theta 0.7, leaf 1000, size check 4", N=4_000_000, dist="gauss", kernel=1, kp=0.0,
            approx=2, ctype=1, degree=6, theta=0.7, leaf=1000, sc=4.0, sample_n=60_000),
    4: dict(workload="256 independent systems in one bt_eval_batch call: N log-uniform 1,000-200,000, uniform in "
                     "the unit cube [0,1]^3, charges U[-1,1], regularized Coulomb eps=1e-3 (self term q/eps "
                     "included), particle-cluster Lagrange n=7, theta 0.7, leaf 2000, mixed precision",
            N=None, dist="batch", nsys=256, nmin=1_000, nmax=200_000, kernel=3, kp=1e-3, approx=1, ctype=1,
            degree=7, theta=0.7, leaf=2000, sc=1.0, sample_n=300_000),
    5: dict(workload="N=16,000,000: 80% in 8 Gaussian blobs (centres U[-0.7,0.7]^3, sigma log-uniform 0.05-0.3, "
                     "clipped to [-1,1]^3), 20% uniform [-1,1]^3, charges U[-1,1], Coulomb, particle-cluster "
                     "Lagrange, theta 0.7, leaf 2000; degree per interaction from the learned selector at 1e-6, "
                     "against fixed degree 10", N=16_000_000, dist="blobs", kernel=1, kp=0.0, approx=1, ctype=1,
            degree=10, theta=0.7, leaf=2000, sc=1.0, sample_n=80_000),
}


def batch_sizes(cfg, seed):
    """Particle counts of a batch: log-uniform between nmin and nmax."""
    rng = np.random.default_rng(seed)
    nsys = cfg.get("nsys_override", cfg["nsys"])
    return np.round(np.exp(rng.uniform(np.log(cfg["nmin"]), np.log(cfg["nmax"]), nsys))).astype(np.int64)


def make_inputs(cfg, seed):
    """Seeded synthetic inputs with the configuration's distribution (numpy
    PCG64): x, y, z, q and, for a batch, the system offsets (else None)."""
    rng = np.random.default_rng(seed)
    if cfg["dist"] == "batch":
        sizes = batch_sizes(cfg, seed)
        n = int(sizes.sum())
        x, y, z = (rng.uniform(0, 1, n) for _ in range(3))
        q = rng.uniform(-1, 1, n)
        return x, y, z, q, np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    n = cfg["N"] if "n_override" not in cfg else cfg["n_override"]
    if cfg["dist"] == "uniform":
        x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
        q = rng.uniform(-1, 1, n)
    elif cfg["dist"] == "gauss":
        x, y, z = (np.clip(rng.normal(0, 0.25, n), -1, 1) for _ in range(3))
        q = rng.choice([-1.0, 1.0], n)
    elif cfg["dist"] == "blobs":
        from barytree_b200.selector import blobs
        x, y, z, q = blobs(n, seed)
    else:
        raise ValueError(cfg["dist"])
    return x, y, z, q, None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms from the
    warm-up through the timed regions."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def wait_first_sample(self, limit_s=5.0):
        """Block until nvidia-smi has written a sample: its start-up (NVML
        initialisation) must not overlap a timed region."""
        t0 = time.perf_counter()
        while self.proc is not None and time.perf_counter() - t0 < limit_s:
            if os.path.getsize(self.path) > 0:
                return
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [c.strip() for c in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# Configurations whose reference measurement runs the reference on the full
# system (particle-cluster, oracle/ref_sampled.c); the others (cluster-cluster,
# the batch of systems) time the reference on smaller independent samples.
FULL_SYSTEM_REFERENCE = (1, 3, 5)


def reference_full_system(cfg, threads, warmup, steps, step_seconds):
    """The reference's own CPU code (oracle/_ref, built from its sources) on
    the configuration's full system, the same seed-0 inputs the GPU arm's rank
    0 evaluates.

    The reference's setup (source tree, target batches, source proxies,
    interaction lists: its own serial routines) runs once and is timed.  Each
    step then evaluates a strided sample of the target batches with the
    reference's InteractionCompute_PC on `threads` host threads (a different
    offset every step); the batches of a step are sized to take about
    `step_seconds`.  The whole-system time on `threads` cores is the setup
    plus the full evaluation, extrapolated from the sampled batches by the
    pointwise interaction counts (the reference's own count):
        t = t_setup + W_total / (r_core * threads),
    with r_core = sampled interactions / the sampled batches' summed thread
    seconds.  Returns None if the reference build is absent."""
    from oracle import oracle as O
    if not O.ref_available() or not os.path.exists(os.path.join(O.REF_DIR, "libBaryTree_refsample.so")):
        return None
    x, y, z, q, _ = make_inputs(cfg, 0)
    n = len(x)
    R = O.RefSampled(x, y, z, x.copy(), y.copy(), z.copy(), q, cfg["kernel"], [cfg["kp"]], cfg["approx"],
                     cfg["theta"], cfg["degree"], cfg["leaf"], cfg["leaf"], cfg["sc"])
    t_setup = sum(R.setup_seconds.values())
    nb, w_total = R.nbatches, int(R.work.sum())
    out = np.zeros(n)
    # warm-up steps: one batch per thread each, which also calibrates the rate
    cpu = work = 0.0
    for s in range(max(1, warmup)):
        sel = np.arange(s * threads, (s + 1) * threads) * 7919 % nb
        _, _, per = R.evaluate(sel, threads, out=out, batch_seconds=True)
        cpu += per.sum()
        work += R.work[sel].sum()
    stride = max(1, int(np.ceil(w_total / ((work / cpu) * threads * step_seconds))))
    rates, walls, nsel, ntgt, wsum, csum = [], [], 0, 0, 0, 0.0
    for s in range(steps):
        sel = np.arange((s * 104729 + 1) % stride, nb, stride)
        _, wall, per = R.evaluate(sel, threads, out=out, batch_seconds=True)
        rates.append(R.work[sel].sum() / per.sum())
        walls.append(wall)
        nsel += len(sel)
        ntgt += int(R.sizes[sel].sum())
        wsum += int(R.work[sel].sum())
        csum += float(per.sum())
    R.close()
    r_core = wsum / csum
    t_eval = w_total / (r_core * threads)
    per_step = [n / (t_setup + w_total / (r * threads)) for r in rates]
    return {"value": n / (t_setup + t_eval), "per_step": per_step, "n": n, "threads": threads,
            "setup_s": t_setup, "setup_phases_s": R.setup_seconds, "eval_s_extrapolated": t_eval,
            "whole_system_s": t_setup + t_eval, "rate_per_core": r_core, "interactions_total": w_total,
            "batches": nb, "batches_per_step": nsel / max(1, steps), "stride": stride,
            "sample_fraction": wsum / (w_total * max(1, steps)), "targets_sampled": ntgt,
            "ms_per_sample_step": 1e3 * statistics.mean(walls) if walls else None,
            "sample": (f"reference BaryTree CPU build (gcc -O3, its own routines) on the full N={n:,} system, seed 0: "
                       f"setup (source tree, target batches, degree-{cfg['degree']} proxies, lists; serial, as in "
                       f"the reference) timed once = {t_setup:.1f} s; per step every {stride}-th of {nb} target "
                       f"batches evaluated by InteractionCompute_PC on {threads} host threads "
                       f"({100 * wsum / (w_total * max(1, steps)):.2f} % of the pointwise interactions per step); "
                       f"whole-system time on {threads} cores = setup + evaluation extrapolated by the interaction "
                       f"count = {t_setup + t_eval:.0f} s")}


def reference_sample_worker(args):
    """One bounded sample of the workload through the reference CPU build:
    smaller independent systems with the configuration's distribution."""
    cfg, seed, n = args
    from oracle import oracle as O
    c = dict(cfg)
    if c["dist"] == "batch":
        # systems of the batch distribution, one after another, up to about n particles
        sizes = batch_sizes(dict(c, nsys_override=64), seed)
        sizes = sizes[: max(1, int(np.searchsorted(np.cumsum(sizes), n)))]
        c["nsys_override"] = len(sizes)
    else:
        c["n_override"] = n
    x, y, z, q, off = make_inputs(c, seed)
    if off is None:
        off = np.array([0, len(x)])
    t0 = time.perf_counter()
    for k in range(len(off) - 1):
        a, b = off[k], off[k + 1]
        O.ref_treecode(x[a:b].copy(), y[a:b].copy(), z[a:b].copy(), None, x[a:b], y[a:b], z[a:b], q[a:b], None,
                       c["kernel"], [c["kp"]], 1, c["approx"], c["ctype"], c["theta"], c["degree"], c["leaf"],
                       c["leaf"], c["sc"], -1.0, 0)
    return int(off[-1]), time.perf_counter() - t0, len(off) - 1


def reference_samples(cfg, cores):
    """The reference on `cores` independent smaller systems, one core each
    (configurations without a full-system reference measurement)."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    n = cfg["sample_n"]
    if cores == 1:
        done, secs, nsys = reference_sample_worker((cfg, 1000, n))
        value = done / secs
        n = done
    else:
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        t0 = time.perf_counter()
        with ctx.Pool(cores) as pool:
            res = pool.map(reference_sample_worker, [(cfg, 1000 + i, n) for i in range(cores)])
        secs = time.perf_counter() - t0
        value = sum(r[0] for r in res) / secs
        nsys = res[0][2]
        n = res[0][0]
    return {"value": value, "n": n, "sample": f"reference BaryTree CPU build (gcc -O3, serial) on {cores} independent "
                                              f"system(s) of N={n} particles" +
                                              (f" in {nsys} systems" if cfg["dist"] == "batch" else "") +
                                              f" with this configuration's distribution and parameters (not the full "
                                              f"configuration); {secs:.1f} s wall"}


# Largest system the embedded CPU baseline runs the reference on: its serial
# setup grows with N (156 s of proxy charges at 16M), so a larger
# configuration is sampled at this N with its distribution; the reference arm
# (--impl reference) measures the full system.
CPU_BASELINE_MAX_N = 2_000_000


def cpu_baseline(cfg, config_id, cores):
    """The reference on this host, bounded to about half a minute: the split
    harness on the configuration's system (reduced to CPU_BASELINE_MAX_N
    particles of the same distribution when larger; one short sampled step)
    where it covers the configuration, else independent smaller systems."""
    if config_id in FULL_SYSTEM_REFERENCE and "n_override" not in cfg:
        c = dict(cfg)
        reduced = c["N"] > CPU_BASELINE_MAX_N
        if reduced:
            c["n_override"] = CPU_BASELINE_MAX_N
        r = reference_full_system(c, cores, 1, 1, 10.0)
        if r is None:
            return None
        sample = r["sample"]
        if reduced:
            sample += (f" [a bounded sample: the configuration's distribution at N={CPU_BASELINE_MAX_N:,}, not the "
                       f"full N={c['N']:,} system, which `bench.py --impl reference` measures]")
        return {"value": r["value"], "unit": "targets/s", "cores": cores, "kind": "reference", "sample": sample,
                "n": r["n"], "whole_system_s": r["whole_system_s"], "setup_s": r["setup_s"]}
    r = reference_samples(cfg, cores)
    if r is None:
        return None
    return {"value": r["value"], "unit": "targets/s", "cores": cores, "kind": "reference", "sample": r["sample"]}


# committed ncu summaries that carry a DRAM traffic figure for a configuration,
# and what that figure is
PROFILE_FOR_CONFIG = {5: ("eval_traffic_blobs16M.md",
                          "ncu capture (one pass per kernel) of the 16M evaluation's four kernels "
                          "(k_eval_targets_mixed_rb, k_pp_sym x2, k_sym_gather), second evaluation of the process: "
                          "dram__bytes_read.sum + dram__bytes_write.sum summed")}


def traffic_from_profiles(config_id, n_override=None):
    """DRAM bytes per launch of the evaluation kernels from the committed ncu
    summary, and where the figure comes from; (None, None) where no summary
    covers the run (a reduced --n is not what the figure describes)."""
    if config_id not in PROFILE_FOR_CONFIG or n_override:
        return None, None
    name, source = PROFILE_FOR_CONFIG[config_id]
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None, None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1]), f"{source} (profiles/{name})"
            except ValueError:
                return None, None
    return None, None


def max_over_ranks(ms, world, device):
    """Per-rank times (ms) reduced to the slowest rank's (the job's time)."""
    if world <= 1:
        return [float(v) for v in ms]
    import torch
    import torch.distributed as dist
    t = torch.tensor(ms, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def combine_shards(pot, world):
    """Sum the ranks' partial potentials in place (each target is nonzero on
    exactly one rank): the one collective of a target-sharded system."""
    if world <= 1:
        return pot
    import torch.distributed as dist
    dist.all_reduce(pot, op=dist.ReduceOp.SUM)
    return pot


def job_throughput(n_per_rank, world, ms_per_step):
    """Whole-job targets/s: every rank evaluates its own system of n_per_rank
    targets (weak scaling), the step lasting as long as the slowest rank."""
    return world * n_per_rank / (ms_per_step * 1e-3)


def roofline(sfu, tflops, fma_peak, prec, rep, ev_ms, w, mufu_per_eval, rsqrt_rate, traffic, traffic_source):
    """Roofline of the particle-output evaluation (PC + PP onto targets): the
    particle-output kernel and, when the targets are the sources, the
    symmetric near-field pair kernels beside it and their gather.

    Neither HBM nor the tensor cores bind it: source tiles are reused from
    shared memory and the work is kernel evaluations.  Mixed Lagrange: the
    special-function (MUFU) pipe binds (one rsqrt per evaluation, two MUFU ops
    for Yukawa), peak = the rsqrt rate measured on this GPU by the library's
    probe.  FP64: the FP64 FMA pipe, peak = the measured DFMA rate."""
    evals = rep["eval_flops"] / w
    r = {"kernel": "evaluation: k_eval_targets(_mixed) + k_pp_sym + k_sym_gather (PC + PP)", "ms_per_launch": ev_ms,
         "evaluations_per_launch": evals, "flops_per_launch": rep["eval_flops"], "traffic": traffic,
         "traffic_source": traffic_source,
         "simt_tflops": tflops, "simt_peak_tflops": fma_peak,
         "simt_frac": tflops / fma_peak if tflops else None,
         "peak_source": "measured by bt_measure_peaks on this GPU (rsqrt probe; FMA = 2 FLOP)"}
    if sfu:
        ach = evals * mufu_per_eval / (ev_ms * 1e-3) / 1e9 if ev_ms > 0 else None
        r.update(bound="sfu (MUFU rsqrt/ex2)", achieved=ach, peak=rsqrt_rate, unit="Gop/s",
                 frac=ach / rsqrt_rate if ach else None)
        # symmetric near-field pairs: one 1/r serves two of the evaluations
        # counted above, so the pipe itself did fewer operations
        sym = rep.get("sym_ptwise", 0)
        if sym and ev_ms > 0:
            phys = (evals - sym / 2) * mufu_per_eval / (ev_ms * 1e-3) / 1e9
            r.update(symmetric_evaluations=sym, mufu_physical=phys, frac_physical=phys / rsqrt_rate,
                     note="achieved counts evaluations as the reference does (each direction of a near-field "
                          "pair); mufu_physical counts the 1/r the GPU computed (one per symmetric pair), as "
                          "MUFU operations, although one grid point in eight (or fewer) of the Lagrange far "
                          "field takes its 1/r on the FP32 pipe instead")
    else:
        r.update(bound="fp64-simt" if prec == 0 else "fp32-simt", achieved=tflops, peak=fma_peak, unit="TFLOP/s",
                 frac=tflops / fma_peak if tflops else None)
    return r


def run_reference_arm(args, cfg, rank, world):
    """The reference's CPU implementation on this host's cores (rank 0 only):
    for configurations 1, 3 and 5 on the full system (reference_full_system),
    else on independent smaller systems (labelled as such)."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    full = args.config in FULL_SYSTEM_REFERENCE and "n_override" not in cfg
    if full:
        r = reference_full_system(cfg, cores, args.warmup, args.steps, args.ref_step_seconds)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref not present"}))
            return
        v = statistics.mean(r["per_step"])
        workload = cfg["workload"]
        extra = {k: r[k] for k in ("whole_system_s", "setup_s", "setup_phases_s", "eval_s_extrapolated",
                                   "rate_per_core", "interactions_total", "batches", "batches_per_step",
                                   "sample_fraction", "ms_per_sample_step")}
        sample = r["sample"]
    else:
        vals = []
        for _ in range(args.warmup):
            reference_samples(cfg, cores)
        for _ in range(args.steps):
            b = reference_samples(cfg, cores)
            if b is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref not present"}))
                return
            vals.append(b["value"])
        v = statistics.mean(vals)
        workload = f"{cfg['workload']} [reference: {b['sample']}]"
        extra = {}
        sample = b["sample"]
    line = {"metric": "targets/s", "value": v, "unit": "targets/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded numpy PCG64 with the configuration's "
                                                         "distribution, seed 0 as the GPU arm's rank 0)",
            "config": {"workload": workload, "config_id": args.config, "precision": "fp64",
                       "degree_policy": "fixed", "degree": cfg["degree"], "full_system": full},
            "cpu_baseline": dict({"value": v, "unit": "targets/s", "cores": cores, "kind": "reference",
                                  "sample": sample}, **extra),
            "e2e": {"value": v, "unit": "targets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def make_parser():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=5, choices=sorted(CONFIGS))
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--degree-policy", choices=["auto", "fixed", "learned"], default="auto",
                    help="auto: learned for the 16M clustered configuration, fixed otherwise")
    ap.add_argument("--tolerance", type=float, default=1e-6)
    ap.add_argument("--no-fp64-plain", action="store_true", help="skip the FP64 fixed-degree comparison step")
    ap.add_argument("--fp64-steps", type=int, default=3, help="timed steps of the FP64 fixed-degree comparison")
    ap.add_argument("--no-baselines", action="store_true",
                    help="skip the learned selection's baselines (lowest fixed degree meeting the tolerance in "
                         "mixed and FP64, the reference's beta path, and the split of the speed-up)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-step-seconds", type=float, default=4.0,
                    help="reference arm: host seconds of sampled evaluation per step")
    ap.add_argument("--no-graph", action="store_true", help="skip the session (graph replay) measurement")
    ap.add_argument("--dispatch", choices=["auto", "queue", "grid"], default="auto",
                    help="mixed evaluation kernels: persistent blocks on a device work queue, or one block per item")
    ap.add_argument("--upward", choices=["auto", "fp64"], default="auto",
                    help="mixed Lagrange upward pass: tensor-core leaf P2M (auto) or FP64 SIMT")
    ap.add_argument("--shard", action="store_true",
                    help="strong scaling: all ranks share one system, each evaluates its target shard, "
                         "one all-reduce combines the potentials (default: one independent system per rank)")
    ap.add_argument("--symmetry", choices=["auto", "off"], default="auto",
                    help="mixed path with targets = sources: near-field leaf pairs once for both sides (auto) or not")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default tile shape instead of autotuning it on this workload")
    ap.add_argument("--n", type=int, default=None,
                    help="particles (default: the configuration's N); smaller systems of the same "
                         "distribution for profiling captures")
    return ap


def eval_kwargs(B, cfg, args, policy, device, shard):
    """Keyword arguments of every library call of one run (treecode_ptr,
    treecode_batch_ptr, Session, autotune)."""
    prec = B.PRECISION_MIXED if args.precision == "mixed" else B.PRECISION_FP64
    return dict(degree_policy=B.DEGREE_LEARNED if policy == "learned" else B.DEGREE_FIXED,
                tolerance=args.tolerance,
                kernel=cfg["kernel"], kernel_param=cfg["kp"], approximation=cfg["approx"],
                compute_type=cfg["ctype"], theta=cfg["theta"], degree=cfg["degree"], max_source_leaf=cfg["leaf"],
                max_target_leaf=cfg["leaf"], size_check=cfg["sc"], precision=prec, device=device,
                dispatch={"auto": B.DISPATCH_AUTO, "queue": B.DISPATCH_QUEUE, "grid": B.DISPATCH_GRID}[args.dispatch],
                upward=B.UPWARD_FP64 if args.upward == "fp64" else B.UPWARD_AUTO,
                shard=shard, symmetry=B.SYMMETRY_OFF if args.symmetry == "off" else B.SYMMETRY_AUTO)


def autotune_kwargs(common):
    """The autotuner takes the run's arguments except precision (always mixed) and dispatch (tuned)."""
    return {k: v for k, v in common.items() if k not in ("precision", "dispatch")}


def main():
    args = make_parser().parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.n:
        cfg["n_override"] = args.n
        cfg["workload"] = f"{cfg['workload']} [reduced to N={args.n:,}]"

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, cfg, rank, world)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import barytree_b200 as B
    B.lib()

    dev = torch.device("cuda", local)
    shard = args.shard and world > 1
    x, y, z, q, off = make_inputs(cfg, seed=0 if args.shard else rank)
    n = len(x)
    batch = off is not None
    if shard and batch:
        raise SystemExit("--shard covers single systems (configurations 1-3 and 5)")
    ranks_n = n if args.shard else world * n        # targets of the whole job
    prec = B.PRECISION_MIXED if args.precision == "mixed" else B.PRECISION_FP64
    policy = args.degree_policy
    if policy == "auto":
        policy = "learned" if args.config == 5 and prec == B.PRECISION_MIXED else "fixed"
    if policy == "learned":
        from barytree_b200 import selector
        selector.install_default()
    common = eval_kwargs(B, cfg, args, policy, local, (rank, world) if shard else None)

    # device-resident inputs (targets are separate arrays with the same coordinates)
    d_in = [torch.from_numpy(a).to(dev) for a in (x, y, z, x.copy(), y.copy(), z.copy(), q)]
    d_out = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)     # > L2 (126 MB)

    def call(ptrs, out_ptr, on_device, **kw):
        if batch:
            return B.treecode_batch_ptr(len(off) - 1, off, off, *ptrs, out_ptr, inputs_on_device=on_device, **kw)
        return B.treecode_ptr(n, n, *ptrs, out_ptr, inputs_on_device=on_device, **kw)

    def step_device():
        rep = call([t.data_ptr() for t in d_in[3:6] + d_in[:3] + d_in[6:]], d_out.data_ptr(), True, **common)
        if shard:
            combine_shards(d_out, world)
        return rep

    # pinned host buffers for the end-to-end path
    h_in = [torch.from_numpy(a.copy()).pin_memory() for a in (x, y, z, x, y, z, q)]
    h_out = torch.empty(n, dtype=torch.float64).pin_memory()

    def step_host():
        rep = call([t.data_ptr() for t in h_in[3:6] + h_in[:3] + h_in[6:]], h_out.data_ptr(), False, **common)
        if shard:
            h_out.copy_(combine_shards(h_out.to(dev), world).cpu())
        return rep

    def timed(step, k):
        """K steps, each bracketed by CUDA events on the current stream; L2 flushed between steps."""
        total, reps = 0.0, []
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            reps.append(step())
            e1.record()
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        return total, reps

    # tile shape of the mixed particle-output kernel, autotuned once on this
    # workload before any timing (like a library's benchmark mode)
    tuning = None
    if prec == B.PRECISION_MIXED and not args.no_autotune:
        t0 = time.perf_counter()
        systems = ([(x[a:b], y[a:b], z[a:b], x[a:b], y[a:b], z[a:b], q[a:b]) for a, b in zip(off[:-1], off[1:])]
                   if batch else [(x, y, z, x, y, z, q)])
        best, trials = B.autotune(systems, **autotune_kwargs(common))
        tuning = {"best": best, "trials": len(trials), "seconds": round(time.perf_counter() - t0, 2),
                  "default_ms": next((t["ms"] for t in trials if t["targets_per_thread"] == 2 and
                                      t["source_tile"] == 1024 and t["dispatch"] == B.DISPATCH_GRID), None)}

    # clocks are sampled from the warm-up through both timed regions; the
    # sampler is started (and has answered once) before the warm-up, because
    # nvidia-smi's start-up stalls the GPU for tens of milliseconds
    clocks = ClockSampler(local)
    clocks.start()
    clocks.wait_first_sample()
    for _ in range(args.warmup):
        step_device()
        step_host()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = B.kernel_launch_count()
    ms_dev, reps = timed(step_device, args.steps)
    launches = B.kernel_launch_count() - launches0
    torch.cuda.synchronize()
    ms_e2e, _ = timed(step_host, args.steps)
    clock_info = clocks.stop()
    if world > 1:
        dist.barrier()
    ms_dev, ms_e2e = max_over_ranks([ms_dev, ms_e2e], world, dev)

    # accuracy of the last step vs the FP64 direct sum (outside timing): 10,000
    # strided targets; for a batch, per system (every target up to 20,000
    # particles, else 10,000 strided) and the worst system reported
    def accuracy(pot_all):
        if not batch:
            idx = np.arange(0, n, max(1, n // 10000))
            d = B.direct(x[idx], y[idx], z[idx], x, y, z, q, cfg["kernel"], cfg["kp"], device=local)
            e = pot_all[idx] - d
            return (float(np.linalg.norm(e) / np.linalg.norm(d)), float(np.max(np.abs(e)) / np.max(np.abs(d))),
                    len(idx))
        l2, mx, cnt = [], [], 0
        for k in range(len(off) - 1):
            a, b = int(off[k]), int(off[k + 1])
            m = b - a
            idx = a + (np.arange(m) if m <= 20000 else np.arange(0, m, m // 10000))
            d = B.direct(x[idx], y[idx], z[idx], x[a:b], y[a:b], z[a:b], q[a:b], cfg["kernel"], cfg["kp"],
                         device=local)
            e = pot_all[idx] - d
            l2.append(float(np.linalg.norm(e) / np.linalg.norm(d)))
            mx.append(float(np.max(np.abs(e)) / np.max(np.abs(d))))
            cnt += len(idx)
        return max(l2), max(mx), cnt

    rel_l2, rel_max, n_checked = accuracy(d_out.cpu().numpy())

    # the plain FP64 treecode at the configuration's fixed degree on the same
    # system and inputs (the denominator of the mixed + learned speed-up)
    fp64_plain = None
    if not args.no_fp64_plain and (prec != B.PRECISION_FP64 or policy != "fixed"):
        plain = dict(common)
        plain.update(precision=B.PRECISION_FP64, degree_policy=B.DEGREE_FIXED, dispatch=B.DISPATCH_AUTO)

        def step_plain():
            rep = call([t.data_ptr() for t in d_in[3:6] + d_in[:3] + d_in[6:]], d_out.data_ptr(), True, **plain)
            if shard:
                combine_shards(d_out, world)
            return rep
        step_plain()
        k_plain = max(1, args.fp64_steps)
        ms_plain, preps = timed(step_plain, k_plain)
        (ms_plain,) = max_over_ranks([ms_plain / k_plain], world, dev)
        fp64_plain = {"value": ranks_n / (ms_plain * 1e-3), "unit": "targets/s", "ms_per_step": ms_plain,
                      "steps": k_plain, "degree": cfg["degree"],
                      "rel_l2_vs_fp64_direct": accuracy(d_out.cpu().numpy())[0],
                      "ms_eval_kernel": preps[-1]["ms_eval_kernel"],
                      "interactions": preps[-1]["pp_ptwise"] + preps[-1]["pc_ptwise"]}

    # what the learned selection gains over the method without it: the lowest
    # fixed degree that meets the tolerance (mixed and FP64), the reference's
    # beta knob at the lowest beta that meets it, and the headline speed-up
    # split into its factors (precision, symmetric pass, degree selection)
    baselines = None
    if (not args.no_baselines and not shard and not batch and prec == B.PRECISION_MIXED and policy == "learned"
            and world == 1):
        def variant(k, **over):
            kw = dict(common)
            kw.update(degree_policy=B.DEGREE_FIXED, **over)

            def st():
                return call([t.data_ptr() for t in d_in[3:6] + d_in[:3] + d_in[6:]], d_out.data_ptr(), True, **kw)
            st()
            ms, vreps = timed(st, k)
            r = vreps[-1]
            return {"targets_per_s": n / (ms / k * 1e-3), "ms_per_step": ms / k, "steps": k,
                    "ms_eval_kernel": r["ms_eval_kernel"], "evaluations": r["pp_ptwise"] + r["pc_ptwise"],
                    "rel_l2_vs_fp64_direct": accuracy(d_out.cpu().numpy())[0],
                    "precision": "fp64" if kw["precision"] == B.PRECISION_FP64 else "mixed",
                    "theta": kw["theta"], "degree": kw["degree"], "leaf": kw["max_source_leaf"],
                    "symmetry": "off" if kw["symmetry"] == B.SYMMETRY_OFF else "auto"}

        def lowest_passing(runs):
            ok = [r for r in runs if r["rel_l2_vs_fp64_direct"] <= args.tolerance]
            return min(ok, key=lambda r: r["ms_per_step"]) if ok else None

        # mixed, fixed degree, from the configuration's degree down until the
        # tolerance is missed (lower degree: fewer far-field terms per pair)
        mixed_sweep = []
        for d in range(cfg["degree"], 1, -1):
            mixed_sweep.append(variant(2, degree=d))
            if mixed_sweep[-1]["rel_l2_vs_fp64_direct"] > args.tolerance:
                break
        mixed_best = lowest_passing(mixed_sweep)
        # FP64, fixed degree, from the mixed path's best degree down
        fp64_sweep = []
        d0 = mixed_best["degree"] if mixed_best else cfg["degree"]
        for d in range(d0, 1, -1):
            fp64_sweep.append(variant(1, degree=d, precision=B.PRECISION_FP64, dispatch=B.DISPATCH_AUTO))
            if fp64_sweep[-1]["rel_l2_vs_fp64_direct"] > args.tolerance:
                break
        # the reference's beta knob (theta and degree from beta, the reference
        # GPU build's leaf size), mixed precision, from beta 0.5 down by 0.1
        beta_sweep = []
        for b10 in range(5, 0, -1):
            bp = B.beta_parameters(b10 / 10, cfg["ctype"], cfg["approx"])
            r = variant(2, theta=bp["theta"], degree=bp["degree"], size_check=bp["size_check"],
                        max_source_leaf=bp["max_source_leaf"], max_target_leaf=bp["max_target_leaf"])
            r["beta"] = bp["beta"]
            beta_sweep.append(r)
            if r["rel_l2_vs_fp64_direct"] > args.tolerance:
                break
        # the speed-up's factors at the configuration's degree: precision
        # (FP64 -> mixed, symmetric pass off), the symmetric pass, the selection
        mixed_nosym = variant(2, degree=cfg["degree"], symmetry=B.SYMMETRY_OFF)
        mixed_sym = mixed_sweep[0]
        baselines = {
            "mixed_fixed_best": mixed_best, "fp64_fixed_best": lowest_passing(fp64_sweep),
            "beta_auto": lowest_passing(beta_sweep),
            "sweeps": {"mixed_fixed": mixed_sweep, "fp64_fixed": fp64_sweep, "beta": beta_sweep,
                       "mixed_fixed_symmetry_off": mixed_nosym},
            "what": ("device-resident steps like value; each variant one untimed step, then timed steps; rel-L2 "
                     "against the FP64 direct sum on the same strided targets; *_best = the fastest run of the "
                     "sweep that meets the tolerance; beta runs use the reference's theta/degree for beta and "
                     f"its GPU build's leaf size {B.BETA_GPU_LEAF}"),
        }

    # the same evaluation through a session: trees, lists and degree selection
    # built once, then per evaluation the charges go host->device, one CUDA
    # graph replays the whole device sequence, potentials come back
    graph = None
    if not args.no_graph and not shard:
        bounds = off if batch else np.array([0, n])
        systems = [(x[a:b], y[a:b], z[a:b], x[a:b], y[a:b], z[a:b], q[a:b]) for a, b in zip(bounds[:-1], bounds[1:])]
        sess = B.Session(systems, **common)
        hout = np.empty(n)                   # the solver's potential vector, reused across evaluations
        sess.evaluate(q, out=hout)
        ms_graph, greps = timed(lambda: sess.evaluate(q, return_report=True, out=hout)[1], args.steps)
        sess.close()
        ms_graph = max_over_ranks([ms_graph], world, dev)[0] / args.steps
        graph = {"value": world * n / (ms_graph * 1e-3), "unit": "targets/s", "ms_per_step": ms_graph,
                 "kernels_per_graph": greps[-1]["kernel_launches"], "ms_eval_kernel": greps[-1]["ms_eval_kernel"],
                 "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                 "what": "bt_session_eval with host charges and potentials (a reused host array): one CUDA graph replay of the whole "
                         "device sequence; trees, lists and degree selection made once by bt_session_create"}

    if rank == 0:
        fp64_peak, fp32_peak, rsqrt_rate = B.measure_peaks(local)
        rep = reps[-1]
        ev_ms = statistics.mean(r["ms_eval_kernel"] for r in reps)
        achieved = rep["eval_flops"] / (ev_ms * 1e-3) / 1e12 if ev_ms > 0 else None
        # Hermite grid outputs evaluate in FP64 in either precision mode
        fp64_kernels = prec == B.PRECISION_FP64 or (cfg["approx"] == 2 and cfg["ctype"] != 1)
        peak = fp64_peak if fp64_kernels else fp32_peak
        # the binding pipe of the mixed Lagrange kernels is the special-function
        # unit: one rsqrt per evaluation (Yukawa: rsqrt + ex2)
        w = {1: 10.0, 2: 13.0, 3: 11.0}[cfg["kernel"]]
        mufu_per_eval = 2 if cfg["kernel"] == 2 else 1
        sfu = prec == B.PRECISION_MIXED and cfg["approx"] == 1
        value = ranks_n / (ms_dev / args.steps * 1e-3)
        e2e = ranks_n / (ms_e2e / args.steps * 1e-3)
        line = {
            "metric": "targets/s", "value": value, "unit": "targets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
            "scaling": "strong" if args.shard else "weak",
            "vs_baseline": None, "dtype": "f64" if prec == B.PRECISION_FP64 else "f32+f64",
            "data": "synthetic (seeded numpy PCG64 with the configuration's distribution)",
            "config": {"workload": cfg["workload"], "config_id": args.config, "precision": args.precision,
                       "degree_policy": policy, "tolerance": args.tolerance, "dispatch": args.dispatch,
                       "tile_shape": tuning, "upward": args.upward, "symmetry": args.symmetry,
                       "l2": "flushed between steps (256 MB write)",
                       "parallelism": (f"one system, target shards over {world} GPU(s), one all-reduce of the "
                                       "potentials" if args.shard else
                                       f"{world} independent " + ("batch(es)" if batch else "system(s)") + ", one per GPU"),
                       "systems": len(off) - 1 if batch else 1,
                       "rel_l2_vs_fp64_direct": rel_l2, "rel_max_vs_fp64_direct": rel_max,
                       "direct_sample_targets": n_checked},
            # the target arrays hold the sources' coordinates, which the library
            # detects and copies once: x, y, z, q go host->device, potentials back
            "e2e": {"value": e2e, "unit": "targets/s", "h2d_bytes_per_step": 4 * 8 * n,
                    "d2h_bytes_per_step": 8 * n, "ms_per_step": ms_e2e / args.steps},
            "roofline": roofline(sfu, achieved, peak, B.PRECISION_FP64 if fp64_kernels else prec, rep, ev_ms, w,
                                 mufu_per_eval, rsqrt_rate,
                                 *(traffic_from_profiles(args.config, args.n) if sfu and policy == "learned"
                                   else (None, None))),
            "phases_ms": {k: rep[k] for k in ("ms_setup", "ms_upward", "ms_compute", "ms_downward", "ms_transfer")},
            "interactions": {k: rep[k] for k in ("pp_ptwise", "pc_ptwise", "cp_ptwise", "cc_ptwise")},
            "clocks": clock_info,
            "gpu_launches": launches,
        }
        if graph is not None:
            line["graph_replay"] = graph
        if fp64_plain is not None:
            line["fp64_plain"] = fp64_plain
            line["speedup_vs_fp64_plain"] = {"value": value / fp64_plain["value"],
                                             "e2e": e2e / fp64_plain["value"]}
        if baselines is not None:
            line["baselines"] = baselines
            ratio = {k: (value / baselines[k]["targets_per_s"] if baselines[k] else None)
                     for k in ("mixed_fixed_best", "fp64_fixed_best", "beta_auto")}
            line["speedup_vs_baselines"] = ratio
            if fp64_plain is not None:
                nosym = baselines["sweeps"]["mixed_fixed_symmetry_off"]["targets_per_s"]
                sym = baselines["sweeps"]["mixed_fixed"][0]["targets_per_s"]
                line["speedup_vs_fp64_plain"]["factors"] = {
                    "precision": nosym / fp64_plain["value"], "symmetric_pass": sym / nosym,
                    "degree_selection": value / sym,
                    "what": (f"at the configuration's degree {cfg['degree']}: FP64 -> mixed (symmetric pass off), "
                             "then the symmetric near-field pass, then the learned selection; their product is "
                             "the speed-up up to run-to-run noise")}
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(cfg, args.config, os.cpu_count() or 1)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
