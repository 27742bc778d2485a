"""CPU checks of bench.py's plumbing: for every configuration and the
options that change the library calls, the keyword arguments the run builds
are accepted by each call it makes (bt_eval through treecode_ptr, the batch
call, sessions and the autotuner), so a run cannot fail on an argument
after minutes on the GPU."""
import inspect
import os

import numpy as np
import pytest

import barytree_b200 as B
import bench
from conftest import ROOT


@pytest.mark.parametrize("config", sorted(bench.CONFIGS))
@pytest.mark.parametrize("argv", [[], ["--precision", "fp64"], ["--dispatch", "queue", "--upward", "fp64"],
                                  ["--shard"], ["--symmetry", "off"]])
def test_every_call_accepts_the_run_arguments(config, argv):
    args = bench.make_parser().parse_args(["--config", str(config)] + argv)
    cfg = bench.CONFIGS[config]
    for policy in ("fixed", "learned"):
        common = bench.eval_kwargs(B, cfg, args, policy, 0, (0, 2) if "--shard" in argv else None)
        ptrs = [0] * 7
        inspect.signature(B.treecode_ptr).bind(10, 10, *ptrs, 0, inputs_on_device=True, **common)
        inspect.signature(B.treecode_batch_ptr).bind(1, np.zeros(2), np.zeros(2), *ptrs, 0,
                                                     inputs_on_device=True, **common)
        inspect.signature(B.Session).bind([], **common)
        inspect.signature(B.autotune).bind([], **bench.autotune_kwargs(common))
        plain = dict(common)
        plain.update(precision=B.PRECISION_FP64, degree_policy=B.DEGREE_FIXED, dispatch=B.DISPATCH_AUTO)
        inspect.signature(B.treecode_ptr).bind(10, 10, *ptrs, 0, inputs_on_device=True, **plain)


def test_ranks_share_the_host_cores_under_torchrun():
    """A rank started by torchrun (OMP_NUM_THREADS=1) gets its share of the
    host's cores for the library's host planning; a single process and an
    explicit thread count are left alone."""
    import subprocess
    import sys
    code = "import os, bench; print(os.environ.get('OMP_NUM_THREADS'))"
    cores = os.cpu_count() or 1
    for local, omp, want in [("2", "1", str(max(1, cores // 2))), ("1", "1", "1"), ("4", "3", "3")]:
        env = dict(os.environ, LOCAL_WORLD_SIZE=local, OMP_NUM_THREADS=omp)
        out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                             check=True).stdout.split()[-1]
        assert out == want, (local, omp, out)
