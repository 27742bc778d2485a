"""GPU tests of the learned degree selector.

* the MLP gradient computed by the library's backward kernels matches the
  CPU FP64 oracle (oracle/mlp_oracle.py): loss to 1e-5 and gradient to 1e-4
  relative (FP32 accumulation over the batch);
* labels made by the treecode fall with the degree, and training on them
  with the library's Adam kernels lowers the loss;
* A/B against the fixed-degree method (degree 10, mixed precision) on a
  clustered system: with the selector the relative L2 error against the FP64
  direct sum stays within the 1e-6 tolerance while the number of kernel
  evaluations drops.
"""
import os

import numpy as np
import pytest

import barytree_b200 as B
from barytree_b200 import selector as S
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def test_mlp_gradient_matches_cpu_oracle():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(777, S.IN)).astype(np.float32) * np.array([1, 1, .2, .1, .1, .3], np.float32) + 1
    Y = rng.normal(size=(777, S.OUT)).astype(np.float32) - 6
    w = S.init_weights(X, seed=3)
    w[2 * S.IN:] += rng.normal(scale=0.05, size=len(w) - 2 * S.IN).astype(np.float32)
    loss_gpu, g_gpu = S.loss_grad(w, X, Y)
    loss_cpu, g_cpu = M.loss_grad(w, X, Y)
    assert abs(loss_gpu - loss_cpu) / loss_cpu < 1e-5
    assert np.linalg.norm(g_gpu - g_cpu) / np.linalg.norm(g_cpu) < 1e-4
    # every layer individually
    p_gpu, p_cpu = M.unpack(g_gpu), M.unpack(g_cpu)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        assert np.linalg.norm(p_gpu[k] - p_cpu[k]) <= 1e-4 * np.linalg.norm(p_cpu[k]) + 1e-9, k
    pred = S.predict(w, X)
    assert np.allclose(pred, M.forward(w, X)[-1], rtol=1e-4, atol=1e-4)


@pytest.fixture(scope="module")
def small_training_set():
    x, y, z, q = S.blobs(300_000, seed=5)
    return S.training_data(x, y, z, q, theta=0.7, leaf=500, nsamples=4000, seed=5)


def test_labels_fall_with_degree(small_training_set):
    f, lab = small_training_set
    assert len(f) > 1000
    assert np.all(np.isfinite(lab)) and np.all(np.isfinite(f))
    med = np.median(lab, axis=0)
    assert med[-1] < med[0] - 3          # degree 12 at least three decades below degree 2
    assert np.mean(np.diff(med) < 0) > 0.8


def test_training_lowers_loss(small_training_set):
    f, lab = small_training_set
    w0 = S.init_weights(f, seed=1)
    l0, _ = S.loss_grad(w0, f, lab)
    w, l1 = S.train(f, lab, w0, epochs=30, batch=256, lr=2e-3, seed=1)
    lf, _ = S.loss_grad(w, f, lab)
    assert lf < 0.2 * l0, (l0, lf)


def _selector_weights():
    if os.path.exists(S.MODEL_PATH):
        return S.load()
    x, y, z, q = S.blobs(1_000_000, seed=21)
    f, lab = S.training_data(x, y, z, q, theta=0.7, leaf=2000, nsamples=8000, seed=21)
    w, _ = S.train(f, lab, S.init_weights(f), epochs=60, batch=256, lr=1e-3)
    return w


def test_learned_vs_fixed_degree_ab():
    S.install(_selector_weights())
    x, y, z, q = S.blobs(1_000_000, seed=77)
    common = dict(theta=0.7, max_source_leaf=2000, max_target_leaf=2000, precision=B.PRECISION_MIXED,
                  return_report=True)
    fixed, rf = B.treecode(x, y, z, x, y, z, q, degree=10, **common)
    learned, rl = B.treecode(x, y, z, x, y, z, q, degree=10, degree_policy=B.DEGREE_LEARNED, tolerance=1e-6, **common)
    idx = np.arange(0, len(x), 97)
    d = B.direct(x[idx], y[idx], z[idx], x, y, z, q)
    err_fixed = np.linalg.norm(fixed[idx] - d) / np.linalg.norm(d)
    err_learned = np.linalg.norm(learned[idx] - d) / np.linalg.norm(d)
    evals_fixed = rf["pp_ptwise"] + rf["pc_ptwise"]
    evals_learned = rl["pp_ptwise"] + rl["pc_ptwise"]
    print(f"fixed n=10: rel-L2 {err_fixed:.2e}, {evals_fixed:.3e} evals, kernel {rf['ms_eval_kernel']:.1f} ms; "
          f"learned: rel-L2 {err_learned:.2e}, {evals_learned:.3e} evals, kernel {rl['ms_eval_kernel']:.1f} ms")
    assert err_learned <= 1e-6
    assert evals_learned < 0.8 * evals_fixed
