"""Learned interpolation-degree selector: training data, training, storage.

The selector is a 6 -> 64 -> 64 -> 64 -> 11 tanh MLP (FP32) that predicts,
for one particle-cluster interaction, log10 of its normalised error at
degrees 2..12 (see include/barytree_b200.h).  Everything heavy runs on the
GPU inside libbarytree_b200.so:

* ``training_data``  -- the treecode labels its own interactions against the
  exact FP64 sum (bt_selector_training_data);
* ``train``          -- Adam with the library's forward/backward kernels
  (bt_selector_train);
* ``install``        -- hands the weights to the library (bt_selector_set).

Usage (writes barytree_b200/models/degree_selector.npz):

    python -m barytree_b200.selector --out barytree_b200/models/degree_selector.npz
"""
from __future__ import annotations

import argparse
import ctypes
import os
import time

import numpy as np

from . import _check, lib

IN, H, OUT = 6, 64, 11
DEGREES = tuple(range(2, 13))
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "degree_selector.npz")
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)


def nweights() -> int:
    return int(lib().bt_selector_nweights())


def blobs(n, seed):
    """Clustered system: 80% in 8 Gaussian blobs (centres U[-0.7,0.7]^3, sigma
    log-uniform in [0.05, 0.3], equal counts, clipped to [-1,1]^3) and 20%
    uniform in [-1,1]^3; charges U[-1,1]."""
    rng = np.random.default_rng(seed)
    nb = int(0.8 * n) // 8 * 8
    nu = n - nb
    c = rng.uniform(-0.7, 0.7, (8, 3))
    sig = np.exp(rng.uniform(np.log(0.05), np.log(0.3), 8))
    parts = [np.clip(rng.normal(c[i], sig[i], (nb // 8, 3)), -1, 1) for i in range(8)]
    parts.append(rng.uniform(-1, 1, (nu, 3)))
    p = np.concatenate(parts)
    q = rng.uniform(-1, 1, n)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), q


def training_data(x, y, z, q, theta=0.7, leaf=2000, nsamples=20000, seed=0, device=0):
    x, y, z, q = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q))
    f = np.zeros((nsamples, IN), dtype=np.float32)
    lab = np.zeros((nsamples, OUT), dtype=np.float32)
    got = lib().bt_selector_training_data(len(x), x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                          z.ctypes.data_as(_dp), q.ctypes.data_as(_dp), float(theta), int(leaf),
                                          int(nsamples), int(seed), f.ctypes.data_as(_fp), lab.ctypes.data_as(_fp),
                                          int(device))
    if got < 0:
        _check(-got)
    return f[:got], lab[:got]


def init_weights(features, seed=0):
    """Glorot-uniform weights, zero biases, input normalisation from the data."""
    rng = np.random.default_rng(seed)
    mean = features.mean(axis=0)
    std = features.std(axis=0) + 1e-6
    parts = [mean, std]
    for fi, fo in ((IN, H), (H, H), (H, H), (H, OUT)):
        lim = np.sqrt(6.0 / (fi + fo))
        parts.append(rng.uniform(-lim, lim, fi * fo))
        parts.append(np.zeros(fo))
    w = np.concatenate(parts).astype(np.float32)
    assert len(w) == nweights()
    return w


def train(features, labels, weights, epochs=60, batch=512, lr=1e-3, seed=0, device=0):
    w = np.ascontiguousarray(weights, dtype=np.float32).copy()
    f = np.ascontiguousarray(features, dtype=np.float32)
    lab = np.ascontiguousarray(labels, dtype=np.float32)
    loss = ctypes.c_float()
    _check(lib().bt_selector_train(f.ctypes.data_as(_fp), lab.ctypes.data_as(_fp), len(f), int(epochs), int(batch),
                                   float(lr), int(seed), w.ctypes.data_as(_fp), ctypes.byref(loss), int(device)))
    return w, float(loss.value)


def loss_grad(weights, features, labels, device=0):
    w = np.ascontiguousarray(weights, dtype=np.float32)
    f = np.ascontiguousarray(features, dtype=np.float32)
    lab = np.ascontiguousarray(labels, dtype=np.float32)
    g = np.zeros(nweights(), dtype=np.float32)
    loss = ctypes.c_float()
    _check(lib().bt_mlp_loss_grad(w.ctypes.data_as(_fp), f.ctypes.data_as(_fp), lab.ctypes.data_as(_fp), len(f),
                                  g.ctypes.data_as(_fp), ctypes.byref(loss), int(device)))
    return float(loss.value), g


def predict(weights, features, device=0):
    w = np.ascontiguousarray(weights, dtype=np.float32)
    f = np.ascontiguousarray(features, dtype=np.float32)
    out = np.zeros((len(f), OUT), dtype=np.float32)
    _check(lib().bt_mlp_predict(w.ctypes.data_as(_fp), f.ctypes.data_as(_fp), len(f), out.ctypes.data_as(_fp),
                                int(device)))
    return out


def install(weights):
    w = np.ascontiguousarray(weights, dtype=np.float32)
    _check(lib().bt_selector_set(w.ctypes.data_as(_fp), len(w)))


def save(path, weights, meta):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, weights=np.asarray(weights, dtype=np.float32), **{k: np.asarray(v) for k, v in meta.items()})


def load(path=MODEL_PATH):
    return np.load(path)["weights"].astype(np.float32)


def install_default():
    """Install the committed selector (barytree_b200/models/degree_selector.npz)."""
    install(load(MODEL_PATH))


def build_default(out=MODEL_PATH, device=0, log=print):
    """The committed selector's training recipe: clustered systems of the
    benchmark's distribution at three sizes plus a uniform one, theta 0.7,
    leaf 2000, 20,000 labelled interactions each."""
    t0 = time.time()
    feats, labs = [], []
    systems = [("blobs", 2_000_000, 11), ("blobs", 4_000_000, 12), ("blobs", 16_000_000, 13), ("uniform", 1_000_000, 14)]
    for kind, n, seed in systems:
        if kind == "blobs":
            x, y, z, q = blobs(n, seed)
        else:
            rng = np.random.default_rng(seed)
            x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
            q = rng.uniform(-1, 1, n)
        f, lab = training_data(x, y, z, q, theta=0.7, leaf=2000, nsamples=20000, seed=seed, device=device)
        feats.append(f)
        labs.append(lab)
        log(f"{kind} N={n}: {len(f)} labelled interactions ({time.time() - t0:.1f} s)")
    f = np.concatenate(feats)
    lab = np.concatenate(labs)
    rng = np.random.default_rng(0)
    idx = rng.permutation(len(f))
    nval = len(f) // 10
    val, trn = idx[:nval], idx[nval:]
    w0 = init_weights(f[trn], seed=0)
    w, tr_loss = train(f[trn], lab[trn], w0, epochs=80, batch=512, lr=1e-3, seed=0, device=device)
    val_loss, _ = loss_grad(w, f[val], lab[val], device=device)
    log(f"trained: train loss {tr_loss:.4f}, validation loss {val_loss:.4f} (log10 units^2), {time.time() - t0:.1f} s")
    save(out, w, {"train_loss": tr_loss, "val_loss": val_loss, "samples": len(f)})
    np.savez(os.path.splitext(out)[0] + "_data.npz", features=f, labels=lab)
    return w


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=MODEL_PATH)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    build_default(a.out, a.device)
