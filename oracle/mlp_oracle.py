"""CPU FP64 oracle of the degree-selector MLP (test infrastructure).

Same network and loss as the library's CUDA kernels (bt_learned.cu): input
normalisation (x - mean) / std clipped to [-4, 4], three tanh layers of 64, a linear layer of 11,
mean-squared error over all outputs.  Forward and backward in numpy FP64, for
checking the GPU gradients.
"""
import numpy as np

IN, H, OUT = 6, 64, 11


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    parts = {}
    for name, size in (("mean", IN), ("std", IN), ("W1", IN * H), ("b1", H), ("W2", H * H), ("b2", H),
                       ("W3", H * H), ("b3", H), ("W4", H * OUT), ("b4", OUT)):
        parts[name] = w[o:o + size]
        o += size
    assert o == len(w)
    parts["W1"] = parts["W1"].reshape(IN, H)
    parts["W2"] = parts["W2"].reshape(H, H)
    parts["W3"] = parts["W3"].reshape(H, H)
    parts["W4"] = parts["W4"].reshape(H, OUT)
    return parts


def forward(w, X):
    p = unpack(w)
    Xn = np.clip((np.asarray(X, dtype=np.float64) - p["mean"]) / p["std"], -4.0, 4.0)
    A1 = np.tanh(Xn @ p["W1"] + p["b1"])
    A2 = np.tanh(A1 @ p["W2"] + p["b2"])
    A3 = np.tanh(A2 @ p["W3"] + p["b3"])
    return Xn, A1, A2, A3, A3 @ p["W4"] + p["b4"]


def loss_grad(w, X, Y):
    """(loss, gradient in the flat weight layout; zero for the normalisation)."""
    p = unpack(w)
    Xn, A1, A2, A3, Yh = forward(w, X)
    Y = np.asarray(Y, dtype=np.float64)
    B = len(X)
    loss = np.mean((Yh - Y) ** 2)
    dO = 2.0 * (Yh - Y) / (B * OUT)
    g = {"W4": A3.T @ dO, "b4": dO.sum(0)}
    d3 = (dO @ p["W4"].T) * (1 - A3 ** 2)
    g["W3"], g["b3"] = A2.T @ d3, d3.sum(0)
    d2 = (d3 @ p["W3"].T) * (1 - A2 ** 2)
    g["W2"], g["b2"] = A1.T @ d2, d2.sum(0)
    d1 = (d2 @ p["W2"].T) * (1 - A1 ** 2)
    g["W1"], g["b1"] = Xn.T @ d1, d1.sum(0)
    flat = np.concatenate([np.zeros(IN), np.zeros(IN)] +
                          [g[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")])
    return loss, flat
