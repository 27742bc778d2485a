"""The far field's software 1/sqrt (f2_rsqrt_sw in barytree_b200/csrc/bt_f2.cuh),
emulated step by step in FP32 on the CPU: C. Lomont's bit-pattern estimate
(2003, constant 0x5f375a86), one Newton step y <- y - y e/2 and one
third-order step y <- y (1 - e/2 + 3 e^2/8), each with e = x y^2 - 1.
Every FP32 multiply and fused multiply-add is rounded once, as on the GPU
(products of FP32 values are exact in FP64; the FP64 sum is rounded to
FP32).

The bound checked is the one the kernels rely on: relative error below
2.5e-7 over the squared distances the far field meets (the MUFU
approximation it stands in for is within about 1.3e-7), and no bias.
"""
import numpy as np

LOMONT = np.uint32(0x5F375A86)


def f32(v):
    return np.asarray(v, dtype=np.float64).astype(np.float32)


def fma32(a, b, c):
    # a*b is exact in FP64 for FP32 a, b; the sum rounds once in FP64 and
    # once more to FP32, which differs from a single rounding only in rare
    # ties far below the bound tested here
    return f32(a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64))


def mul32(a, b):
    return f32(a.astype(np.float64) * b.astype(np.float64))


def rsqrt_sw(x):
    x = f32(x)
    m1, mh = f32(np.full_like(x, -1.0)), f32(np.full_like(x, -0.5))
    y = (LOMONT - (x.view(np.uint32) >> np.uint32(1))).astype(np.uint32).view(np.float32)
    e = fma32(x, mul32(y, y), m1)
    y = fma32(mul32(y, e), mh, y)
    e = fma32(x, mul32(y, y), m1)
    p = fma32(e, f32(np.full_like(x, 0.375)), mh)
    return fma32(mul32(y, e), p, y)


def test_software_rsqrt_accuracy_over_far_field_range():
    rng = np.random.default_rng(7)
    # squared distances of well-separated pairs in leaf-relative FP32
    # coordinates: from 1e-12 to 1e6, log-uniform, plus every mantissa
    # pattern near powers of two (where the estimate's error peaks)
    x = f32(10.0 ** rng.uniform(-12, 6, 400_000))
    k = np.arange(-40, 20, dtype=np.float64)
    edges = f32(np.concatenate([2.0 ** k * (1 + d) for d in (-1e-7, 0.0, 1e-7, 0.5, 0.999)]))
    x = np.concatenate([x, edges[edges > 0]])
    y = rsqrt_sw(x).astype(np.float64)
    ref = 1.0 / np.sqrt(x.astype(np.float64))
    rel = (y - ref) / ref
    assert np.all(np.isfinite(y))
    assert np.max(np.abs(rel)) < 2.5e-7, np.max(np.abs(rel))
    assert abs(np.mean(rel)) < 2e-8


def test_lomont_estimate_and_newton_step_bounds():
    x = f32(10.0 ** np.linspace(-10, 10, 200_001))
    y0 = (LOMONT - (x.view(np.uint32) >> np.uint32(1))).astype(np.uint32).view(np.float32)
    rel0 = y0.astype(np.float64) * np.sqrt(x.astype(np.float64)) - 1.0
    assert np.max(np.abs(rel0)) < 3.5e-2
    e = fma32(x, mul32(y0, y0), f32(np.full_like(x, -1.0)))
    y1 = fma32(mul32(y0, e), f32(np.full_like(x, -0.5)), y0)
    rel1 = y1.astype(np.float64) * np.sqrt(x.astype(np.float64)) - 1.0
    assert np.max(np.abs(rel1)) < 1.8e-3
