"""The FP32 patch bound of the FP32C CPA search (patch_rejects in
csrc/wq3d_kernels.cu) restated with numpy float32 arithmetic, one rounding
per operation as the kernel (built with --fmad=false) does it, and checked
against the same bound in exact rational arithmetic: a target the FP32
form rejects must be rejected by the exact bound too, or the per-ray
screen could lose a pair it would have kept."""
from fractions import Fraction as Fr

import numpy as np

f = np.float32
U32 = f(5.9604645e-8)  # 2^-24


def rejects_fp32(w, lo, hi, W, c0):
    ub = mag = wm = f(0)
    for m in range(8):
        a, b = f(w[m] * lo[m]), f(w[m] * hi[m])
        ub = f(ub + max(a, b))
        mag = f(mag + max(abs(a), abs(b)))
        wm = f(wm + f(W[m] * max(abs(lo[m]), abs(hi[m]))))
    t = f(ub + f(f(f(14) * U32) * mag))
    t = f(t + f(f(f(43) * U32) * wm))
    t = f(t + f(f(1.0003) * c0))
    return bool(t < 0)


def rejects_exact(w, lo, hi, W, c0):
    """sum_k max(w_k lo_k, w_k hi_k) + 41 u sum_k W_k max|range_k| + 1.0001 c0 < 0"""
    ub = sum(max(Fr(float(w[m])) * Fr(float(lo[m])), Fr(float(w[m])) * Fr(float(hi[m]))) for m in range(8))
    wm = sum(Fr(float(W[m])) * max(abs(Fr(float(lo[m]))), abs(Fr(float(hi[m])))) for m in range(8))
    return ub + 41 * Fr(1, 2 ** 24) * wm + Fr(10001, 10000) * Fr(float(c0)) < 0


def test_fp32_patch_bound_never_rejects_more_than_the_exact_bound():
    rng = np.random.default_rng(20261203)
    n_fp32 = n_exact = 0
    for _ in range(3000):
        w = (rng.standard_normal(8) * 10.0 ** rng.uniform(-3, 8, 8)).astype(f)
        lo = (rng.standard_normal(8) * 10.0 ** rng.uniform(-4, 3, 8)).astype(f)
        hi = (lo + np.abs(rng.standard_normal(8)) * 10.0 ** rng.uniform(-6, 2, 8)).astype(f)
        # move the constant feature's weight so the bound sits near zero
        if abs(lo[0]) > 1e-3:
            ub = sum(max(float(w[m]) * float(lo[m]), float(w[m]) * float(hi[m])) for m in range(8))
            w[0] = f(w[0] - f(ub / abs(float(lo[0])) * rng.uniform(0.9, 1.1)))
        W = (np.abs(w) * f(1.0001)).astype(f)
        c0 = f(1.0)
        r32 = rejects_fp32(w, lo, hi, W, c0)
        rex = rejects_exact(w, lo, hi, W, c0)
        assert not (r32 and not rex), (w, lo, hi)
        n_fp32 += r32
        n_exact += rex
    # the FP32 form is conservative but nearly as sharp
    assert n_fp32 > 0.98 * n_exact > 0


def one_product_form_sum(w, lo, hi, W, c0):
    """The kernel's form: per-patch magnitudes and weighted-range sum
    hoisted, one product per term chosen by the weight's sign."""
    M = [max(abs(lo[m]), abs(hi[m])) for m in range(8)]
    wm = f(0)
    for m in range(8):
        wm = f(wm + f(W[m] * M[m]))
    K = f(f(f(43) * U32) * wm)
    Cc = f(f(1.0003) * c0)
    ub = mag = f(0)
    for m in range(8):
        ub = f(ub + f(w[m] * (hi[m] if w[m] >= 0 else lo[m])))
        mag = f(mag + f(abs(w[m]) * M[m]))
    t = f(f(f(ub + f(f(f(14) * U32) * mag)) + K) + Cc)
    return t


def full_form_sum(w, lo, hi, W, c0):
    ub = mag = wm = f(0)
    for m in range(8):
        a, b = f(w[m] * lo[m]), f(w[m] * hi[m])
        ub = f(ub + max(a, b))
        mag = f(mag + max(abs(a), abs(b)))
        wm = f(wm + f(W[m] * max(abs(lo[m]), abs(hi[m]))))
    t = f(ub + f(f(f(14) * U32) * mag))
    t = f(t + f(f(f(43) * U32) * wm))
    return f(t + f(f(1.0003) * c0))


def test_one_product_form_equals_full_form():
    rng = np.random.default_rng(11)
    for _ in range(5000):
        w = (rng.standard_normal(8) * 10.0 ** rng.uniform(-3, 8, 8)).astype(f)
        w[rng.random(8) < 0.1] = f(0)
        lo = (rng.standard_normal(8) * 10.0 ** rng.uniform(-4, 3, 8)).astype(f)
        hi = (lo + np.abs(rng.standard_normal(8)) * 10.0 ** rng.uniform(-6, 2, 8)).astype(f)
        W = (np.abs(w) * f(1.0001)).astype(f)
        c0 = f(rng.uniform(1.0, 3.0))
        a = one_product_form_sum(w, lo, hi, W, c0)
        b = full_form_sum(w, lo, hi, W, c0)
        assert a == b, (a, b)
