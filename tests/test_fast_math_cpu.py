"""The Remez-fitted atan2 of csrc/fast_math.cuh (the phase output of boxcar and
Goldstein), checked on the CPU: the coefficients are read from the header
itself and evaluated in float32 in the kernel's operation order (Horner with
one rounding per step, the quotient from a reciprocal one ulp off), against
numpy's double-precision arctan2.  The header states 6e-7 rad."""
import os
import re

import numpy as np

HEADER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "despeckcl_b200", "csrc", "fast_math.cuh")
f32 = np.float32


def _coefficients():
    src = open(HEADER).read()
    body = src[src.index("atan2_fast"):]
    first = float(re.search(r"float p = ([-0-9.eE]+)f;", body).group(1))
    rest = [float(v) for v in re.findall(r"p = fmaf\(p, s, ([-0-9.eE]+)f\);", body)]
    return [first] + rest  # highest degree first


def _atan2_f32(y, x, coef, rng):
    y = y.astype(f32)
    x = x.astype(f32)
    ax, ay = np.abs(x), np.abs(y)
    mx, mn = np.maximum(ax, ay), np.minimum(ax, ay)
    inv = (f32(1) / np.maximum(mx, f32(1.17549435e-38))).astype(f32)
    # the hardware reciprocal is within one ulp: take either neighbour
    inv = np.where(rng.random(inv.shape) < 0.5, np.nextafter(inv, f32(np.inf)), inv).astype(f32)
    a = (mn * inv).astype(f32)
    s = (a * a).astype(f32)
    p = np.full_like(s, f32(coef[0]))
    for c in coef[1:]:
        p = (p.astype(np.float64) * s + c).astype(f32)  # one rounding, like fmaf
    r = (a * p).astype(f32)
    r = np.where(ay > ax, (f32(1.57079637) - r).astype(f32), r)
    r = np.where(np.signbit(x), (f32(3.14159274) - r).astype(f32), r)
    return np.copysign(r, y)


def test_atan2_fast_within_its_stated_bound():
    coef = _coefficients()
    assert len(coef) == 7
    rng = np.random.default_rng(5)
    n = 2_000_000
    x = rng.standard_normal(n) * 10.0 ** rng.uniform(-30, 30, n)
    y = rng.standard_normal(n) * 10.0 ** rng.uniform(-30, 30, n)
    got = _atan2_f32(y, x, coef, rng).astype(np.float64)
    want = np.arctan2(y.astype(f32).astype(np.float64), x.astype(f32).astype(np.float64))
    err = np.abs(np.angle(np.exp(1j * (got - want))))
    assert err.max() <= 6e-7, err.max()


def test_atan2_fast_axes_and_signs():
    coef = _coefficients()
    rng = np.random.default_rng(6)
    y = np.array([0.0, 0.0, 1.0, -1.0, 1.0, -1.0, -0.0, 0.0])
    x = np.array([1.0, -1.0, 0.0, 0.0, 1.0, -1.0, -1.0, 0.0])
    got = _atan2_f32(y, x, coef, rng).astype(np.float64)
    want = np.arctan2(y, x)
    assert np.all(np.abs(got - want) <= 6e-7), (got, want)
