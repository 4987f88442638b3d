"""sfp32::atan_r (csrc/sfp_device32.cuh), the float32 form's branch-free
atan of the Gaussian pulse's Gouy phase, emulated in float32 with its own
coefficients read from the header: within 4 ulp of the exact arctan over
every magnitude, exact sign symmetry, atan(0) = 0, and the limits at
+-infinity."""
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HDR = os.path.join(os.path.dirname(HERE), "sfparticles_b200", "csrc", "sfp_device32.cuh")


def _coefficients():
    src = open(HDR).read()
    body = re.search(r"SFP_DEVICE_INLINE float atan_r\(float a\) \{(.*?)\n\}", src, re.S).group(1)
    first = float(re.search(r"float p = ([-0-9.e]+)f;", body).group(1))
    rest = [float(v) for v in re.findall(r"p = fmaf\(p, u, ([-0-9.e]+)f\);", body)]
    return [first] + rest


def atan_r(a):
    """The device function, step by step in float32 (fmaf as one rounding)."""
    f32 = np.float32
    a = np.asarray(a, dtype=f32)
    ax = np.abs(a)
    big = ax > f32(1.0)
    with np.errstate(divide="ignore"):
        t = np.where(big, (f32(1.0) / ax).astype(f32), ax).astype(f32)
    u = (t * t).astype(f32)
    c = _coefficients()
    p = np.full_like(t, f32(c[0]))
    for k in c[1:]:
        p = (p.astype(np.float64) * u.astype(np.float64) + np.float64(f32(k))).astype(f32)
    r = (t * p).astype(f32)
    r = np.where(big, (f32(1.5707963267948966) - r).astype(f32), r)
    return np.copysign(r, a).astype(f32)


def test_coefficients_found():
    c = _coefficients()
    assert len(c) == 9 and c[-1] == 1.0


def test_within_four_ulp_everywhere():
    rng = np.random.default_rng(3)
    a = np.concatenate([np.linspace(-2, 2, 400001), np.exp(rng.uniform(-30, 30, 200000)),
                        -np.exp(rng.uniform(-30, 30, 200000)), [1.0, -1.0, 1 + 2 ** -23, 1 - 2 ** -24]])
    a = a.astype(np.float32)
    got = atan_r(a).astype(np.float64)
    ref = np.arctan(a.astype(np.float64))
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    err = np.abs(got - ref) / np.maximum(ulp, np.finfo(np.float32).tiny)
    assert err.max() <= 4.0, (err.max(), a[np.argmax(err)])


def test_sign_zero_and_limits():
    a = np.float32([0.0, -0.0, np.inf, -np.inf, 3.0e38, -3.0e38, 1e-30])
    r = atan_r(a)
    assert r[0] == 0.0 and r[1] == 0.0 and np.signbit(r[1])
    assert abs(float(r[2]) - np.pi / 2) < 1e-7 and abs(float(r[3]) + np.pi / 2) < 1e-7
    assert abs(float(r[4]) - np.pi / 2) < 1e-7 and r[6] == np.float32(1e-30)
    x = np.float32(np.linspace(0.01, 50, 1001))
    assert np.array_equal(atan_r(-x), -atan_r(x))
