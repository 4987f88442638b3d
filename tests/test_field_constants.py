"""Host-side checks of the float32 Gaussian pulse's mathematics.

The float32 form evaluates gaussian_laser_pulse from twelve float32
constants that fields.py packs into slots 10-15 of the parameter block, with
no divisions: the curvature term k0 r^2 / (2 R(x)) as (k0 / (2 zR^2)) r^2 x / q
and r^2 / w(x)^2 as (1/w0^2) r^2 / q, q = 1 + (x/zR)^2, 1/q = rsqrt(q)^2.
Here that evaluation is restated in numpy float32 (slot order as the device
reads it) and compared with the float64 formula of the reference
(fields.py:152-168), and the float32 far-field cut is shown to be exact:
where it sets the field to 0, the envelope is below float32's smallest
subnormal."""
import math

import numpy as np

from sfparticles_b200.constants import C
from sfparticles_b200.fields import gaussian_laser_pulse

F32 = np.float32
CUT32 = 10.5  # |phi| / kc of the float32 cut


def _pulse(a0=200.0, w0=3e-6, ctau=6.4e-6, d=-1, x0=20e-6, pol=0.4, cep=0.3):
    p = gaussian_laser_pulse(a0, w0, ctau, direction=d, x0=x0, pol_angle=pol, cep=cep).params()
    return p, np.frombuffer(np.ascontiguousarray(p[10:16]).tobytes(), dtype="<f4")


def _field64(P, x, y, z, t):
    """Ey of the reference formula in float64 (x != 0)."""
    E0, k0, zR, w0, ctau, d, x0, cep, cp = P[:9]
    r2 = y * y + z * z
    wx = w0 * np.sqrt(1 + (x / zR) ** 2)
    Rx = x * (1 + (zR / x) ** 2)
    phi = k0 * ((x - x0) - d * C * t) + k0 * r2 / 2 / Rx - np.arctan(x / zR)
    kc = k0 * ctau
    return E0 * np.cos(phi + cep) * w0 / wx * np.exp(-r2 / wx ** 2) * np.exp(-(phi / kc) ** 2) * cp, phi / kc


def _field32(P, G, x, y, z, t):
    """Ey of the float32 evaluation, operation by operation."""
    E0, k0, inv_zR, cq, inv_w02, inv_kc2, dirc, cep, cp, sp, cut_r, kc = (F32(v) for v in G)
    d, x0 = P[5], P[6]
    xf, yf, zf = x.astype(F32), y.astype(F32), z.astype(F32)
    xr = ((x - x0) - (d * C) * t).astype(F32)
    r2 = yf * yf + zf * zf
    cut = k0 * np.abs(xr) - cut_r * r2 - F32(1.5708) > F32(CUT32) * kc
    xz = xf * inv_zR
    q = F32(1) + xz * xz
    rs = F32(1) / np.sqrt(q)
    rq = rs * rs
    phi = k0 * xr + (cq * r2) * (xf * rq) - np.arctan(xz)
    env = np.exp(-((r2 * inv_w02) * rq + (phi * phi) * inv_kc2))
    Ey = E0 * np.cos(phi + cep) * rs * env * cp
    return np.where(cut, F32(0), Ey), cut


def test_packed_constants_reproduce_the_float64_field():
    P, G = _pulse()
    rng = np.random.default_rng(5)
    n = 200_000
    t = 0.0
    x = P[6] + rng.uniform(-3, 3, n) * P[4]  # within three pulse lengths of the centre
    x = np.where(np.abs(x) < 1e-12, 1e-12, x)
    y, z = rng.normal(0, 2e-6, n), rng.normal(0, 2e-6, n)
    e64, _ = _field64(P, x, y, z, t)
    e32, cut = _field32(P, G, x, y, z, t)
    assert not cut.any()
    # float32 phase: |phi| up to ~1e2 rad carries ~1e-5 rad of rounding
    err = np.abs(e32.astype(np.float64) - e64).max() / np.abs(e64).max()
    assert err < 5e-5, err


def test_float32_cut_is_exact():
    """Wherever the float32 cut sets the field to 0, exp(-(phi/kc)^2) of the
    float64 formula is below float32's smallest subnormal (2^-149)."""
    for d in (1, -1):
        P, G = _pulse(d=d, w0=2e-6, ctau=3e-6)
        rng = np.random.default_rng(9 + d)
        n = 400_000
        t = rng.uniform(0, 200e-15, n)
        x = P[6] + d * C * t + rng.uniform(-15, 15, n) * P[4]
        x = np.where(np.abs(x) < 1e-12, 1e-12, x)
        y, z = rng.normal(0, 5e-6, n), rng.normal(0, 5e-6, n)
        _, cut = _field32(P, G, x, y, z, t)
        _, u = _field64(P, x, y, z, t)
        assert cut.sum() > n // 4
        assert (u[cut] ** 2 > 149 * math.log(2)).all()
