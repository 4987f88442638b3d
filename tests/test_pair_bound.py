"""The pair-rate bound behind the photon kernel's exact skip of pair tests
(rejection sampling): csrc/sfp_capi.cu k_pair_bound, exposed as
sfp_pair_rate_bound, with the chi bins of sfp_pair_bin (csrc/sfp_run.cuh).

A photon is pushed without its pair test when bound(bin of chi) * dt / gamma
is below the smallest second draw; that is exact only if 4 * the pair rate
(qed/rejection_sampling_tables.py:56-78) never exceeds the bound at any delta
for any chi of the bin.  Restated here in numpy and checked on the CPU
against the oracle's restatement of the reference's rate (pinned to the
reference's own outputs elsewhere); on the GPU, the device table against
this restatement.
"""
import ctypes

import numpy as np
import pytest

import oracle as orc
from gpu_helpers import cuda_or_skip

BINS = 256
BASE = (127 - 16) << 3
ALPHA, M_E, C, HBAR = 0.0072973525643, 9.1093837139e-31, 299792458.0, 1.0545718176461565e-34
FACTOR = ((ALPHA * M_E) * (C * C)) / HBAR


def chi_bin(chi):
    """sfp_pair_bin: the float's exponent and 3 mantissa bits from 2^-16."""
    k = (np.asarray(chi, dtype=np.float32).view(np.uint32).astype(np.int64) >> 20) - BASE
    return np.clip(k, 0, BINS - 1)


def bin_upper(k):
    return float(np.uint32((k + BASE + 1) << 20).view(np.float32))


def bin_lower(k):
    return float(np.uint32((k + BASE) << 20).view(np.float32))


def bound_table(iA, dA, zmax):
    """k_pair_bound restated (float64, then rounded up to float32)."""
    zN = iA.size
    out = np.empty(BINS, dtype=np.float32)
    dz = zmax / (zN - 1)
    for k in range(BINS):
        if k == BINS - 1:
            out[k] = np.inf
            continue
        chi = bin_upper(k)
        zmin = (4.0 / chi) ** (2.0 / 3.0)
        if zmin * (1.0 - 1e-4) > zmax:
            out[k] = 0.0
            continue
        j0 = max(int(np.floor(zmin / dz)) - 1, 0)
        j = np.arange(j0, zN - 1)
        zl = np.maximum(j * dz, zmin * (1.0 - 1e-4))
        zr = (j + 1) * dz
        ia = np.maximum(iA[j], iA[j + 1])
        dpos = np.maximum(np.maximum(dA[j], dA[j + 1]), 0.0)
        dabs = np.maximum(np.abs(dA[j]), np.abs(dA[j + 1]))
        b = np.max(ia + np.where(dpos > 0, 2.0 / zl * dpos, 0.0) + chi * np.sqrt(zr) * dabs)
        v = np.float32(4.0 * FACTOR * b)
        if float(v) < 4.0 * FACTOR * b:
            v = np.nextafter(v, np.float32(np.inf))
        out[k] = v
    return out


@pytest.fixture(scope="module")
def rs():
    from sfparticles_b200.qed import tables
    iA, dA, zN, zmax = tables.rs_tables()
    return np.ascontiguousarray(iA, dtype=np.float64), np.ascontiguousarray(dA, dtype=np.float64), int(zN), float(zmax)


def test_bins_cover_chi_in_order():
    rng = np.random.default_rng(1)
    chi = np.exp(rng.uniform(np.log(1e-7), np.log(1e6), 20000)).astype(np.float32)
    k = chi_bin(chi)
    order = np.argsort(chi)
    assert np.all(np.diff(k[order]) >= 0)  # the bins follow chi
    inside = chi < 2.0 ** 16 * (1 - 1 / 16)
    assert all(chi[i] < bin_upper(k[i]) for i in np.flatnonzero(inside)[:2000])
    assert chi_bin(np.float32(1e-9)) == 0 and chi_bin(np.float32(1e9)) == BINS - 1


def test_the_bound_is_four_times_the_rate_or_more_over_every_delta(rs):
    iA, dA, zN, zmax = rs
    B = bound_table(iA, dA, zmax)
    L = orc.lib()
    deltas = np.concatenate([np.linspace(1e-4, 1 - 1e-4, 401), [0.5, 0.5 - 1e-9, 0.5 + 1e-9]])
    pi, pd = iA.ctypes.data_as(ctypes.c_void_p), dA.ctypes.data_as(ctypes.c_void_p)
    checked = 0
    for k in range(0, BINS - 1, 3):
        lo, hi = bin_lower(k), bin_upper(k)
        for chi in (lo, 0.5 * (lo + hi), float(np.nextafter(np.float32(hi), np.float32(0)))):
            rate = np.array([L.orc_pair_prob_rate_from_table(chi, d, pi, pd, zN, zmax) for d in deltas])
            assert np.all(4.0 * rate <= float(B[k])), (k, chi, float(B[k]), rate.max())
            if B[k] == 0.0:
                assert np.all(rate == 0.0)
            checked += 1
    assert checked > 200
    # the bound is not loose by orders of magnitude where pairs are likely
    k = int(chi_bin(np.float32(1.0)))
    rmax = max(L.orc_pair_prob_rate_from_table(bin_upper(k), 0.5, pi, pd, zN, zmax), 1e-300)
    assert float(B[k]) < 40 * rmax


@pytest.mark.gpu
def test_device_table_matches_the_restatement(rs):
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib
    iA, dA, zN, zmax = rs
    ti = torch.as_tensor(iA, device="cuda")
    td = torch.as_tensor(dA, device="cuda")
    out = torch.full((BINS,), -1.0, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.call("sfp_pair_rate_bound", ctypes.c_void_p(ti.data_ptr()), ctypes.c_void_p(td.data_ptr()), zN, zmax,
              ctypes.c_void_p(out.data_ptr()), st)
    got = out.cpu().numpy()
    ref = bound_table(iA, dA, zmax)
    assert np.array_equal(np.isinf(got), np.isinf(ref)) and np.array_equal(got == 0, ref == 0)
    fin = np.isfinite(ref) & (ref > 0)
    np.testing.assert_allclose(got[fin], ref[fin], rtol=5e-7)


def _host_bound(fields, tmp_path):
    """The generated sfp_field_bound(P), compiled for the host."""
    import subprocess
    src = fields.cuda_source()
    a = src.index("SFP_DEVICE_INLINE double sfp_field_bound")
    code = ("#include <cmath>\nusing std::fabs; using std::sqrt; using std::fmod;\n#define SFP_DEVICE_INLINE inline\n"
            + src[a:] + '\nextern "C" double bound(const double* P) { return sfp_field_bound(P); }\n')
    # a new file name per field: the loader would hand back an earlier library of the same path
    name = "b%d" % len(list(tmp_path.glob("b*.so")))
    (tmp_path / f"{name}.cpp").write_text(code)
    so = tmp_path / f"{name}.so"
    subprocess.check_call(["g++", "-O1", "-shared", "-fPIC", str(tmp_path / f"{name}.cpp"), "-o", str(so)])
    lib = ctypes.CDLL(str(so))
    lib.bound.restype = ctypes.c_double
    lib.bound.argtypes = [ctypes.c_void_p]
    p = np.ascontiguousarray(fields.params(), dtype=np.float64)
    return float(lib.bound(p.ctypes.data))


def test_field_bound_covers_the_fields(tmp_path):
    """The photon kernel skips the field evaluation of a photon whose energy
    alone bounds its chi below any pair test (chi <= gamma (|E| + c|B|)_max
    / E_s).  The generated bound must cover |E| + c|B| of the field at every
    point: checked against the oracle's fields over the pulse, its peak
    included, for a Gaussian pulse plus a static field and a simple pulse of
    even temporal order; a simple pulse of odd order gets no bound."""
    from sfparticles_b200 import fields as F
    rng = np.random.default_rng(5)
    ctau = C * 25e-15 / (2 * np.sqrt(np.log(2) / 2))
    cases = [
        (F.gaussian_laser_pulse(200.0, 3e-6, ctau, direction=-1, x0=0.0) + F.static_field(Ex=3e12, By=5e3),
         orc.gaussian_laser_pulse(200.0, 3e-6, ctau, direction=-1, x0=0.0) + orc.static_field(Ex=3e12, By=5e3)),
        (F.simple_laser_pulse(50.0, 2e-6, ctau, t_order=2, direction=1, x0=0.0),
         orc.simple_laser_pulse(50.0, 2e-6, ctau, t_order=2, direction=1, x0=0.0)),
    ]
    for prod, ref in cases:
        b = _host_bound(prod, tmp_path)
        assert 0.0 < b < 1e299
        worst = 0.0
        for t in (-20e-15, 0.0, 7e-15):
            n = 200_000
            # points around the pulse centre (x = x0 + dir c t), the focus and the axis
            x = rng.normal(0.0, 3e-6, n) + rng.choice([-1.0, 1.0], n) * C * t
            y, z = rng.normal(0.0, 1.5e-6, n), rng.normal(0.0, 1.5e-6, n)
            Ex, Ey, Ez, Bx, By, Bz = orc.field_eval(ref, x, y, z, t)
            m = np.sqrt(Ex ** 2 + Ey ** 2 + Ez ** 2) + C * np.sqrt(Bx ** 2 + By ** 2 + Bz ** 2)
            assert np.all(m <= b), (float(m.max()), b)
            worst = max(worst, float(m.max()))
        assert worst > 0.5 * b  # the pulse's peak was sampled: the bound is not loose by much
    odd = F.simple_laser_pulse(50.0, 2e-6, ctau, t_order=3)
    assert _host_bound(odd, tmp_path) >= 1e299
