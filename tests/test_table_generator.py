"""The QED table generator's mathematics on the CPU: the package's Airy
functions (csrc/sfp_airy.h), its restatement of QUADPACK's QAGS / QAGI
(csrc/sfp_quadpack.h) and the rate functor (csrc/sfp_table_math.h) --
the code the GPU generator runs (csrc/sfp_tables.cu) -- compiled for the
host with g++, against
* scipy.integrate.quad run on the same integrand (a C function handed to
  quad as a LowLevelCallable): bit for bit, which pins the restatement of
  the reference's integrator;
* mpmath's Airy functions (1e-13 relative, 2e-13 where exp(-(2/3) z^1.5)
  carries the rounding of its argument);
* the reference's own table entries (tests/golden/ref_tables.npz: the
  shipped rejection-sampling table; ref_od.npz: 18 optical-depth rows from
  the reference's generator): 1e-12 relative on every entry above 1e-250
  (rates in 1/s; below, the reference's scipy flushes Airy values to 0).
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import golden

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sfparticles_b200", "csrc")
SRC = r'''
#include "sfp_table_math.h"
extern "C" double ai_c(double x) { return sfp_airy::Ai(x); }
extern "C" void airy_c(double z, double* ai, double* aip) { sfp_airy::airy(z, *ai, *aip); }
extern "C" double int_ai_c(double z) { return sfp_quad::quad_inf(sfp_tab::AiFn{}, z); }
static double g_chi = 1.0, g_factor = 1.0;
static int g_kind = 0;
extern "C" void set_rate(int kind, double factor, double chi) { g_kind = kind; g_factor = factor; g_chi = chi; }
extern "C" double rate_c(double d) { return sfp_tab::RateFn{g_chi, g_factor, g_kind}(d); }
extern "C" double quad_rate_c(double a, double b) { return sfp_quad::quad(sfp_tab::RateFn{g_chi, g_factor, g_kind}, a, b); }
extern "C" void rs_rows(const double* z, long n, double* ia, double* aip) {
    for (long i = 0; i < n; ++i) sfp_tab::airy_terms(z[i], ia[i], aip[i]);
}
extern "C" void od_row(int kind, double factor, double chi, const double* delta, long n, double* total, double* cum) {
    const sfp_tab::RateFn P{chi, factor, kind};
    *total = sfp_quad::quad(P, 0.0, 1.0);
    double acc = sfp_quad::quad(P, 0.0, delta[0]);
    cum[0] = acc;
    for (long i = 1; i < n; ++i) { acc = acc + P(delta[i]) * (delta[i] - delta[i - 1]); cum[i] = acc; }
}
'''
D = ctypes.c_double
DP = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def lib():
    with tempfile.TemporaryDirectory() as d:
        cpp, so = os.path.join(d, "t.cpp"), os.path.join(d, "t.so")
        with open(cpp, "w") as f:
            f.write(SRC)
        subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC", f"-I{CSRC}", "-o", so,
                        cpp], check=True, capture_output=True)
        L = ctypes.CDLL(so)
        for nm in ("ai_c", "int_ai_c", "rate_c"):
            getattr(L, nm).restype, getattr(L, nm).argtypes = D, [D]
        L.quad_rate_c.restype, L.quad_rate_c.argtypes = D, [D, D]
        L.set_rate.argtypes = [ctypes.c_int, D, D]
        L.airy_c.argtypes = [D, DP, DP]
        L.od_row.argtypes = [ctypes.c_int, D, D, DP, ctypes.c_long, DP, DP]
        yield L


def _cb(L, name):
    from scipy import LowLevelCallable
    return LowLevelCallable(ctypes.cast(getattr(L, name), ctypes.CFUNCTYPE(D, D)))


def test_quadrature_is_scipys_quad_bit_for_bit(lib):
    from scipy.integrate import quad
    from sfparticles_b200.qed import tables as T
    ai = _cb(lib, "ai_c")
    for z in np.linspace(0.0, 100.0, 257):  # QAGI
        assert quad(ai, z, np.inf)[0] == lib.int_ai_c(z), z
    rate = _cb(lib, "rate_c")
    for kind, factor in ((0, T.photon_factor()), (1, T.pair_factor())):  # QAGS, nested over QAGI
        for chi in np.logspace(-3, 3, 13):
            lib.set_rate(kind, factor, chi)
            for a, b in ((0.0, 1.0), (0.0, 1e-6), (0.2, 0.7)):
                assert quad(rate, a, b)[0] == lib.quad_rate_c(a, b), (kind, chi, a, b)


def test_airy_functions_against_mpmath(lib):
    import mpmath as mp
    mp.mp.dps = 40
    a, d = D(), D()
    for z in np.concatenate([np.linspace(0.0, 2.0, 41), np.linspace(2.0001, 100.0, 120)]):
        lib.airy_c(z, ctypes.byref(a), ctypes.byref(d))
        ea, ed = float(mp.airyai(z)), float(mp.airyai(z, derivative=1))
        tol = 1e-13 if z < 50 else 2e-13
        assert abs(a.value - ea) <= tol * abs(ea) and abs(d.value - ed) <= tol * abs(ed), z
    lib.airy_c(108.0, ctypes.byref(a), ctypes.byref(d))
    assert a.value == 0.0 and d.value == 0.0


def _rel_above_floor(got, ref, floor=1e-250):
    got, ref = np.asarray(got, float), np.asarray(ref, float)
    big = np.abs(ref) > floor
    assert np.all(np.abs(got[~big]) <= floor), "an entry the reference flushes to zero is not negligible"
    return float(np.max(np.abs(got[big] - ref[big]) / np.abs(ref[big]))) if big.any() else 0.0


def test_rejection_sampling_table_matches_the_reference(lib):
    g = golden("ref_tables.npz")
    z = np.linspace(0.0, float(g["z_range"][1]), int(g["z_N"]))
    ia, dA = np.zeros(z.size), np.zeros(z.size)
    lib.rs_rows(z.ctypes.data_as(DP), ctypes.c_long(z.size), ia.ctypes.data_as(DP), dA.ctypes.data_as(DP))
    assert _rel_above_floor(ia, g["int_Ai"]) < 1e-12
    assert _rel_above_floor(dA, g["Aip"]) < 1e-12


def test_optical_depth_rows_match_the_reference(lib):
    from sfparticles_b200.qed import tables as T
    o = golden("ref_od.npz")
    delta = np.logspace(float(o["log_delta_min"]), 0, 1024)
    tot, cum = np.zeros(1), np.zeros(1024)
    n_pair_rows = 0
    for j, chi in enumerate(o["chi_rows"]):
        lib.od_row(0, T.photon_factor(), chi, delta.ctypes.data_as(DP), 1024, tot.ctypes.data_as(DP),
                   cum.ctypes.data_as(DP))
        assert _rel_above_floor(tot, o["photon_total"][j:j + 1]) < 1e-12, chi
        assert _rel_above_floor(cum, o["photon_cum"][j]) < 1e-12, chi
        lib.od_row(1, T.pair_factor(), chi, delta.ctypes.data_as(DP), 1024, tot.ctypes.data_as(DP),
                   cum.ctypes.data_as(DP))
        assert _rel_above_floor(tot, o["pair_total"][j:j + 1]) < 1e-12, chi
        ref = o["pair_cum"][j]
        if np.isfinite(ref).all():  # the reference's rows below chi ~ 0.43 are NaN
            assert _rel_above_floor(cum, ref) < 1e-12, chi
            n_pair_rows += 1
        assert np.isfinite(cum).all()
    assert n_pair_rows >= 5
