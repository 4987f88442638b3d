"""QED rate tables: generation and loading.

Generation runs either on the GPU (generate_on_gpu: libsfp's own QUADPACK
restatement and Airy functions, no scipy) or on the CPU with scipy at build
time (rs_table_gen / od_table_gen); the two agree to ~1e-13.

Two table families, as in the reference:

* rejection sampling (qed/rejection_sampling_tables.py:14-26, 91-112):
  on z = linspace(0, 100, 1024): int_Ai(z) = integral_z^inf Ai(t) dt and Ai'(z);
* optical depth (qed/optical_depth_tables.py:136-233): on log10 chi rows the
  total rates W(chi) = integral_0^1 dW/ddelta ddelta (photon emission and pair
  creation, 1/s) and the cumulative rates integral_0^delta_j dW/ddelta on
  1024 log-spaced delta columns from 1e-6 to 1.

The differential rates are the nonlinear-Compton / Breit-Wheeler LCFA forms
in Airy functions used by the reference (optical_depth_tables.py:246-268):

  dW_gamma/ddelta = -alpha m c^2/hbar [Ai_1(z) + (2/z + chi_gamma sqrt z) Ai'(z)],
  z = (chi_gamma / (chi_e chi_e'))^(2/3), chi_gamma = delta chi_e, chi_e' = chi_e - chi_gamma;
  dW_pair/ddelta  =  alpha m c^2/hbar [Ai_1(z) + (2/z - chi_gamma sqrt z) Ai'(z)],
  z = (chi_gamma / (chi_e chi_e'))^(2/3), chi_e = delta chi_gamma.

The optical-depth rows reproduce the reference grid (256 rows over log10 chi
in [-3, 2]) and extend it with the same spacing up to log10 chi = 3
(307 rows), so that chi > 100 is tabulated instead of read past the end.
Cumulative columns: first entry by quadrature from 0, then the reference's
left-Riemann accumulation integ[i] = integ[i-1] + P(delta_i)(delta_i - delta_{i-1}).

One deliberate difference: Ai, Ai' and integral Ai are taken as exactly 0
from z = 108 on (AIRY_ZERO_Z), where their float64 values are 0.  The
reference evaluates them there with scipy, which returns NaN for z ~ 1e8 and
above; that leaves its cumulative pair rows for chi_gamma below ~0.43 all NaN
and its optical-depth pair creation there with a NaN energy fraction.  Every
finite entry of the reference's tables is unchanged.
"""
from __future__ import annotations

import os
import time

import numpy as np

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
RS_FILE = os.path.join(DATA, "rs_tables.npz")
OD_FILE = os.path.join(DATA, "od_tables.npz")

# scipy.constants (CODATA 2022)
_C = 299792458.0
_ME = float.fromhex("0x1.279dcc922bcd9p-100")
_HBAR = float.fromhex("0x1.185a7057c690dp-113")
_ALPHA = float.fromhex("0x1.de3d429c6dc9dp-8")

RS_Z_N = 1024
RS_Z_MAX = 100.0

OD_LOG_CHI_MIN = -3.0
OD_LOG_CHI_MAX_REF = 2.0
OD_CHI_N_REF = 256
OD_LOG_CHI_MAX = 3.0
OD_DELTA_N = 1024
OD_LOG_DELTA_MIN = -6.0


def _Ai(z):
    from scipy.special import airy
    return airy(z)[0]


def _Aip(z):
    from scipy.special import airy
    return airy(z)[1]


def int_Ai(z: float) -> float:
    """integral_z^inf Ai(t) dt by adaptive quadrature."""
    from scipy.integrate import quad
    return quad(_Ai, z, np.inf)[0]


# Ai(z), Ai'(z) and integral_z^inf Ai are all below half the smallest float64
# subnormal from z = 108 on (Ai(z) ~ exp(-(2/3) z^1.5) / (2 sqrt(pi) z^0.25),
# exp(-(2/3) 108^1.5) = 1e-325), so all three are exactly 0.0 in float64
# there.  scipy's airy returns NaN from z ~ 1e8 on, which the rates reach at
# delta -> 0 (pair creation for chi_gamma below ~0.43): the reference's
# generator (optical_depth_tables.py:126-187) keeps those NaNs, and every
# cumulative pair row below chi_gamma ~ 0.43 comes out NaN.
AIRY_ZERO_Z = 108.0


def _airy_terms(z: float):
    """(integral_z^inf Ai, Ai'(z)), exactly 0 from AIRY_ZERO_Z on."""
    if z >= AIRY_ZERO_Z:
        return 0.0, 0.0
    return int_Ai(z), _Aip(z)


def photon_rate_delta(chi_e: float, delta: float) -> float:
    """dW_gamma/ddelta [1/s] at photon energy fraction delta."""
    if delta == 1.0:
        return 0.0
    factor = -_ALPHA * _ME * _C ** 2 / _HBAR
    chi_gamma = delta * chi_e
    chi_ep = chi_e - chi_gamma
    z = (chi_gamma / chi_e / chi_ep) ** (2 / 3)
    iA, dA = _airy_terms(z)
    return factor * (iA + (2.0 / z + chi_gamma * np.sqrt(z)) * dA)


def pair_rate_delta(chi_gamma: float, delta: float) -> float:
    """dW_pair/ddelta [1/s] at electron energy fraction delta."""
    if delta == 1.0:
        return 0.0
    factor = _ALPHA * _ME * _C ** 2 / _HBAR
    chi_e = delta * chi_gamma
    chi_ep = chi_gamma - chi_e
    z = (chi_gamma / chi_e / chi_ep) ** (2 / 3)
    iA, dA = _airy_terms(z)
    return factor * (iA + (2.0 / z - chi_gamma * np.sqrt(z)) * dA)


def photon_rate_total(chi_e: float) -> float:
    from scipy.integrate import quad
    return quad(lambda d: photon_rate_delta(chi_e, d), 0, 1)[0]


def pair_rate_total(chi_gamma: float) -> float:
    from scipy.integrate import quad
    return quad(lambda d: pair_rate_delta(chi_gamma, d), 0, 1)[0]


def _cumulative(rate_fn, chi: float, delta_N: int, log_delta_min: float) -> np.ndarray:
    from scipy.integrate import quad
    delta = np.logspace(log_delta_min, 0, delta_N)
    out = np.zeros(delta_N)
    out[0] = quad(lambda d: rate_fn(chi, d), 0, delta[0])[0]
    for i in range(1, delta_N):
        out[i] = out[i - 1] + rate_fn(chi, delta[i]) * (delta[i] - delta[i - 1])
    return out


def photon_cumulative(chi_e, delta_N=OD_DELTA_N, log_delta_min=OD_LOG_DELTA_MIN):
    return _cumulative(photon_rate_delta, chi_e, delta_N, log_delta_min)


def pair_cumulative(chi_gamma, delta_N=OD_DELTA_N, log_delta_min=OD_LOG_DELTA_MIN):
    return _cumulative(pair_rate_delta, chi_gamma, delta_N, log_delta_min)


def rs_table_gen(z_N: int = RS_Z_N, z_max: float = RS_Z_MAX, processes: int | None = None):
    z = np.linspace(0.0, z_max, z_N)
    iA = np.array(_pmap(int_Ai, list(z), processes))
    dA = _Aip(z)
    return iA, dA


def od_chi_rows():
    """log10 chi rows: the reference grid np.logspace(-3, 2, 256) extended
    with the same spacing to log10 chi = 3."""
    step = (OD_LOG_CHI_MAX_REF - OD_LOG_CHI_MIN) / (OD_CHI_N_REF - 1)
    n_ext = int(round((OD_LOG_CHI_MAX - OD_LOG_CHI_MAX_REF) / step))
    base = np.logspace(OD_LOG_CHI_MIN, OD_LOG_CHI_MAX_REF, OD_CHI_N_REF)
    ext = 10.0 ** (OD_LOG_CHI_MIN + step * np.arange(OD_CHI_N_REF, OD_CHI_N_REF + n_ext))
    return np.concatenate([base, ext]), step


def od_table_gen(processes: int | None = None, verbose: bool = False):
    chi, step = od_chi_rows()
    t0 = time.time()
    ph_tot = np.array(_pmap(photon_rate_total, list(chi), processes))
    pa_tot = np.array(_pmap(pair_rate_total, list(chi), processes))
    if verbose:
        print(f"  od totals: {time.time() - t0:.1f}s", flush=True)
    ph_cum = np.stack(_pmap(photon_cumulative, list(chi), processes))
    pa_cum = np.stack(_pmap(pair_cumulative, list(chi), processes))
    if verbose:
        print(f"  od cumulative: {time.time() - t0:.1f}s", flush=True)
    return dict(photon_rate_total=ph_tot, pair_rate_total=pa_tot, photon_cumulative=ph_cum,
                pair_cumulative=pa_cum, log_chi_min=OD_LOG_CHI_MIN, log_chi_delta=step,
                log_delta_min=OD_LOG_DELTA_MIN, log_delta_delta=(0 - OD_LOG_DELTA_MIN) / (OD_DELTA_N - 1),
                chi=chi)


def _pmap(fn, items, processes=None):
    n = processes if processes is not None else (os.cpu_count() or 1)
    if n <= 1 or len(items) < 8:
        return [fn(v) for v in items]
    import multiprocessing as mp
    ctx = mp.get_context("spawn")  # never fork a process that may hold a CUDA context
    with ctx.Pool(n) as pool:
        return pool.map(fn, items, chunksize=max(1, len(items) // (4 * n)))


def photon_factor() -> float:
    """-alpha m c^2 / hbar, evaluated as the reference writes it."""
    return -_ALPHA * _ME * _C ** 2 / _HBAR


def pair_factor() -> float:
    return _ALPHA * _ME * _C ** 2 / _HBAR


def generate_on_gpu(z_N: int = RS_Z_N, z_max: float = RS_Z_MAX, delta_N: int = OD_DELTA_N,
                    log_delta_min: float = OD_LOG_DELTA_MIN, chi=None):
    """Both table families computed on the GPU by libsfp (sfp_table_rs,
    sfp_table_od: QUADPACK's QAGS / QAGI as scipy runs them, with the
    package's own Airy functions), without scipy.  Grids as the reference
    builds them (numpy linspace / logspace); `chi` defaults to the product's
    307 optical-depth rows.  Returns (rs dict, od dict) with the keys of
    rs_tables' file and od_table_gen."""
    import ctypes
    import torch
    from .. import _lib
    from ..particles import _device, _stream_ptr
    dev = _device()

    def p(t):
        return ctypes.c_void_p(t.data_ptr())

    z = torch.as_tensor(np.linspace(0.0, z_max, z_N), device=dev)
    ia = torch.empty_like(z)
    dA = torch.empty_like(z)
    _lib.call("sfp_table_rs", p(z), z_N, p(ia), p(dA), _stream_ptr())
    if chi is None:
        chi, step = od_chi_rows()
    else:
        step = (OD_LOG_CHI_MAX_REF - OD_LOG_CHI_MIN) / (OD_CHI_N_REF - 1)
    chi_d = torch.as_tensor(np.asarray(chi, dtype=np.float64), device=dev)
    delta = torch.as_tensor(np.logspace(log_delta_min, 0, delta_N), device=dev)
    n = chi_d.numel()
    out = {}
    for kind, name, factor in ((0, "photon", photon_factor()), (1, "pair", pair_factor())):
        tot = torch.empty(n, dtype=torch.float64, device=dev)
        cum = torch.empty((n, delta_N), dtype=torch.float64, device=dev)
        first = torch.empty(n, dtype=torch.float64, device=dev)
        _lib.call("sfp_table_od", kind, factor, p(chi_d), n, p(delta), delta_N, p(tot), p(cum), p(first),
                  _stream_ptr())
        out[f"{name}_rate_total"] = tot.cpu().numpy()
        out[f"{name}_cumulative"] = cum.cpu().numpy()
    rs = dict(int_Ai=ia.cpu().numpy(), Aip=dA.cpu().numpy(), z_N=z_N, z_max=z_max)
    od = dict(out, log_chi_min=OD_LOG_CHI_MIN, log_chi_delta=step, log_delta_min=log_delta_min,
              log_delta_delta=(0 - log_delta_min) / (delta_N - 1), chi=np.asarray(chi, dtype=np.float64))
    return rs, od


def ensure_tables(verbose: bool = False):
    os.makedirs(DATA, exist_ok=True)
    if not os.path.exists(RS_FILE):
        t = time.time()
        iA, dA = rs_table_gen()
        np.savez(RS_FILE, int_Ai=iA, Aip=dA, z_N=RS_Z_N, z_max=RS_Z_MAX)
        if verbose:
            print(f"rejection-sampling tables: {time.time() - t:.1f}s", flush=True)
    if not os.path.exists(OD_FILE):
        t = time.time()
        tab = od_table_gen(verbose=verbose)
        np.savez_compressed(OD_FILE, **tab)
        if verbose:
            print(f"optical-depth tables: {time.time() - t:.1f}s", flush=True)


_cache = {}


def rs_tables():
    """(int_Ai, Aip, z_N, z_max) of the rejection-sampling method."""
    if "rs" not in _cache:
        if not os.path.exists(RS_FILE):
            ensure_tables()
        d = np.load(RS_FILE)
        _cache["rs"] = (np.ascontiguousarray(d["int_Ai"]), np.ascontiguousarray(d["Aip"]), int(d["z_N"]),
                        float(d["z_max"]))
    return _cache["rs"]


def od_tables():
    """dict of the optical-depth tables (see od_table_gen)."""
    if "od" not in _cache:
        if not os.path.exists(OD_FILE):
            ensure_tables()
        d = np.load(OD_FILE)
        _cache["od"] = {k: d[k] for k in d.files}
    return _cache["od"]
