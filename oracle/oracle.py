"""CPU oracle for the sfparticles per-particle step -- TEST INFRASTRUCTURE ONLY.

This module is the checker the CUDA path is compared against.  The product
package ``sfparticles_b200`` never imports it; only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` do.

It wraps ``liboracle.so`` (``oracle/sfp_oracle.c``, a C restatement of the
reference's Numba kernels with the same operation order) and restates the
reference's Python orchestration on top of it:

* preset parameter derivation: ``fields.py:69-271`` (``simple_laser_pulse``,
  ``gaussian_laser_pulse``, ``focused_gaussian_laser_pulse``, ``static_field``)
  and ``Fields.__add__`` (``fields.py:52-61``) as a postfix op list;
* species bookkeeping: ``particles.py:43-516`` (``_extend`` growth rule
  ``particles.py:487-500``, ``_create_photon`` ``:399-431``, ``_create_pair``
  ``:433-473``, ``_push_momentum`` ``:244-281`` / ``:575-604``, ``_prune``);
* the step loop: ``simulation.py:102-144``.

Conventions where the reference is undefined: appended slots start with zero
spin and zero optical depth (the reference copies stale values cyclically via
``numpy.resize``); random draws come from the keyed Philox stream shared with
the GPU instead of Numba's MT19937.  Optical-depth tables are passed in
(``make_od_table``); the tests pass the ones sfparticles_b200.qed.tables
ships, whose pair rows below chi_gamma ~ 0.43 are finite where the
reference's generator leaves them NaN.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# scipy.constants (CODATA 2022), identical to the reference's imports
C = 299792458.0
M_E = float.fromhex("0x1.279dcc922bcd9p-100")
E_CHARGE = float.fromhex("0x1.7a4da290c1653p-63")
HBAR = float.fromhex("0x1.185a7057c690dp-113")
EPS0 = float.fromhex("0x1.37876f1591150p-37")
PI = math.pi
ALPHA = float.fromhex("0x1.de3d429c6dc9dp-8")

TERM_PARAMS = 16
FIELD_STATIC, FIELD_SIMPLE, FIELD_GAUSSIAN, FIELD_FOCUSED = 0, 1, 2, 3

RR_NONE, RR_PHOTON, RR_LL, RR_CLL = 1, 2, 3, 4

_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with oracle/Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "sfp_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        d, i64, i32, u32, u64 = ctypes.c_double, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64
        P = ctypes.c_void_p
        L.orc_philox4x32_10.argtypes = [P, P, P]
        L.orc_uniform2.argtypes = [u64, u32, u32, u32, i64, P]
        L.orc_uniform2_batch.argtypes = [u64, u32, u32, u32, P, i64, P]
        L.orc_field_eval.argtypes = [P, i32, P, P, P, P, P, d, i64, P, P, P, P, P, P, P]
        L.orc_push_position.argtypes = [P] * 7 + [i64, P, d]
        L.orc_boris.argtypes = [P] * 10 + [d, i64, P, d]
        L.orc_boris_tbmt.argtypes = [P] * 13 + [d, d, i64, P, d]
        L.orc_LL_push.argtypes = [P] * 5 + [i64, P, d]
        L.orc_CLL_push.argtypes = [P] * 5 + [i64, P, d]
        L.orc_update_chi.argtypes = [P] * 11 + [i64, P]
        L.orc_photon_recoil.argtypes = [P] * 6 + [i64, P]
        L.orc_pick_hard_photon.argtypes = [P, P, P, d, i64]
        L.orc_bool_sum.argtypes = [P, i64]
        L.orc_bool_sum.restype = i64
        L.orc_find_event_index.argtypes = [P, i64, i64, P]
        L.orc_create_photon.argtypes = [P] * 16 + [i64, i64]
        L.orc_create_pair.argtypes = [P] * 17 + [i64, i64, i32]
        L.orc_photon_prob_rate_from_table.argtypes = [d, d, P, P, i32, d]
        L.orc_photon_prob_rate_from_table.restype = d
        L.orc_pair_prob_rate_from_table.argtypes = [d, d, P, P, i32, d]
        L.orc_pair_prob_rate_from_table.restype = d
        L.orc_photon_from_rejection_sampling.argtypes = [P, P, d, i64, P, P, P, P, P, i32, d, u64, u32, u32]
        L.orc_pair_from_rejection_sampling.argtypes = [P, P, d, i64, P, P, P, P, P, i32, d, u64, u32, u32]
        L.orc_od_interp1d.argtypes = [d, P]
        L.orc_od_interp1d.restype = d
        L.orc_od_bisect.argtypes = [d, d, P]
        L.orc_od_bisect.restype = d
        L.orc_od_bisect_batch.argtypes = [P, P, i64, P, P]
        L.orc_update_tau.argtypes = [P, P, P, d, i64, P, P, P, P, u64, u32, u32]
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


# --------------------------------------------------------------------------
# RNG
# --------------------------------------------------------------------------

def philox4x32_10(ctr: Sequence[int], key: Sequence[int]) -> List[int]:
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(_p(c), _p(k), _p(o))
    return [int(v) for v in o]


def uniform2(seed: int, stream: int, step: int, purpose: int, slots: np.ndarray) -> np.ndarray:
    """(len(slots), 2) uniforms in (0,1) for the keyed Philox stream."""
    s = np.ascontiguousarray(slots, dtype=np.int64)
    out = np.zeros((s.size, 2))
    lib().orc_uniform2_batch(seed & (2**64 - 1), stream, step & 0xFFFFFFFF, purpose, _p(s), s.size, _p(out))
    return out


# --------------------------------------------------------------------------
# Field presets: derived parameters restated from fields.py
# --------------------------------------------------------------------------

@dataclass
class FieldTerms:
    """Postfix program over preset terms (Fields.__add__ tree, fields.py:52-61)."""
    ops: List[int] = field(default_factory=list)
    kinds: List[int] = field(default_factory=list)
    params: List[List[float]] = field(default_factory=list)

    def __add__(self, other: "FieldTerms") -> "FieldTerms":
        n = len(self.kinds)
        ops = list(self.ops) + [o + n if o >= 0 else o for o in other.ops] + [-1]
        return FieldTerms(ops, self.kinds + other.kinds, self.params + other.params)

    def arrays(self):
        ops = np.asarray(self.ops, dtype=np.int32)
        kinds = np.asarray(self.kinds, dtype=np.int32)
        prm = np.zeros((max(1, len(self.params)), TERM_PARAMS))
        for i, p in enumerate(self.params):
            prm[i, : len(p)] = p
        return ops, kinds, prm


def _single(kind: int, p: List[float]) -> FieldTerms:
    return FieldTerms([0], [kind], [p])


def static_field(Ex=0, Ey=0, Ez=0, Bx=0, By=0, Bz=0) -> FieldTerms:
    """fields.py:268-271"""
    return _single(FIELD_STATIC, [float(Ex), float(Ey), float(Ez), float(Bx), float(By), float(Bz)])


def simple_laser_pulse(a0, w0, ctau, t_order=2, direction=1, x0=0, wavelength=0.8e-6, pol_angle=0, cep=0):
    """fields.py:69-118 (omega0, k0, a0_norm, E0 computed as in the closure setup)."""
    assert direction in (1, -1)
    omega0 = 2 * PI * C / wavelength
    k0 = omega0 / C
    a0_norm = E_CHARGE / (M_E * C * omega0)
    E0 = a0 / a0_norm
    is_int = isinstance(t_order, (int, np.integer))
    return _single(FIELD_SIMPLE, [E0, k0, float(w0), float(ctau), float(direction), float(x0), float(cep),
                                  math.cos(pol_angle), math.sin(pol_angle), float(t_order), 1.0 if is_int else 0.0])


def gaussian_laser_pulse(a0, w0, ctau, direction=1, x0=0.0, l0=0.8e-6, pol_angle=0.0, cep=0.0):
    """fields.py:120-170"""
    assert direction in (1, -1)
    omega0 = 2 * PI * C / l0
    k0 = 2 * PI / l0
    zR = PI * w0 ** 2 / l0
    a0_norm = E_CHARGE / (M_E * C * omega0)
    E0 = a0 / a0_norm
    return _single(FIELD_GAUSSIAN, [E0, k0, zR, float(w0), float(ctau), float(direction), float(x0), float(cep),
                                    math.cos(pol_angle), math.sin(pol_angle)])


def focused_gaussian_laser_pulse(a0, w0, ctau, direction=1, xfoc=0.0, x0=0.0, l0=0.8e-6, pol_angle=0.0, cep=0.0):
    """fields.py:173-265"""
    assert direction in (1, -1)
    omega0 = 2 * PI * C / l0
    k0 = 2 * PI / l0
    zR = PI * w0 ** 2 / l0
    eps = w0 / zR
    a0_norm = E_CHARGE / (M_E * C * omega0)
    E0 = a0 / a0_norm
    return _single(FIELD_FOCUSED, [E0, k0, zR, float(w0), float(ctau), float(direction), float(xfoc), float(x0),
                                   float(cep), math.cos(pol_angle), math.sin(pol_angle), eps])


def field_eval(terms: FieldTerms, x, y, z, t, to_be_pruned=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.float64)
    n = x.size
    pr = np.zeros(n, dtype=np.uint8) if to_be_pruned is None else np.ascontiguousarray(to_be_pruned, dtype=np.uint8)
    out = [np.zeros(n) for _ in range(6)]
    ops, kinds, prm = terms.arrays()
    lib().orc_field_eval(_p(ops), ops.size, _p(kinds), _p(prm), _p(x), _p(y), _p(z), float(t), n, _p(pr),
                         *[_p(o) for o in out])
    return tuple(out)


# --------------------------------------------------------------------------
# QED tables
# --------------------------------------------------------------------------

class ODTable(ctypes.Structure):
    _fields_ = [
        ("chi_N", ctypes.c_int32), ("delta_N", ctypes.c_int32),
        ("log_chi_min", ctypes.c_double), ("log_chi_delta", ctypes.c_double),
        ("log_delta_min", ctypes.c_double), ("log_delta_delta", ctypes.c_double),
        ("log_chi_max", ctypes.c_double),
        ("rate_total", ctypes.c_void_p), ("cumulative", ctypes.c_void_p),
    ]


def make_od_table(rate_total: np.ndarray, cumulative: np.ndarray, log_chi_min: float, log_chi_delta: float,
                  log_delta_min: float, log_delta_delta: float):
    rate_total = np.ascontiguousarray(rate_total, dtype=np.float64)
    cumulative = np.ascontiguousarray(cumulative, dtype=np.float64)
    t = ODTable(rate_total.size, cumulative.shape[1], log_chi_min, log_chi_delta, log_delta_min, log_delta_delta,
                log_chi_min + (rate_total.size - 1) * log_chi_delta, _p(rate_total), _p(cumulative))
    t._keep = (rate_total, cumulative)
    return t


# --------------------------------------------------------------------------
# Species and step loop (particles.py / simulation.py restated)
# --------------------------------------------------------------------------

class Species:
    """particles.py:43-146 state; arrays are float64 SoA of length buffer_size."""

    def __init__(self, name, q, m, N=0, props=None, RR=RR_PHOTON, push=True, spin=False, ae=1.14e-3, spin_props=None):
        self.name = name
        self.q = q * E_CHARGE
        self.m = m * M_E
        self.massless = m == 0
        self.RR = RR
        self.push = push
        self.spin = spin
        self.ae = ae
        self.radiating = False
        self.bw = False
        self.photon = None
        self.electron = None
        self.positron = None
        N = int(N)
        if props is None:
            props = [np.zeros(N) for _ in range(6)]
        self.x, self.y, self.z, self.ux, self.uy, self.uz = [np.array(p, dtype=np.float64) for p in props]
        if m > 0:
            self.inv_gamma = 1.0 / np.sqrt(1 + self.ux ** 2 + self.uy ** 2 + self.uz ** 2)
        else:
            self.inv_gamma = 1.0 / np.sqrt(self.ux ** 2 + self.uy ** 2 + self.uz ** 2)
        self.attrs = ["x", "y", "z", "ux", "uy", "uz", "inv_gamma", "chi", "Ex", "Ey", "Ez", "Bx", "By", "Bz",
                      "to_be_pruned"]
        self.chi = np.zeros(N)
        for a in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
            setattr(self, a, np.zeros(N))
        self.to_be_pruned = np.zeros(N, dtype=np.uint8)
        if spin:
            if spin_props is None:
                spin_props = [np.zeros(N) for _ in range(3)]
            self.sx, self.sy, self.sz = [np.array(p, dtype=np.float64) for p in spin_props]
            self.attrs += ["sx", "sy", "sz"]
        self.N_buffered = N
        self.buffer_size = N
        self.od = False

    def set_photon(self, photon: "Species", od=False):
        assert not self.massless and self.RR not in (RR_LL, RR_CLL)
        self.radiating = True
        self.photon = photon
        self.event = np.zeros(self.buffer_size, dtype=np.uint8)
        self.delta = np.zeros(self.buffer_size)
        self.attrs += ["event", "delta"]
        if od:
            self.od = True
            self.tau = np.zeros(self.buffer_size)
            self.attrs += ["tau"]

    def set_pair(self, electron: "Species", positron: "Species", od=False):
        assert self.massless
        self.bw = True
        self.electron = electron
        self.positron = positron
        self.event = np.zeros(self.buffer_size, dtype=np.uint8)
        self.delta = np.zeros(self.buffer_size)
        self.attrs += ["event", "delta"]
        if od:
            self.od = True
            self.tau = np.zeros(self.buffer_size)
            self.attrs += ["tau"]

    def extend(self, N_new: int):
        """particles.py:476-500; tails are zero-filled (see module docstring)."""
        if (self.buffer_size - self.N_buffered) < N_new:
            new = self.buffer_size + int(self.N_buffered / 4) + N_new
            for a in self.attrs:
                old = getattr(self, a)
                arr = np.zeros(new, dtype=old.dtype)
                arr[: old.size] = old
                setattr(self, a, arr)
            self.to_be_pruned[self.buffer_size:] = 1
            self.buffer_size = new

    def npart(self) -> int:
        return self.N_buffered - int(lib().orc_bool_sum(_p(self.to_be_pruned), self.N_buffered))

    def prune(self):
        sel = self.to_be_pruned[: self.N_buffered] == 0
        for a in self.attrs:
            setattr(self, a, getattr(self, a)[: self.N_buffered][sel].copy())
        self.N_buffered = self.buffer_size = int(sel.sum())

    # -- kernels --------------------------------------------------------
    def eval_field(self, terms: FieldTerms, t: float):
        ops, kinds, prm = terms.arrays()
        lib().orc_field_eval(_p(ops), ops.size, _p(kinds), _p(prm), _p(self.x), _p(self.y), _p(self.z), float(t),
                             self.N_buffered, _p(self.to_be_pruned), _p(self.Ex), _p(self.Ey), _p(self.Ez),
                             _p(self.Bx), _p(self.By), _p(self.Bz))

    def calc_chi(self):
        lib().orc_update_chi(_p(self.Ex), _p(self.Ey), _p(self.Ez), _p(self.Bx), _p(self.By), _p(self.Bz),
                             _p(self.ux), _p(self.uy), _p(self.uz), _p(self.inv_gamma), _p(self.chi),
                             self.N_buffered, _p(self.to_be_pruned))

    def push_position(self, dt):
        lib().orc_push_position(_p(self.x), _p(self.y), _p(self.z), _p(self.ux), _p(self.uy), _p(self.uz),
                                _p(self.inv_gamma), self.N_buffered, _p(self.to_be_pruned), dt)

    def push_momentum(self, dt):
        """particles.py:244-281 (Particles) and :575-604 (SpinParticles)."""
        if self.massless:
            return
        if self.spin:
            lib().orc_boris_tbmt(_p(self.ux), _p(self.uy), _p(self.uz), _p(self.inv_gamma), _p(self.sx),
                                 _p(self.sy), _p(self.sz), _p(self.Ex), _p(self.Ey), _p(self.Ez), _p(self.Bx),
                                 _p(self.By), _p(self.Bz), self.q, self.ae, self.N_buffered,
                                 _p(self.to_be_pruned), dt)
        else:
            lib().orc_boris(_p(self.ux), _p(self.uy), _p(self.uz), _p(self.inv_gamma), _p(self.Ex), _p(self.Ey),
                            _p(self.Ez), _p(self.Bx), _p(self.By), _p(self.Bz), self.q, self.N_buffered,
                            _p(self.to_be_pruned), dt)
        if self.RR == RR_LL:
            self.calc_chi()
            lib().orc_LL_push(_p(self.ux), _p(self.uy), _p(self.uz), _p(self.inv_gamma), _p(self.chi),
                              self.N_buffered, _p(self.to_be_pruned), dt)
        if self.RR == RR_CLL and not self.spin:
            self.calc_chi()
            lib().orc_CLL_push(_p(self.ux), _p(self.uy), _p(self.uz), _p(self.inv_gamma), _p(self.chi),
                               self.N_buffered, _p(self.to_be_pruned), dt)


class OracleSim:
    """simulation.py:12-160 restated over the C kernels.

    ``qed`` is ("rs", int_Ai, Aip) or ("od", photon_table, pair_table).
    RNG: key = seed, counter = (slot, purpose, step, stream = species index).
    """

    def __init__(self, species: List[Species], dt: float, terms: FieldTerms, qed, seed: int = 0,
                 t0: float = 0.0, photon_threshold: float = 2.0, z_max: float = 100.0):
        self.all = species
        self.dt = dt
        self.terms = terms
        self.qed = qed
        self.seed = seed
        self.t = t0
        self.step = 0
        self.thr = photon_threshold
        self.z_max = z_max
        self.push_list = [p for p in species if p.push]
        self.bw_list = [p for p in species if p.bw]
        self.rad_list = [p for p in species if p.radiating]
        self.particle_steps = 0

    def _stream(self, p):
        return self.all.index(p)

    def _events(self, p, photon: bool):
        L = lib()
        kind = self.qed[0]
        stream = self._stream(p)
        if kind == "rs":
            iA, dA = self.qed[1], self.qed[2]
            fn = L.orc_photon_from_rejection_sampling if photon else L.orc_pair_from_rejection_sampling
            fn(_p(p.inv_gamma), _p(p.chi), self.dt, p.N_buffered, _p(p.to_be_pruned), _p(p.event), _p(p.delta),
               _p(iA), _p(dA), iA.size, self.z_max, self.seed, stream, self.step)
        else:
            tab = self.qed[1] if photon else self.qed[2]
            L.orc_update_tau(_p(p.tau), _p(p.inv_gamma), _p(p.chi), self.dt, p.N_buffered, _p(p.to_be_pruned),
                             _p(p.event), _p(p.delta), ctypes.byref(tab), self.seed, stream, self.step)

    def _create_photon(self, p):
        L = lib()
        n = int(L.orc_bool_sum(_p(p.event), p.N_buffered))
        if n == 0:
            return
        pho = p.photon
        idx = np.zeros(n, dtype=np.int64)
        L.orc_find_event_index(_p(p.event), n, p.N_buffered, _p(idx))
        pho.extend(n)
        L.orc_create_photon(_p(p.x), _p(p.y), _p(p.z), _p(p.ux), _p(p.uy), _p(p.uz), _p(pho.x), _p(pho.y),
                            _p(pho.z), _p(pho.ux), _p(pho.uy), _p(pho.uz), _p(pho.inv_gamma),
                            _p(pho.to_be_pruned), _p(idx), _p(p.delta), pho.N_buffered, n)
        pho.N_buffered += n
        if p.RR == RR_PHOTON:
            L.orc_photon_recoil(_p(p.ux), _p(p.uy), _p(p.uz), _p(p.inv_gamma), _p(p.event), _p(p.delta),
                                p.N_buffered, _p(p.to_be_pruned))

    def _create_pair(self, p):
        L = lib()
        n = int(L.orc_bool_sum(_p(p.event), p.N_buffered))
        if n == 0:
            return
        ele, pos = p.electron, p.positron
        idx = np.zeros(n, dtype=np.int64)
        L.orc_find_event_index(_p(p.event), n, p.N_buffered, _p(idx))
        ele.extend(n)
        pos.extend(n)
        for dst, inv in ((ele, 0), (pos, 1)):
            L.orc_create_pair(_p(p.x), _p(p.y), _p(p.z), _p(p.ux), _p(p.uy), _p(p.uz), _p(p.to_be_pruned),
                              _p(dst.x), _p(dst.y), _p(dst.z), _p(dst.ux), _p(dst.uy), _p(dst.uz),
                              _p(dst.inv_gamma), _p(dst.to_be_pruned), _p(idx), _p(p.delta), dst.N_buffered, n, inv)
        ele.N_buffered += n
        pos.N_buffered += n

    def run(self, nstep: int):
        L = lib()
        for _ in range(nstep):
            self.particle_steps += sum(p.N_buffered for p in self.all)
            for p in self.push_list:
                p.eval_field(self.terms, self.t)
            for p in self.bw_list:
                p.calc_chi()
                self._events(p, photon=False)
            for p in self.rad_list:
                p.calc_chi()
                self._events(p, photon=True)
                L.orc_pick_hard_photon(_p(p.event), _p(p.delta), _p(p.inv_gamma), self.thr, p.N_buffered)
            for p in self.rad_list:
                self._create_photon(p)
            for p in self.bw_list:
                self._create_pair(p)
            for p in self.push_list:
                p.push_position(0.5 * self.dt)
                p.eval_field(self.terms, self.t + 0.5 * self.dt)
                p.push_momentum(self.dt)
                p.push_position(0.5 * self.dt)
            self.t += self.dt
            self.step += 1
