"""Analytic electromagnetic fields, compiled into the particle push.

Mirrors sfparticles/fields.py: ``Fields(field_func)`` wraps a callable
``(x, y, z, t) -> (Ex, Ey, Ez, Bx, By, Bz)`` (SI units), ``Fields.__add__``
sums two fields componentwise (fields.py:52-61), and the presets
``simple_laser_pulse`` (fields.py:69-118), ``gaussian_laser_pulse``
(fields.py:120-170), ``focused_gaussian_laser_pulse`` (fields.py:173-265) and
``static_field`` (fields.py:268-271) keep their signatures.

Where the reference JIT-compiles the callable with Numba (fields.py:26-50),
here a Fields object is a *program*: a tree of terms whose structure becomes
CUDA C++ (``sfp_field_program``) compiled by NVRTC into the step kernel, and
whose numeric parameters live in a small device array.  Presets are built-in
device functions (sfparticles_b200/csrc/sfp_device.cuh); a user callable is
translated from its Python source (``sfparticles_b200.translate``).
"""
from __future__ import annotations

import hashlib
import math
from typing import Callable, List, Optional

import numpy as np

from .constants import C, E_CHARGE, M_E, PI

KIND_STATIC, KIND_SIMPLE, KIND_GAUSSIAN, KIND_FOCUSED, KIND_USER = "static", "simple", "gaussian", "focused", "user"
_DEVICE_FN = {KIND_STATIC: "sfp::field_static", KIND_SIMPLE: "sfp::field_simple",
              KIND_GAUSSIAN: "sfp::field_gaussian", KIND_FOCUSED: "sfp::field_focused"}
_DEVICE_FN32 = {KIND_STATIC: "sfp32::field_static", KIND_SIMPLE: "sfp32::field_simple",
                KIND_GAUSSIAN: "sfp32::field_gaussian", KIND_FOCUSED: "sfp32::field_focused"}
N_PARAMS = 16


class _Term:
    __slots__ = ("kind", "params", "user_code", "user_name")

    def __init__(self, kind: str, params: List[float], user_code: str = "", user_name: str = ""):
        self.kind = kind
        self.params = [float(p) for p in params] + [0.0] * (N_PARAMS - len(params))
        self.user_code = user_code
        self.user_name = user_name


class Fields:
    """A field program.  ``Fields(callable)`` or a preset; ``a + b`` sums."""

    def __init__(self, field_func: Optional[Callable] = None, *, _tree=None):
        if _tree is None:
            if field_func is None or not callable(field_func):
                raise TypeError("Fields needs a callable (x, y, z, t) -> (Ex, Ey, Ez, Bx, By, Bz)")
            from .translate import translate_field_function
            code, name = translate_field_function(field_func)
            _tree = _Term(KIND_USER, [], user_code=code, user_name=name)
        self._tree = _tree
        self.field_func_input = field_func
        self._params_dev = {}

    # Fields.__add__, fields.py:52-61: componentwise sum, left then right
    def __add__(self, other: "Fields") -> "Fields":
        if not isinstance(other, Fields):
            return NotImplemented
        return Fields(_tree=("add", self._tree, other._tree))

    # -- program pieces ---------------------------------------------------
    def terms(self) -> List[_Term]:
        out = []

        def walk(n):
            if isinstance(n, _Term):
                out.append(n)
            else:
                walk(n[1])
                walk(n[2])

        walk(self._tree)
        return out

    def params(self) -> np.ndarray:
        return np.asarray([p for t in self.terms() for p in t.params], dtype=np.float64)

    def structure(self) -> str:
        def walk(n):
            if isinstance(n, _Term):
                if n.kind == KIND_USER:
                    return "user:" + hashlib.sha256(n.user_code.encode()).hexdigest()[:16]
                return n.kind
            return f"add({walk(n[1])},{walk(n[2])})"

        return walk(self._tree)

    def cuda_source(self) -> str:
        """CUDA C++ of ``sfp_field_program`` (float64) and
        ``sfp_field_program32`` (float32 result) for this structure."""
        helpers = []
        user_fn = {}

        def program(real: str, fns) -> str:
            lines = []
            counter = [0, 0]
            # float32 sums of Gaussian terms share the terms' transverse factors
            # (sfp32::GaussXY: equal for terms of one beam geometry)
            share = real == "float" and sum(t.kind == KIND_GAUSSIAN for t in self.terms()) >= 2
            if share:
                lines.append("    sfp32::GaussXY G; bool G_have = false;")

            def emit(n) -> str:
                if isinstance(n, _Term):
                    k = counter[0]
                    counter[0] += 1
                    v = f"T{counter[1]}"
                    counter[1] += 1
                    if n.kind == KIND_USER:
                        if id(n) not in user_fn:
                            user_fn[id(n)] = f"sfp_user_field_{len(helpers)}"
                            helpers.append(n.user_code.replace("__SFP_USER_FN__", user_fn[id(n)]))
                        fname = user_fn[id(n)]
                        if real == "double":
                            lines.append(f"    double {v}[6]; {fname}(x, y, z, t, P + {k * N_PARAMS}, {v});")
                        else:
                            lines.append(f"    float {v}[6]; {{ double D[6]; {fname}(x, y, z, t, P + {k * N_PARAMS}, D);"
                                         f" for (int i = 0; i < 6; ++i) {v}[i] = (float)D[i]; }}")
                    elif n.kind == KIND_STATIC:
                        lines.append(f"    {real} {v}[6]; {fns[n.kind]}(P + {k * N_PARAMS}, {v});")
                    elif share and n.kind == KIND_GAUSSIAN:
                        lines.append(f"    {real} {v}[6]; sfp32::field_gaussian_g(P + {k * N_PARAMS}, x, y, z, t, G, G_have, {v});")
                    else:
                        lines.append(f"    {real} {v}[6]; {fns[n.kind]}(P + {k * N_PARAMS}, x, y, z, t, {v});")
                    return v
                a = emit(n[1])
                b = emit(n[2])
                v = f"T{counter[1]}"
                counter[1] += 1
                lines.append(f"    {real} {v}[6];")
                lines.append(f"    for (int k = 0; k < 6; ++k) {v}[k] = {a}[k] + {b}[k];")
                return v

            res = emit(self._tree)
            name = "sfp_field_program" if real == "double" else "sfp_field_program32"
            return (f"SFP_DEVICE_INLINE void {name}(double x, double y, double z, double t,\n"
                    f"                                  const double* __restrict__ P, {real} F[6]) {{\n"
                    + "\n".join(lines) + "\n"
                    f"    for (int k = 0; k < 6; ++k) F[k] = {res}[k];\n"
                    "}\n")

        p64 = program("double", _DEVICE_FN)
        p32 = program("float", _DEVICE_FN32)
        return "\n".join(helpers) + "\n" + p64 + p32 + self._bound_source()

    def _bound_source(self) -> str:
        """CUDA C++ of ``sfp_field_bound(P)``: an upper bound of |E| + c|B| over
        all space and time, the sum of the terms' bounds.  A Gaussian or simple
        pulse has |E| <= |E0| (its transverse and temporal envelopes and the
        focusing factor w0/w are at most 1; for the simple pulse only with an
        even temporal order) and c|B| = |E|; a static field has its own
        magnitudes; a focused pulse or a user callable has no bound here
        (1e300).  The photon kernel turns it into a bound of chi per unit of
        gamma (chi <= gamma (|E| + c|B|) / E_s)."""
        lines = ["SFP_DEVICE_INLINE double sfp_field_bound(const double* __restrict__ P) {", "    double b = 0.0;"]
        for k, t in enumerate(self.terms()):
            o = k * N_PARAMS
            if t.kind == KIND_GAUSSIAN:
                lines.append(f"    b += 2.0 * fabs(P[{o}]);")
            elif t.kind == KIND_SIMPLE:
                lines.append(f"    b += fmod(P[{o + 9}], 2.0) == 0.0 ? 2.0 * fabs(P[{o}]) : 1e300;")
            elif t.kind == KIND_STATIC:
                lines.append(f"    b += sqrt(P[{o}] * P[{o}] + P[{o + 1}] * P[{o + 1}] + P[{o + 2}] * P[{o + 2}]) + "
                             f"299792458.0 * sqrt(P[{o + 3}] * P[{o + 3}] + P[{o + 4}] * P[{o + 4}] + "
                             f"P[{o + 5}] * P[{o + 5}]);")
            else:
                lines.append("    b += 1e300;")
        lines += ["    return b;", "}", ""]
        return "\n".join(lines)

    def params_device(self, device=None):
        """Parameter array on the CUDA device (cached per device)."""
        import torch
        dev = torch.device("cuda") if device is None else torch.device(device)
        key = str(dev)
        t = self._params_dev.get(key)
        if t is None:
            t = torch.as_tensor(self.params(), dtype=torch.float64, device=dev).contiguous()
            self._params_dev[key] = t
        return t

    def __repr__(self):
        return f"Fields({self.structure()})"


def _preset(kind: str, params: List[float]) -> Fields:
    return Fields(_tree=_Term(kind, params))


def _pack_float32(values: List[float]) -> List[float]:
    """float64 parameter slots holding float32 values in pairs (little
    endian: value 2j in the low half of slot j).  Finite float32 values never
    pack into a NaN or infinity."""
    import struct
    v = list(values) + [0.0] * (len(values) % 2)
    return [struct.unpack("<d", struct.pack("<ff", v[j], v[j + 1]))[0] for j in range(0, len(v), 2)]


def _check_direction(direction):
    assert direction == 1 or direction == -1, "direction must be +1 (+x) or -1 (-x)"


def simple_laser_pulse(a0, w0, ctau, t_order=2, direction=1, x0=0, wavelength=0.8e-6, pol_angle=0, cep=0):
    """Plane-wave-like pulse without focusing (fields.py:69-118).

    Parameters are those of the reference: a0, w0 (1/e radius), ctau (1/e
    length), t_order (envelope exponent), direction (+1/-1 along x), x0,
    wavelength, pol_angle [rad], cep [rad].
    """
    _check_direction(direction)
    omega0 = 2 * PI * C / wavelength
    k0 = omega0 / C
    a0_norm = E_CHARGE / (M_E * C * omega0)
    E0 = a0 / a0_norm
    is_int = isinstance(t_order, (int, np.integer)) and not isinstance(t_order, bool)
    f = _preset(KIND_SIMPLE, [E0, k0, w0, ctau, direction, x0, cep, math.cos(pol_angle), math.sin(pol_angle),
                              t_order, 1.0 if is_int else 0.0])
    f.field_func_input = ("simple_laser_pulse", dict(a0=a0, w0=w0, ctau=ctau, t_order=t_order, direction=direction,
                                                     x0=x0, wavelength=wavelength, pol_angle=pol_angle, cep=cep))
    return f


def gaussian_laser_pulse(a0, w0, ctau, direction=1, x0=0.0, l0=0.8e-6, pol_angle=0.0, cep=0.0):
    """Paraxial Gaussian pulse (fields.py:120-170).  Singular at x = 0 exactly,
    as in the reference (its curvature radius x(1 + (zR/x)^2))."""
    _check_direction(direction)
    omega0 = 2 * PI * C / l0
    k0 = 2 * PI / l0
    zR = PI * w0 ** 2 / l0
    a0_norm = E_CHARGE / (M_E * C * omega0)
    E0 = a0 / a0_norm
    cp, sp = math.cos(pol_angle), math.sin(pol_angle)
    kc = k0 * ctau
    # slots 10-15: the float32 form's constants, two float32 per slot, so that
    # its per-particle evaluation converts and divides nothing
    f32 = [E0, k0, 1.0 / zR, k0 / (2.0 * zR * zR), 1.0 / (w0 * w0), 1.0 / (kc * kc), direction / C, cep, cp, sp,
           k0 / (4.0 * zR), kc]
    f = _preset(KIND_GAUSSIAN, [E0, k0, zR, w0, ctau, direction, x0, cep, cp, sp] + _pack_float32(f32))
    f.field_func_input = ("gaussian_laser_pulse", dict(a0=a0, w0=w0, ctau=ctau, direction=direction, x0=x0, l0=l0,
                                                       pol_angle=pol_angle, cep=cep))
    return f


def focused_gaussian_laser_pulse(a0, w0, ctau, direction=1, xfoc=0.0, x0=0.0, l0=0.8e-6, pol_angle=0.0, cep=0.0):
    """Tightly focused Gaussian pulse with corrections to order eps^5
    (fields.py:173-265; Salamin & Keitel, PRL 88, 095005)."""
    _check_direction(direction)
    omega0 = 2 * PI * C / l0
    k0 = 2 * PI / l0
    zR = PI * w0 ** 2 / l0
    eps = w0 / zR
    a0_norm = E_CHARGE / (M_E * C * omega0)
    E0 = a0 / a0_norm
    f = _preset(KIND_FOCUSED, [E0, k0, zR, w0, ctau, direction, xfoc, x0, cep, math.cos(pol_angle),
                               math.sin(pol_angle), eps])
    f.field_func_input = ("focused_gaussian_laser_pulse", dict(a0=a0, w0=w0, ctau=ctau, direction=direction,
                                                               xfoc=xfoc, x0=x0, l0=l0, pol_angle=pol_angle, cep=cep))
    return f


def static_field(Ex=0, Ey=0, Ez=0, Bx=0, By=0, Bz=0):
    """Uniform static field (fields.py:268-271)."""
    f = _preset(KIND_STATIC, [Ex, Ey, Ez, Bx, By, Bz])
    f.field_func_input = ("static_field", dict(Ex=Ex, Ey=Ey, Ez=Ez, Bx=Bx, By=By, Bz=Bz))
    return f


def preset_structures():
    """Representative programs whose modules build() compiles ahead of time."""
    g = gaussian_laser_pulse(1.0, 1e-6, 1e-6)
    return [static_field(), g, simple_laser_pulse(1.0, 1e-6, 1e-6), focused_gaussian_laser_pulse(1.0, 1e-6, 1e-6),
            g + gaussian_laser_pulse(1.0, 1e-6, 1e-6)]
