"""User field callables for the ``Fields(callable)`` tests (test
infrastructure).

Each is a plain Python function of (x, y, z, t) returning six SI field
components, the form the reference's ``Fields`` accepts and JIT-compiles with
Numba (sfparticles/fields.py:11-50).  tests/golden/make_golden.py evaluates
these same functions through the reference's ``Fields`` and ``Simulation``
and records the outputs; the tests translate them to CUDA with
``sfparticles_b200.translate`` and compare.

* ``gaussian_callable`` restates ``gaussian_laser_pulse``
  (fields.py:120-170) as a user function, written the way a user would;
* ``mixed_callable`` touches every statement and expression form the
  translator accepts (if/elif/else, augmented and tuple assignment,
  conditional expressions, chained comparisons, and/or/not, ``%`` and
  ``//``, integer and real powers, math and numpy functions, module
  attributes, closure constants);
* ``lambda_field`` is a lambda.
"""
import math
from math import atan, cos, exp, sin, sqrt

import numpy as np

C = 299792458.0
PI = math.pi
E_CHARGE = 1.602176634e-19
M_E = 9.1093837139e-31


def gaussian_callable(a0, w0, ctau, direction=1, x0=0.0, l0=0.8e-6, pol_angle=0.0, cep=0.0):
    omega0 = 2 * PI * C / l0
    k0 = 2 * PI / l0
    zR = PI * w0 ** 2 / l0
    E0 = a0 / (E_CHARGE / (M_E * C * omega0))
    cpol, spol = cos(pol_angle), sin(pol_angle)

    def user_gaussian(x, y, z, t):
        r2 = y ** 2 + z ** 2
        wx = w0 * sqrt(1 + (x / zR) ** 2)
        Rx = x * (1 + (zR / x) ** 2)
        gouy = atan(x / zR)
        phi = k0 * (x - x0 - direction * C * t) + k0 * r2 / 2 / Rx - gouy
        E = E0 * cos(phi + cep) * w0 / wx * exp(-r2 / wx ** 2) * exp(-phi ** 2 / (k0 * ctau) ** 2)
        Ey = E * cpol
        Ez = E * spol
        return (0.0, Ey, Ez, 0.0, -Ez / C * direction, Ey / C * direction)

    return user_gaussian


def mixed_callable(e0, b0, L, k):
    def user_mixed(x, y, z, t):
        """A smooth-edged, sheared field: one of each translated construct."""
        r = np.sqrt(y * y + z * z)
        s, c2 = math.sin(k * x), np.cos(k * x)
        env = 0.0
        if abs(x) > L:
            env = 0.0
        elif x < -0.5 * L:
            env = (x + L) / (0.5 * L)
        else:
            env = 1.0
            pass
        env *= np.exp(-(r / L) ** 2)
        g = env if 0.0 <= env <= 1.0 else 0.0
        ph = (k * x) % (2 * math.pi) - math.pi
        cells = (x + 2 * L) // L
        w = (1.0 + cells * cells) ** -2
        side = 1.0 if (y > 0 and z > 0) or not (r < 0.25 * L) else -1.0
        Ex = e0 * g * s * w
        Ey = e0 * g * c2 * max(0.2, min(0.8, 0.5 + y / L))
        Ez = e0 * g * np.tanh(ph) * side
        Bx = b0 * g * math.pow(1.0 + abs(t) * 1e13, 1.5)
        By = b0 * g * np.hypot(s, c2) * exp(-abs(z) / L)
        Bz = b0 * (g - 0.5) ** 3 + b0 * atan(y / L)
        return Ex, Ey, Ez, Bx, By, Bz

    return user_mixed


def lambda_field():
    e1, b1 = 2.0e11, 300.0
    return lambda x, y, z, t: (0.0, e1 * cos(1e6 * x), 0.0, 0.0, 0.0, b1 * sin(1e6 * y))


# builders by name, with their keyword arguments, for the fixtures and tests
GAUSSIAN = dict(a0=80.0, w0=3e-6, ctau=5e-6, direction=-1, x0=3e-6)
STATIC = dict(Ex=0.0, Ey=2.0e11, Ez=0.0, Bx=0.0, By=0.0, Bz=150.0)
MIXED = dict(e0=3.0e12, b0=5.0e3, L=4e-6, k=2.0e6)
BUILDERS = {"gaussian": gaussian_callable, "mixed": mixed_callable, "lambda": lambda_field}
