"""Fields(callable): the translator of Python field functions to CUDA
(sfparticles_b200.translate), on the CPU.

The reference JIT-compiles any Numba-compilable f(x, y, z, t) returning six
components (sfparticles/fields.py:11-50).  Here the callable is translated to
C++; these tests check, without a GPU:

* that the accepted subset translates and NVRTC compiles it for sm_100a;
* that the translated code computes what the Python function computes: the
  generated function is compiled for the host with g++ (with the product's
  own ``ipow`` / ``py_mod`` helpers from csrc/sfp_device.cuh) and evaluated
  against the Python callable at seeded points, 1e-13 relative;
* that every construct outside the subset raises FieldTranslationError
  naming it.
The device results against the reference's own outputs are
tests/test_gpu_user_fields.py.
"""
import ctypes
import math
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import user_fields as U
from sfparticles_b200.fields import Fields, static_field
from sfparticles_b200.translate import FieldTranslationError, translate_field_function

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "sfparticles_b200", "csrc")


def _helpers_from_device_header() -> str:
    """ipow and py_mod exactly as csrc/sfp_device.cuh defines them."""
    src = open(os.path.join(CSRC, "sfp_device.cuh")).read()
    m = re.search(r"template <int N>\s*\nSFP_DEVICE_INLINE double ipow\(.*?\n}\n.*?"
                  r"SFP_DEVICE_INLINE double py_mod\(.*?\n}\n", src, re.S)
    assert m, "ipow / py_mod not found in sfp_device.cuh"
    return m.group(0).replace("#pragma unroll", "")


def _host_eval(func, pts):
    """Compile the translation of `func` for the host and evaluate it at pts (4 x n)."""
    code, _ = translate_field_function(func)
    src = ("#include <cmath>\n#define SFP_DEVICE_INLINE static inline\nusing namespace std;\n"
           "namespace sfp {\n" + _helpers_from_device_header() + "}\n"
           + code.replace("__SFP_USER_FN__", "user_fn") +
           'extern "C" void eval_points(const double* x, const double* y, const double* z, const double* t,\n'
           '                            long n, double* out) {\n'
           "    for (long i = 0; i < n; ++i) {\n"
           "        double F[6];\n"
           "        user_fn(x[i], y[i], z[i], t[i], nullptr, F);\n"
           "        for (int c = 0; c < 6; ++c) out[c * n + i] = F[c];\n"
           "    }\n}\n")
    with tempfile.TemporaryDirectory() as d:
        cpp, so = os.path.join(d, "f.cpp"), os.path.join(d, "f.so")
        with open(cpp, "w") as f:
            f.write(src)
        subprocess.run(["g++", "-O1", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC", "-o", so, cpp],
                       check=True, capture_output=True)
        lib = ctypes.CDLL(so)
        n = pts.shape[1]
        a = [np.ascontiguousarray(p, dtype=np.float64) for p in pts]
        out = np.zeros(6 * n)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.eval_points(*[x.ctypes.data_as(dp) for x in a], ctypes.c_long(n), out.ctypes.data_as(dp))
        return out.reshape(6, n)


def _py_eval(func, pts):
    return np.array([func(*pts[:, j]) for j in range(pts.shape[1])], dtype=float).T


def _points(builder, n=200, seed=3):
    rng = np.random.default_rng(seed)
    if builder == "mixed":
        L = U.MIXED["L"]
        return np.stack([rng.uniform(-1.5 * L, 1.5 * L, n), rng.normal(0, L, n), rng.normal(0, L, n),
                         rng.uniform(-3e-14, 3e-14, n)])
    t = rng.uniform(-4e-14, 4e-14, n)
    x = 3e-6 - 299792458.0 * t + rng.normal(0, 5e-6, n)
    return np.stack([x, rng.normal(0, 2e-6, n), rng.normal(0, 2e-6, n), t])


@pytest.mark.parametrize("builder", ["gaussian", "mixed", "lambda"])
def test_translation_computes_the_python_function(builder):
    kw = {"gaussian": U.GAUSSIAN, "mixed": U.MIXED, "lambda": {}}[builder]
    func = U.BUILDERS[builder](**kw)
    pts = _points(builder)
    got = _host_eval(func, pts)
    ref = _py_eval(func, pts)
    scale = np.max(np.abs(ref), axis=1, keepdims=True) + 1e-300
    assert np.all(np.abs(got - ref) / scale < 1e-13), np.max(np.abs(got - ref) / scale)
    assert np.count_nonzero(ref) > 0


def test_every_branch_of_the_mixed_function_is_taken():
    """The points of the host check reach each if/elif/else arm and both
    sides of the conditional expressions."""
    L = U.MIXED["L"]
    x = _points("mixed")[0]
    assert (np.abs(x) > L).any() and ((x < -0.5 * L) & (x >= -L)).any() and ((x >= -0.5 * L) & (x <= L)).any()


def test_translated_modules_compile_for_sm100a():
    """NVRTC compiles the field-evaluation module of each user function and
    of a user + preset sum (no GPU needed)."""
    from sfparticles_b200 import program
    for f in (Fields(U.gaussian_callable(**U.GAUSSIAN)) + static_field(**U.STATIC),
              Fields(U.mixed_callable(**U.MIXED)), Fields(U.lambda_field())):
        program.get_module(f, form=None, qed=None, load=False)
        assert f.structure().startswith(("user:", "add(user:"))


def test_integer_powers_unroll_like_numba():
    def f(x, y, z, t):
        return (x ** 2, x ** 7, x ** -3, x ** 0.5, x ** y, 0.0)

    code, _ = translate_field_function(f)
    assert "sfp::ipow<2>(x)" in code and "sfp::ipow<7>(x)" in code
    assert "(1.0 / sfp::ipow<3>(x))" in code
    assert "pow(x, 0.5)" in code and "pow(x, y)" in code


def test_closure_numbers_are_folded_and_structure_is_stable():
    a = U.gaussian_callable(**U.GAUSSIAN)
    b = U.gaussian_callable(**U.GAUSSIAN)
    c = U.gaussian_callable(**{**U.GAUSSIAN, "a0": 81.0})
    ca, na = translate_field_function(a)
    cb, nb = translate_field_function(b)
    cc, nc = translate_field_function(c)
    assert ca == cb and na == nb
    assert na != nc  # constants are part of the translated program
    assert repr(U.C) in ca


def _bad_for(x, y, z, t):
    s = 0.0
    for k in range(3):
        s += k
    return (s, 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_while(x, y, z, t):
    while x > 0:
        x -= 1.0
    return (x, 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_kw(x, y, z, t):
    return (math.copysign(x, y=1.0), 0.0, 0.0, 0.0, 0.0, 0.0)


def _helper(v):
    return v


def _bad_call(x, y, z, t):
    return (_helper(x), 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_name(x, y, z, t):
    return (undefined_q * x, 0.0, 0.0, 0.0, 0.0, 0.0)  # noqa: F821


_LIST = [1.0, 2.0]


def _bad_global(x, y, z, t):
    return (_LIST, 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_arity(x, y, z):
    return (x, y, z, 0.0, 0.0, 0.0)


def _bad_five(x, y, z, t):
    return (x, y, z, t, 0.0)


def _bad_no_return(x, y, z, t):
    v = x + y


def _bad_after_return(x, y, z, t):
    return (x, y, z, t, 0.0, 0.0)
    v = 1.0


def _bad_string(x, y, z, t):
    return ("a", 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_subscript(x, y, z, t):
    return (_LIST[0], 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_attr_target(x, y, z, t):
    math.foo = 1.0
    return (x, 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_bitand(x, y, z, t):
    return (x & y, 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_is(x, y, z, t):
    return (1.0 if x is y else 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)


def _bad_varargs(x, y, z, *t):
    return (x, y, z, 0.0, 0.0, 0.0)


def _bad_complex(x, y, z, t):
    return (1j * x, 0.0, 0.0, 0.0, 0.0, 0.0)


@pytest.mark.parametrize("func,message", [
    (_bad_for, "unsupported statement For"),
    (_bad_while, "unsupported statement While"),
    (_bad_kw, "keyword arguments are not supported"),
    (_bad_call, "unsupported call '_helper'"),
    (_bad_name, "unknown name 'undefined_q'"),
    (_bad_global, "name '_LIST' is not a number"),
    (_bad_arity, "exactly four positional arguments"),
    (_bad_varargs, "exactly four positional arguments"),
    (_bad_five, "must return six values"),
    (_bad_no_return, "must end with a return"),
    (_bad_after_return, "statement after return"),
    (_bad_string, "unsupported constant 'a'"),
    (_bad_subscript, "unsupported expression Subscript"),
    (_bad_attr_target, "unsupported assignment"),
    (_bad_bitand, "unsupported operator BitAnd"),
    (_bad_is, "unsupported comparison"),
    (_bad_complex, "unsupported constant 1j"),
])
def test_unsupported_constructs_are_named(func, message):
    with pytest.raises(FieldTranslationError, match=re.escape(message)):
        Fields(func)


def test_a_function_without_source_is_refused():
    with pytest.raises(FieldTranslationError, match="cannot read the source"):
        Fields(math.hypot)


def test_fields_needs_a_callable():
    with pytest.raises(TypeError):
        Fields(3.0)
