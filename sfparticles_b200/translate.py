"""Translate a Python field callable into a CUDA C++ device function.

The reference accepts any Numba-compilable ``f(x, y, z, t)`` returning six
field components (fields.py:11-50).  Here the callable becomes CUDA C++ that
NVRTC compiles into the push.  Accepted subset (anything else raises
``FieldTranslationError`` naming the construct; there is no fallback):

* positional arguments x, y, z, t (any names), float64 arithmetic
  ``+ - * / ** // %``, unary ``-``/``+``, comparisons, ``and``/``or``/``not``,
  conditional expressions;
* statements: assignment to names (also tuple unpacking of tuples), augmented
  assignment, ``if``/``elif``/``else``, ``pass``, one final ``return`` of six values;
* calls of math / numpy scalar functions (sin, cos, tan, asin, acos, atan,
  atan2, sinh, cosh, tanh, exp, log, log10, log2, sqrt, cbrt, fabs/abs, floor,
  ceil, pow, hypot, copysign, fmin/min, fmax/max);
* names from the closure or globals bound to numbers (folded as constants),
  ``math.pi``/``math.e``/``numpy.pi`` and the functions above via a module.

Integer literal exponents ``a**n`` are unrolled as Numba does
(exponentiation by squaring); other exponents call ``pow``.
"""
from __future__ import annotations

import ast
import hashlib
import inspect
import math
import numbers
import textwrap

import numpy as np


class FieldTranslationError(ValueError):
    pass


_FUNCS = {
    "sin": "sin", "cos": "cos", "tan": "tan", "asin": "asin", "acos": "acos", "atan": "atan", "arcsin": "asin",
    "arccos": "acos", "arctan": "atan", "atan2": "atan2", "arctan2": "atan2", "sinh": "sinh", "cosh": "cosh",
    "tanh": "tanh", "exp": "exp", "expm1": "expm1", "log": "log", "log10": "log10", "log2": "log2", "log1p": "log1p",
    "sqrt": "sqrt", "cbrt": "cbrt", "fabs": "fabs", "abs": "fabs", "absolute": "fabs", "floor": "floor",
    "ceil": "ceil", "pow": "pow", "power": "pow", "hypot": "hypot", "copysign": "copysign", "fmin": "fmin",
    "fmax": "fmax", "min": "fmin", "max": "fmax", "minimum": "fmin", "maximum": "fmax",
}
_MATH_FUNCS = {getattr(math, k): v for k, v in _FUNCS.items() if hasattr(math, k)}
_MATH_FUNCS.update({getattr(np, k): v for k, v in _FUNCS.items() if hasattr(np, k) and callable(getattr(np, k))})
_MATH_FUNCS[abs] = "fabs"
_MATH_FUNCS[min] = "fmin"
_MATH_FUNCS[max] = "fmax"
_MODULES = (math, np)


def _lit(v) -> str:
    if isinstance(v, (bool, np.bool_)):
        return "1.0" if v else "0.0"
    v = float(v)
    if math.isnan(v):
        return "__longlong_as_double(0x7ff8000000000000ll)"
    if math.isinf(v):
        return "(1.0/0.0)" if v > 0 else "(-1.0/0.0)"
    return "(" + repr(v) + ")" if v < 0 else repr(v) if "e" in repr(v) or "." in repr(v) else repr(v) + ".0"


def _parse_lambda(src: str):
    """The first lambda expression in `src`, the source lines that define
    it.  Those lines need not form a statement on their own (``return
    lambda ...``, a lambda inside a call), so the text from ``lambda`` on is
    parsed as an expression, trimmed from the end until it parses."""
    i = src.find("lambda")
    if i < 0:
        return None
    s = src[i:].rstrip()
    for end in range(len(s), 0, -1):
        if s[end - 1] not in ")]},\n \t" and end != len(s):
            continue  # only trim at the closing characters an enclosing expression can leave
        try:
            tree = ast.parse(s[:end], mode="eval")
        except SyntaxError:
            continue
        if isinstance(tree.body, ast.Lambda):
            return tree.body
    return None


class _Translator:
    def __init__(self, func):
        self.func = func
        try:
            src = textwrap.dedent(inspect.getsource(func))
        except (OSError, TypeError) as e:
            raise FieldTranslationError(f"cannot read the source of {func!r}: {e}") from e
        node = None
        if func.__name__ == "<lambda>":
            node = _parse_lambda(src)
        else:
            try:
                tree = ast.parse(src)
            except SyntaxError as e:
                raise FieldTranslationError(f"cannot parse the source of {func.__name__}: {e}") from e
            for n in ast.walk(tree):
                if isinstance(n, ast.FunctionDef) and n.name == func.__name__:
                    node = n
                    break
        if node is None:
            raise FieldTranslationError(f"cannot find the definition of {func.__name__}")
        self.node = node
        cv = inspect.getclosurevars(func)
        self.env = dict(cv.builtins)
        self.env.update(cv.globals)
        self.env.update(cv.nonlocals)
        args = node.args
        if args.vararg or args.kwarg or args.kwonlyargs or len(args.args) != 4:
            raise FieldTranslationError("field function must take exactly four positional arguments (x, y, z, t)")
        self.vars = {}
        for a, c in zip(args.args, ("x", "y", "z", "t")):
            self.vars[a.arg] = c
        self.locals = []
        self.ret = None

    def var(self, name, create=False):
        if name in self.vars:
            return self.vars[name]
        if not create:
            return None
        c = f"v{len(self.locals)}"
        self.locals.append(c)
        self.vars[name] = c
        return c

    # -- expressions ------------------------------------------------------
    def resolve(self, node):
        """Python object of a Name / Attribute chain from closure/globals, or None."""
        if isinstance(node, ast.Name):
            if node.id in self.vars:
                return None
            if node.id in self.env:
                return self.env[node.id]
            raise FieldTranslationError(f"unknown name '{node.id}' (line {node.lineno})")
        if isinstance(node, ast.Attribute):
            base = self.resolve(node.value)
            if base is None:
                return None
            if not hasattr(base, node.attr):
                raise FieldTranslationError(f"'{node.attr}' not found (line {node.lineno})")
            return getattr(base, node.attr)
        return None

    def expr(self, n) -> str:
        if isinstance(n, ast.Constant):
            if isinstance(n.value, (bool, int, float)):
                return _lit(n.value)
            raise FieldTranslationError(f"unsupported constant {n.value!r} (line {n.lineno})")
        if isinstance(n, ast.Name):
            v = self.var(n.id)
            if v is not None:
                return v
            obj = self.resolve(n)
            if isinstance(obj, (numbers.Number, np.number)) and not isinstance(obj, complex):
                return _lit(obj)
            raise FieldTranslationError(f"name '{n.id}' is not a number (line {n.lineno})")
        if isinstance(n, ast.Attribute):
            obj = self.resolve(n)
            if isinstance(obj, (numbers.Number, np.number)) and not isinstance(obj, complex):
                return _lit(obj)
            raise FieldTranslationError(f"attribute '{ast.unparse(n)}' is not a number (line {n.lineno})")
        if isinstance(n, ast.UnaryOp):
            a = self.expr(n.operand)
            if isinstance(n.op, ast.USub):
                return f"(-{a})"
            if isinstance(n.op, ast.UAdd):
                return f"(+{a})"
            if isinstance(n.op, ast.Not):
                return f"((double)!({a} != 0.0))"
            raise FieldTranslationError(f"unsupported unary operator (line {n.lineno})")
        if isinstance(n, ast.BinOp):
            if isinstance(n.op, ast.Pow):
                return self.power(n)
            a, b = self.expr(n.left), self.expr(n.right)
            if isinstance(n.op, ast.Add):
                return f"({a} + {b})"
            if isinstance(n.op, ast.Sub):
                return f"({a} - {b})"
            if isinstance(n.op, ast.Mult):
                return f"({a} * {b})"
            if isinstance(n.op, ast.Div):
                return f"({a} / {b})"
            if isinstance(n.op, ast.FloorDiv):
                return f"floor({a} / {b})"
            if isinstance(n.op, ast.Mod):
                return f"sfp::py_mod({a}, {b})"
            raise FieldTranslationError(f"unsupported operator {type(n.op).__name__} (line {n.lineno})")
        if isinstance(n, ast.Compare):
            if len(n.ops) != 1:
                parts = []
                left = n.left
                for op, right in zip(n.ops, n.comparators):
                    parts.append(self.expr(ast.Compare(left=left, ops=[op], comparators=[right])))
                    left = right
                return "((double)(" + " && ".join(f"({p} != 0.0)" for p in parts) + "))"
            ops = {ast.Lt: "<", ast.LtE: "<=", ast.Gt: ">", ast.GtE: ">=", ast.Eq: "==", ast.NotEq: "!="}
            op = ops.get(type(n.ops[0]))
            if op is None:
                raise FieldTranslationError(f"unsupported comparison (line {n.lineno})")
            return f"((double)({self.expr(n.left)} {op} {self.expr(n.comparators[0])}))"
        if isinstance(n, ast.BoolOp):
            j = " && " if isinstance(n.op, ast.And) else " || "
            return "((double)(" + j.join(f"({self.expr(v)} != 0.0)" for v in n.values) + "))"
        if isinstance(n, ast.IfExp):
            return f"(({self.expr(n.test)} != 0.0) ? {self.expr(n.body)} : {self.expr(n.orelse)})"
        if isinstance(n, ast.Call):
            if n.keywords:
                raise FieldTranslationError(f"keyword arguments are not supported (line {n.lineno})")
            fobj = self.resolve(n.func)
            cname = _MATH_FUNCS.get(fobj) if fobj is not None else None
            if cname is None:
                raise FieldTranslationError(f"unsupported call '{ast.unparse(n.func)}' (line {n.lineno})")
            args = [self.expr(a) for a in n.args]
            if cname in ("fmin", "fmax") and len(args) > 2:
                acc = args[0]
                for a in args[1:]:
                    acc = f"{cname}({acc}, {a})"
                return acc
            return f"{cname}({', '.join(args)})"
        raise FieldTranslationError(f"unsupported expression {type(n).__name__} (line {getattr(n, 'lineno', '?')})")

    def _const_int(self, n):
        if isinstance(n, ast.Constant) and isinstance(n.value, int) and not isinstance(n.value, bool):
            return n.value
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, ast.USub):
            v = self._const_int(n.operand)
            return None if v is None else -v
        if isinstance(n, (ast.Name, ast.Attribute)) and (not isinstance(n, ast.Name) or self.var(n.id) is None):
            obj = self.resolve(n)
            if isinstance(obj, (int, np.integer)) and not isinstance(obj, bool):
                return int(obj)
        return None

    def power(self, n) -> str:
        base = self.expr(n.left)
        k = self._const_int(n.right)
        if k is not None and abs(k) <= 64:
            if k >= 0:
                return f"sfp::ipow<{k}>({base})"
            return f"(1.0 / sfp::ipow<{-k}>({base}))"
        return f"pow({base}, {self.expr(n.right)})"

    # -- statements -------------------------------------------------------
    def stmts(self, body, out, indent):
        for s in body:
            self.stmt(s, out, indent)

    def assign_name(self, name, value_code, out, indent):
        v = self.var(name, create=True)
        out.append(f"{indent}{v} = {value_code};")

    def stmt(self, s, out, indent):
        if self.ret is not None:
            raise FieldTranslationError(f"statement after return (line {s.lineno})")
        if isinstance(s, ast.Assign):
            for tgt in s.targets:
                if isinstance(tgt, ast.Name):
                    self.assign_name(tgt.id, self.expr(s.value), out, indent)
                elif isinstance(tgt, (ast.Tuple, ast.List)) and isinstance(s.value, (ast.Tuple, ast.List)) and len(
                        tgt.elts) == len(s.value.elts):
                    tmps = []
                    for e in s.value.elts:
                        tv = f"w{len(self.locals)}"
                        self.locals.append(tv)
                        out.append(f"{indent}{tv} = {self.expr(e)};")
                        tmps.append(tv)
                    for e, tv in zip(tgt.elts, tmps):
                        if not isinstance(e, ast.Name):
                            raise FieldTranslationError(f"unsupported assignment target (line {s.lineno})")
                        self.assign_name(e.id, tv, out, indent)
                else:
                    raise FieldTranslationError(f"unsupported assignment (line {s.lineno})")
            return
        if isinstance(s, ast.AugAssign):
            if not isinstance(s.target, ast.Name):
                raise FieldTranslationError(f"unsupported augmented assignment (line {s.lineno})")
            cur = ast.Name(id=s.target.id, ctx=ast.Load(), lineno=s.lineno)
            val = self.expr(ast.BinOp(left=cur, op=s.op, right=s.value, lineno=s.lineno))
            self.assign_name(s.target.id, val, out, indent)
            return
        if isinstance(s, ast.If):
            out.append(f"{indent}if ({self.expr(s.test)} != 0.0) {{")
            self.stmts(s.body, out, indent + "    ")
            if s.orelse:
                out.append(f"{indent}}} else {{")
                self.stmts(s.orelse, out, indent + "    ")
            out.append(f"{indent}}}")
            return
        if isinstance(s, ast.Pass):
            return
        if isinstance(s, ast.Expr) and isinstance(s.value, ast.Constant) and isinstance(s.value.value, str):
            return  # docstring
        if isinstance(s, ast.Return):
            val = s.value
            if not isinstance(val, (ast.Tuple, ast.List)) or len(val.elts) != 6:
                raise FieldTranslationError("the field function must return six values (Ex, Ey, Ez, Bx, By, Bz)")
            for i, e in enumerate(val.elts):
                out.append(f"{indent}F[{i}] = {self.expr(e)};")
            out.append(f"{indent}return;")
            if indent == "    ":
                self.ret = True
            return
        raise FieldTranslationError(f"unsupported statement {type(s).__name__} (line {s.lineno})")

    def translate(self) -> str:
        out = []
        if isinstance(self.node, ast.Lambda):
            self.stmt(ast.Return(value=self.node.body, lineno=self.node.lineno), out, "    ")
        else:
            self.stmts(self.node.body, out, "    ")
        if self.ret is None:
            raise FieldTranslationError("the field function must end with a return of six values")
        decl = f"    double {', '.join(l + ' = 0.0' for l in self.locals)};" if self.locals else ""
        return ("SFP_DEVICE_INLINE void __SFP_USER_FN__(double x, double y, double z, double t,\n"
                "                                      const double* __restrict__ P, double F[6]) {\n"
                "    (void)P; (void)x; (void)y; (void)z; (void)t;\n"
                f"{decl}\n" + "\n".join(out) + "\n}\n")


def translate_field_function(func):
    """CUDA C++ (function named ``__SFP_USER_FN__``) and a stable name."""
    code = _Translator(func).translate()
    name = "user_" + hashlib.sha256(code.encode()).hexdigest()[:12]
    return code, name
