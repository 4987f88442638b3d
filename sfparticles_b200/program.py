"""NVRTC modules: a field program compiled together with the step kernels.

A module is identified by (field structure, arithmetic form, QED method);
numeric field parameters are runtime data, so every gaussian-pulse
simulation shares one module.  Compiled cubins are cached on disk under
``_jit_cache`` next to this file (override with SFPARTICLES_B200_CACHE) and
keyed by a hash of the full source and options, so ``build()`` can compile
the presets ahead of time without a GPU.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import re
import threading

from . import _lib

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
CACHE = os.environ.get("SFPARTICLES_B200_CACHE", os.path.join(PKG, "_jit_cache"))
TILE = 256

_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"\s*$', re.M)
_modules = {}
_lock = threading.Lock()


def _read(name: str) -> str:
    for d in (CSRC, INCLUDE):
        p = os.path.join(d, name)
        if os.path.exists(p):
            with open(p) as f:
                return f.read()
    raise FileNotFoundError(name)


def _inline(text: str, seen: set) -> str:
    def rep(m):
        name = m.group(1)
        if name in seen:
            return ""
        seen.add(name)
        return _inline(_read(name), seen)

    return _INCLUDE_RE.sub(rep, text.replace("#pragma once", ""))


def module_source(field_src: str, form, qed, n_const=None) -> str:
    """Source of a module.  ``n_const``: the length of the field's parameter
    block when the module serves runs of one instance, which then read the
    block from the module's constant bank (``sfp_cfield``)."""
    seen = set()
    head = _inline('#include "sfp_types.h"\n#include "sfp_device.cuh"\n#include "sfp_device32.cuh"\n', seen)
    parts = [head, "// ---- field program ----\n", field_src]
    if form is None:
        parts.append("#define SFP_WANT_FIELD_EVAL 1\n")
    else:
        parts.append(f"#define SFP_WANT_STEP 1\n#define SFP_STEP_FORM_{form.upper()} 1\n#define SFP_STEP_QED_{qed.upper()} 1\n")
        if n_const:
            parts.append(f"#define SFP_CONST_FIELD_N {int(n_const)}\n")
    parts.append(_inline('#include "sfp_step.cuh"\n', seen))
    return "".join(parts)


def options(form=None):
    """NVRTC options of a module.  The float32 form's step modules flush
    float32 denormals and take float32 square roots and divisions from the
    hardware approximations (within 2 ulp): its error budget is set by
    float32 itself, and the exact IEEE sequences cost issue slots in kernels
    that are issue-bound.  Float64 arithmetic is unaffected by these flags."""
    opts = ["-arch=sm_100a", "-std=c++17", "-lineinfo", f"-DSFP_TILE={TILE}", "--fmad=true"]
    if form == "fp32":
        opts += ["-ftz=true", "-prec-sqrt=false", "-prec-div=false"]
    return opts


def _key(src: str, opts) -> str:
    h = hashlib.sha256()
    h.update(src.encode())
    h.update("\0".join(opts).encode())
    return h.hexdigest()[:32]


def compile_image(src: str, opts) -> bytes:
    L = _lib.load()
    arr = (ctypes.c_char_p * len(opts))(*[o.encode() for o in opts])
    img = ctypes.c_void_p()
    size = ctypes.c_size_t()
    log = ctypes.c_void_p()
    rc = L.sfp_nvrtc_compile(src.encode(), b"sfp_module.cu", ctypes.cast(arr, ctypes.c_void_p), len(opts),
                             ctypes.byref(img), ctypes.byref(size), ctypes.byref(log))
    if log.value:
        L.sfp_free(log)
    if rc != 0:
        raise _lib.SFPError("NVRTC: " + L.sfp_last_error().decode(errors="replace"))
    data = ctypes.string_at(img.value, size.value)
    L.sfp_free(img)
    return data


def get_image(fields, form, qed, single=False) -> bytes:
    # the constant bank holds 64 KiB: a field of more than 256 terms keeps
    # its parameters in global memory (the run finds no sfp_cfield)
    n = len(fields.params())
    n_const = n if (single and form is not None and 0 < n <= 4096) else None
    src = module_source(fields.cuda_source(), form, qed, n_const)
    opts = options(form)
    key = _key(src, opts)
    path = os.path.join(CACHE, f"{key}.cubin")
    if os.path.exists(path):
        with open(path, "rb") as f:
            return f.read()
    data = compile_image(src, opts)
    os.makedirs(CACHE, exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "wb") as f:
        f.write(data)
    os.replace(tmp, path)
    return data


class Module:
    """A loaded NVRTC module (sfp_module*)."""

    def __init__(self, image: bytes):
        L = _lib.load()
        self._image = image
        h = ctypes.c_void_p()
        _lib.check(L.sfp_module_load(image, len(image), ctypes.byref(h)), "sfp_module_load")
        self.handle = h

    def __del__(self):
        try:
            if self.handle:
                _lib.load().sfp_module_unload(self.handle)
        except Exception:
            pass


def get_module(fields, form="fp64", qed="rs", load=True, single=False):
    """Module for (fields structure, form, qed); form=None gives the
    field-evaluation module used by the per-op path.  ``single``: a step
    module for runs of one instance (field parameters in its constant bank,
    copied there by the run); otherwise each instance's parameters are read
    from global memory."""
    single = bool(single) and form is not None
    key = (fields.structure(), form, qed, single)
    with _lock:
        m = _modules.get(key)
        if m is not None:
            return m
        img = get_image(fields, form, qed, single)
        if not load:
            return None
        m = Module(img)
        _modules[key] = m
        return m
