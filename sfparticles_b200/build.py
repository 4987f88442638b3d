"""Build steps of sfparticles_b200.

* ``build_library()``  -- nvcc: csrc/sfp_capi.cu + csrc/sfp_mlp.cu -> libsfp.so (sm_100a, in-tree)
* ``build_tables()``   -- QED tables into qed/data (scipy, CPU)
* ``prebuild_modules()`` -- NVRTC: field-specialised step modules for the
  presets into the module cache (NVRTC needs no GPU)
* ``build()``          -- all of the above
"""
from __future__ import annotations

import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    p = os.path.join(CUDA_HOME, "bin", "nvcc")
    return p if os.path.exists(p) else (shutil.which("nvcc") or "nvcc")


def library_sources():
    return [os.path.join(CSRC, "sfp_capi.cu"), os.path.join(CSRC, "sfp_mlp.cu"), os.path.join(CSRC, "sfp_tables.cu")]


def library_headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def build_library(force: bool = False, verbose: bool = False) -> str:
    out = os.path.join(PKG, "libsfp.so")
    deps = library_sources() + library_headers()
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc(), *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           f"-I{INCLUDE}", f"-I{CSRC}", "-o", out + ".tmp", *library_sources(),
           f"-L{CUDA_HOME}/lib64", "-lnvrtc", "-Xlinker", f"-rpath={CUDA_HOME}/lib64"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def build_tables(verbose: bool = True):
    from .qed import tables
    tables.ensure_tables(verbose=verbose)


def prebuild_modules(verbose: bool = False):
    """Compile the field-specialised step modules of the presets (NVRTC)."""
    from . import fields, program
    for f in fields.preset_structures():
        for form in ("fp64", "fp32"):
            for qed in ("rs", "od"):
                for single in (True, False):
                    program.get_module(f, form=form, qed=qed, load=False, single=single)
        program.get_module(f, form=None, qed=None, load=False)


def build(verbose: bool = False):
    build_library(verbose=verbose)
    build_tables(verbose=verbose)
    prebuild_modules(verbose=verbose)


if __name__ == "__main__":
    build(verbose=True)
