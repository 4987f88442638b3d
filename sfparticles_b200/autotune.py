"""Autotuner of the step kernels.

Every NVRTC step module holds several variants of the two persistent step
kernels, both over warp tiles of 1024 particles streamed through a
``stages``-deep ring of asynchronous copies:

* ``sfp_massive_<form>_<qed>_s<stages>_b<blocks>`` -- e+- tiles;
* ``sfp_photon_<form>_<qed>_s<stages>_b<blocks>`` -- photon tiles;

``blocks`` is the register budget: at least that many blocks of 256 threads
stay resident per SM.  Which variant is fastest depends on the particle mix,
the field program and the form, so ``tune`` measures them: it builds a sample
of the simulation's current state (up to ``sample`` particles per species,
copied, so the user's run is not advanced), times a few steps of each
variant with CUDA events on the launching stream, and selects the fastest
of each kernel (the two kernels run one after the other and touch disjoint
memory, so they are tuned independently).  Results are cached per (GPU,
form, QED method, field structure, population bucket) in ``autotune.json``
beside the NVRTC module cache.
"""
from __future__ import annotations

import json
import math
import os
import threading

import numpy as np

from . import program

# (massive variants (stages, blocks), photon variants (stages, blocks)); the
# NVRTC step module compiles exactly these
VARIANTS = {
    ("fp64", "rs"): ([(2, 2), (3, 2)], [(3, 3), (2, 3), (3, 2)]),
    ("fp64", "od"): ([(2, 2), (3, 2)], [(3, 3), (2, 3)]),
    ("fp32", "rs"): ([(2, 3), (3, 3), (3, 2), (4, 2), (2, 4)], [(3, 4), (2, 4), (3, 3), (4, 3)]),
    ("fp32", "od"): ([(2, 3), (3, 2)], [(3, 4), (3, 3)]),
}
DEFAULT = {
    ("fp64", "rs"): ((2, 2), (3, 2)),
    ("fp64", "od"): ((2, 2), (3, 3)),
    ("fp32", "rs"): ((2, 4), (3, 3)),
    ("fp32", "od"): ((2, 3), (3, 3)),
}

_lock = threading.Lock()


def _cache_path():
    return os.path.join(program.CACHE, "autotune.json")


def _load():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(d):
    os.makedirs(program.CACHE, exist_ok=True)
    tmp = _cache_path() + f".{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, _cache_path())


def cache_key(sim) -> str:
    import torch
    name = torch.cuda.get_device_name()
    n = sum(p.N_buffered for p in sim.all_particles)
    bucket = int(math.log2(max(n, 1)))
    mix = "-".join(("g" if p.m == 0 else "e") for p in sim.all_particles)
    return f"{name}|{sim.form}|{sim.qed_method}|{sim.fields.structure()}|{mix}|2^{bucket}"


def _sample_sim(sim, sample):
    """A copy of the simulation's current state, at most `sample` alive
    particles per species, same fields / form / QED method."""
    from .particles import Particles, SpinParticles
    from .simulation import Simulation
    import torch
    copies = {}
    for p in sim.all_particles:
        p._to_gpu()
        pr = p._d("_to_be_pruned")[: p.N_buffered]
        keep = torch.nonzero(pr == 0).flatten()[:sample]
        props = [p._d(k)[keep].cpu().numpy() for k in ("x", "y", "z", "ux", "uy", "uz")]
        n = int(keep.numel())
        q = round(p.q / 1.602176634e-19)
        m = 0 if p.m == 0 else 1
        if "sx" in p.attrs:
            props += [p._d(k)[keep].cpu().numpy() for k in ("sx", "sy", "sz")]
            c = SpinParticles(p.name, q, m, N=n, props=props if n else None, RR=p.RR, ae=p.ae, push=p.push)
        else:
            c = Particles(p.name, q, m, N=n, props=props if n else None, RR=p.RR, push=p.push)
        copies[id(p)] = c
    for p in sim.all_particles:
        c = copies[id(p)]
        if p.radiating:
            c.set_photon(copies[id(p.photon_ref())])
        if p.bw:
            c.set_pair(copies[id(p.bw_electron_ref())], copies[id(p.bw_positron_ref())])
    s = Simulation(*[copies[id(p)] for p in sim.all_particles], dt=sim.dt, fields=sim.fields, print_every=None,
                   photon_threshold=sim.photon_threshold, seed=sim.seed, form=sim.form, graph_chunk=0)
    s.t = sim.t
    s.step = sim.step
    return s


def measure(sim, variants=None, steps: int = 3):
    """Median kernel times [ms] on `sim`'s current state: ({massive variant:
    ms}, {photon variant: ms}).  Advances `sim` by
    (len(massive) + len(photon)) * steps steps."""
    mv, pv = variants or VARIANTS[(sim.form, sim.qed_method)]
    tm, tp = {}, {}
    m0, p0 = (sim.m_stages, sim.min_blocks), (sim.p_stages, sim.p_min_blocks)
    for v in mv:
        sim.set_kernel(massive=v, photon=p0)
        ms, _, _ = sim.time_step_kernel(steps)
        tm[tuple(v)] = float(np.median([m[0] for m in ms]))
    for v in pv:
        sim.set_kernel(massive=m0, photon=v)
        ms, _, _ = sim.time_step_kernel(steps)
        tp[tuple(v)] = float(np.median([m[1] for m in ms]))
    return tm, tp


def tune(sim, sample: int = 2_000_000, steps: int = 3, use_cache: bool = True):
    """Select the fastest massive- and photon-kernel variants for `sim` (see
    the module doc).  Returns ((massive, photon), times), times a dict
    'm<stages>_b<blocks>' / 'p<stages>_b<blocks>' -> ms."""
    key = cache_key(sim)
    with _lock:
        cache = _load() if use_cache else {}
        if key in cache and "best" in cache[key] and len(cache[key]["best"]) == 2:
            m, p = (tuple(v) for v in cache[key]["best"])
            sim.set_kernel(massive=m, photon=p)
            return (m, p), cache[key].get("ms", {})
    s = _sample_sim(sim, sample)
    try:
        tm, tp = measure(s, steps=steps)
    finally:
        s.finish()
    # a kernel with no work (0 ms everywhere) keeps the default
    m = min(tm, key=tm.get) if any(tm.values()) else (sim.m_stages, sim.min_blocks)
    p = min(tp, key=tp.get) if any(tp.values()) else (sim.p_stages, sim.p_min_blocks)
    sim.set_kernel(massive=m, photon=p)
    times = {**{f"m{a}_b{b}": v for (a, b), v in tm.items()}, **{f"p{a}_b{b}": v for (a, b), v in tp.items()}}
    if use_cache:
        with _lock:
            cache = _load()
            cache[key] = {"best": [list(m), list(p)], "ms": times}
            _store(cache)
    return (m, p), times
