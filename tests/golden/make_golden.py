#!/usr/bin/env python
"""Generate the golden fixtures in tests/golden/ from the reference package.

Runs only where the reference source is available (default
/root/reference, override with SFP_REFERENCE); the fixtures it writes are
committed so that tests never need the reference at run time.  Uses the
test-only h5py stand-in in tests/golden/_h5shim to load the reference's
shipped rate table.

What is recorded, and from which reference code:

* ref_tables.npz   -- the shipped Airy tables (qed/rejection_sampling_tables.h5)
                      and the 256 golden total-rate values of tests/test_tables.py
* ref_pushers.npz  -- cpu.py kernels on seeded random inputs
* ref_fields.npz   -- fields.py presets and Fields.__add__ at seeded points
* ref_user_fields.npz, ref_sim_user_sum.npz -- user callables (tests/user_fields.py)
                      through Fields(callable) and Fields.__add__, and a whole run
* ref_rates.npz    -- photon/pair_prob_rate_from_table on a (chi, delta) grid
* ref_rs_events.npz-- rejection samplers (their Python bodies, .py_func) fed the
                      Philox draws of the oracle through a stand-in `random`
* ref_sim_*.npz    -- whole Simulation.start runs with those samplers injected,
                      so orchestration order, appends, recoil and child pushes
                      are the reference's own
* ref_od.npz       -- optical-depth table rows from the reference generators and
                      the inverse-CDF / rate interpolation (py_func) on them, for
                      the photon rows and the finite pair rows
* ref_stats.json   -- un-injected reference runs (Numba's own RNG) for
                      statistical comparison

Usage:  python tests/golden/make_golden.py [--only NAME ...]
"""
from __future__ import annotations

import argparse
import ast
import json
import math
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("SFP_REFERENCE", "/root/reference")

os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "sfp_golden_numba"))
sys.path.insert(0, os.path.join(HERE, "_h5shim"))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(REPO, "oracle"))

import oracle as orc  # noqa: E402

um, fs = 1e-6, 1e-15


def out(name):
    return os.path.join(HERE, name)


# ---------------------------------------------------------------------------
def gen_tables():
    from sfparticles.qed import rejection_sampling_tables as rst
    src = open(os.path.join(REF, "tests", "test_tables.py")).read()
    vals = None
    for node in ast.walk(ast.parse(src)):
        if isinstance(node, ast.Assign) and getattr(node.targets[0], "id", "") == "prob_rate_table":
            if isinstance(node.value, ast.List):
                vals = [ast.literal_eval(e) for e in node.value.elts]
    assert vals is not None and len(vals) == 256
    np.savez(out("ref_tables.npz"), int_Ai=rst._int_Ai_table, Aip=rst._Aip_table, z_N=int(rst._z_N),
             z_range=np.asarray(rst._z_range, dtype=float), z_delta=float(rst._z_delta),
             test_tables_rate=np.asarray(vals), test_tables_chi_range=np.array([-3.0, 2.0]), test_tables_chi_N=256)


# ---------------------------------------------------------------------------
def gen_pushers():
    from scipy.constants import e
    from sfparticles import cpu
    rng = np.random.default_rng(20240601)
    N = 512
    res = {}

    def mom(n):
        mag = 10 ** rng.uniform(-2, 4.3, n)
        d = rng.normal(size=(3, n))
        d /= np.linalg.norm(d, axis=0)
        return mag * d

    u = mom(N)
    E = rng.normal(size=(3, N)) * 10 ** rng.uniform(11, 15, N)
    B = rng.normal(size=(3, N)) * 10 ** rng.uniform(3, 7, N)
    pr = rng.random(N) < 0.1
    dt = 3.3e-17
    res.update(u=u, E=E, B=B, pruned=pr, dt=dt)
    for q, tag in ((-e, "m"), (e, "p")):
        ux, uy, uz = [a.copy() for a in u]
        ig = 1 / np.sqrt(1 + ux ** 2 + uy ** 2 + uz ** 2)
        cpu.boris(ux, uy, uz, ig, *E, *B, q, N, pr, dt)
        res[f"boris_{tag}"] = np.stack([ux, uy, uz, ig])
    s = rng.normal(size=(3, N))
    s /= np.linalg.norm(s, axis=0)
    res["s"] = s
    for ae in (1.14e-3, 0.3):
        ux, uy, uz = [a.copy() for a in u]
        sx, sy, sz = [a.copy() for a in s]
        ig = 1 / np.sqrt(1 + ux ** 2 + uy ** 2 + uz ** 2)
        cpu.boris_tbmt(ux, uy, uz, ig, sx, sy, sz, *E, *B, -e, ae, N, pr, dt)
        res[f"tbmt_{ae}"] = np.stack([ux, uy, uz, ig, sx, sy, sz])
    chi = 10 ** rng.uniform(-3, 1.3, N)
    res["chi_in"] = chi
    for fn, tag in ((cpu.LL_push, "LL"), (cpu.CLL_push, "CLL")):
        ux, uy, uz = [a.copy() for a in u]
        ig = 1 / np.sqrt(1 + ux ** 2 + uy ** 2 + uz ** 2)
        fn(ux, uy, uz, ig, chi, N, pr, dt)
        res[tag] = np.stack([ux, uy, uz, ig])
    ux, uy, uz = [a.copy() for a in u]
    ig = 1 / np.sqrt(1 + ux ** 2 + uy ** 2 + uz ** 2)
    res["ig_in"] = ig
    chi_o = np.zeros(N)
    cpu.update_chi(*E, *B, ux, uy, uz, ig, chi_o, N, pr)
    res["update_chi"] = chi_o
    x = rng.normal(size=(3, N)) * 1e-5
    res["x"] = x
    xx, yy, zz = [a.copy() for a in x]
    cpu.push_position(xx, yy, zz, ux, uy, uz, ig, N, pr, dt)
    res["push_position"] = np.stack([xx, yy, zz])
    ev = rng.random(N) < 0.3
    ev &= ~pr
    delta = rng.random(N)
    res["event"] = ev
    res["delta"] = delta
    ux, uy, uz = [a.copy() for a in u]
    ig2 = ig.copy()
    cpu.photon_recoil(ux, uy, uz, ig2, ev, delta, N, pr)
    res["photon_recoil"] = np.stack([ux, uy, uz, ig2])
    ev2 = ev.copy()
    cpu.pick_hard_photon(ev2, delta, ig, 2.0, N)
    res["pick_hard_photon"] = ev2
    n_ev = int(cpu.bool_sum(ev, N))
    res["bool_sum"] = n_ev
    idx = cpu.find_event_index(ev, n_ev, N)
    res["find_event_index"] = idx
    M0 = 7
    dst = [np.zeros(M0 + n_ev) for _ in range(7)]
    dpr = np.ones(M0 + n_ev, dtype=bool)
    cpu.create_photon(*x, *u, *dst[:6], dst[6], dpr, idx, delta, M0, n_ev)
    res["create_photon"] = np.stack(dst)
    res["create_photon_pruned"] = dpr
    for inv in (False, True):
        dst = [np.zeros(M0 + n_ev) for _ in range(7)]
        dpr = np.ones(M0 + n_ev, dtype=bool)
        spr = pr.copy()
        cpu.create_pair(*x, *u, spr, *dst[:6], dst[6], dpr, idx, delta, M0, n_ev, inv)
        res[f"create_pair_{int(inv)}"] = np.stack(dst)
        res[f"create_pair_{int(inv)}_pruned"] = dpr
        res[f"create_pair_{int(inv)}_src_pruned"] = spr
    np.savez(out("ref_pushers.npz"), **res)


# ---------------------------------------------------------------------------
FIELD_CASES = [
    ("static_field", dict(Ex=1.5e12, Ey=-3e11, Ez=2e10, Bx=1e3, By=-4e2, Bz=7e3)),
    ("simple_laser_pulse", dict(a0=50.0, w0=3e-6, ctau=6e-6, t_order=2, direction=1, x0=-5e-6, wavelength=0.8e-6,
                                pol_angle=0.3, cep=0.2)),
    ("simple_laser_pulse", dict(a0=700.0, w0=5e-6, ctau=5e-6, t_order=4, direction=-1, x0=15e-6)),
    ("gaussian_laser_pulse", dict(a0=50.0, w0=3e-6, ctau=6.366e-6, direction=-1, x0=12e-6)),
    ("gaussian_laser_pulse", dict(a0=200.0, w0=3e-6, ctau=6.366e-6, direction=1, x0=-8e-6, l0=1.0e-6,
                                  pol_angle=math.pi / 2, cep=math.pi / 2)),
    ("focused_gaussian_laser_pulse", dict(a0=100.0, w0=2e-6, ctau=5e-6, direction=1, xfoc=1e-6, x0=-3e-6,
                                          pol_angle=0.7, cep=0.1)),
    ("focused_gaussian_laser_pulse", dict(a0=30.0, w0=1.5e-6, ctau=4e-6, direction=-1, xfoc=-2e-6, x0=6e-6)),
]
# sums (indices into FIELD_CASES), as nested pairs
FIELD_SUMS = [[3, 4], [[1, 3], 0], [5, [6, 2]]]


def _build_ref_field(fields_mod, spec):
    if isinstance(spec, int):
        name, kw = FIELD_CASES[spec]
        return getattr(fields_mod, name)(**kw)
    return _build_ref_field(fields_mod, spec[0]) + _build_ref_field(fields_mod, spec[1])


def field_points(rng, n, x0, direction, t_span=40 * fs):
    t = rng.uniform(-t_span, t_span, n)
    x = x0 + direction * 299792458.0 * t + rng.normal(0, 5e-6, n)
    x = np.where(np.abs(x) < 1e-9, 1e-9, x)
    y = rng.normal(0, 2e-6, n)
    z = rng.normal(0, 2e-6, n)
    return x, y, z, t


def gen_fields():
    from sfparticles import fields as F
    rng = np.random.default_rng(7)
    n = 256
    res = {"cases": json.dumps(FIELD_CASES), "sums": json.dumps(FIELD_SUMS)}
    for i, spec in enumerate(list(range(len(FIELD_CASES))) + FIELD_SUMS):
        fld = _build_ref_field(F, spec)
        kw = FIELD_CASES[spec if isinstance(spec, int) else 3][1]
        x, y, z, t = field_points(rng, n, kw.get("x0", 0.0), kw.get("direction", 1))
        outv = np.zeros((6, n))
        for j in range(n):  # t varies per point; the launcher takes one t
            o = [np.zeros(1) for _ in range(6)]
            fld.field_func(x[j:j + 1], y[j:j + 1], z[j:j + 1], float(t[j]), 1, np.zeros(1, dtype=bool), *o)
            outv[:, j] = [a[0] for a in o]
        res[f"pts_{i}"] = np.stack([x, y, z, t])
        res[f"out_{i}"] = outv
    np.savez(out("ref_fields.npz"), **res)


def gen_user_fields():
    """User callables (tests/user_fields.py) through the reference's
    Fields(callable) (fields.py:11-50), alone and summed with a preset
    (Fields.__add__, fields.py:52-61) at seeded points, and one whole
    deterministic Simulation.start in the summed field."""
    import sfparticles
    from sfparticles import fields as F
    from sfparticles.particles import RadiationReactionType as RRT
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import user_fields as U
    rng = np.random.default_rng(11)
    n = 256
    cases = {"gaussian": ("gaussian", U.GAUSSIAN, False), "gaussian_plus_static": ("gaussian", U.GAUSSIAN, True),
             "mixed": ("mixed", U.MIXED, False), "lambda": ("lambda", {}, False)}
    res = {"cases": json.dumps(cases), "static": json.dumps(U.STATIC)}
    for name, (builder, kw, plus_static) in cases.items():
        fld = F.Fields(U.BUILDERS[builder](**kw))
        if plus_static:
            fld = fld + F.static_field(**U.STATIC)
        x, y, z, t = field_points(rng, n, kw.get("x0", 0.0), kw.get("direction", 1))
        if builder == "mixed":
            x = rng.uniform(-1.5 * kw["L"], 1.5 * kw["L"], n)
        outv = np.zeros((6, n))
        for j in range(n):
            o = [np.zeros(1) for _ in range(6)]
            fld.field_func(x[j:j + 1], y[j:j + 1], z[j:j + 1], float(t[j]), 1, np.zeros(1, dtype=bool), *o)
            outv[:, j] = [a[0] for a in o]
        res[f"pts_{name}"] = np.stack([x, y, z, t])
        res[f"out_{name}"] = outv
    np.savez(out("ref_user_fields.npz"), **res)
    # whole run: 32 electrons with Landau-Lifshitz through the user Gaussian + a static field
    case = dict(kind="det", n_e=32, gamma0=2000.0, a0=U.GAUSSIAN["a0"], w0=U.GAUSSIAN["w0"],
                ctau=U.GAUSSIAN["ctau"], dt_T0=1 / 50, steps=300, field="user", lead=U.GAUSSIAN["x0"], spin=False,
                rr="LL", pairs=False, seed=0, thr=2.0)
    rng = np.random.default_rng(sum(map(ord, "user_sum")))
    props, spin = sim_initial(case, rng)
    fld = F.Fields(U.gaussian_callable(**U.GAUSSIAN)) + F.static_field(**U.STATIC)
    ele = sfparticles.Particles("ele", -1, 1, N=case["n_e"], props=tuple(np.array(a) for a in props), RR=RRT.LL)
    dt = 0.8e-6 / 299792458.0 * case["dt_T0"]
    sim = sfparticles.Simulation(ele, dt=dt, fields=fld, print_every=None, photon_threshold=case["thr"])
    sim.start(case["steps"])
    terms = [["user:gaussian", U.GAUSSIAN], ["static_field", U.STATIC]]
    np.savez(out("ref_sim_user_sum.npz"), case=json.dumps(case), field_terms=json.dumps(terms),
             field_comb=json.dumps([0, 1]), dt=dt, init=np.stack(props), spin_init=np.stack(spin),
             s0_state=np.stack([getattr(ele, k) for k in ("x", "y", "z", "ux", "uy", "uz")]), s0_name="ele",
             n_species=1)


# ---------------------------------------------------------------------------
def gen_rates():
    from sfparticles.qed import rejection_sampling as rs
    from sfparticles.qed import rejection_sampling_tables as rst
    rng = np.random.default_rng(11)
    chi = 10 ** rng.uniform(-3, 2.5, 4000)
    delta = np.concatenate([rng.random(2000) ** 3, rng.random(2000)])
    ph = np.array([rs.photon_prob_rate_from_table(c, d, rst._int_Ai_table, rst._Aip_table) for c, d in zip(chi, delta)])
    pa = np.array([rs.pair_prob_rate_from_table(c, d, rst._int_Ai_table, rst._Aip_table) for c, d in zip(chi, delta)])
    # photon z beyond the table is undefined in the reference (reads past the end)
    z_ph = ((delta * chi) / chi / (chi - delta * chi)) ** (2 / 3)
    np.savez(out("ref_rates.npz"), chi=chi, delta=delta, photon=ph, pair=pa, photon_valid=z_ph <= 100.0)


# ---------------------------------------------------------------------------
class _QueueRandom:
    """Stands in for the `random` module inside the reference samplers."""

    def __init__(self, draws):
        self.d = draws
        self.i = 0

    def rand(self, n=None):
        if n is None:
            v = self.d[self.i]
            self.i += 1
            return v
        v = np.asarray(self.d[self.i:self.i + n])
        self.i += n
        return v


class _NP:
    """Stands in for the `np` module inside the reference's _bisect_interp:
    np.random.rand() serves the given draws, everything else is numpy."""

    def __init__(self, r):
        self.random = _QueueRandom(r)

    def __getattr__(self, k):
        return getattr(np, k)


def run_rs_injected(photon, inv_gamma, chi, dt, N, pruned, event, delta, seed, stream, step):
    """Call the reference sampler body with the oracle's keyed Philox draws."""
    from sfparticles.qed import rejection_sampling as rs
    live = np.nonzero((~pruned[:N]) & (chi[:N] != 0.0))[0]
    draws = orc.uniform2(seed, stream, step, 0, live).reshape(-1)
    fn = rs.photon_from_rejection_sampling if photon else rs.pair_from_rejection_sampling
    saved = rs.random
    rs.random = _QueueRandom(draws)
    try:
        fn.py_func(inv_gamma, chi, dt, N, pruned, event, delta)
    finally:
        used = rs.random.i
        rs.random = saved
    assert used == draws.size


def gen_rs_events():
    rng = np.random.default_rng(5)
    N = 4096
    res = {}
    for photon in (True, False):
        ig = 10 ** rng.uniform(-4, -2, N)
        chi = 10 ** rng.uniform(-1, 1.3, N)
        chi[rng.random(N) < 0.05] = 0.0
        pr = rng.random(N) < 0.1
        ev = np.zeros(N, dtype=bool)
        de = np.full(N, -1.0)
        dt = 3e-13 if photon else 1e-12
        seed, stream, step = 0x1234_5678_9ABC, 3 if photon else 5, 17
        run_rs_injected(photon, ig, chi, dt, N, pr, ev, de, seed, stream, step)
        tag = "photon" if photon else "pair"
        res.update({f"{tag}_ig": ig, f"{tag}_chi": chi, f"{tag}_pruned": pr, f"{tag}_dt": dt,
                    f"{tag}_key": np.array([seed, stream, step], dtype=np.uint64),
                    f"{tag}_event": ev, f"{tag}_delta": de})
    np.savez(out("ref_rs_events.npz"), **res)


# ---------------------------------------------------------------------------
SIM_CASES = {
    # laser-beam collision with photon emission and pair creation
    "cascade": dict(kind="rs", n_e=48, gamma0=4000.0, a0=600.0, w0=3e-6, ctau=5e-6, dt_T0=1 / 100, steps=260,
                    field="gaussian", lead=1.2e-6, spin=False, rr="PHOTON", pairs=True, seed=99, thr=2.0),
    # emission with TBMT spin (no pairs: the reference gives pair children no spin)
    "spin_photon": dict(kind="rs", n_e=32, gamma0=3000.0, a0=300.0, w0=3e-6, ctau=5e-6, dt_T0=1 / 100, steps=200,
                        field="gaussian", lead=1.0e-6, spin=True, rr="PHOTON", pairs=False, seed=7, thr=1.0),
    # deterministic Landau-Lifshitz + spin, no emission
    "spin_LL": dict(kind="det", n_e=32, gamma0=2000.0, a0=200.0, w0=3e-6, ctau=5e-6, dt_T0=1 / 50, steps=300,
                    field="gaussian", lead=3e-6, spin=True, rr="LL", pairs=False, seed=0, thr=2.0),
    # spin with RR=CLL: the reference's spin push has no CLL branch (particles.py:596-604),
    # so this is the plain Boris-TBMT push
    "spin_CLL": dict(kind="det", n_e=32, gamma0=2000.0, a0=200.0, w0=3e-6, ctau=5e-6, dt_T0=1 / 50, steps=300,
                     field="gaussian", lead=3e-6, spin=True, rr="CLL", pairs=False, seed=0, thr=2.0),
    # Landau-Lifshitz without spin, through the plane-wave-like pulse (Gaussian in time)
    "simple_LL": dict(kind="det", n_e=32, gamma0=2000.0, a0=150.0, w0=3e-6, ctau=5e-6, dt_T0=1 / 50, steps=300,
                      field="simple", t_order=2, lead=3e-6, spin=False, rr="LL", pairs=False, seed=0, thr=2.0),
    # emission off through the same pulse with a fourth-order temporal envelope
    "simple_t4": dict(kind="det", n_e=32, gamma0=500.0, a0=20.0, w0=3e-6, ctau=6e-6, dt_T0=1 / 50, steps=300,
                      field="simple", t_order=4, lead=4e-6, spin=False, rr="NONE", pairs=False, seed=0, thr=2.0),
    # deterministic quantum-corrected LL with a focused pulse
    "CLL_focused": dict(kind="det", n_e=32, gamma0=1500.0, a0=150.0, w0=2.5e-6, ctau=5e-6, dt_T0=1 / 50, steps=300,
                        field="focused", lead=3e-6, spin=False, rr="CLL", pairs=False, seed=0, thr=2.0),
    # emission off: the plain Boris push through a sum of two pulses
    "push_only": dict(kind="det", n_e=64, gamma0=500.0, a0=20.0, w0=3e-6, ctau=6e-6, dt_T0=1 / 50, steps=400,
                      field="cp", lead=4e-6, spin=False, rr="NONE", pairs=False, seed=0, thr=2.0),
}


def sim_initial(case, rng):
    n = case["n_e"]
    g = case["gamma0"] * (1 + 0.01 * rng.normal(size=n))
    x = rng.normal(-case["lead"], 0.5e-6, n)
    y = rng.normal(0, 0.5e-6, n)
    z = rng.normal(0, 0.5e-6, n)
    ux = np.sqrt(g ** 2 - 1)
    s = rng.normal(size=(3, n))
    s /= np.linalg.norm(s, axis=0)
    return [x, y, z, ux, np.zeros(n), np.zeros(n)], list(s)


def sim_field_spec(case):
    """(name, kwargs) list and combination for the case's field."""
    a0, w0, ctau = case["a0"], case["w0"], case["ctau"]
    x0 = case["lead"]
    if case["field"] == "gaussian":
        return [("gaussian_laser_pulse", dict(a0=a0, w0=w0, ctau=ctau, direction=-1, x0=x0))], 0
    if case["field"] == "focused":
        return [("focused_gaussian_laser_pulse", dict(a0=a0, w0=w0, ctau=ctau, direction=-1, x0=x0))], 0
    if case["field"] == "cp":
        a = a0 / math.sqrt(2)
        return [("gaussian_laser_pulse", dict(a0=a, w0=w0, ctau=ctau, direction=-1, x0=x0, pol_angle=0.0)),
                ("gaussian_laser_pulse", dict(a0=a, w0=w0, ctau=ctau, direction=-1, x0=x0, pol_angle=math.pi / 2,
                                              cep=math.pi / 2))], [0, 1]
    if case["field"] == "simple":
        return [("simple_laser_pulse", dict(a0=a0, w0=w0, ctau=ctau, t_order=case["t_order"], direction=-1,
                                            x0=x0))], 0
    raise ValueError(case["field"])


def gen_sims(names=None):
    import sfparticles
    from sfparticles import fields as F
    from sfparticles import particles as P
    from sfparticles.particles import RadiationReactionType as RRT

    saved_ph, saved_pair = P.Particles._photon_event, P.Particles._pair_event
    for name, case in SIM_CASES.items():
        if names and name not in names:
            continue
        rng = np.random.default_rng(sum(map(ord, name)))
        props, spin = sim_initial(case, rng)
        terms, comb = sim_field_spec(case)
        flds = [getattr(F, nm)(**kw) for nm, kw in terms]
        fld = flds[0] if comb == 0 else flds[0] + flds[1]
        rr = getattr(RRT, case["rr"])
        n = case["n_e"]
        if case["spin"]:
            ele = sfparticles.SpinParticles("ele", -1, 1, N=n, RR=rr)
            ele.x, ele.y, ele.z, ele.ux, ele.uy, ele.uz = [np.array(a) for a in props]
            ele.inv_gamma = 1 / np.sqrt(1 + ele.ux ** 2 + ele.uy ** 2 + ele.uz ** 2)
            ele.sx, ele.sy, ele.sz = [np.array(a) for a in spin]
        else:
            ele = sfparticles.Particles("ele", -1, 1, N=n, props=tuple(np.array(a) for a in props), RR=rr)
        species = [ele]
        if case["rr"] == "PHOTON":
            pho = sfparticles.Particles("pho", 0, 0)
            ele.set_photon(pho)
            species.append(pho)
            if case["pairs"]:
                pos = sfparticles.Particles("pos", 1, 1)
                pos.set_photon(pho)
                pho.set_pair(ele, pos)
                species = [ele, pos, pho]
        T0 = 0.8e-6 / 299792458.0
        dt = T0 * case["dt_T0"]
        sim = sfparticles.Simulation(*species, dt=dt, fields=fld, print_every=None,
                                     photon_threshold=case["thr"])
        seed = case["seed"]
        stream_of = {id(p): i for i, p in enumerate(species)}

        def ph_event(self, dt_):
            run_rs_injected(True, self.inv_gamma, self.chi, dt_, self.N_buffered, self._to_be_pruned, self.event,
                            self.photon_delta, seed, stream_of[id(self)], sim.step)
            return self.event, self.photon_delta

        def pair_event(self, dt_):
            run_rs_injected(False, self.inv_gamma, self.chi, dt_, self.N_buffered, self._to_be_pruned, self.event,
                            self.pair_delta, seed, stream_of[id(self)], sim.step)
            return self.event, self.pair_delta

        P.Particles._photon_event, P.Particles._pair_event = ph_event, pair_event
        t0 = time.time()
        try:
            sim.start(case["steps"])
        finally:
            P.Particles._photon_event, P.Particles._pair_event = saved_ph, saved_pair
        res = {"case": json.dumps(case), "field_terms": json.dumps(terms), "field_comb": json.dumps(comb),
               "dt": dt, "init": np.stack(props), "spin_init": np.stack(spin)}
        for i, p in enumerate(species):
            keys = ["x", "y", "z", "ux", "uy", "uz"] + (["sx", "sy", "sz"] if hasattr(p, "sx") else [])
            res[f"s{i}_state"] = np.stack([getattr(p, k) for k in keys])
            res[f"s{i}_name"] = p.name
        res["n_species"] = len(species)
        np.savez(out(f"ref_sim_{name}.npz"), **res)
        print(f"  sim {name}: {[p.N_buffered for p in species]} in {time.time() - t0:.1f}s")


# ---------------------------------------------------------------------------
def gen_od():
    """Reference OD generators on a subset of rows, and its sampling pieces."""
    from sfparticles.qed import optical_depth_tables as odt
    chi_N, lo, hi, delta_N, ldm = 256, -3.0, 2.0, 1024, -6
    chi_all = np.logspace(lo, hi, chi_N)
    rows = np.arange(0, chi_N, 15)
    t0 = time.time()
    ph_tot = np.array([odt.integral_photon_prob_over_delta(c) for c in chi_all[rows]])
    pa_tot = np.array([odt.integral_pair_prob_over_delta(c) for c in chi_all[rows]])
    ph_cum = np.stack([odt.integral_photon_prob_along_delta(c, delta_N, ldm) for c in chi_all[rows]])
    pa_cum = np.stack([odt.integral_pair_prob_along_delta(c, delta_N, ldm) for c in chi_all[rows]])
    print(f"  od rows: {time.time() - t0:.1f}s")
    # sampling pieces on a small synthetic table (the reference's functions are
    # generic in the table contents): rows = the generated subset
    sub_N = len(rows)
    sub_delta = (hi - lo) / (chi_N - 1) * 15
    g = odt.__dict__
    g.update(_chi_N=sub_N, _log_chi_range=np.array([lo, lo + sub_delta * (sub_N - 1)]), _log_chi_delta=sub_delta,
             _delta_N=delta_N, _log_delta_range=np.array([ldm, 0.0]), _log_delta_delta=(0 - ldm) / (delta_N - 1))
    rng = np.random.default_rng(3)
    chis = 10 ** rng.uniform(lo, lo + sub_delta * (sub_N - 1) - 1e-9, 2000)
    rs_ = rng.random(2000)

    interp = np.array([odt._linear_interp1d.py_func(c, ph_tot) for c in chis])
    bis = []
    saved = g["np"]
    for c, r in zip(chis, rs_):
        g["np"] = _NP([r])
        try:
            bis.append(odt._bisect_interp.py_func(c, ph_cum))
        finally:
            g["np"] = saved
    # the same pieces on the pair rows, at chi whose two bracketing rows are
    # finite (the reference's rows below chi_gamma ~ 0.43 are NaN)
    first = int(np.nonzero(np.isfinite(pa_cum).all(axis=1))[0][0])
    chis_p = 10 ** rng.uniform(lo + sub_delta * first, lo + sub_delta * (sub_N - 1) - 1e-9, 1000)
    rs_p = rng.random(1000)
    interp_p = np.array([odt._linear_interp1d.py_func(c, pa_tot) for c in chis_p])
    bis_p = []
    for c, r in zip(chis_p, rs_p):
        g["np"] = _NP([r])
        try:
            bis_p.append(odt._bisect_interp.py_func(c, pa_cum))
        finally:
            g["np"] = saved
    np.savez(out("ref_od.npz"), chi_rows=chi_all[rows], rows=rows, photon_total=ph_tot, pair_total=pa_tot,
             photon_cum=ph_cum, pair_cum=pa_cum, sub_log_chi_min=lo, sub_log_chi_delta=sub_delta,
             log_delta_min=float(ldm), log_delta_delta=(0 - ldm) / (delta_N - 1),
             q_chi=chis, q_r=rs_, q_interp=interp, q_bisect=np.array(bis),
             q_chi_pair=chis_p, q_r_pair=rs_p, q_interp_pair=interp_p, q_bisect_pair=np.array(bis_p))


# ---------------------------------------------------------------------------
# Whole optical-depth runs.  The reference picks the method when it is
# imported (qed/__init__.py), so they run in a child process with
# SFPARTICLES_OPTICAL_DEPTH=1, from a scratch copy of the reference package
# in which the rate tables are written as optical_depth_tables.h5 (served by
# the h5py stand-in).  The tables are the reference grid (rows 0-255,
# log10 chi in [-3, 2]) of sfparticles_b200's shipped tables, which equal the
# reference generator's rows wherever those are finite.  Both cases keep chi
# below 100 (the reference's interpolation reads past its last row above it)
# and give no appended particle an optical depth, where the reference copies
# stale values cyclically (numpy.resize) and the oracle starts at zero.
OD_SIM_CASES = {
    # electrons emit by optical depth, with recoil, in a laser pulse; photons make no pairs
    "od_emission": dict(kind="od", n_e=48, gamma0=4000.0, a0=600.0, w0=3e-6, ctau=5e-6, dt_T0=1 / 100, steps=260,
                        field="gaussian", lead=1.2e-6, seed=31, thr=2.0),
    # the same with Thomas-BMT spin (the avalanche's electrons)
    "od_spin_emission": dict(kind="od", n_e=32, gamma0=3000.0, a0=300.0, w0=3e-6, ctau=5e-6, dt_T0=1 / 100,
                             steps=200, field="gaussian", lead=1.0e-6, seed=33, thr=1.0, spin=True),
    # photons convert to pairs by optical depth in a static field; the pairs do not radiate
    "od_pairs": dict(kind="od", n_g=2000, gamma_lo=3000.0, gamma_hi=30000.0, chi_ref=1.5, gamma_ref=1e4,
                     dt=1.5e-15, steps=40, seed=32, thr=2.0),
}


def _od_injected(kind, sim, species, seed):
    """update_tau_e / update_tau_gamma of the reference (their Python bodies,
    one particle per call) fed the oracle's keyed draws: purpose 1 gives the
    reset draw (used when tau == 0) and the draw after an event, purpose 2
    the inverse-CDF draw of _bisect_interp."""
    from sfparticles.qed import optical_depth as od
    from sfparticles.qed import optical_depth_tables as odt
    fn = (od.update_tau_e if kind == "e" else od.update_tau_gamma).py_func
    name = "photon_delta_from_chi_delta_table" if kind == "e" else "pair_delta_from_chi_delta_table"
    table = odt._integral_photon_prob_along_delta if kind == "e" else odt._integral_pair_prob_along_delta
    G, T = fn.__globals__, odt.__dict__

    def run(tau, inv_gamma, chi, dt, N, pruned, event, delta):
        stream = next(i for i, p in enumerate(species) if getattr(p, "tau", None) is tau)
        slots = np.arange(N)
        ra = orc.uniform2(seed, stream, sim.step, 1, slots)
        rb = orc.uniform2(seed, stream, sim.step, 2, slots)
        saved = G["random"], G[name], T["np"]

        def draw(c, r):
            T["np"] = _NP([r])
            try:
                return odt._bisect_interp.py_func(c, table)
            finally:
                T["np"] = saved[2]

        try:
            for ip in range(N):
                G["random"] = _QueueRandom(np.array(([ra[ip, 0]] if tau[ip] == 0.0 else []) + [ra[ip, 1]]))
                G[name] = lambda c, r=rb[ip, 0]: draw(c, r)
                fn(tau[ip:ip + 1], inv_gamma[ip:ip + 1], chi[ip:ip + 1], dt, 1, pruned[ip:ip + 1],
                   event[ip:ip + 1], delta[ip:ip + 1])
        finally:
            G["random"], G[name] = saved[0], saved[1]

    return run


def od_pairs_initial(case, rng):
    """Photons along +x at the origin, energies log-uniform."""
    n = case["n_g"]
    g = np.exp(rng.uniform(math.log(case["gamma_lo"]), math.log(case["gamma_hi"]), n))
    return [np.zeros(n), np.zeros(n), np.zeros(n), g, np.zeros(n), np.zeros(n)]


def od_pairs_bz(case):
    """Static B_z that gives chi_ref to a photon of gamma_ref moving along x."""
    from scipy.constants import c, e, hbar, m_e
    return case["chi_ref"] * m_e ** 2 * c ** 2 / e / hbar / case["gamma_ref"]


def _od_sims_child():
    import sfparticles
    from sfparticles import fields as F
    from sfparticles import particles as P
    assert P._use_optical_depth
    saved = P.update_tau_e, P.update_tau_gamma
    for name, case in OD_SIM_CASES.items():
        rng = np.random.default_rng(sum(map(ord, name)))
        seed = case["seed"]
        spin = None
        if "n_e" in case:
            props, spin = sim_initial(case, rng)
            terms, comb = sim_field_spec(case)
            fld = getattr(F, terms[0][0])(**terms[0][1])
            if case.get("spin"):
                # SpinParticles cannot take props in the reference: set the state after construction
                ele = sfparticles.SpinParticles("ele", -1, 1, N=case["n_e"])
                ele.x, ele.y, ele.z, ele.ux, ele.uy, ele.uz = [np.array(a) for a in props]
                ele.inv_gamma = 1 / np.sqrt(1 + ele.ux ** 2 + ele.uy ** 2 + ele.uz ** 2)
                ele.sx, ele.sy, ele.sz = [np.array(a) for a in spin]
            else:
                ele = sfparticles.Particles("ele", -1, 1, N=case["n_e"], props=tuple(np.array(a) for a in props))
            pho = sfparticles.Particles("pho", 0, 0)
            ele.set_photon(pho)
            species = [ele, pho]
            dt = 0.8e-6 / 299792458.0 * case["dt_T0"]
        else:
            props = od_pairs_initial(case, rng)
            terms, comb = [("static_field", dict(Bz=od_pairs_bz(case)))], 0
            fld = F.static_field(Bz=od_pairs_bz(case))
            pho = sfparticles.Particles("pho", 0, 0, N=case["n_g"], props=tuple(np.array(a) for a in props))
            ele = sfparticles.Particles("ele", -1, 1)
            pos = sfparticles.Particles("pos", 1, 1)
            pho.set_pair(ele, pos)
            species = [ele, pos, pho]
            dt = case["dt"]
        sim = sfparticles.Simulation(*species, dt=dt, fields=fld, print_every=None, photon_threshold=case["thr"])
        P.update_tau_e = _od_injected("e", sim, species, seed)
        P.update_tau_gamma = _od_injected("g", sim, species, seed)
        t0 = time.time()
        try:
            sim.start(case["steps"])
        finally:
            P.update_tau_e, P.update_tau_gamma = saved
        res = {"case": json.dumps(case), "field_terms": json.dumps(terms), "field_comb": json.dumps(comb),
               "dt": dt, "init": np.stack(props)}
        if case.get("spin"):
            res["spin_init"] = np.stack(spin)
        for i, p in enumerate(species):
            keys = ["x", "y", "z", "ux", "uy", "uz"] + (["sx", "sy", "sz"] if hasattr(p, "sx") else [])
            res[f"s{i}_state"] = np.stack([getattr(p, k) for k in keys])
            res[f"s{i}_name"] = p.name
        res["n_species"] = len(species)
        np.savez(out(f"ref_sim_{name}.npz"), **res)
        print(f"  sim {name}: {[p.N_buffered for p in species]} in {time.time() - t0:.1f}s")


def gen_od_sims():
    """Prepare the scratch reference copy with its OD tables and run the child."""
    import shutil
    import subprocess
    sys.path.insert(0, REPO)
    from sfparticles_b200.qed import tables
    d = tables.od_tables()
    n = 256
    with tempfile.TemporaryDirectory() as tmp:
        shutil.copytree(os.path.join(REF, "sfparticles"), os.path.join(tmp, "sfparticles"),
                        ignore=shutil.ignore_patterns("__pycache__"))
        with open(os.path.join(tmp, "sfparticles", "qed", "optical_depth_tables.h5"), "wb") as f:
            np.savez(f, photon_prob_rate_total=d["photon_rate_total"][:n], pair_prob_rate_total=d["pair_rate_total"][:n],
                     integral_photon_prob_along_delta=d["photon_cumulative"][:n],
                     integral_pair_prob_along_delta=d["pair_cumulative"][:n],
                     attr_chi_N=np.int64(n), attr_log_chi_range=np.array([-3.0, 2.0]),
                     attr_log_chi_delta=np.float64(d["log_chi_delta"]), attr_delta_N=np.int64(1024),
                     attr_log_delta_range=np.array([float(d["log_delta_min"]), 0.0]),
                     attr_log_delta_delta=np.float64(d["log_delta_delta"]))
        env = dict(os.environ, SFPARTICLES_OPTICAL_DEPTH="1", SFP_REFERENCE=tmp)
        subprocess.run([sys.executable, os.path.abspath(__file__), "--od-child"], env=env, check=True)


# ---------------------------------------------------------------------------
def gen_stats():
    """Reference runs with its own RNG (not reproducible), for 3-sigma checks."""
    import sfparticles
    from sfparticles import fields as F
    res = {}
    # reference tests/test_qed.py-style: static B field for a chi target, one step
    from scipy.constants import c, e, hbar, m_e
    gamma = 10000
    ux = math.sqrt(gamma ** 2 - 1)
    N = 1_000_000
    counts = {}
    for chi_e in (0.5, 2.0):
        dt = 1e-17 / chi_e
        reps = []
        for _ in range(4):
            ele = sfparticles.Particles("ele", -1, 1, N=N, props=(np.zeros(N), np.zeros(N), np.zeros(N),
                                                                  np.full(N, ux), np.zeros(N), np.zeros(N)),
                                        RR=sfparticles.RadiationReactionType.NONE)
            pho = sfparticles.Particles("pho", 0, 0)
            ele.set_photon(pho)
            fld = F.static_field(Bz=chi_e * m_e ** 2 * c ** 2 / e / hbar / ux)
            ele._eval_field(fld, 0)
            ele._calculate_chi()
            ele._photon_event(dt)
            ele._create_photon(pho)
            reps.append([pho.Npart, int(np.histogram(pho.ux / gamma, bins=[0.01, 0.011])[0][0]),
                         int(np.histogram(pho.ux / gamma, bins=[0.1, 0.11])[0][0])])
        counts[str(chi_e)] = reps
    res["static_photon"] = dict(N=N, gamma=gamma, counts=counts)
    # C1-shaped small run: 1000 electrons, a0=50 Gaussian, dt=T0/50, 1500 steps
    T0 = 0.8e-6 / c
    ctau = c * 25e-15 / (2 * math.sqrt(math.log(2) / 2))
    L = c * (1500 * T0 / 50) / 2
    runs = []
    for rep in range(6):
        rng = np.random.default_rng(1000 + rep)
        n = 1000
        g = 2000 * (1 + 0.01 * rng.normal(size=n))
        props = (rng.normal(-L, 5e-6, n), rng.normal(0, 1e-6, n), rng.normal(0, 1e-6, n), np.sqrt(g ** 2 - 1),
                 np.zeros(n), np.zeros(n))
        ele = sfparticles.Particles("ele", -1, 1, N=n, props=props)
        pho = sfparticles.Particles("pho", 0, 0)
        pos = sfparticles.Particles("pos", 1, 1)
        ele.set_photon(pho)
        pos.set_photon(pho)
        pho.set_pair(ele, pos)
        fld = F.gaussian_laser_pulse(50.0, 3e-6, ctau, direction=-1, x0=L)
        sim = sfparticles.Simulation(ele, pos, pho, dt=T0 / 50, fields=fld, print_every=None)
        sim.start(1500)
        eph = 1.0 / pho.inv_gamma
        hist = np.histogram(np.log10(eph), bins=16, range=(np.log10(2.0), np.log10(2000.0)))[0]
        runs.append(dict(n_photon=int(pho.Npart), n_pos=int(pos.Npart), mean_gamma_e=float(np.mean(1 / ele.inv_gamma)),
                         hist=hist.tolist(), e_photon_sum=float(eph.sum())))
    res["c1_small"] = dict(n=1000, a0=50.0, steps=1500, ctau=ctau, L=L, runs=runs,
                           hist_range=[math.log10(2.0), math.log10(2000.0)], bins=16)
    with open(out("ref_stats.json"), "w") as f:
        json.dump(res, f, indent=1)


PARTS = dict(tables=gen_tables, pushers=gen_pushers, fields=gen_fields, user_fields=gen_user_fields, rates=gen_rates,
             rs_events=gen_rs_events, sims=gen_sims, od=gen_od, od_sims=gen_od_sims, stats=gen_stats)

if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--od-child", action="store_true", help=argparse.SUPPRESS)
    a = ap.parse_args()
    if a.od_child:
        _od_sims_child()
        sys.exit(0)
    for k, fn in PARTS.items():
        if a.only and k not in a.only:
            continue
        t = time.time()
        print(f"[golden] {k} ...", flush=True)
        fn()
        print(f"[golden] {k} done in {time.time() - t:.1f}s", flush=True)
