#!/usr/bin/env python
"""Benchmark: particle-steps/s of the fused B200 step on the scaled-cascade
workload (1e7 electrons, gamma0 = 2000 +- 1 %, sigma_perp = 1 um,
sigma_par = 5 um, head-on with a linearly polarised Gaussian pulse a0 = 200,
lambda = 0.8 um, w0 = 3 um, 25 fs intensity FWHM; photon emission and pair
creation; dt = T0/100; 3000 steps).  Synthetic, seeded inputs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One "step" is one simulation step of the whole cascade (all species).
Prints one JSON line (rank 0).  Under torchrun every rank runs its own full
collision (seed = 1000 + rank): weak scaling with no data-path collective;
--split-beam instead gives each rank its slice of one beam (strong
scaling).  After the timed window every rank joins one all-reduce of the
job's counters and photon spectrum; the time is the max over ranks of
CUDA-event time.  On one GPU the line also carries, under `workloads`,
summaries of the plain config (C1), the learned sampler (C3), the batched
instances (C4) and the avalanche (C5), each measured after the window
(`--no-extras` skips them; `--workload cN` prints one in full).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

C = 299792458.0
LAMBDA = 0.8e-6
T0 = LAMBDA / C
FWHM = 25e-15
CTAU = C * FWHM / (2 * math.sqrt(math.log(2) / 2))  # 1/e field half-width from the intensity FWHM
A0 = 200.0
W0 = 3e-6
GAMMA0 = 2000.0
STEPS_FULL = 3000
DT = T0 / 100
# algorithmic bytes per unit of work (float64 state in HBM, each byte moved once)
BYTES_EPM = 97      # pushed e+-: x,y,z,ux,uy,uz read + written (96) + alive flag read
BYTES_PHOTON = 49   # photon in the step: x,y,z,ux,uy,uz + flag read; its push is the position epoch's advance,
                    # so nothing is written (photons fly straight: positions are stored as of an epoch)
BYTES_SYNC = 73     # photon positions written out (sfp_run_sync_positions): state + flag read, x,y,z written
BYTES_DEAD = 1      # pruned slot: flag read
BYTES_APPEND = 49   # appended particle: x,y,z,ux,uy,uz + flag written
BYTES_EMIT_MARK = 9  # emitter in the massive kernel: delta (8) + mark (1) written instead of its state
BYTES_EMIT = 154    # emitter in the appends kernel: parent state + delta read (56), photon written (49), parent
                    # state + flag written (49)
BYTES_PAIR = 155    # pair event in the appends kernel: parent state + delta read (56), flag (1), e- and e+
                    # written (98)
# DRAM bytes (read + write) over algorithmic bytes of one launch, from a
# one-kernel ncu capture of the collision window at 1e6 e- (photon kernel:
# 2.38e7 photons, 1.17 GB of state, larger than L2, so traffic scales with
# the units processed): 1.1695e9 read + 0.0036e9 written against 1.1680e9.
# Only kernels whose state exceeds L2 in that capture are listed.
NCU_TRAFFIC_RATIO = {"photon": (1.169452e9 + 3.648256e6) / 1.167978920e9}

WORKLOAD = "scaled cascade: 1e7 e- (gamma0 2000 +-1%, sigma_perp 1um, sigma_par 5um) x LP Gaussian a0=200 " \
           "(0.8um, w0 3um, 25fs FWHM), photons + pairs, dt=T0/100, 3000 steps"
# upper edge of the photon spectrum bins: above every photon (the beam's gamma stays below 2200)
SPECTRUM_HI = 2500.0


def window_label(start, steps):
    return f"{WORKLOAD}; timed window: steps {start}-{start + steps}" + (
        " (the collision: beam and pulse centres meet at the focus at step 1500)"
        if start < STEPS_FULL // 2 < start + steps else "")


def beam(n, seed, steps=STEPS_FULL, dt=DT):
    rng = np.random.default_rng(seed)
    L = C * (steps * dt) / 2
    g = GAMMA0 * (1 + 0.01 * rng.normal(size=n))
    x = rng.normal(-L, 5e-6, n)
    y = rng.normal(0, 1e-6, n)
    z = rng.normal(0, 1e-6, n)
    return (x, y, z, np.sqrt(g * g - 1), np.zeros(n), np.zeros(n)), L


def make_sim(n, seed, form="fp64", massive=(0, 0), photon=(0, 0), graph_chunk=64, engine="fused", share=None,
             a0=A0, dt=DT, steps=STEPS_FULL):
    """The scaled cascade with `n` electrons drawn from `seed`; `share` =
    (start, count) keeps that slice of the beam (Philox key `seed` either way).
    a0, dt, steps: the pulse amplitude, the time step and the run length the
    beam's offset is set for (the plain config: a0=50, dt=T0/50, 1500)."""
    import sfparticles_b200 as S
    from sfparticles_b200.fields import gaussian_laser_pulse
    props, L = beam(n, seed, steps, dt)
    if share is not None:
        a, c = share
        props = tuple(np.ascontiguousarray(v[a:a + c]) for v in props)
        n = c
    ele = S.Particles("electron", -1, 1, N=n, props=props)
    pos = S.Particles("positron", 1, 1)
    pho = S.Particles("photon", 0, 0)
    ele.set_photon(pho)
    pos.set_photon(pho)
    pho.set_pair(ele, pos)
    fld = gaussian_laser_pulse(a0, W0, CTAU, direction=-1, x0=L)
    sim = S.Simulation(ele, pos, pho, dt=dt, fields=fld, print_every=None, seed=seed, form=form,
                       m_stages=massive[0], min_blocks=massive[1], p_stages=photon[0], p_min_blocks=photon[1],
                       graph_chunk=graph_chunk, engine=engine)
    return sim


WORKLOAD_C4 = "batched uneven instances: 256 collisions, a0 log-U[10,500], electrons log-U[1e3,1e6], gamma0 " \
              "U[500,5000] (rng default_rng(0)), Philox seed = index, w0 3um, 25fs, photons + pairs, dt=T0/100, 2000 steps"


def make_c4(form="fp32", n_inst=256, steps=2000, scale=1.0):
    """The batched-instances workload as an Ensemble (scale shrinks every
    member's electron count, for tests and warm-up)."""
    import sfparticles_b200 as S
    from sfparticles_b200.fields import gaussian_laser_pulse
    rng = np.random.default_rng(0)
    a0s = 10 ** rng.uniform(1, math.log10(500), n_inst)
    ns = np.round(10 ** rng.uniform(3, 6, n_inst) * scale).astype(int)
    g0s = rng.uniform(500, 5000, n_inst)
    sims = []
    L = C * (steps * DT) / 2
    for k in range(n_inst):
        r = np.random.default_rng(10_000 + k)
        n = max(int(ns[k]), 1)
        g = g0s[k] * (1 + 0.01 * r.normal(size=n))
        props = (r.normal(-L, 5e-6, n), r.normal(0, 1e-6, n), r.normal(0, 1e-6, n), np.sqrt(g * g - 1),
                 np.zeros(n), np.zeros(n))
        ele = S.Particles("electron", -1, 1, N=n, props=props)
        pos = S.Particles("positron", 1, 1)
        pho = S.Particles("photon", 0, 0)
        ele.set_photon(pho)
        pos.set_photon(pho)
        pho.set_pair(ele, pos)
        fld = gaussian_laser_pulse(float(a0s[k]), W0, CTAU, direction=-1, x0=L)
        sims.append(S.Simulation(ele, pos, pho, dt=DT, fields=fld, print_every=None, seed=k, form=form))
    ens = S.Ensemble(sims)
    ens.electrons_initial = int(sum(max(int(n), 1) for n in ns))
    return ens


_SINK = None  # a list while the default run collects the other workloads' lines


def _emit(line):
    """Print a workload's JSON line, or keep it for the default line's `workloads`."""
    if _SINK is not None:
        _SINK.append(line)
    else:
        print(json.dumps(line), flush=True)


def run_c4(args):
    """Batched uneven instances on one GPU: value, per-kernel roofline."""
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    w = make_c4(args.form, n_inst=8, steps=args.steps, scale=1e-3)
    w.run_on_device(args.warmup)
    w.finish()
    del w
    ens = make_c4(args.form, steps=args.steps)
    ens._begin()
    torch.cuda.synchronize()
    launches0 = ens.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        e0.record()
        ens.run_on_device(args.steps)
        ens._sync_positions()  # the photon positions written out: part of the timed work
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = ens.kernel_launches - launches0
    ps = ens.particle_steps
    allp = ens.species
    counts = {k: int(sum(p.N_buffered for p in allp if p.name == k)) for k in ("electron", "positron", "photon")}
    alive = {k: int(sum(p.Npart for p in allp if p.name == k)) for k in ("electron", "positron", "photon")}
    torch.cuda.nvtx.range_push("roofline")
    kms, before, after = ens.time_step_kernel(args.roofline_steps)
    torch.cuda.nvtx.range_pop()
    k_ms = [float(np.mean([k[j] for k in kms])) for j in range(3)]
    names = [p.name for p in allp]
    n_ph_app = sum(a - b for a, b, nm in zip(after, before, names) if nm == "photon") / args.roofline_steps
    n_pairs = sum(a - b for a, b, nm in zip(after, before, names) if nm == "positron") / args.roofline_steps
    buf = {k: int(sum(n for n, nm in zip(before, names) if nm == k)) for k in ("electron", "positron", "photon")}
    n_epm = alive["electron"] + alive["positron"]
    alg = {"massive": n_epm * BYTES_EPM + (buf["electron"] + buf["positron"] - n_epm) * BYTES_DEAD
           + n_ph_app * BYTES_APPEND,
           "photon": alive["photon"] * BYTES_PHOTON + (buf["photon"] - alive["photon"]) * BYTES_DEAD
           + 2 * n_pairs * BYTES_APPEND}
    peak, peak_kind = measured_peak_hbm()
    per_kernel = {}
    for j, k in enumerate(("massive", "photon")):
        gbs = alg[k] / (k_ms[j] * 1e-3) / 1e9 if k_ms[j] > 0 else 0.0
        per_kernel[k] = {"avg_ms": k_ms[j], "alg_bytes_per_launch": alg[k], "achieved_gbs": gbs, "frac": gbs / peak}
    per_kernel["appends"] = {"avg_ms": k_ms[2]}
    dominant = max(("massive", "photon"), key=lambda k: per_kernel[k]["avg_ms"])
    dk = per_kernel[dominant]
    ens.finish()
    value = ps / (ms * 1e-3)
    line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32/f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD_C4, "form": args.form, "instances": len(ens.sims),
                       "electrons_initial": ens.electrons_initial,
                       "final_counts": counts, "l2": "state larger than L2 (no flush needed)"},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": dk["achieved_gbs"], "peak": peak,
                         "unit": "GB/s", "frac": dk["frac"], "traffic": None, "peak_kind": peak_kind,
                         "per_kernel": per_kernel, "launches_timed": args.roofline_steps},
            "cpu_baseline": None, "e2e": None, "gpu_launches": launches, "clocks": clk.summary(),
            "particle_steps": ps}
    _emit(line)


WORKLOAD_C3 = "learned photon-energy sampler: 5e7 queries per step, log10 chi ~ U[-3,0] (the small plain config's " \
              "emitters reach chi ~ 0.6), u ~ U(0,1); MLP 2-64-64-64-1 SiLU, BF16 weights, FP32 accumulation"
MLP_FLOP_PER_QUERY = 2 * (2 * 64 + 2 * 64 * 64 + 64)  # 16768


def measured_peak_bf16():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def run_c3(args):
    """Learned sampler vs the table sampler on a batch of emission events."""
    import torch
    import sfparticles_b200  # noqa: F401 (loads the library)
    from sfparticles_b200 import mlp
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    n = args.queries
    g = torch.Generator(device=dev).manual_seed(3)
    lc = torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 3.0 - 3.0
    u = torch.rand(n, dtype=torch.float64, device=dev, generator=g)
    s = mlp.PhotonSampler.trained()
    out = {}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clk_summary = None
    for name, fn in (("table", lambda: mlp.sample_table(lc, u)), ("mlp_warp", lambda: s.sample(lc, u, kernel="warp")),
                     ("mlp", lambda: s.sample(lc, u))):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        with ClockSampler(dev.index) as clk:
            e0.record()
            for _ in range(args.steps):
                fn()
            e1.record()
            torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / args.steps
        if name == "mlp":
            clk_summary = clk.summary()
    # end to end through the public API: host arrays in, host delta out
    hl = lc.cpu().pin_memory()
    hu = u.cpu().pin_memory()
    hd = torch.empty(n, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record()
    for _ in range(args.steps):
        dl = hl.to(dev, non_blocking=True)
        du = hu.to(dev, non_blocking=True)
        hd.copy_(s.sample(dl, du), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3) / args.steps
    # training throughput of the hand-written kernels (one epoch over 1e7 samples)
    t = mlp.PhotonSampler(mlp.init_params(0))
    feat, targ = t.make_samples(10_000_000, seed=5)
    gbuf = torch.zeros(mlp.NPARAM, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    e0.record()
    for lo in range(0, 10_000_000, 65536):
        m = min(65536, 10_000_000 - lo)
        t.grad(feat[lo:lo + m], targ[lo:lo + m])
    e1.record()
    torch.cuda.synchronize()
    train_sps = 1e7 / (e0.elapsed_time(e1) * 1e-3)
    # accuracy vs the table at fixed chi
    acc = {}
    for lc0 in (-2.5, -1.0, 0.0, 1.0, 2.5):
        m = 1_000_000
        a = torch.full((m,), lc0, dtype=torch.float64, device=dev)
        b = torch.rand(m, dtype=torch.float64, device=dev, generator=g)
        dt = mlp.sample_table(a, b).cpu().numpy()
        dm = s.sample(a, b).cpu().numpy()
        xs = np.concatenate([np.sort(dt), np.sort(dm)])
        ks = float(np.max(np.abs(np.searchsorted(np.sort(dt), xs, side="right") / m
                                 - np.searchsorted(np.sort(dm), xs, side="right") / m)))
        acc[f"log10chi={lc0:+.1f}"] = {"ks": ks, "moment_ratio_minus_1": [
            float(np.mean(dm ** k) / np.mean(dt ** k) - 1.0) for k in (1, 2, 3)]}
    peak, peak_kind = measured_peak_bf16()
    tflops = MLP_FLOP_PER_QUERY * n / (out["mlp"] * 1e-3) / 1e12
    value = n / (out["mlp"] * 1e-3)
    line = {"metric": "delta samples/s", "value": value, "unit": "samples/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["mlp"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16/f32", "data": "synthetic",
            "config": {"workload": WORKLOAD_C3, "queries_per_step": n,
                       "l2": "inputs 0.8 GB + output 0.4 GB per step, larger than L2 (no flush needed)"},
            "roofline": {"bound": "tensor", "kernel": "k_mlp_infer_tc", "achieved": tflops, "peak": peak,
                         "unit": "TFLOP/s", "frac": tflops / peak, "traffic": None, "peak_kind": peak_kind,
                         "flop_per_query": MLP_FLOP_PER_QUERY},
            "table_sampler": {"ms_per_step": out["table"], "samples_per_s": n / (out["table"] * 1e-3)},
            "warp_mma_sync_sampler": {"ms_per_step": out["mlp_warp"], "samples_per_s": n / (out["mlp_warp"] * 1e-3)},
            "mlp_over_table_speed": out["table"] / out["mlp"],
            "training": {"samples_per_s_fwd_bwd": train_sps},
            "accuracy_vs_table": acc,
            "e2e": {"value": n / (e2e_ms * 1e-3), "unit": "samples/s", "h2d_bytes_per_step": 16 * n,
                    "d2h_bytes_per_step": 8 * n},
            "cpu_baseline": None if args.no_cpu else c3_cpu_baseline(lc, u, mlp), "gpu_launches": args.steps,
            "clocks": clk_summary}
    _emit(line)


def c3_cpu_baseline(lc, u, mlp, m=1_000_000, budget_s=10.0):
    """The oracle's restatement of the reference's inverse-CDF bisection
    (_bisect_interp, optical_depth_tables.py:59-102; C, OpenMP, all host
    threads) on the first `m` queries of the same batch, checked against the
    GPU table sampler on them."""
    import ctypes
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc
    from sfparticles_b200.qed import tables
    d = tables.od_tables()
    tab = orc.make_od_table(d["photon_rate_total"], d["photon_cumulative"], float(d["log_chi_min"]),
                            float(d["log_chi_delta"]), float(d["log_delta_min"]), float(d["log_delta_delta"]))
    a = np.ascontiguousarray(lc[:m].cpu().numpy())
    b = np.ascontiguousarray(u[:m].cpu().numpy())
    out = np.empty(m)
    L = orc.lib()
    L.orc_od_bisect_batch(orc._p(a), orc._p(b), m, ctypes.byref(tab), orc._p(out))  # warm-up
    reps = 0
    t0 = time.perf_counter()
    while reps < 3 or (time.perf_counter() - t0 < budget_s and reps < 50):
        L.orc_od_bisect_batch(orc._p(a), orc._p(b), m, ctypes.byref(tab), orc._p(out))
        reps += 1
    dt = time.perf_counter() - t0
    gpu = mlp.sample_table(lc[:m], u[:m]).cpu().numpy()
    return {"value": m * reps / dt, "unit": "samples/s", "cores": omp_threads(), "kind": "port",
            "sample": f"{m} queries of the same batch, {reps} passes in {dt:.2f} s, through the oracle's "
                      "_bisect_interp (the table sampler the network replaces)",
            "max_rel_diff_vs_gpu_table_sampler": float(np.max(np.abs(gpu - out) / np.abs(out)))}


WORKLOAD_C5 = "spin + radiation-reaction avalanche: 5e6 e- at rest (uniform 2um cube, spin +z) between two " \
              "counter-propagating circularly polarised Gaussian pulses a0=800 (0.8um, w0 4um, 30fs FWHM; each the sum " \
              "of two linear pulses, pol 0 / pi/2, cep offset pi/2, amplitude a0/sqrt2), Boris-TBMT spin push, photon " \
              "emission (optical depth, learned sampler) + recoil + pairs, dt=T0/100, until 2500 steps or 1e9 particles"


def make_c5(n, form="fp32", sampler="mlp", seed=0):
    import sfparticles_b200 as S
    from sfparticles_b200 import qed
    from sfparticles_b200.fields import gaussian_laser_pulse
    rng = np.random.default_rng(seed)
    qed.set_method("od")
    try:
        props = (rng.uniform(-1e-6, 1e-6, n), rng.uniform(-1e-6, 1e-6, n), rng.uniform(-1e-6, 1e-6, n),
                 np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n), np.ones(n))
        ele = S.SpinParticles("electron", -1, 1, N=n, props=props)
        pos = S.SpinParticles("positron", 1, 1)  # pairs are created without spin
        pho = S.Particles("photon", 0, 0)
        ele.set_photon(pho)
        pos.set_photon(pho)
        pho.set_pair(ele, pos)
    finally:
        qed.set_method("rs")
    ctau = C * 30e-15 / (2 * math.sqrt(math.log(2) / 2))
    a = 800.0 / math.sqrt(2.0)
    xm = 10e-6  # the pulse centres start 10 um from the target and meet there after ~33 fs
    fld = None
    for d, x0 in ((1, -xm), (-1, xm)):
        for pol, cep in ((0.0, 0.0), (math.pi / 2, math.pi / 2)):
            f = gaussian_laser_pulse(a, 4e-6, ctau, direction=d, x0=x0, pol_angle=pol, cep=cep)
            fld = f if fld is None else fld + f
    return S.Simulation(ele, pos, pho, dt=DT, fields=fld, print_every=None, seed=seed, form=form, sampler=sampler)


def run_c5(args):
    """The avalanche config: particle-steps/s until the step limit or the particle cap."""
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    w = make_c5(1000, args.form)
    w.run_on_device(args.warmup)
    w.finish()
    del w
    sim = make_c5(args.electrons_c5, args.form)
    sim._begin()
    torch.cuda.synchronize()
    launches0 = sim.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    done = 0
    with ClockSampler(dev.index) as clk:
        e0.record()
        while done < args.steps and sum(p.N_buffered for p in sim.all_particles) < args.particle_cap:
            k = min(64, args.steps - done)
            sim.run_on_device(k)
            done += k
        sim._sync_positions()  # the photon positions written out: part of the timed work
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    counts = {p.name: p.N_buffered for p in sim.all_particles}
    alive = {p.name: p.Npart for p in sim.all_particles}
    torch.cuda.nvtx.range_push("roofline")  # profilers select these launches by this range
    kms, before, after = sim.time_step_kernel(args.roofline_steps)
    torch.cuda.nvtx.range_pop()
    k_ms = [float(np.mean([q[j] for q in kms])) for j in range(3)] if kms else [0.0, 0.0, 0.0]
    ps = sim.particle_steps
    launches = sim.kernel_launches - launches0
    sim.finish()
    n_epm = alive["electron"] + alive["positron"]
    alg_m = n_epm * (BYTES_EPM + 16 + 48)  # + optical depth, + spin (read and written)
    alg_p = alive["photon"] * (BYTES_PHOTON + 8)  # + optical depth
    peak, peak_kind = measured_peak_hbm()
    per_kernel = {
        "massive": {"avg_ms": k_ms[0], "alg_bytes_per_launch": alg_m,
                    "achieved_gbs": alg_m / (k_ms[0] * 1e-3) / 1e9 if k_ms[0] else 0.0},
        "photon": {"avg_ms": k_ms[1], "alg_bytes_per_launch": alg_p,
                   "achieved_gbs": alg_p / (k_ms[1] * 1e-3) / 1e9 if k_ms[1] else 0.0},
        "appends": {"avg_ms": k_ms[2]}}
    dominant = max(("massive", "photon"), key=lambda k: per_kernel[k]["avg_ms"])
    dk = per_kernel[dominant]
    line = {"metric": "particle-steps/s", "value": ps / (ms * 1e-3), "unit": "particle-steps/s", "n_gpus": 1,
            "steps": done, "warmup": args.warmup, "ms_per_step": ms / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32/f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD_C5, "form": args.form, "electrons_initial": args.electrons_c5,
                       "particle_cap": args.particle_cap, "steps_run": done, "final_counts": counts,
                       "l2": "state larger than L2 (no flush needed)"},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": dk["achieved_gbs"], "peak": peak,
                         "unit": "GB/s", "frac": dk["achieved_gbs"] / peak, "traffic": None, "peak_kind": peak_kind,
                         "per_kernel": per_kernel, "launches_timed": len(kms)},
            "cpu_baseline": None, "e2e": None, "gpu_launches": launches, "clocks": clk.summary(),
            "particle_steps": ps}
    _emit(line)


WORKLOAD_OPS = "the reference's step loop over the one-for-one float64 kernels (engine 'ops'): the scaled-cascade " \
               "beam at the given electron count, over the window that config.start_step opens"


def run_ops(args):
    """The plain float64 path on its own: particle-steps/s of the per-op
    kernels (each launched once per species per step, fields materialised),
    over the same window as the default line (advanced to it untimed, the
    last `--warmup` steps of the advance serving as warm-up)."""
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    sim = make_sim(args.electrons, 1000, "fp64", engine="ops")
    for p in sim.all_particles:
        p._to_gpu()
    S0 = max(window_start(args), args.warmup)
    sim._loop_ops(S0, None)
    torch.cuda.synchronize()
    ps0 = sim.particle_steps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        torch.cuda.nvtx.range_push("ops")  # profilers select these launches by this range
        e0.record()
        sim._loop_ops(args.steps, None)
        e1.record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ps = sim.particle_steps - ps0
    line = {"metric": "particle-steps/s", "value": ps / (ms * 1e-3), "unit": "particle-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_OPS, "electrons": args.electrons, "start_step": S0,
                       "steps_timed": args.steps,
                       "l2": "80 MB per array at 1e7 electrons, larger than L2 for every kernel"},
            "roofline": None, "cpu_baseline": None, "e2e": None, "clocks": clk.summary(), "particle_steps": ps}
    print(json.dumps(line), flush=True)


WORKLOAD_C1 = "plain method, small: 1e4 e- (gamma0 2000 +-1%, sigma_perp 1um, sigma_par 5um) x LP Gaussian a0=50 " \
              "(0.8um, w0 3um, 25fs FWHM), photons + pairs, float64, dt=T0/50, 1500 steps, beam seed 0; the whole run"
C1_N, C1_A0, C1_DT, C1_STEPS = 10_000, 50.0, T0 / 50, 1500


def run_c1(args):
    """The plain config at full size in float64 (the reference arithmetic):
    the whole 1500-step run device-resident (CUDA events), the same run
    through Simulation.start from host arrays (e2e), and the oracle port on
    the same run on the host cores beside it.  The state (<30 MB) sits in
    L2: the run is launch- and latency-bound, so no roofline is claimed."""
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    kw = dict(a0=C1_A0, dt=C1_DT, steps=C1_STEPS)
    w = make_sim(1000, 1, "fp64", **kw)  # warm-up: module load, graphs
    w.run_on_device(max(args.warmup, 3))
    w.finish()
    del w
    sim = make_sim(C1_N, 0, "fp64", **kw)
    sim._begin()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ps0, l0 = sim.particle_steps, sim.kernel_launches
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        e0.record()
        sim.run_on_device(C1_STEPS)
        sim._sync_positions()  # the photon positions written out: part of the timed work
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ps = sim.particle_steps - ps0
    launches = sim.kernel_launches - l0
    counts = {p.name: p.N_buffered for p in sim.all_particles}
    sim._end()
    del sim
    _release()
    # end to end: Simulation.start from host arrays, results back in host arrays
    sim2 = make_sim(C1_N, 0, "fp64", **kw)
    h2d = sum(a.nbytes for p in sim2.all_particles for a in p._arr.values())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record()
    sim2.start(C1_STEPS)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    d2h = sum(a.nbytes for p in sim2.all_particles for a in p._arr.values())
    e2e_ms = max(e0.elapsed_time(e1), wall * 1e3)
    e2e = {"value": sim2.particle_steps / (e2e_ms * 1e-3), "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "wall_s": wall, "note": "one step = the whole 1500-step run"}
    del sim2
    cpu = None
    if not args.no_cpu:
        osim = make_oracle_sim(C1_N, 0, **kw)
        t0 = time.perf_counter()
        osim.run(C1_STEPS)
        dt_cpu = time.perf_counter() - t0
        osim_counts = {p.name: p.N_buffered for p in osim.all}
        cpu = {"value": osim.particle_steps / dt_cpu, "unit": "particle-steps/s", "cores": omp_threads(),
               "kind": "port", "sample": f"the full run: {osim.particle_steps:.3g} particle-steps in {dt_cpu:.2f} s",
               "final_counts": osim_counts}
    line = {"metric": "particle-steps/s", "value": ps / (ms * 1e-3), "unit": "particle-steps/s", "n_gpus": 1,
            "steps": C1_STEPS, "warmup": max(args.warmup, 3), "ms_per_step": ms / C1_STEPS, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_C1, "electrons": C1_N, "form": "fp64", "final_counts": counts,
                       "l2": "the whole state (<30 MB) is L2-resident: launch- and latency-bound, no flush"},
            "roofline": None, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
            "particle_steps": ps}
    _emit(line)


WORKLOAD_KERNELS ="the per-op kernels one by one (the reference's one-for-one kernel boundary): N e- and N photons " \
                   "at the collision (beam and pulse centred on the focus at t = 0, gamma0 2000 +-1%, photons at " \
                   "gamma 500 along the beam, a0 200), float64 state; the learned sampler's training kernels on " \
                   "2^22 samples"

# algorithmic bytes of each per-op kernel: (per particle, per event); an
# element is 8 B, a flag 1 B; see the kernels in csrc/sfp_capi.cu
KERNEL_BYTES = {
    "sfp_field_eval_kernel": (73, 0),   # x,y,z (24) + flag (1) read, 6 components written (48)
    "k_update_chi": (89, 0),            # 6 components, u, 1/gamma (80) + flag read, chi written
    "k_rs": (26, 0),                    # flag, chi, 1/gamma read (17), event + delta written (9)
    "k_pick_hard": (1, 16),             # event read; per event delta + 1/gamma read
    "k_bool_sum": (1, 0),
    "k_fei": (2, 8),                    # count + scatter passes read the events, indices written
    "k_create_photon": (0, 121),        # index, parent x,u, delta read (64), photon x,u,1/gamma + flag written (57)
    "k_photon_recoil": (2, 64),         # flag + event; per event delta (8), u r/w (48), 1/gamma written
    "k_push_position": (81, 0),         # flag, x,y,z r/w (48), u, 1/gamma read (32)
    "k_boris": (105, 0),                # flag, 6 components (48), u r/w (48), 1/gamma written
    "k_ll": (73, 0),                    # flag, u r/w (48), 1/gamma r/w (16), chi read
    "k_boris_tbmt": (153, 0),           # k_boris + spin r/w (48)
    "k_update_tau": (42, 0),            # flag, tau r/w (16), 1/gamma, chi read (16), event + delta written
    "k_inv_gamma": (32, 0),
    "k_create_pair": (0, 122),          # as k_create_photon + the photon's flag written
}


def run_kernels(args):
    """Each per-op entry point launched alone, CUDA events around every
    launch (median of 5 after 2 warm-ups), achieved GB/s from its
    algorithmic bytes against the measured HBM peak.  Under an NVTX range
    "kernels" so profilers can select these launches."""
    import ctypes
    import torch
    from sfparticles_b200 import _lib, mlp, program
    from sfparticles_b200.fields import gaussian_laser_pulse
    from sfparticles_b200.qed import device_tables
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    HBM_PEAK, HBM_PEAK_KIND = measured_peak_hbm()
    n = args.electrons
    rng = np.random.default_rng(7)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    g = GAMMA0 * (1 + 0.01 * rng.normal(size=n))
    e = {"x": T(rng.normal(0, 2e-6, n)), "y": T(rng.normal(0, 1e-6, n)), "z": T(rng.normal(0, 1e-6, n)),
         "ux": T(np.sqrt(g * g - 1)), "uy": T(np.zeros(n)), "uz": T(np.zeros(n))}
    e["ig"] = 1.0 / torch.sqrt(1.0 + e["ux"] ** 2)
    ph = {"x": T(rng.normal(0, 2e-6, n)), "y": T(rng.normal(0, 1e-6, n)), "z": T(rng.normal(0, 1e-6, n)),
          "ux": T(np.full(n, 500.0)), "uy": T(np.zeros(n)), "uz": T(np.zeros(n))}
    ph["ig"] = 1.0 / ph["ux"]
    for d in (e, ph):
        for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "chi", "delta"):
            d[k] = torch.zeros(n, dtype=torch.float64, device=dev)
        d["pr"] = torch.zeros(n, dtype=torch.uint8, device=dev)
        d["ev"] = torch.zeros(n, dtype=torch.uint8, device=dev)
    e["tau"] = T(rng.exponential(size=n))
    spin = {k: T(v) for k, v in (("sx", np.zeros(n)), ("sy", np.zeros(n)), ("sz", np.ones(n)))}
    dst = {k: torch.empty(n, dtype=torch.float64, device=dev) for k in ("x", "y", "z", "ux", "uy", "uz", "ig")}
    dst["pr"] = torch.empty(n, dtype=torch.uint8, device=dev)
    fld = gaussian_laser_pulse(A0, W0, CTAU, direction=-1, x0=0.0)
    mod = program.get_module(fld, form=None, qed=None)
    prm = fld.params_device(dev)
    rs = device_tables.rs_table(dev)
    od_ph, _ = device_tables.od_tables(dev)
    ws = torch.empty(int(_lib.load().sfp_find_event_index_workspace(n)) + 8, dtype=torch.uint8, device=dev)
    idx = torch.empty(n, dtype=torch.int64, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    F = lambda d: [P(d[k]) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")]  # noqa: E731
    U = lambda d: [P(d[k]) for k in ("ux", "uy", "uz")]  # noqa: E731
    X = lambda d: [P(d[k]) for k in ("x", "y", "z")]  # noqa: E731
    q = -1.602176634e-19
    rows = []
    n_ev = {"e": 0, "ph": 0}

    def count(d):
        cnt.zero_()
        _lib.call("sfp_bool_sum", P(d["ev"]), n, P(cnt), st)
        return int(cnt.item())

    def fei(d, key):
        k = n_ev[key]
        _lib.call("sfp_find_event_index", P(d["ev"]), k, n, P(idx), P(ws), ws.numel(), st)

    def timed(name, fn, events=0, reps=5, bytes_name=None, prep=None):
        """`prep` (outside the events) restores what the kernel changes."""
        for _ in range(2):
            if prep:
                prep()
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        torch.cuda.synchronize()
        for a, b in ev:
            if prep:
                prep()
            a.record()
            fn()
            b.record()
        torch.cuda.synchronize()
        ms = float(np.median([a.elapsed_time(b) for a, b in ev]))
        per, per_ev = KERNEL_BYTES[bytes_name or name]
        alg = per * n + per_ev * events
        gbs = alg / (ms * 1e-3) / 1e9
        rows.append({"kernel": name, "ms": ms, "alg_bytes": alg, "events": events, "achieved_gbs": gbs,
                     "frac": gbs / HBM_PEAK})

    torch.cuda.nvtx.range_push("kernels")
    # the e- side of a step at the pulse's peak
    timed("sfp_field_eval_kernel", lambda: _lib.call("sfp_field_eval", mod.handle, P(prm), *X(e), 0.0, n, P(e["pr"]),
                                                     *F(e), st))
    timed("k_update_chi", lambda: _lib.call("sfp_update_chi", *F(e), *U(e), P(e["ig"]), P(e["chi"]), n, P(e["pr"]),
                                            st))
    timed("k_rs", lambda: _lib.call("sfp_photon_from_rejection_sampling", P(e["ig"]), P(e["chi"]), DT, n,
                                    P(e["pr"]), P(e["ev"]), P(e["delta"]), ctypes.byref(rs), 1, 0, 7, st))
    n_ev["e"] = count(e)
    e_ev_all = e["ev"].clone()
    timed("k_pick_hard", lambda: _lib.call("sfp_pick_hard_photon", P(e["ev"]), P(e["delta"]), P(e["ig"]), 2.0, n, st),
          events=n_ev["e"], prep=lambda: e["ev"].copy_(e_ev_all))
    n_ev["e"] = count(e)
    timed("k_bool_sum", lambda: _lib.call("sfp_bool_sum", P(e["ev"]), n, P(cnt), st))
    timed("k_fei", lambda: fei(e, "e"), events=n_ev["e"])
    fei(e, "e")
    k = n_ev["e"]
    timed("k_create_photon", lambda: _lib.call("sfp_create_photon", *X(e), *U(e), *X(dst), *U(dst), P(dst["ig"]),
                                               P(dst["pr"]), P(idx), P(e["delta"]), 0, k, st), events=k)
    timed("k_photon_recoil", lambda: _lib.call("sfp_photon_recoil", *U(e), P(e["ig"]), P(e["ev"]), P(e["delta"]),
                                               n, P(e["pr"]), st), events=k)
    timed("k_push_position", lambda: _lib.call("sfp_push_position", *X(e), *U(e), P(e["ig"]), n, P(e["pr"]),
                                               DT / 2, st))
    timed("k_boris", lambda: _lib.call("sfp_boris", *U(e), P(e["ig"]), *F(e), q, n, P(e["pr"]), DT, st))
    timed("k_ll(LL)", lambda: _lib.call("sfp_LL_push", *U(e), P(e["ig"]), P(e["chi"]), n, P(e["pr"]), DT, st),
          bytes_name="k_ll")
    timed("k_ll(CLL)", lambda: _lib.call("sfp_CLL_push", *U(e), P(e["ig"]), P(e["chi"]), n, P(e["pr"]), DT, st),
          bytes_name="k_ll")
    timed("k_boris_tbmt", lambda: _lib.call("sfp_boris_tbmt", *U(e), P(e["ig"]), P(spin["sx"]), P(spin["sy"]),
                                            P(spin["sz"]), *F(e), q, 1.14e-3, n, P(e["pr"]), DT, st))
    timed("k_update_tau", lambda: _lib.call("sfp_update_tau", P(e["tau"]), P(e["ig"]), P(e["chi"]), DT, n,
                                            P(e["pr"]), P(e["ev"]), P(e["delta"]), ctypes.byref(od_ph), 1, 0, 7, st))
    timed("k_inv_gamma", lambda: _lib.call("sfp_inv_gamma", *U(e), P(e["ig"]), n, 0, st))
    # the photon side: fields, chi, pair events, the pairs
    _lib.call("sfp_field_eval", mod.handle, P(prm), *X(ph), 0.0, n, P(ph["pr"]), *F(ph), st)
    _lib.call("sfp_update_chi", *F(ph), *U(ph), P(ph["ig"]), P(ph["chi"]), n, P(ph["pr"]), st)
    timed("k_rs(pair)", lambda: _lib.call("sfp_pair_from_rejection_sampling", P(ph["ig"]), P(ph["chi"]), DT, n,
                                          P(ph["pr"]), P(ph["ev"]), P(ph["delta"]), ctypes.byref(rs), 1, 2, 7, st),
          bytes_name="k_rs")
    n_ev["ph"] = count(ph)
    fei(ph, "ph")
    kp = n_ev["ph"]
    pr0 = ph["pr"].clone()
    timed("k_create_pair", lambda: _lib.call("sfp_create_pair", *X(ph), *U(ph), P(ph["pr"]), *X(dst), *U(dst),
                                             P(dst["ig"]), P(dst["pr"]), P(idx), P(ph["delta"]), 0, kp, 0, st),
          events=kp, prep=lambda: ph["pr"].copy_(pr0))
    # the learned sampler's training kernels
    ns = 1 << 22
    feats = torch.empty(ns * 2, dtype=torch.float32, device=dev)
    targ = torch.empty(ns, dtype=torch.float32, device=dev)
    tab = mlp._photon_table()
    lo, hi = mlp.LOG_CHI_RANGE
    params = torch.as_tensor(mlp.init_params(3), device=dev)
    grad = torch.zeros_like(params)
    m1, v1 = torch.zeros_like(params), torch.zeros_like(params)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    train = []

    def ttime(name, fn, nbytes, flops=None):
        for _ in range(2):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for _ in range(5):
            fn()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 5
        r = {"kernel": name, "ms": ms, "alg_bytes": nbytes, "achieved_gbs": nbytes / (ms * 1e-3) / 1e9,
             "frac": nbytes / (ms * 1e-3) / 1e9 / HBM_PEAK}
        if flops:
            r["tflops"] = flops / (ms * 1e-3) / 1e12
        train.append(r)

    ttime("k_mlp_samples", lambda: _lib.call("sfp_mlp_make_samples", ctypes.byref(tab), 1, 0, lo, hi, ns, P(feats),
                                             P(targ), st), 12 * ns)
    ttime("k_mlp_grad", lambda: _lib.call("sfp_mlp_grad", P(params), P(feats), P(targ), ns, P(grad), P(loss), st),
          12 * ns, flops=3 * 16768 * ns)
    ttime("k_mlp_adam", lambda: _lib.call("sfp_mlp_adam", P(params), P(grad), P(m1), P(v1), 1, 1e-3, 0.9, 0.999,
                                          1e-8, 1.0, st), 28 * params.numel())
    torch.cuda.nvtx.range_pop()
    line = {"metric": "GB/s per kernel", "workload": "kernels", "n_gpus": 1, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_KERNELS, "particles": n, "electron_events": n_ev["e"],
                       "pair_events": n_ev["ph"],
                       "l2": f"{n * 8 / 1e6:.0f} MB per array, every kernel's traffic larger than L2"},
            "peak_gbs": HBM_PEAK, "peak_kind": HBM_PEAK_KIND, "kernels": rows, "training": train}
    print(json.dumps(line), flush=True)


def make_oracle_sim(n, seed, a0=A0, dt=DT, steps=STEPS_FULL):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc
    from sfparticles_b200.qed import tables
    props, L = beam(n, seed, steps, dt)
    ele = orc.Species("electron", -1, 1, N=n, props=props)
    pos = orc.Species("positron", 1, 1)
    pho = orc.Species("photon", 0, 0)
    ele.set_photon(pho)
    pos.set_photon(pho)
    pho.set_pair(ele, pos)
    iA, dA, _, zmax = tables.rs_tables()
    terms = orc.gaussian_laser_pulse(a0, W0, CTAU, direction=-1, x0=L)
    return orc.OracleSim([ele, pos, pho], dt, terms, ("rs", iA, dA), seed=seed, z_max=zmax)


def cpu_sample(n_e, start, max_steps, budget_s):
    """Oracle port (C, OpenMP, all host threads) on a bounded sample of the
    same window: `n_e` electrons of the same beam advanced untimed to step
    `start`, then up to `max_steps` steps timed (fewer if `budget_s` runs
    out).  Returns (rate, steps timed, particle-steps, seconds)."""
    sim = make_oracle_sim(n_e, 12345)
    sim.run(max(start, 1))  # untimed: the approach (and one step of warm-up)
    ps0 = sim.particle_steps
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps and time.perf_counter() - t0 < budget_s:
        sim.run(1)
        steps += 1
    dt = time.perf_counter() - t0
    ps = sim.particle_steps - ps0
    return ps / dt, steps, ps, dt


def window_state_sample(sim, every):
    """Every `every`-th alive particle of each species of a device-resident
    run, as host arrays (x, y, z, ux, uy, uz), with the run's t and step."""
    out = {}
    for p in sim.all_particles:
        N = p.N_buffered
        if N == 0:
            out[p.name] = None
            continue
        keep = (p._d("_to_be_pruned")[:N] == 0).nonzero().flatten()[::every]
        out[p.name] = tuple(p._d(k)[keep].cpu().numpy() for k in ("x", "y", "z", "ux", "uy", "uz"))
    return {"species": out, "t": float(sim.t), "step": int(sim.step), "every": every}


def cpu_sample_from_state(state, seed, max_steps, budget_s):
    """Oracle port (C, OpenMP, all host threads) stepping a subsample of the
    GPU run's own state at the window's start over the same steps (up to
    `max_steps`, fewer if `budget_s` runs out).  Returns (rate, steps timed,
    particle-steps, seconds, counts at the start)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc
    from sfparticles_b200.qed import tables
    sp = state["species"]

    def species(name, q, m):
        props = sp.get(name)
        return orc.Species(name, q, m, N=0 if props is None else len(props[0]), props=props)

    ele, pos, pho = species("electron", -1, 1), species("positron", 1, 1), species("photon", 0, 0)
    ele.set_photon(pho)
    pos.set_photon(pho)
    pho.set_pair(ele, pos)
    iA, dA, _, zmax = tables.rs_tables()
    _, L = beam(1, 0)
    terms = orc.gaussian_laser_pulse(A0, W0, CTAU, direction=-1, x0=L)
    osim = orc.OracleSim([ele, pos, pho], DT, terms, ("rs", iA, dA), seed=seed, t0=state["t"], z_max=zmax)
    osim.step = state["step"]
    counts = {p.name: p.N_buffered for p in osim.all}
    ps0 = osim.particle_steps
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps and time.perf_counter() - t0 < budget_s:
        osim.run(1)
        steps += 1
    dt = time.perf_counter() - t0
    ps = osim.particle_steps - ps0
    return ps / dt, steps, ps, dt, counts


def window_start(args):
    """First step of the timed window.  `--start-step` if given; else, when
    the window is shorter than the 3000-step run, the steps centred on the
    collision (the beam and pulse centres meet at the focus at step 1500), so
    the window times the cascade -- photon emission and pair creation --
    rather than the approach; else step 0."""
    if args.start_step is not None and args.start_step >= 0:
        return min(args.start_step, STEPS_FULL)
    if args.steps >= STEPS_FULL:
        return 0
    return max(0, STEPS_FULL // 2 - args.steps // 2)


def omp_threads():
    v = os.environ.get("OMP_NUM_THREADS")
    return int(v) if v else (os.cpu_count() or 1)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once sampling runs (short regions get samples)
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 3.0:
                time.sleep(0.01)
            self.rows.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for nm, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_ours(args, rank, world):
    import torch
    import sfparticles_b200 as S
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    from sfparticles_b200 import shard
    # weak scaling: a full collision per rank; --split-beam: rank r's slice of one beam
    seed = 1000 + rank
    share = None
    if args.split_beam and world > 1:
        share = shard.split_counts(args.electrons, world)[rank]
        seed = 1000
    S0 = window_start(args)
    # warm-up: compile / load the module, W steps of a small instance, then a fresh timed instance
    wsim = make_sim(max(1000, args.electrons // 1000), seed, args.form)
    wsim.run_on_device(args.warmup)
    wsim.finish()
    del wsim
    sim = make_sim(args.electrons, seed, args.form, (args.m_stages, args.min_blocks), (args.p_stages, args.p_min_blocks),
                   graph_chunk=0 if args.no_graphs else 64, share=share)
    if share is not None:
        sim.seed = shard.rank_seed(seed, rank)  # the slice's own Philox key
    sim._begin()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    phases = {}  # device ms and particle-steps of the timed phases of the 3000-step run

    def timed(name, n):
        ps_a = sim.particle_steps
        torch.cuda.synchronize()
        e0.record()
        sim.run_on_device(n)
        sim._sync_positions()  # the photon positions written out: part of the timed work
        e1.record()
        torch.cuda.synchronize()
        phases[name] = (e0.elapsed_time(e1), sim.particle_steps - ps_a, n)

    # the approach, untimed for the headline: up to the variant search, which
    # measures the kernel variants on the state the window starts from
    from sfparticles_b200 import autotune
    nvar = sum(len(v) for v in autotune.VARIANTS[(args.form, "rs")]) * 2
    tune = not args.no_variants and S0 >= nvar
    tm, tp = {}, {}
    if S0 - (nvar if tune else 0) > 0:
        timed("approach", S0 - (nvar if tune else 0))
    if tune:
        tm, tp = autotune.measure(sim, steps=2)
        sim.set_kernel(massive=min(tm, key=tm.get), photon=min(tp, key=tp.get))
    assert sim.step == S0, (sim.step, S0)
    sim.reserve(args.steps)  # room for the window at twice the rate seen, so no growth inside it
    start_counts = {p.name: p.N_buffered for p in sim.all_particles}
    # the CPU baseline's sample: a subsample of this state, stepped by the oracle after the GPU work
    cpu_state = window_state_sample(sim, args.cpu_every) if (rank == 0 and world == 1 and not args.no_cpu) else None
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches0 = sim.kernel_launches
    ps0 = sim.particle_steps
    with ClockSampler(dev.index) as clk:
        e0.record()
        sim.run_on_device(args.steps)
        sim._sync_positions()  # the photon positions written out: part of the timed work
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = sim.kernel_launches - launches0
    ps = sim.particle_steps - ps0
    phases["window"] = (ms, ps, args.steps)
    counts = {p.name: p.N_buffered for p in sim.all_particles}
    # job-wide counters and photon spectrum at the window's end: one all-reduce over the ranks
    jd = shard.reduce_diagnostics(sim.all_particles, ps, bins=64, lo=2.0, hi=SPECTRUM_HI, device=dev)
    job = {"buffered": jd["buffered"], "alive": jd["alive"], "window_particle_steps": jd["particle_steps"],
           "photons_in_spectrum": float(jd["spectrum"].sum()), "spectrum_range": [2.0, SPECTRUM_HI],
           "spectrum": [float(v) for v in jd["spectrum"]], "ranks": world}
    spectrum = None
    if not args.no_compare:
        from sfparticles_b200 import diagnostics as D
        spectrum = D.photon_spectrum_device(sim.all_particles[2], 64, 2.0, SPECTRUM_HI)
    # roofline of each step kernel at the window's end state: CUDA events around every launch
    alive = {p.name: p.Npart for p in sim.all_particles}
    buffered = {p.name: p.N_buffered for p in sim.all_particles}
    torch.cuda.nvtx.range_push("roofline")  # profilers select these launches by this range
    kms, before, after = sim.time_step_kernel(args.roofline_steps)
    torch.cuda.nvtx.range_pop()
    k_ms = [float(np.mean([k[j] for k in kms])) for j in range(3)]
    n_ph_app = (after[2] - before[2]) / args.roofline_steps  # photons appended per step
    n_pairs = (after[1] - before[1]) / args.roofline_steps    # pairs per step
    n_epm = alive["electron"] + alive["positron"]
    dead_m = buffered["electron"] + buffered["positron"] - n_epm
    # algorithmic bytes of each launch: the massive kernel streams every e+- (state read, a
    # non-emitter's written back, an emitter's delta and mark written), the appends kernel reads
    # each emitter / converted photon again and writes the children and the emitter's new state
    n_emit = n_ph_app
    alg = {
        "massive": n_epm * (BYTES_EPM - 48) + (n_epm - n_emit) * 48 + n_emit * BYTES_EMIT_MARK
        + dead_m * BYTES_DEAD,
        "photon": alive["photon"] * BYTES_PHOTON + (buffered["photon"] - alive["photon"]) * BYTES_DEAD,
        "appends": n_emit * BYTES_EMIT + n_pairs * BYTES_PAIR,
    }
    names = {
        "massive": f"sfp_massive_{args.form}_rs_s{sim.m_stages}_b{sim.min_blocks}",
        "photon": f"sfp_photon_{args.form}_rs_s{sim.p_stages}_b{sim.p_min_blocks}",
        "appends": f"sfp_scan_kernel+sfp_appends_{args.form}",
    }
    per_kernel = {}
    for j, k in enumerate(("massive", "photon", "appends")):
        gbs = alg[k] / (k_ms[j] * 1e-3) / 1e9 if k_ms[j] > 0 else 0.0
        per_kernel[k] = {"kernel": names[k], "avg_ms": k_ms[j], "alg_bytes_per_launch": alg[k],
                         "achieved_gbs": gbs}
    dominant = max(per_kernel, key=lambda k: per_kernel[k]["avg_ms"])
    # the e+- push as SURVEY-style work: 97 B per e+- and 49 B per appended photon over the two
    # launches that do it (the appends time also covers the step's pairs)
    push_alg = n_epm * BYTES_EPM + dead_m * BYTES_DEAD + n_ph_app * BYTES_APPEND
    push_ms = k_ms[0] + k_ms[2]
    per_kernel["push_path"] = {"kernel": "massive + appends", "avg_ms": push_ms, "alg_bytes_per_launch": push_alg,
                               "achieved_gbs": push_alg / (push_ms * 1e-3) / 1e9 if push_ms > 0 else 0.0}
    step_units = {"electrons+positrons_alive": n_epm, "photons_alive": alive["photon"],
                  "photons_appended_per_step": n_ph_app, "pairs_per_step": n_pairs}
    # the rest of the 3000-step run, for the whole-run rate (second field)
    whole = None
    if not args.no_whole_run and sim.step < STEPS_FULL:
        timed("rest", STEPS_FULL - sim.step)
    if "approach" in phases or "rest" in phases:
        wms = sum(v[0] for v in phases.values())
        wps = sum(v[1] for v in phases.values())
        wst = sum(v[2] for v in phases.values())
        whole = {"value": wps / (wms * 1e-3), "unit": "particle-steps/s", "steps_timed": wst, "ms": wms,
                 "particle_steps": wps, "final_step": sim.step,
                 "final_counts": {p.name: p.N_buffered for p in sim.all_particles},
                 "note": f"steps 0-{sim.step} timed in phases; the {sim.step - wst} variant-search and roofline "
                         "steps are excluded from both time and work"}
    sim._end()
    del sim
    _release()

    # end to end through the public API from host arrays: the same window
    e2e = None
    if not args.no_e2e:
        sim2 = make_sim(args.electrons, seed, args.form, share=share)
        if share is not None:
            sim2.seed = shard.rank_seed(seed, rank)
        if S0 > 0:
            sim2.start(S0)  # untimed: the approach, ending in host arrays
        h2d = sum(a.nbytes for p in sim2.all_particles for a in p._arr.values())
        ps_a = sim2.particle_steps
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record()
        sim2.start(args.steps)
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ms2 = e0.elapsed_time(e1)
        d2h = sum(a.nbytes for p in sim2.all_particles for a in p._arr.values())
        # whole job: the slowest rank's time, every rank's work and copies
        from sfparticles_b200.shard import reduce_job, sum_over_ranks
        ms2, ps2 = reduce_job(max(ms2, wall * 1e3), sim2.particle_steps - ps_a, device=dev)
        h2d, d2h = sum_over_ranks([h2d, d2h], device=dev)
        e2e = dict(value=ps2 / (ms2 * 1e-3), unit="particle-steps/s",
                   h2d_bytes_per_step=h2d / args.steps, d2h_bytes_per_step=d2h / args.steps,
                   wall_s=wall, window=f"steps {S0}-{S0 + args.steps}: Simulation.start({args.steps}) from host "
                                       f"arrays after an untimed start({S0})")
        del sim2
        _release()

    # the chosen form vs the plain float64 form: same beam, seed and window
    compare = None
    if not args.no_compare and args.form != "fp64":
        from sfparticles_b200 import diagnostics as D
        s = make_sim(args.electrons, seed, "fp64", share=share)
        if share is not None:
            s.seed = shard.rank_seed(seed, rank)
        s._begin()
        # the float64 form gets the same variant search, on its own state before the window
        nvar64 = sum(len(v) for v in autotune.VARIANTS[("fp64", "rs")]) * 2
        tune64 = not args.no_variants and S0 >= nvar64
        if S0 - (nvar64 if tune64 else 0) > 0:
            s.run_on_device(S0 - (nvar64 if tune64 else 0))
        if tune64:
            tm64, tp64 = autotune.measure(s, steps=2)
            s.set_kernel(massive=min(tm64, key=tm64.get), photon=min(tp64, key=tp64.get))
        s.reserve(args.steps)
        torch.cuda.synchronize()
        ps_a = s.particle_steps
        e0.record()
        s.run_on_device(args.steps)
        s._sync_positions()
        e1.record()
        torch.cuda.synchronize()
        fms = e0.elapsed_time(e1)
        fps = s.particle_steps - ps_a
        spec64 = D.photon_spectrum_device(s.all_particles[2], 64, 2.0, SPECTRUM_HI)
        c64 = {p.name: p.N_buffered for p in s.all_particles}
        s._end()
        del s
        _release()
        pairs_form = counts["positron"] - start_counts["positron"]
        pairs_64 = c64["positron"] - start_counts["positron"]
        v64 = fps / (fms * 1e-3)
        compare = {"electrons": args.electrons, "window": f"steps {S0}-{S0 + args.steps}", "fp64_value": v64,
                   "form_value": ps / (ms * 1e-3), "speedup_vs_fp64": (ps / ms) / (fps / fms),
                   "spectrum_rel_l1": D.spectrum_rel_l1(spectrum, spec64), "spectrum_bins": 64,
                   "spectrum_range": [2.0, SPECTRUM_HI], "photons_in_spectrum": float(spec64.sum()),
                   "pair_yield_rel": D.rel_diff(counts["positron"], c64["positron"]),
                   "pairs_fp64": c64["positron"], "pairs_form": counts["positron"],
                   "pairs_created_in_window_fp64": pairs_64, "pairs_created_in_window_form": pairs_form,
                   "photons_fp64": c64["photon"], "photons_form": counts["photon"],
                   "note": "fused float64 step (the reference arithmetic) over the same window after the same "
                           "approach; spectrum of all photons alive at the window's end"}

    # max over ranks of the device time; sum of work
    from sfparticles_b200.shard import reduce_job
    ms, tot_ps = reduce_job(ms, ps, device=dev)
    peak, peak_kind = measured_peak_hbm()
    dk = per_kernel[dominant]
    for v in per_kernel.values():
        v["frac"] = v["achieved_gbs"] / peak
    return dict(ms=ms, particle_steps=tot_ps, counts=counts, launches=launches, clocks=clk.summary(),
                roofline={"bound": "hbm", "achieved": dk["achieved_gbs"], "peak": peak, "unit": "GB/s",
                          "frac": dk["achieved_gbs"] / peak, "peak_kind": peak_kind,
                          "traffic": (dk["alg_bytes_per_launch"] * NCU_TRAFFIC_RATIO[dominant]
                                      if dominant in NCU_TRAFFIC_RATIO else None),
                          "traffic_note": "ncu DRAM bytes of a 1e6-electron capture scaled by units processed",
                          "kernel": dk["kernel"], "kernel_avg_ms": dk["avg_ms"],
                          "alg_bytes_per_launch": dk["alg_bytes_per_launch"], "launches_timed": args.roofline_steps,
                          "units_at_window_end": step_units, "per_kernel": per_kernel,
                          "variants_ms": {**{f"massive_s{a}_b{b}": v for (a, b), v in tm.items()},
                                          **{f"photon_s{a}_b{b}": v for (a, b), v in tp.items()}}},
                e2e=e2e, compare=compare, start_step=S0, start_counts=start_counts, whole=whole, job=job,
                cpu_state=cpu_state)


def _release():
    """Return a finished workload's device blocks and page-locked host blocks
    (its final state's copies) before the next workload: tens of GB each at
    the C4 and C5 sizes, more than the host holds if they accumulate."""
    import gc
    import torch
    gc.collect()
    torch.cuda.empty_cache()
    if hasattr(torch._C, "_host_emptyCache"):
        torch._C._host_emptyCache()


def _summary(line):
    """The parts of a workload's line that the default line carries."""
    if not line:
        return None
    keep = ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "dtype", "gpu_launches", "clocks",
            "mlp_over_table_speed")
    s = {k: line[k] for k in keep if k in line}
    s["workload"] = (line.get("config") or {}).get("workload")
    r = line.get("roofline")
    if r:
        s["roofline"] = {k: r.get(k) for k in ("bound", "kernel", "achieved", "peak", "unit", "frac")}
    for k in ("cpu_baseline", "e2e"):
        v = line.get(k)
        if v:
            s[k] = {kk: v.get(kk) for kk in ("value", "unit", "cores", "kind", "sample", "h2d_bytes_per_step",
                                              "d2h_bytes_per_step") if kk in v}
    if "table_sampler" in line:
        s["table_sampler_samples_per_s"] = line["table_sampler"]["samples_per_s"]
    return s


def run_extras(args):
    """The other configs, measured after the default line's window on the
    same GPU, one after the other: C1 (the plain config's whole run, with the
    oracle port on the same run), C3 (the learned sampler), C4 (256 batched
    instances, 2000 steps), C5 (the avalanche to 1e9 particles).  Each entry
    summarises the line `bench.py --workload cN` prints in full; a workload
    that fails records its error and the others still run."""
    import copy
    global _SINK
    out = {}
    _release()  # the default line's runs
    for name, fn, steps in (("c1", run_c1, None), ("c3", run_c3, 20), ("c4", run_c4, 2000), ("c5", run_c5, 2500)):
        a = copy.copy(args)
        a.workload = name
        a.warmup = 3
        if steps is not None:
            a.steps = steps
        _SINK = []
        try:
            fn(a)
            out[name] = _summary(_SINK[-1] if _SINK else None)
        except Exception as exc:  # recorded in the line; the headline stands
            out[name] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
        finally:
            _SINK = None
            _release()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=STEPS_FULL)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "ops", "kernels"],
                    help="c1: the plain config (1e4 e-, float64, the whole run); c2: the scaled cascade (default); c3: the learned photon-energy sampler on 5e7 "
                         "queries per step; c4: 256 batched uneven instances (2000 steps); c5: the spin + "
                         "radiation-reaction avalanche to 1e9 particles; ops: the per-op float64 kernels; "
                         "kernels: each per-op kernel launched alone (GB/s per kernel)")
    ap.add_argument("--queries", type=int, default=50_000_000, help="c3: queries per step")
    ap.add_argument("--electrons-c5", type=int, default=5_000_000, help="c5: electrons at rest")
    ap.add_argument("--particle-cap", type=int, default=1_000_000_000, help="c5: stop at this many particles")
    ap.add_argument("--electrons", type=int, default=10_000_000)
    ap.add_argument("--form", default="fp32", choices=["fp64", "fp32"])
    ap.add_argument("--start-step", type=int, default=None,
                    help="c2: first step of the timed window (default: centred on the collision at step 1500 "
                         "when --steps < 3000, else 0); the steps before it run untimed")
    ap.add_argument("--no-whole-run", action="store_true", help="c2: skip the rest of the 3000-step run")
    ap.add_argument("--split-beam", action="store_true",
                    help="c2 under torchrun: split one beam of --electrons over the ranks (strong scaling) instead "
                         "of a full collision per rank (weak scaling)")
    ap.add_argument("--no-compare", action="store_true", help="c2: skip the float64 run over the same window")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--m-stages", type=int, default=0)
    ap.add_argument("--min-blocks", type=int, default=0)
    ap.add_argument("--p-stages", type=int, default=0)
    ap.add_argument("--p-min-blocks", type=int, default=0)
    ap.add_argument("--no-graphs", action="store_true", help="one eager launch per kernel (for profilers)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="c2 on one GPU: skip the summaries of C1, C3, C4 and C5 in the line")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--roofline-steps", type=int, default=8)
    ap.add_argument("--cpu-electrons", type=int, default=100_000,
                    help="--impl reference: electrons of the CPU sample (advanced on the CPU to the window)")
    ap.add_argument("--cpu-every", type=int, default=10,
                    help="cpu_baseline: every n-th particle of the GPU run's state at the window's start")
    ap.add_argument("--cpu-budget", type=float, default=30.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.workload == "c3":
        if args.impl != "ours" or world != 1:
            print(json.dumps({"impl": args.impl, "workload": "c3",
                              "unavailable": "the learned-sampler mode runs one GPU, product arm only"}))
            return
        if args.steps == STEPS_FULL:
            args.steps = 20
        run_c3(args)
        return
    if args.workload == "c1":
        if args.impl != "ours" or world != 1:
            print(json.dumps({"impl": args.impl, "workload": "c1",
                              "unavailable": "the plain-config mode runs one GPU, product arm only"}))
            return
        run_c1(args)
        return
    if args.workload == "kernels":
        if args.impl != "ours" or world != 1:
            print(json.dumps({"impl": args.impl, "workload": "kernels",
                              "unavailable": "the per-kernel mode runs one GPU, product arm only"}))
            return
        run_kernels(args)
        return
    if args.workload == "ops":
        if args.impl != "ours" or world != 1:
            print(json.dumps({"impl": args.impl, "workload": "ops",
                              "unavailable": "the per-op mode runs one GPU, product arm only"}))
            return
        if args.steps == STEPS_FULL:
            args.steps = 20
        run_ops(args)
        return
    if args.workload == "c5":
        if args.impl != "ours" or world != 1:
            print(json.dumps({"impl": args.impl, "workload": "c5",
                              "unavailable": "the avalanche mode runs one GPU, product arm only"}))
            return
        if args.steps == STEPS_FULL:
            args.steps = 2500
        run_c5(args)
        return
    if args.workload == "c4":
        if args.impl != "ours" or world != 1:
            print(json.dumps({"impl": args.impl, "workload": "c4",
                              "unavailable": "the batched-instances mode runs one GPU, product arm only"}))
            return
        if args.steps == STEPS_FULL:
            args.steps = 2000
        run_c4(args)
        return

    if args.impl == "reference":
        # the reference's CPU algorithm (oracle port) on the host cores; rank 0 only
        if rank != 0:
            return
        S0 = window_start(args)
        rate, steps, ps, dt = cpu_sample(args.cpu_electrons, max(S0, args.warmup), args.steps, args.cpu_budget * 3)
        S0 = max(S0, args.warmup, 1)
        cores = omp_threads()
        sample = (f"{args.cpu_electrons} e- of the same beam (1/{args.electrons // args.cpu_electrons} of it), "
                  f"advanced untimed to step {S0}, then steps {S0}-{S0 + steps} timed: {ps:.3g} particle-steps "
                  f"in {dt:.2f}s")
        line = {"impl": "reference", "metric": "particle-steps/s", "value": rate, "unit": "particle-steps/s",
                "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(steps, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": window_label(S0, steps), "sample_electrons": args.cpu_electrons,
                           "start_step": S0, "steps_timed": steps},
                "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    r = run_ours(args, rank, world)
    # CPU baseline (rank 0, N=1): the oracle port steps a subsample of the GPU run's state at the window's start
    cpu = None
    if r.get("cpu_state") is not None:
        st = r.pop("cpu_state")
        rate, steps, ps, dt, c0 = cpu_sample_from_state(st, 1000, args.steps, args.cpu_budget)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": omp_threads(), "kind": "port",
               "sample": f"every {st['every']}th alive particle of each species of the GPU run at step {st['step']} "
                         f"({', '.join(f'{k} {v}' for k, v in c0.items())}), stepped by the oracle over steps "
                         f"{st['step']}-{st['step'] + steps}: {ps:.3g} particle-steps in {dt:.2f} s",
               "start_step": st["step"], "steps_timed": steps}
    if rank == 0:
        value = r["particle_steps"] / (r["ms"] * 1e-3)
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps,
                "higher_is_better": True, "scaling": "strong" if (args.split_beam and world > 1) else "weak",
                "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32/f64",
                "data": "synthetic",
                "config": {"workload": window_label(r["start_step"], args.steps),
                           "electrons_per_gpu": (args.electrons // world if (args.split_beam and world > 1)
                                                 else args.electrons),
                           "form": args.form, "start_step": r["start_step"], "steps_timed": args.steps,
                           "l2": "state > 1 GB per step, larger than L2 (no flush needed)",
                           "counts_at_window_start": r["start_counts"], "counts_at_window_end": r["counts"]},
                "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": r["e2e"], "gpu_launches": r["launches"],
                "clocks": r["clocks"], "particle_steps": r["particle_steps"], "whole_run": r["whole"],
                "job_diagnostics": r["job"], "vs_fp64": r["compare"]}
        if world == 1 and not args.no_extras:
            line["workloads"] = run_extras(args)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
