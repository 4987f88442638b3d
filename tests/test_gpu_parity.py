"""GPU parity: libsfp.so kernels (through the C-ABI) vs the CPU oracle and
the reference fixtures.

Tolerances: the device code computes in float64 with the reference's
operation order but lets the compiler fuse multiply-adds and uses CUDA's
libm, so single operations agree to ~1e-15 relative and whole runs to the
1e-10 relative bound of deterministic pushes; integer/index results and
event decisions are compared exactly.
"""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle as orc
from conftest import golden
from gpu_helpers import (build_fields_pair, cuda_or_skip, dev, golden_case_fields, host, product_rs_tables, ptr,
                         sim_case_species, stream)

pytestmark = pytest.mark.gpu

RTOL_OP = 1e-13     # one kernel application (FMA contraction vs the reference order)
RTOL_RUN = 1e-10    # whole deterministic runs


def _rel(a, b, axis_scale=True):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    if a.size == 0:
        return 0.0
    scale = np.max(np.abs(b), axis=-1, keepdims=True) if axis_scale and b.ndim > 1 else np.max(np.abs(b))
    return float(np.max(np.abs(a - b) / (scale + 1e-300)))


def test_per_op_pushers_match_reference():
    cuda_or_skip()
    from sfparticles_b200 import _lib
    g = golden("ref_pushers.npz")
    u, E, B, pr, dt = g["u"], g["E"], g["B"], g["pruned"], float(g["dt"])
    N = u.shape[1]
    Ed = [dev(a) for a in E]
    Bd = [dev(a) for a in B]
    prd = dev(pr)
    for q, tag in ((-orc.E_CHARGE, "m"), (orc.E_CHARGE, "p")):
        ud = [dev(a) for a in u]
        ig = dev(1 / np.sqrt(1 + (u ** 2).sum(0)))
        _lib.call("sfp_boris", *map(ptr, ud + [ig] + Ed + Bd), q, N, ptr(prd), dt, stream())
        got = np.stack([host(t) for t in ud + [ig]])
        assert _rel(got, g[f"boris_{tag}"]) < RTOL_OP
    for ae in (1.14e-3, 0.3):
        ud = [dev(a) for a in u]
        sd = [dev(a) for a in g["s"]]
        ig = dev(1 / np.sqrt(1 + (u ** 2).sum(0)))
        _lib.call("sfp_boris_tbmt", *map(ptr, ud + [ig] + sd + Ed + Bd), -orc.E_CHARGE, ae, N, ptr(prd), dt, stream())
        got = np.stack([host(t) for t in ud + [ig] + sd])
        assert _rel(got, g[f"tbmt_{ae}"]) < RTOL_OP
    chi = dev(g["chi_in"])
    for fn, tag in (("sfp_LL_push", "LL"), ("sfp_CLL_push", "CLL")):
        ud = [dev(a) for a in u]
        ig = dev(1 / np.sqrt(1 + (u ** 2).sum(0)))
        _lib.call(fn, *map(ptr, ud + [ig, chi]), N, ptr(prd), dt, stream())
        assert _rel(np.stack([host(t) for t in ud + [ig]]), g[tag]) < RTOL_OP
    ud = [dev(a) for a in u]
    ig = dev(g["ig_in"])
    chi_o = dev(np.zeros(N))
    _lib.call("sfp_update_chi", *map(ptr, Ed + Bd + ud + [ig, chi_o]), N, ptr(prd), stream())
    ref = g["update_chi"]
    assert np.max(np.abs(host(chi_o) - ref) / (np.abs(ref) + 1e-300)) < 1e-12
    xd = [dev(a) for a in g["x"]]
    _lib.call("sfp_push_position", *map(ptr, xd + ud + [ig]), N, ptr(prd), dt, stream())
    assert _rel(np.stack([host(t) for t in xd]), g["push_position"]) < RTOL_OP


def test_per_op_events_and_appends_match_reference():
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib
    g = golden("ref_pushers.npz")
    u, pr = g["u"], g["pruned"]
    N = u.shape[1]
    ev = dev(g["event"])
    delta = dev(g["delta"])
    ud = [dev(a) for a in u]
    ig = dev(g["ig_in"])
    prd = dev(pr)
    _lib.call("sfp_photon_recoil", *map(ptr, ud + [ig, ev, delta]), N, ptr(prd), stream())
    assert _rel(np.stack([host(t) for t in ud + [ig]]), g["photon_recoil"]) < RTOL_OP
    ev2 = dev(g["event"])
    ig_in = dev(g["ig_in"])
    _lib.call("sfp_pick_hard_photon", ptr(ev2), ptr(delta), ptr(ig_in), 2.0, N, stream())
    np.testing.assert_array_equal(host(ev2).astype(bool), g["pick_hard_photon"])
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.call("sfp_bool_sum", ptr(ev), N, ptr(cnt), stream())
    n = int(cnt.item())
    assert n == int(g["bool_sum"])
    L = _lib.load()
    ws = torch.empty(int(L.sfp_find_event_index_workspace(N)) // 8 + 1, dtype=torch.int64, device="cuda")
    idx = torch.empty(n, dtype=torch.int64, device="cuda")
    _lib.call("sfp_find_event_index", ptr(ev), n, N, ptr(idx), ptr(ws), ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(idx), g["find_event_index"])
    x = [dev(a) for a in g["x"]]
    uu = [dev(a) for a in u]
    M0 = 7
    dst = [dev(np.zeros(M0 + n)) for _ in range(7)]
    dpr = dev(np.ones(M0 + n, dtype=np.uint8))
    _lib.call("sfp_create_photon", *map(ptr, x + uu + dst), ptr(dpr), ptr(idx), ptr(delta), M0, n, stream())
    assert _rel(np.stack([host(t) for t in dst]), g["create_photon"]) < RTOL_OP
    np.testing.assert_array_equal(host(dpr).astype(bool), g["create_photon_pruned"])
    for inv in (0, 1):
        dst = [dev(np.zeros(M0 + n)) for _ in range(7)]
        dpr = dev(np.ones(M0 + n, dtype=np.uint8))
        spr = dev(pr)
        _lib.call("sfp_create_pair", *map(ptr, x + uu), ptr(spr), *map(ptr, dst), ptr(dpr), ptr(idx), ptr(delta), M0,
                  n, inv, stream())
        assert _rel(np.stack([host(t) for t in dst]), g[f"create_pair_{inv}"]) < RTOL_OP
        np.testing.assert_array_equal(host(dpr).astype(bool), g[f"create_pair_{inv}_pruned"])
        np.testing.assert_array_equal(host(spr).astype(bool), g[f"create_pair_{inv}_src_pruned"])


@pytest.mark.parametrize("N,p", [(0, 0.5), (1, 1.0), (4095, 0.3), (4096, 1.0), (4097, 0.0), (5_000_017, 0.013),
                                 (3_000_000, 1.0)])
def test_find_event_index_ragged_sizes(N, p):
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib
    rng = np.random.default_rng(N)
    ev = rng.random(N) < p
    evd = dev(ev)
    n = int(ev.sum())
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.call("sfp_bool_sum", ptr(evd), N, ptr(cnt), stream())
    assert int(cnt.item()) == n
    L = _lib.load()
    ws = torch.empty(int(L.sfp_find_event_index_workspace(N)) // 8 + 1, dtype=torch.int64, device="cuda")
    idx = torch.full((max(n, 1),), -1, dtype=torch.int64, device="cuda")
    _lib.call("sfp_find_event_index", ptr(evd), n, N, ptr(idx), ptr(ws), ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(idx)[:n], np.nonzero(ev)[0])


def test_field_programs_match_reference():
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib, program
    g = golden("ref_fields.npz")
    cases = json.loads(str(g["cases"]))
    sums = json.loads(str(g["sums"]))
    for i, spec in enumerate(list(range(len(cases))) + sums):
        f, _ = build_fields_pair(spec, cases)
        mod = program.get_module(f, form=None, qed=None)
        x, y, z, t = g[f"pts_{i}"]
        ref = g[f"out_{i}"]
        got = np.zeros_like(ref)
        prm = f.params_device()
        xd, yd, zd = dev(x), dev(y), dev(z)
        pr = dev(np.zeros(1, dtype=np.uint8))
        out = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(6)]
        for j in range(x.size):  # one time per point, as the fixture was made
            _lib.call("sfp_field_eval", mod.handle, ptr(prm), ptr(xd[j:j + 1]), ptr(yd[j:j + 1]), ptr(zd[j:j + 1]),
                      float(t[j]), 1, ptr(pr), *map(ptr, out), stream())
            got[:, j] = [o.item() for o in out]
        err = _rel(got, ref)
        assert err < 1e-13, (spec, err)


@pytest.mark.parametrize("kind", ["photon", "pair"])
def test_rejection_samplers_match_oracle(kind):
    cuda_or_skip()
    from sfparticles_b200 import _lib
    from sfparticles_b200.qed import device_tables
    g = golden("ref_rs_events.npz")
    iA, dA, zN, zmax = product_rs_tables()
    ig, chi, pr = g[f"{kind}_ig"], g[f"{kind}_chi"], g[f"{kind}_pruned"]
    N = ig.size
    seed, st, step = [int(v) for v in g[f"{kind}_key"]]
    dt = float(g[f"{kind}_dt"])
    # oracle on the same (product) table
    L = orc.lib()
    ev_o = np.zeros(N, dtype=np.uint8)
    de_o = np.full(N, -1.0)
    fn = L.orc_photon_from_rejection_sampling if kind == "photon" else L.orc_pair_from_rejection_sampling
    igc, chic, prc = np.ascontiguousarray(ig), np.ascontiguousarray(chi), pr.astype(np.uint8)
    fn(orc._p(igc), orc._p(chic), dt, N, orc._p(prc), orc._p(ev_o), orc._p(de_o), orc._p(iA), orc._p(dA), zN, zmax,
       seed, st, step)
    evd, ded = dev(np.zeros(N, dtype=np.uint8)), dev(np.full(N, -1.0))
    tab = device_tables.rs_table("cuda")
    name = "sfp_photon_from_rejection_sampling" if kind == "photon" else "sfp_pair_from_rejection_sampling"
    igd, chid, prd = dev(ig), dev(chi), dev(pr)
    _lib.call(name, ptr(igd), ptr(chid), dt, N, ptr(prd), ptr(evd), ptr(ded), ctypes.byref(tab), seed, st,
              step, stream())
    np.testing.assert_array_equal(host(evd), ev_o)
    np.testing.assert_allclose(host(ded), de_o, rtol=1e-14, atol=0)
    assert ev_o.sum() > 50


def test_optical_depth_update_matches_oracle():
    cuda_or_skip()
    from sfparticles_b200 import _lib
    from sfparticles_b200.qed import device_tables, tables
    d = tables.od_tables()
    rng = np.random.default_rng(9)
    N = 200_000
    chi = 10 ** rng.uniform(-3.5, 3.2, N)
    ig = 10 ** rng.uniform(-4, -1, N)
    tau = np.where(rng.random(N) < 0.3, 0.0, rng.exponential(1.0, N))
    pr = (rng.random(N) < 0.05).astype(np.uint8)
    dt = 2e-15
    seed, st, step = 77, 2, 5
    for kind, key in (("photon", 0), ("pair", 1)):
        t_o = orc.make_od_table(d[f"{kind}_rate_total"], d[f"{kind}_cumulative"], float(d["log_chi_min"]),
                                float(d["log_chi_delta"]), float(d["log_delta_min"]), float(d["log_delta_delta"]))
        tau_o = tau.copy()
        ev_o = np.zeros(N, dtype=np.uint8)
        de_o = np.zeros(N)
        chic, igc = np.ascontiguousarray(chi), np.ascontiguousarray(ig)
        orc.lib().orc_update_tau(orc._p(tau_o), orc._p(igc), orc._p(chic), dt, N, orc._p(pr), orc._p(ev_o),
                                 orc._p(de_o), ctypes.byref(t_o), seed, st, step)
        tab = device_tables.od_tables("cuda")[key]
        taud, evd, ded = dev(tau), dev(np.zeros(N, dtype=np.uint8)), dev(np.zeros(N))
        igd, chid, prd = dev(ig), dev(chi), dev(pr)
        _lib.call("sfp_update_tau", ptr(taud), ptr(igd), ptr(chid), dt, N, ptr(prd), ptr(evd), ptr(ded),
                  ctypes.byref(tab), seed, st, step, stream())
        np.testing.assert_array_equal(host(evd), ev_o)
        np.testing.assert_allclose(host(ded), de_o, rtol=1e-11, atol=0)
        np.testing.assert_allclose(host(taud), tau_o, rtol=1e-11, atol=1e-13)
        assert 100 < ev_o.sum() < N


def _run_gpu_case(g, graph_chunk=64):
    import sfparticles_b200 as S
    case = json.loads(str(g["case"]))
    species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
    sim = S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                       photon_threshold=case["thr"], seed=case["seed"], graph_chunk=graph_chunk)
    sim.start(case["steps"])
    return case, species, sim


def _oracle_case(g):
    from test_oracle_golden import oracle_case_sim
    case, sim, species = oracle_case_sim(g)
    iA, dA, zN, zmax = product_rs_tables()
    sim.qed = ("rs", iA, dA)
    sim.run(case["steps"])
    for p in species:
        p.prune()
    return species


@pytest.mark.parametrize("name", ["cascade", "spin_photon", "spin_LL", "spin_CLL", "CLL_focused", "push_only",
                                  "simple_LL", "simple_t4"])
def test_fused_step_matches_oracle(name):
    """Fused Simulation.start on the GPU vs the oracle step loop, same Philox
    keys: identical particle counts and order, states within tolerance."""
    cuda_or_skip()
    g = golden(f"ref_sim_{name}.npz")
    case, species, sim = _run_gpu_case(g)
    ospecies = _oracle_case(g)
    for p, o in zip(species, ospecies):
        keys = ["x", "y", "z", "ux", "uy", "uz"] + (["sx", "sy", "sz"] if o.spin else [])
        got = np.stack([getattr(p, k) for k in keys])
        ref = np.stack([getattr(o, k) for k in keys])
        assert got.shape == ref.shape, (p.name, got.shape, ref.shape)
        assert _rel(got, ref) < RTOL_RUN, (p.name, _rel(got, ref))
    assert sim.particle_steps > 0


@pytest.mark.parametrize("name", ["od_emission", "od_spin_emission", "od_pairs"])
def test_fused_optical_depth_matches_oracle_and_reference(name):
    """Optical-depth runs (emission with recoil in a laser pulse; pair creation
    by photons in a static field): the fused float64 step vs the oracle and vs
    the reference's own Simulation.start fed the same keyed draws."""
    cuda_or_skip()
    import sfparticles_b200 as S
    from sfparticles_b200 import qed
    from test_oracle_golden import oracle_od_case_sim
    g = golden(f"ref_sim_{name}.npz")
    case = json.loads(str(g["case"]))
    init = tuple(np.array(a) for a in g["init"])
    qed.set_method("od")
    try:
        if "n_e" in case:
            if case.get("spin"):
                ele = S.SpinParticles("ele", -1, 1, N=case["n_e"],
                                      props=init + tuple(np.array(a) for a in g["spin_init"]))
            else:
                ele = S.Particles("ele", -1, 1, N=case["n_e"], props=init)
            pho = S.Particles("pho", 0, 0)
            ele.set_photon(pho)
            species = [ele, pho]
        else:
            ele, pos = S.Particles("ele", -1, 1), S.Particles("pos", 1, 1)
            pho = S.Particles("pho", 0, 0, N=case["n_g"], props=init)
            pho.set_pair(ele, pos)
            species = [ele, pos, pho]
    finally:
        qed.set_method("rs")
    sim = S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                       photon_threshold=case["thr"], seed=case["seed"])
    sim.start(case["steps"])
    _, osim, ospecies = oracle_od_case_sim(g)
    osim.run(case["steps"])
    for i, (p, o) in enumerate(zip(species, ospecies)):
        o.prune()
        keys = ["x", "y", "z", "ux", "uy", "uz"] + (["sx", "sy", "sz"] if o.spin else [])
        got = np.stack([getattr(p, k) for k in keys])
        ref = np.stack([getattr(o, k) for k in keys])
        assert got.shape == ref.shape == g[f"s{i}_state"].shape, (p.name, got.shape, ref.shape)
        assert got.shape[1] > 0, p.name
        assert _rel(got, ref) < RTOL_RUN, (p.name, _rel(got, ref))
        assert _rel(got, g[f"s{i}_state"]) < RTOL_RUN, (p.name, _rel(got, g[f"s{i}_state"]))


@pytest.mark.parametrize("name", ["spin_LL", "spin_CLL", "CLL_focused", "push_only", "simple_LL", "simple_t4"])
def test_fused_deterministic_push_matches_reference(name):
    """Emission off: the GPU run vs the reference's own Simulation.start, 1e-10.
    simple_LL is Landau-Lifshitz on a plain (non-spin) species, whose chi is
    recomputed after the Boris push with the t+dt/2 fields
    (particles.py:264-281); simple_t4 is simple_laser_pulse with a
    fourth-order temporal envelope (fields.py:69-118)."""
    cuda_or_skip()
    g = golden(f"ref_sim_{name}.npz")
    case, species, sim = _run_gpu_case(g)
    for i, p in enumerate(species):
        keys = ["x", "y", "z", "ux", "uy", "uz"] + (["sx", "sy", "sz"] if "sx" in p.attrs else [])
        got = np.stack([getattr(p, k) for k in keys])
        assert _rel(got, g[f"s{i}_state"]) < RTOL_RUN


def test_graph_replay_equals_eager_launches():
    cuda_or_skip()
    g = golden("ref_sim_cascade.npz")
    _, a, _ = _run_gpu_case(g, graph_chunk=16)
    _, b, _ = _run_gpu_case(g, graph_chunk=0)
    for p, q in zip(a, b):
        for k in ("x", "y", "z", "ux", "uy", "uz"):
            np.testing.assert_array_equal(getattr(p, k), getattr(q, k))


def test_repeated_start_continues_the_run():
    """start(a); start(b) == start(a + b) (simulation.py:89-102 keeps step and t)."""
    cuda_or_skip()
    import sfparticles_b200 as S
    g = golden("ref_sim_push_only.npz")  # deterministic: pruning between starts renumbers slots
    case = json.loads(str(g["case"]))

    def run(parts):
        species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
        sim = S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                           photon_threshold=case["thr"], seed=case["seed"])
        for n in parts:
            sim.start(n)
        return species, sim

    a, sa = run([case["steps"]])
    b, sb = run([100, case["steps"] - 100])
    assert sa.step == sb.step and sa.t == sb.t
    for p, q in zip(a, b):
        assert p.N_buffered == q.N_buffered
        np.testing.assert_array_equal(np.stack([p.x, p.ux]), np.stack([q.x, q.ux]))


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_photon_positions_read_from_a_live_run(form):
    """A device-resident run stores photon positions as of its position
    epoch (the step kernels advance them in registers) and writes them out
    when they are read.  Read in the middle of a run they equal those of a
    run stopped at that step; a run read there continues to the end state of
    one never read, up to float64 rounding of the two advances."""
    cuda_or_skip()
    import sfparticles_b200 as S
    g = golden("ref_sim_cascade.npz")
    case = json.loads(str(g["case"]))
    n1, n2 = case["steps"] // 2, case["steps"] - case["steps"] // 2

    def new():
        species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
        return S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                            photon_threshold=case["thr"], seed=case["seed"], form=form)

    a = new()
    a.run_on_device(n1)
    pho = a.all_particles[2]
    assert pho.m == 0
    alive = ~pho._to_be_pruned[: pho.N_buffered]
    mid = np.stack([getattr(pho, k)[: pho.N_buffered][alive] for k in ("x", "y", "z")])
    assert mid.shape[1] > 100  # photons exist at the read
    c = new()
    c.run_on_device(n1)
    c.finish()
    np.testing.assert_array_equal(mid, np.stack([c.all_particles[2].x, c.all_particles[2].y, c.all_particles[2].z]))
    a.run_on_device(n2)
    a.finish()
    b = new()
    b.run_on_device(n1 + n2)
    b.finish()
    for p, q in zip(a.all_particles, b.all_particles):
        assert p.N_buffered == q.N_buffered, (p.name, p.N_buffered, q.N_buffered)
        got = np.stack([getattr(p, k) for k in ("x", "y", "z", "ux", "uy", "uz")])
        ref = np.stack([getattr(q, k) for k in ("x", "y", "z", "ux", "uy", "uz")])
        assert _rel(got, ref) < 1e-12, (p.name, _rel(got, ref))


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_kernel_variants_give_the_same_results(form):
    """Every variant of the massive kernel (items per thread, register
    budget) and of the photon kernel (sub-tiles in flight, register budget)
    computes the same arithmetic in the same append order: the same event
    counts and the same states up to the compiler's different FMA
    contraction per variant (1e-10 relative in float64, 1e-4 in float32)."""
    cuda_or_skip()
    import itertools
    import sfparticles_b200 as S
    from sfparticles_b200.autotune import VARIANTS
    g = golden("ref_sim_cascade.npz")
    case = json.loads(str(g["case"]))
    mv, pv = VARIANTS[(form, "rs")]
    bound = 1e-10 if form == "fp64" else 1e-4
    ref = None
    for m, p in itertools.zip_longest(mv, pv, fillvalue=None):
        m = m or mv[0]
        p = p or pv[0]
        species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
        sim = S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                           photon_threshold=case["thr"], seed=case["seed"], form=form, m_stages=m[0], min_blocks=m[1],
                           p_stages=p[0], p_min_blocks=p[1])
        sim.start(case["steps"])
        got = [np.stack([getattr(q, k) for k in ("x", "y", "z", "ux", "uy", "uz")]) for q in species]
        if ref is None:
            ref = got
            continue
        for a, b in zip(got, ref):
            assert a.shape == b.shape, (m, p, a.shape, b.shape)
            err = _rel(a, b)
            print(f"{form} massive {m} photon {p}: max rel diff {err:.2e}")
            assert err < bound, (m, p, err)


def test_autotune_selects_a_compiled_variant(tmp_path, monkeypatch):
    cuda_or_skip()
    import sfparticles_b200 as S
    from sfparticles_b200 import autotune, program
    monkeypatch.setattr(program, "CACHE", str(tmp_path))
    g = golden("ref_sim_cascade.npz")
    case = json.loads(str(g["case"]))
    species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
    sim = S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                       photon_threshold=case["thr"], seed=case["seed"], form="fp32")
    sim.run_on_device(100)
    step, t = sim.step, sim.t
    best, times = autotune.tune(sim, sample=10_000, steps=2)
    mv, pv = autotune.VARIANTS[("fp32", "rs")]
    assert tuple(best[0]) in mv and tuple(best[1]) in pv and len(times) == len(mv) + len(pv)
    assert (sim.m_stages, sim.min_blocks) == tuple(best[0]) and (sim.p_stages, sim.p_min_blocks) == tuple(best[1])
    assert (sim.step, sim.t) == (step, t)  # tuning ran on a copy
    assert os.path.exists(os.path.join(str(tmp_path), "autotune.json"))
    sim.run_on_device(10)
    sim.finish()


@pytest.mark.parametrize("name", ["cascade", "spin_photon", "CLL_focused"])
def test_ops_engine_matches_fused_fp64(name):
    """The reference's step loop over the one-for-one kernels (engine 'ops')
    and the fused step draw the same Philox numbers, so they take the same
    events and give the same states within the float64 bound."""
    cuda_or_skip()
    import sfparticles_b200 as S
    g = golden(f"ref_sim_{name}.npz")
    case = json.loads(str(g["case"]))
    out = []
    for engine in ("fused", "ops"):
        species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
        sim = S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                           photon_threshold=case["thr"], seed=case["seed"], engine=engine)
        sim.start(case["steps"])
        out.append((species, sim))
    (a, sa), (b, sb) = out
    assert sa.step == sb.step and sa.particle_steps == sb.particle_steps
    for p, q in zip(a, b):
        assert p.N_buffered == q.N_buffered, (p.name, p.N_buffered, q.N_buffered)
        keys = ["x", "y", "z", "ux", "uy", "uz"] + (["sx", "sy", "sz"] if "sx" in p.attrs else [])
        for k in keys:
            assert _rel(getattr(q, k), getattr(p, k)) < RTOL_RUN, (name, p.name, k)


@pytest.mark.parametrize("preset", ["gaussian_laser_pulse", "simple_laser_pulse"])
def test_far_field_cut_is_exact(preset):
    """Far outside the pulse the field kernels return 0 without evaluating
    the pulse; across the cut (|phi| / kc from 20 to 40) they agree with the
    oracle, which always evaluates the formula: 0 where it underflows, to
    1e-13 where it does not."""
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib, fields as F, program
    from sfparticles_b200.constants import C
    kw = dict(a0=200.0, w0=3e-6, ctau=6.366e-6, direction=-1, x0=4.5e-5)
    f, o = getattr(F, preset)(**kw), getattr(orc, preset)(**kw)
    k0 = 2 * np.pi / 0.8e-6
    t = 1e-13
    # phase distance from the pulse centre in units of kc, both sides
    s = np.concatenate([np.linspace(20, 40, 2001), -np.linspace(20, 40, 2001)])
    x = kw["x0"] - C * t + s * kw["ctau"]
    rng = np.random.default_rng(3)
    y, z = rng.normal(0, 2e-6, x.size), rng.normal(0, 2e-6, x.size)
    ref = np.stack(orc.field_eval(o, x, y, z, t))
    mod = program.get_module(f, form=None, qed=None)
    prm = f.params_device()
    xd, yd, zd = dev(x), dev(y), dev(z)
    pr = dev(np.zeros(x.size, dtype=np.uint8))
    out = [torch.full((x.size,), np.nan, dtype=torch.float64, device="cuda") for _ in range(6)]
    _lib.call("sfp_field_eval", mod.handle, ptr(prm), ptr(xd), ptr(yd), ptr(zd), float(t), x.size, ptr(pr),
              *map(ptr, out), stream())
    got = np.stack([host(q) for q in out])
    # near the cut the envelope is a float64 denormal (exp(-729..-745)), good
    # to a few digits only: compare with an absolute floor far below any field
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-280)
    far = np.abs(s) > 29.0
    assert far.any() and (~far).any()
    assert np.all(ref[:, far] == 0.0) and np.all(got[:, far] == 0.0), preset
