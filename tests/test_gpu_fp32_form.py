"""The float32 form of the fused step vs the float64 form and the reference.

Deterministic pushes (emission off) are compared with the reference's own
runs; the error of each output is printed and bounded.  Monte-Carlo results
are compared with the float64 form on the same seeds: both forms draw the
same Philox numbers, so they take the same events except within float32
rounding of an acceptance threshold, and the photon spectrum and pair yield
must agree to 1 %.
"""
import json
import math

import numpy as np
import pytest

from conftest import golden
from gpu_helpers import cuda_or_skip, golden_case_fields, sim_case_species

pytestmark = pytest.mark.gpu

# error bounds of the float32 form for deterministic runs, relative to each
# component's largest magnitude
FP32_RUN_BOUND = {"push_only": 1e-4, "spin_LL": 2e-4, "spin_CLL": 2e-4, "CLL_focused": 2e-4, "simple_LL": 2e-4,
                  "simple_t4": 1e-4}


def _run(g, form, seed=None):
    import sfparticles_b200 as S
    case = json.loads(str(g["case"]))
    species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
    sim = S.Simulation(*species, dt=float(g["dt"]), fields=golden_case_fields(g), print_every=None,
                       photon_threshold=case["thr"], seed=case["seed"] if seed is None else seed, form=form)
    sim.start(case["steps"])
    return species, sim


@pytest.mark.parametrize("name", sorted(FP32_RUN_BOUND))
def test_fp32_deterministic_push_error_vs_reference(name):
    """The float32 form's error against the reference's own float64 run, per
    output: max |error| / max |reference| of each component, printed as one
    table row (run with -s to see it) and bounded."""
    cuda_or_skip()
    g = golden(f"ref_sim_{name}.npz")
    species, _ = _run(g, "fp32")
    for i, p in enumerate(species):
        keys = ["x", "y", "z", "ux", "uy", "uz"] + (["sx", "sy", "sz"] if "sx" in p.attrs else [])
        ref = g[f"s{i}_state"]
        errs = {}
        for j, k in enumerate(keys):
            got = getattr(p, k)
            scale = np.max(np.abs(ref[j])) + 1e-300
            errs[k] = float(np.max(np.abs(got - ref[j])) / scale)
        print(f"\nFP32 error | {name} | {p.name} | " + " | ".join(f"{k} {v:.1e}" for k, v in errs.items()))
        for k, err in errs.items():
            assert err < FP32_RUN_BOUND[name], (name, k, err)


def _c2_shaped(n, seed, form, steps=3000, a0=200.0):
    import sfparticles_b200 as S
    from sfparticles_b200.constants import C
    from sfparticles_b200.fields import gaussian_laser_pulse
    T0 = 0.8e-6 / C
    dt = T0 / 100
    L = C * (steps * dt) / 2
    rng = np.random.default_rng(seed)
    g = 2000 * (1 + 0.01 * rng.normal(size=n))
    props = (rng.normal(-L, 5e-6, n), rng.normal(0, 1e-6, n), rng.normal(0, 1e-6, n), np.sqrt(g * g - 1),
             np.zeros(n), np.zeros(n))
    ele = S.Particles("ele", -1, 1, N=n, props=props)
    pos = S.Particles("pos", 1, 1)
    pho = S.Particles("pho", 0, 0)
    ele.set_photon(pho)
    pos.set_photon(pho)
    pho.set_pair(ele, pos)
    ctau = C * 25e-15 / (2 * math.sqrt(math.log(2) / 2))
    fld = gaussian_laser_pulse(a0, 3e-6, ctau, direction=-1, x0=L)
    sim = S.Simulation(ele, pos, pho, dt=dt, fields=fld, print_every=None, seed=seed, form=form)
    sim.start(steps)
    return ele, pos, pho, sim


def test_fp32_spectrum_and_pair_yield_within_one_percent_of_fp64():
    """Scaled-cascade shape (a0 = 200, dt = T0/100, 3000 steps), 8 seeds of
    5e5 electrons (~2e5 pairs per form): photon spectrum (64 log bins above
    the 2 m c^2 threshold) relative L1 and pair-yield difference <= 1 %.
    Once two runs differ in one emission, later slots -- and so the Philox
    streams keyed by them -- differ too, so the pair yields are compared at
    their statistical floor: the 1 % bound is ~3 sigma of the difference."""
    cuda_or_skip()
    from sfparticles_b200 import diagnostics as D
    spec64 = spec32 = None
    pairs64 = pairs32 = 0
    for seed in range(8):
        e64, p64, g64, s64 = _c2_shaped(500_000, 500 + seed, "fp64")
        e32, p32, g32, s32 = _c2_shaped(500_000, 500 + seed, "fp32")
        hi = max(D.photon_energies(g64).max(), D.photon_energies(g32).max())
        h64, _ = D.photon_spectrum(g64, 64, 2.0, hi)
        h32, _ = D.photon_spectrum(g32, 64, 2.0, hi)
        spec64 = h64 if spec64 is None else spec64 + h64
        spec32 = h32 if spec32 is None else spec32 + h32
        pairs64 += p64.N_buffered
        pairs32 += p32.N_buffered
    l1 = D.spectrum_rel_l1(spec32, spec64)
    dpair = D.rel_diff(pairs32, pairs64)
    print(f"photons fp64 {spec64.sum():.0f} fp32 {spec32.sum():.0f}; spectrum rel L1 {l1:.4f}; "
          f"pairs fp64 {pairs64} fp32 {pairs32} rel diff {dpair:.4f}")
    floor = math.sqrt(1.0 / pairs64 + 1.0 / pairs32)
    print(f"pair-yield statistical floor (1 sigma of the difference): {floor:.4f}")
    assert spec64.sum() > 1e7 and pairs64 > 1e5
    assert l1 <= 0.01, l1
    assert dpair <= 0.01, dpair


def test_fp64_gpu_statistics_match_reference_runs():
    """1000 electrons of the config-1 beam against a0 = 50, 1500 steps, on the
    GPU (float64 form): photon number, spectrum and mean energy vs the
    reference's own runs (its Numba generator), 3 sigma."""
    cuda_or_skip()
    import os
    import sfparticles_b200 as S
    from sfparticles_b200.fields import gaussian_laser_pulse
    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, "ref_stats.json")) as f:
        spec = json.load(f)["c1_small"]
    got = []
    for form in ("fp64", "fp32"):
        rows = []
        for s in range(6):
            rng = np.random.default_rng(300 + s)
            n, L = spec["n"], spec["L"]
            g = 2000 * (1 + 0.01 * rng.normal(size=n))
            props = (rng.normal(-L, 5e-6, n), rng.normal(0, 1e-6, n), rng.normal(0, 1e-6, n), np.sqrt(g ** 2 - 1),
                     np.zeros(n), np.zeros(n))
            ele = S.Particles("ele", -1, 1, N=n, props=props)
            pho = S.Particles("pho", 0, 0)
            pos = S.Particles("pos", 1, 1)
            ele.set_photon(pho)
            pos.set_photon(pho)
            pho.set_pair(ele, pos)
            fld = gaussian_laser_pulse(spec["a0"], 3e-6, spec["ctau"], direction=-1, x0=L)
            T0 = 0.8e-6 / 299792458.0
            sim = S.Simulation(ele, pos, pho, dt=T0 / 50, fields=fld, print_every=None, seed=900 + s, form=form)
            sim.start(spec["steps"])
            eph = pho.gamma
            hist = np.histogram(np.log10(eph), bins=spec["bins"], range=tuple(spec["hist_range"]))[0]
            rows.append(dict(n_photon=pho.N_buffered, mean_gamma_e=float(np.mean(ele.gamma)), hist=hist))
        got.append(rows)
    ref = spec["runs"]
    for rows in got:
        for key in ("n_photon", "mean_gamma_e"):
            r = np.array([x[key] for x in ref], dtype=float)
            o = np.array([x[key] for x in rows], dtype=float)
            sigma = math.sqrt(r.var(ddof=1) / r.size + o.var(ddof=1) / o.size)
            assert abs(r.mean() - o.mean()) < 3 * sigma, (key, r.mean(), o.mean(), sigma)
        rh = np.array([x["hist"] for x in ref], dtype=float)
        oh = np.array([x["hist"] for x in rows], dtype=float)
        l1 = np.abs(rh.mean(0) - oh.mean(0)).sum() / rh.mean(0).sum()
        assert l1 < 0.03, l1
