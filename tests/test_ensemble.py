"""Ensemble: many collisions in one set of launches (batched uneven
instances).  Each member must give exactly the results it gets alone."""
import math

import numpy as np
import pytest

from gpu_helpers import cuda_or_skip

C = 299792458.0
T0 = 0.8e-6 / C


def member(S, n, a0, g0, seed, steps, form="fp64", dt=T0 / 100):
    """One collision of the batched-instances shape: n electrons (gamma0 g0
    +- 1 %, sigma_perp 1 um, sigma_par 5 um) head-on with a Gaussian pulse of
    amplitude a0 (w0 3 um, 25 fs), meeting mid-run."""
    from sfparticles_b200.fields import gaussian_laser_pulse
    rng = np.random.default_rng(seed)
    L = C * steps * dt / 2
    g = g0 * (1 + 0.01 * rng.normal(size=n))
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
    return S.Simulation(ele, pos, pho, dt=dt, fields=fld, print_every=None, seed=seed, form=form)


def test_ensemble_rejects_mismatched_members():
    import sfparticles_b200 as S
    from sfparticles_b200.fields import simple_laser_pulse
    a = member(S, 10, 50.0, 1000.0, 1, 100)
    b = member(S, 10, 50.0, 1000.0, 2, 100, dt=T0 / 50)
    with pytest.raises(ValueError, match="dt"):
        S.Ensemble([a, b])
    c = member(S, 10, 50.0, 1000.0, 3, 100, form="fp32")
    with pytest.raises(ValueError, match="form"):
        S.Ensemble([a, c])
    d = member(S, 10, 50.0, 1000.0, 4, 100)
    d.fields = simple_laser_pulse(10.0, 3e-6, 5e-6)
    with pytest.raises(ValueError, match="structure"):
        S.Ensemble([a, d])
    with pytest.raises(ValueError, match="more than one"):
        S.Ensemble([a, a])


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_ensemble_members_equal_standalone_runs(form):
    """Six members with uneven sizes and parameters drawn like the batched
    workload (a0 log-uniform in [10, 500], n log-uniform in [1, 3000], gamma0
    uniform in [500, 5000]), photon emission and pair creation; every
    species of every member is identical to the member's standalone run on
    the same kind of step module (field parameters read from global memory).
    A standalone run on its default module (parameters in the constant bank)
    is the same arithmetic compiled apart: equal up to the compiler's
    different FMA contraction (1e-10 relative in float64, 1e-4 in float32)."""
    cuda_or_skip()
    import sfparticles_b200 as S
    rng = np.random.default_rng(0)
    steps = 300
    spec = [(int(round(10 ** rng.uniform(0, math.log10(3000)))), 10 ** rng.uniform(1, math.log10(500)),
             rng.uniform(500, 5000), 70 + k) for k in range(6)]
    spec[0] = (3000, 500.0, 5000.0, 70)  # one member that surely creates pairs
    alone, alone_const = [], []
    for n, a0, g0, seed in spec:
        for const, out in ((False, alone), (True, alone_const)):
            sim = member(S, n, a0, g0, seed, steps, form)
            sim._const_field = const
            sim.start(steps)
            out.append(sim)
    ens = S.Ensemble([member(S, n, a0, g0, seed, steps, form) for n, a0, g0, seed in spec])
    ens.start(steps)
    assert ens.step == steps
    total_pairs = 0
    for a, b in zip(alone, ens.sims):
        for p, q in zip(a.all_particles, b.all_particles):
            assert p.N_buffered == q.N_buffered, (p.name, p.N_buffered, q.N_buffered)
            for k in ("x", "y", "z", "ux", "uy", "uz"):
                np.testing.assert_array_equal(getattr(p, k), getattr(q, k))
        total_pairs += a.all_particles[1].N_buffered
    assert total_pairs > 0 and ens.particle_steps == sum(s.particle_steps for s in alone)
    bound = 1e-10 if form == "fp64" else 1e-4
    for a, b in zip(alone_const, ens.sims):
        for p, q in zip(a.all_particles, b.all_particles):
            assert p.N_buffered == q.N_buffered, (p.name, p.N_buffered, q.N_buffered)
            for k in ("x", "y", "z", "ux", "uy", "uz"):
                u, v = getattr(p, k), getattr(q, k)
                err = float(np.max(np.abs(u - v)) / (np.max(np.abs(v)) + 1e-300)) if v.size else 0.0
                assert err < bound, (p.name, k, err)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_live_runs_sharing_a_module_keep_their_own_field_parameters(form):
    """Two simulations of the same field structure share one step module,
    which holds the field parameters of one-instance runs in its constant
    bank.  Both runs stay on the device and advance alternately in chunks;
    each must equal its run alone, bit for bit."""
    cuda_or_skip()
    import sfparticles_b200 as S
    steps, chunk = 300, 50
    spec = [(2000, 400.0, 3000.0, 81), (1500, 30.0, 1500.0, 82)]
    alone = []
    for n, a0, g0, seed in spec:
        sim = member(S, n, a0, g0, seed, steps, form)
        sim.run_on_device(steps)
        sim.finish()
        alone.append(sim)
    pair = [member(S, n, a0, g0, seed, steps, form) for n, a0, g0, seed in spec]
    for _ in range(steps // chunk):
        for sim in pair:
            sim.run_on_device(chunk)
    assert pair[0]._keep[0] is pair[1]._keep[0]  # one module for both runs
    for sim in pair:
        sim.finish()
    for a, b in zip(alone, pair):
        assert a.step == b.step == steps
        for p, q in zip(a.all_particles, b.all_particles):
            assert p.N_buffered == q.N_buffered, (p.name, p.N_buffered, q.N_buffered)
            for k in ("x", "y", "z", "ux", "uy", "uz"):
                np.testing.assert_array_equal(getattr(p, k), getattr(q, k))
    # the two collisions differ (a0 400 against 30): the parameters were not shared
    assert alone[0].all_particles[2].N_buffered != alone[1].all_particles[2].N_buffered
