"""The spin + radiation-reaction avalanche configuration at a small size:
spin electrons at rest between two counter-propagating circularly polarised
pulses (a0 = 800, each the sum of two linear pulses), photon emission with
recoil (optical depth) and pair creation, float32 form; with the learned
photon-energy sampler and with the table."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

C = 299792458.0
T0 = 0.8e-6 / C


def _avalanche(sampler, n=20_000, seed=4):
    import sfparticles_b200 as S
    from sfparticles_b200 import qed
    from sfparticles_b200.fields import gaussian_laser_pulse
    rng = np.random.default_rng(seed)
    qed.set_method("od")
    try:
        props = (rng.uniform(-1e-6, 1e-6, n), rng.uniform(-1e-6, 1e-6, n), rng.uniform(-1e-6, 1e-6, n),
                 np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n), np.ones(n))
        ele = S.SpinParticles("ele", -1, 1, N=n, props=props)
        pos = S.SpinParticles("pos", 1, 1)
        pho = S.Particles("pho", 0, 0)
        ele.set_photon(pho)
        pos.set_photon(pho)
        pho.set_pair(ele, pos)
    finally:
        qed.set_method("rs")
    ctau = C * 30e-15 / (2 * math.sqrt(math.log(2) / 2))
    a = 800.0 / math.sqrt(2.0)
    fld = None
    for d, x0 in ((1, -3e-6), (-1, 3e-6)):  # centres 3 um from the target: they meet after ~375 steps
        for pol, cep in ((0.0, 0.0), (math.pi / 2, math.pi / 2)):
            f = gaussian_laser_pulse(a, 4e-6, ctau, direction=d, x0=x0, pol_angle=pol, cep=cep)
            fld = f if fld is None else fld + f
    sim = S.Simulation(ele, pos, pho, dt=T0 / 100, fields=fld, print_every=None, seed=seed, form="fp32",
                       sampler=sampler)
    sim.start(700)
    return sim


@pytest.mark.parametrize("sampler", ["table", "mlp"])
def test_avalanche_runs_and_conserves_what_it_must(sampler):
    from gpu_helpers import cuda_or_skip
    cuda_or_skip()
    sim = _avalanche(sampler)
    ele, pos, pho = sim.all_particles
    print(f"{sampler}: e- {ele.N_buffered} e+ {pos.N_buffered} photons {pho.N_buffered} "
          f"particle-steps {sim.particle_steps}")
    # pairs come in e-/e+ pairs; the avalanche has started
    assert pos.N_buffered > 0 and pho.N_buffered > 0
    assert ele.N_buffered == 20_000 + pos.N_buffered
    for p in (ele, pos, pho):
        for k in ("x", "y", "z", "ux", "uy", "uz"):
            assert np.all(np.isfinite(getattr(p, k))), (p.name, k)
    # spins stay unit vectors under Thomas-BMT for the initial electrons; pairs start spinless
    s = np.sqrt(ele.sx ** 2 + ele.sy ** 2 + ele.sz ** 2)
    assert np.allclose(s[:20_000][s[:20_000] > 0], 1.0, atol=1e-3)
    assert np.all(np.abs(pos.sx) + np.abs(pos.sy) + np.abs(pos.sz) < 1e-12)
    # photons pass the hard-photon cut delta * gamma >= 2 and take u = delta * u_parent; with
    # gamma >= 2 that is |u| >= 2 |u_parent| / gamma >= sqrt(3)
    assert np.all(np.sqrt(pho.ux ** 2 + pho.uy ** 2 + pho.uz ** 2) >= 1.7)
