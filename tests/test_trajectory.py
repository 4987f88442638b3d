"""Device-side trajectories (sfparticles_b200.trajectory): the record logic
on CPU tensors standing in for a species' device arrays, and the recording
through a run on the GPU against the reference's per-step call_back."""
import math

import numpy as np
import pytest

import sfparticles_b200 as S
from sfparticles_b200.trajectory import Trajectory


class _FakeSpecies:
    """A species whose 'device' arrays are CPU tensors."""

    def __init__(self, n_buf, cap, spin=False):
        import torch
        self.name = "fake"
        self.attrs = ["x", "y", "z", "ux", "uy", "uz", "inv_gamma", "_to_be_pruned"] + (["sx", "sy", "sz"] if spin
                                                                                       else [])
        self.N_buffered = n_buf
        self._arr = {a: torch.arange(cap, dtype=torch.float64) + 1000.0 * k for k, a in enumerate(self.attrs)}

    def _d(self, name):
        return self._arr[name]


def test_capture_gathers_slots_and_marks_unfilled_ones_nan():
    p = _FakeSpecies(n_buf=5, cap=10)
    tr = Trajectory(p, [0, 4, 5, 9], every=3, attrs=("x", "uz"))
    assert [tr.due(s) for s in range(7)] == [True, False, False, True, False, False, True]
    assert [tr.steps_to_next(s) for s in (0, 1, 2, 3)] == [3, 2, 1, 3]
    tr.capture(3)
    assert not tr.due(3)  # one record per step, however the loop is chunked
    p.N_buffered = 10
    p._arr["x"] += 0.5
    tr.capture(6)
    out = tr.numpy()
    np.testing.assert_array_equal(out["step"], [3, 6])
    np.testing.assert_array_equal(out["x"][0, :2], [0.0, 4.0])
    assert np.isnan(out["x"][0, 2:]).all()
    np.testing.assert_array_equal(out["x"][1], [0.5, 4.5, 5.5, 9.5])
    np.testing.assert_array_equal(out["uz"][1], [5000.0, 5004.0, 5005.0, 5009.0])


def test_capture_of_an_empty_species_and_default_attributes():
    p = _FakeSpecies(n_buf=0, cap=0, spin=True)
    tr = Trajectory(p, [0, 1])
    assert tr.attrs == ("x", "y", "z", "ux", "uy", "uz", "sx", "sy", "sz")
    tr.capture(1)
    out = tr.numpy()
    assert out["sz"].shape == (1, 2) and np.isnan(out["sz"]).all()
    assert Trajectory(_FakeSpecies(1, 1), [0]).numpy()["x"].shape == (0, 1)


def test_trajectory_arguments_are_checked():
    p = _FakeSpecies(2, 2)
    with pytest.raises(ValueError):
        Trajectory(p, [0], every=0)
    with pytest.raises(ValueError):
        Trajectory(p, [-1])
    with pytest.raises(ValueError):
        Trajectory(p, [0], attrs=("inv_gamma",))  # scratch, not kept by the fused step
    with pytest.raises(ValueError):
        Trajectory(p, [0], attrs=("sx",))  # not a spin species
    ele = S.Particles("ele", -1, 1, N=2, props=(np.zeros(2),) * 6)
    other = S.Particles("other", -1, 1, N=2, props=(np.zeros(2),) * 6)
    from sfparticles_b200.fields import static_field
    sim = S.Simulation(ele, dt=1e-17, fields=static_field(), print_every=None)
    with pytest.raises(AssertionError):
        sim.record(other, [0])
    tr = sim.record(ele, [0, 1], every=5)
    assert tr.species is ele and tr.every == 5


@pytest.mark.gpu
def test_recorded_trajectory_equals_per_step_call_back():
    """A small cascade: records every 7 steps (device chunks cut at 7, 14, ...)
    equal, bit for bit, what the reference's per-step call_back reads from the
    arrays at the same steps; slots of pairs not yet created are NaN."""
    from gpu_helpers import cuda_or_skip
    cuda_or_skip()
    from sfparticles_b200.constants import C
    from sfparticles_b200.fields import gaussian_laser_pulse

    def make(seed=11, n=2000, steps=60):
        T0 = 0.8e-6 / C
        dt = T0 / 100
        L = C * (steps * dt) / 2
        rng = np.random.default_rng(seed)
        g = 2000 * (1 + 0.01 * rng.normal(size=n))
        props = (rng.normal(-L, 1e-6, n), rng.normal(0, 1e-6, n), rng.normal(0, 1e-6, n), np.sqrt(g * g - 1),
                 np.zeros(n), np.zeros(n))
        ele = S.Particles("ele", -1, 1, N=n, props=props)
        pos = S.Particles("pos", 1, 1)
        pho = S.Particles("pho", 0, 0)
        ele.set_photon(pho)
        pos.set_photon(pho)
        pho.set_pair(ele, pos)
        ctau = C * 25e-15 / (2 * math.sqrt(math.log(2) / 2))
        fld = gaussian_laser_pulse(400.0, 2e-6, ctau, direction=-1, x0=L)
        sim = S.Simulation(ele, pos, pho, dt=dt, fields=fld, print_every=None, seed=seed, form="fp32")
        return sim, ele, pos, pho

    slots = [0, 17, 1999, 2000, 2100]  # 2000+ are pair electrons, created during the run or never
    sim, ele, pos, pho = make()
    tr = sim.record(ele, slots, every=7)
    trp = sim.record(pho, [0, 5, 10_000], every=7, attrs=("x", "ux"))
    sim.start(60)
    got, gotp = tr.numpy(), trp.numpy()

    sim2, ele2, pos2, pho2 = make()
    want = {a: [] for a in ("x", "y", "z", "ux", "uy", "uz")}
    wantp = {"x": [], "ux": []}

    def cb(istep):
        if (istep + 1) % 7:
            return
        for a in want:
            arr = getattr(ele2, a)
            want[a].append([arr[i] if i < ele2.N_buffered else np.nan for i in slots])
        for a in wantp:
            arr = getattr(pho2, a)
            wantp[a].append([arr[i] if i < pho2.N_buffered else np.nan for i in (0, 5, 10_000)])

    sim2.start(60, call_back=cb)
    np.testing.assert_array_equal(got["step"], np.arange(7, 61, 7))
    for a in want:
        np.testing.assert_array_equal(got[a], np.array(want[a]))
    for a in wantp:
        np.testing.assert_array_equal(gotp[a], np.array(wantp[a]))
    assert np.isfinite(got["x"][:, :3]).all()
