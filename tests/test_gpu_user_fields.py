"""Fields(callable) on the GPU: user field functions translated to CUDA and
compiled by NVRTC into the field-evaluation kernel and into the fused step,
against the reference's own outputs for the same Python functions
(Fields(callable) and Fields.__add__, sfparticles/fields.py:11-61, compiled
by Numba when tests/golden/make_golden.py recorded them).

Tolerances: 1e-13 relative for one field evaluation (CUDA's libm against
LLVM's), 1e-10 relative for the whole deterministic run.
"""
import json

import numpy as np
import pytest

import user_fields as U
from conftest import golden
from gpu_helpers import cuda_or_skip, dev, golden_case_fields, ptr, sim_case_species, stream

pytestmark = pytest.mark.gpu


def _rel(a, b):
    scale = np.max(np.abs(b), axis=-1, keepdims=True) + 1e-300
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)) / scale))


def _product_fields(builder, kw, plus_static):
    from sfparticles_b200.fields import Fields, static_field
    f = Fields(U.BUILDERS[builder](**kw))
    return f + static_field(**U.STATIC) if plus_static else f


@pytest.mark.parametrize("name", ["gaussian", "gaussian_plus_static", "mixed", "lambda"])
def test_user_field_evaluation_matches_reference(name):
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib, program
    g = golden("ref_user_fields.npz")
    builder, kw, plus_static = json.loads(str(g["cases"]))[name]
    f = _product_fields(builder, kw, plus_static)
    mod = program.get_module(f, form=None, qed=None)
    x, y, z, t = g[f"pts_{name}"]
    ref = g[f"out_{name}"]
    got = np.zeros_like(ref)
    prm = f.params_device()
    xd, yd, zd = dev(x), dev(y), dev(z)
    pr = dev(np.zeros(1, dtype=np.uint8))
    out = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(6)]
    for j in range(x.size):  # one time per point, as the fixture was made
        _lib.call("sfp_field_eval", mod.handle, ptr(prm), ptr(xd[j:j + 1]), ptr(yd[j:j + 1]), ptr(zd[j:j + 1]),
                  float(t[j]), 1, ptr(pr), *map(ptr, out), stream())
        got[:, j] = [o.item() for o in out]
    assert _rel(got, ref) < 1e-13, _rel(got, ref)


def test_user_field_whole_run_matches_reference():
    """32 electrons with Landau-Lifshitz radiation reaction through the user
    Gaussian + a static field, 300 steps of the fused float64 step, against
    the reference's Simulation.start with the same callable; and the same
    run through the equivalent preset sum."""
    cuda_or_skip()
    import sfparticles_b200 as S
    from sfparticles_b200.fields import gaussian_laser_pulse, static_field
    g = golden("ref_sim_user_sum.npz")
    case = json.loads(str(g["case"]))
    results = []
    for fields in (golden_case_fields(g), gaussian_laser_pulse(**U.GAUSSIAN) + static_field(**U.STATIC)):
        species = sim_case_species(case, g["init"], g["spin_init"], "gpu")
        sim = S.Simulation(*species, dt=float(g["dt"]), fields=fields, print_every=None,
                           photon_threshold=case["thr"], seed=case["seed"])
        sim.start(case["steps"])
        (ele,) = species
        results.append(np.stack([getattr(ele, k) for k in ("x", "y", "z", "ux", "uy", "uz")]))
    user, preset = results
    assert user.shape == g["s0_state"].shape
    assert _rel(user, g["s0_state"]) < 1e-10, _rel(user, g["s0_state"])
    assert _rel(preset, user) < 1e-10, _rel(preset, user)
