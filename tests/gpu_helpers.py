"""Shared helpers of the GPU parity tests (test infrastructure)."""
import ctypes
import json

import numpy as np
import pytest

import oracle as orc


def cuda_or_skip():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sfparticles_b200 import _lib
    _lib.load()
    return torch.device("cuda")


def dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a)
    if dtype is None:
        dtype = torch.uint8 if a.dtype == bool or a.dtype == np.uint8 else torch.float64
    if dtype == torch.uint8:
        a = a.astype(np.uint8)
    return torch.as_tensor(a, device="cuda").to(dtype).contiguous()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def host(t):
    return t.cpu().numpy()


def product_rs_tables():
    from sfparticles_b200.qed import tables
    iA, dA, zN, zmax = tables.rs_tables()
    return iA, dA, zN, zmax


def build_fields_pair(spec, cases):
    """(product Fields, oracle FieldTerms) for a preset spec / nested sum."""
    from sfparticles_b200 import fields as F
    if isinstance(spec, int):
        name, kw = cases[spec]
        return getattr(F, name)(**kw), getattr(orc, name)(**kw)
    a, oa = build_fields_pair(spec[0], cases)
    b, ob = build_fields_pair(spec[1], cases)
    return a + b, oa + ob


def sim_case_species(case, init, spin_init, api):
    """Build the species of a whole-simulation fixture case with the
    product API (api='gpu') -- same layout as tests/golden/make_golden.py."""
    import sfparticles_b200 as S
    rr = getattr(S.RadiationReactionType, case["rr"])
    n = case["n_e"]
    if case["spin"]:
        ele = S.SpinParticles("ele", -1, 1, N=n, props=tuple(np.array(a) for a in list(init) + list(spin_init)),
                              RR=rr)
    else:
        ele = S.Particles("ele", -1, 1, N=n, props=tuple(np.array(a) for a in init), RR=rr)
    species = [ele]
    if case["rr"] == "PHOTON":
        pho = S.Particles("pho", 0, 0)
        ele.set_photon(pho)
        species.append(pho)
        if case["pairs"]:
            pos = S.Particles("pos", 1, 1)
            pos.set_photon(pho)
            pho.set_pair(ele, pos)
            species = [ele, pos, pho]
    return species


def golden_case_fields(g):
    """Product Fields of a whole-run fixture: presets by name, user callables
    (tests/user_fields.py) as "user:<builder>"."""
    from sfparticles_b200 import fields as F
    terms = json.loads(str(g["field_terms"]))
    comb = json.loads(str(g["field_comb"]))

    def build(nm, kw):
        if nm.startswith("user:"):
            import user_fields
            return F.Fields(user_fields.BUILDERS[nm[5:]](**kw))
        return getattr(F, nm)(**kw)

    flds = [build(nm, kw) for nm, kw in terms]
    return flds[0] if comb == 0 else flds[0] + flds[1]
