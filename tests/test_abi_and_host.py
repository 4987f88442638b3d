"""CPU-only tests: the C-ABI library loads and exports every declared entry
point, NVRTC modules compile for sm_100a without a GPU, and the host-side
API mirrors the reference (tests/test_particles.py of the reference)."""
import os
import re
from itertools import product

import numpy as np
import pytest

import sfparticles_b200 as S
from sfparticles_b200 import _lib, fields, program
from sfparticles_b200.constants import E_CHARGE as e, M_E as m_e
from sfparticles_b200.particles import RadiationReactionType

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for h in ("sfp.h",):
        src = open(os.path.join(REPO, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(sfp_[a-zA-Z0-9_]+)\s*\(", src):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    declared = header_symbols()
    assert len(declared) >= 30
    for s in declared:
        assert hasattr(L, s), s
    assert set(_lib.declared_symbols()) >= declared, declared - set(_lib.declared_symbols())
    assert b"sm_100a" in L.sfp_version()


def test_library_reports_errors_without_a_device():
    L = _lib.load()
    rc = L.sfp_bool_sum(None, 10, None, None)
    assert rc != 0 and b"NULL" in L.sfp_last_error()


@pytest.mark.parametrize("form,qed", [(None, None), ("fp64", "rs"), ("fp64", "od")])
def test_nvrtc_modules_compile_without_gpu(form, qed):
    f = fields.gaussian_laser_pulse(50, 3e-6, 6e-6) + fields.static_field(Bz=1.0)
    img = program.compile_image(program.module_source(f.cuda_source(), form, qed), program.options(form))
    assert img[:4] == b"\x7fELF"


def test_nvrtc_compile_error_is_reported():
    with pytest.raises(_lib.SFPError, match="NVRTC"):
        program.compile_image("this is not C++", program.options())


# --- reference tests/test_particles.py, on the host-side API ---------------

def test_particles_init():
    p = S.Particles('e', q=-1, m=1, N=2)
    assert p.q == -e and p.m == m_e and p.N_buffered == 2
    for prop, i in product(['', 'u', 'E', 'B'], ['x', 'y', 'z']):
        assert (getattr(p, prop + i) == np.zeros(2)).all()
    with pytest.raises(AssertionError):
        S.Particles('pho', q=0, m=0, N=2)
    with pytest.raises(AssertionError):
        S.Particles('pho', q=1, m=0)
    with pytest.raises(AssertionError):
        S.Particles('ele', q=-1, m=1, RR='LL')


def test_set_photon_rejects_LL():
    ele = S.Particles('ele', q=-1, m=1, RR=RadiationReactionType.LL)
    pho = S.Particles('pho', q=0, m=0)
    with pytest.raises(AssertionError):
        ele.set_photon(pho)


def test_spin_init():
    p = S.SpinParticles('e', q=-1, m=1, N=2)
    assert hasattr(p, 'sx') and hasattr(p, 'sy') and hasattr(p, 'sz')
    assert (p.sx == 0).all() and (p.sy == 0).all() and (p.sz == 0).all()


def test_spin_init_with_props():
    # the reference raises TypeError here (particles.py:566); supported in this API
    p = S.SpinParticles('e', -1, 1, N=2, props=[[1.0, 2.0]] * 6 + [[0.0, 0.0], [0.0, 0.0], [1.0, 1.0]])
    assert (p.sz == 1).all() and (p.x == [1, 2]).all()


def test_prop_init_list():
    p = S.Particles('e', q=-1, m=1, N=3, props=[[1, 2, 3]] * 6)
    assert p.N_buffered == 3
    for prop, i in product(['', 'u'], ['x', 'y', 'z']):
        assert (getattr(p, prop + i) == np.array([1, 2, 3.0])).all()


def test_prop_init_scalar():
    with pytest.raises(AssertionError):
        S.Particles('pho', q=1, m=0, N=2, props=[[0, 0, 0]] * 6)
    p = S.Particles('e', q=-1, m=1, N=1, props=[1] * 6)
    assert p.N_buffered == 1
    for prop, i in product(['', 'u'], ['x', 'y', 'z']):
        assert (getattr(p, prop + i) == np.array([1.0])).all()


def test_extend_growth_rule():
    N, n1, n2 = 5, 10, 30
    ee = S.Particles('e', -1, 1, N)
    pho = S.Particles('pho', 0, 0)
    ee.set_photon(pho)
    ee._extend(n1)
    assert ee.N_buffered == N
    assert ee.buffer_size == int(N / 4) + N + n1
    assert ee.x.shape[0] == ee.buffer_size
    ee._extend(n2)
    assert ee.N_buffered == N
    assert ee.buffer_size == (int(N / 4) + N + n1) + int(N / 4) + n2
    for attr in ee.attrs:
        assert len(getattr(ee, attr)) == ee.buffer_size, attr
    assert ee._to_be_pruned[N:].all() and not ee._to_be_pruned[:N].any()
    assert not ee.event.any()


def test_prune_on_host():
    p = S.Particles('e', -1, 1, N=4, props=[[1, 2, 3, 4]] * 6)
    pr = p._to_be_pruned
    pr[1] = True
    p._prune()
    assert p.N_buffered == p.buffer_size == 3 and (p.x == [1, 3, 4]).all()


def test_simulation_classification_and_asserts():
    ele = S.Particles('ele', -1, 1, N=2)
    pos = S.Particles('pos', 1, 1)
    pho = S.Particles('pho', 0, 0)
    ele.set_photon(pho)
    pos.set_photon(pho)
    pho.set_pair(ele, pos)
    f = fields.static_field(Bz=1.0)
    sim = S.Simulation(ele, pos, pho, dt=1e-17, fields=f, print_every=None)
    assert sim.particles_bw == [pho] and sim.particles_rad == [ele, pos] and len(sim.particles_push) == 3
    with pytest.raises(AssertionError):
        S.Simulation(ele, pho, dt=1e-17, fields=f)  # positron missing


def test_constants_match_scipy():
    from scipy import constants as sc
    from sfparticles_b200 import constants as K
    assert (K.C, K.M_E, K.E_CHARGE, K.HBAR, K.EPSILON_0, K.ALPHA) == (sc.c, sc.m_e, sc.e, sc.hbar, sc.epsilon_0,
                                                                       sc.alpha)


def test_use_gpu_zero_is_refused(monkeypatch):
    import subprocess
    import sys
    r = subprocess.run([sys.executable, "-c", "import sfparticles_b200"], env={**os.environ, "SFPARTICLES_USE_GPU": "0"},
                       capture_output=True, text=True, cwd=REPO)
    assert r.returncode != 0 and "GPU implementation" in r.stderr


def test_gaussian_float32_block():
    """gaussian_laser_pulse: slots 0-9 are the float64 parameters; slots 10-15
    pack the float32 form's derived constants two per slot, each the float64
    value rounded once to float32, and none packs into a NaN or infinity."""
    import math
    from sfparticles_b200.constants import C, PI
    a0, w0, ctau, d, x0, l0, pol, cep = 150.0, 4e-6, 7e-6, -1, 3e-5, 0.8e-6, 0.7, 0.25
    p = fields.gaussian_laser_pulse(a0, w0, ctau, direction=d, x0=x0, l0=l0, pol_angle=pol, cep=cep).params()
    assert p.size == _lib.SFP_FIELD_PARAMS and np.isfinite(p).all()
    k0, zR = 2 * PI / l0, PI * w0 ** 2 / l0
    E0 = a0 / (e / (m_e * C * (2 * PI * C / l0)))
    np.testing.assert_array_equal(p[:10], [E0, k0, zR, w0, ctau, d, x0, cep, math.cos(pol), math.sin(pol)])
    kc = k0 * ctau
    want = np.array([E0, k0, 1 / zR, k0 / (2 * zR * zR), 1 / (w0 * w0), 1 / (kc * kc), d / C, cep, math.cos(pol),
                     math.sin(pol), k0 / (4 * zR), kc], dtype=np.float32)
    got = np.frombuffer(np.ascontiguousarray(p[10:16]).tobytes(), dtype="<f4")
    np.testing.assert_array_equal(got, want)
