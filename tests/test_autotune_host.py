"""The autotuner's host side: the variant lists match the kernels the step
source instantiates, every default is a tuned variant, and the result cache
round-trips (sfparticles_b200.autotune)."""
import os
import re

from sfparticles_b200 import autotune, program

_SRC = os.path.join(os.path.dirname(program.__file__), "csrc", "sfp_step.cuh")


def _instantiated():
    text = open(_SRC).read()
    found = {}
    for kind, form, qed, a, b in re.findall(r"^SFP_(MASSIVE|PHOTON)_KERNEL\((\w+), (\w+), \w+, \w+, (\d+), (\d+)\)",
                                            text, re.M):
        found.setdefault((form, qed), ([], []))[0 if kind == "MASSIVE" else 1].append((int(a), int(b)))
    return found


def test_variant_lists_are_the_instantiated_kernels():
    found = _instantiated()
    assert set(found) == set(autotune.VARIANTS)
    for key, (mv, pv) in autotune.VARIANTS.items():
        assert sorted(mv) == sorted(found[key][0]), key
        assert sorted(pv) == sorted(found[key][1]), key


def test_defaults_are_tuned_variants():
    assert set(autotune.DEFAULT) == set(autotune.VARIANTS)
    for key, (m, p) in autotune.DEFAULT.items():
        mv, pv = autotune.VARIANTS[key]
        assert m in mv and p in pv, key


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setattr(program, "CACHE", str(tmp_path))
    assert autotune._load() == {}
    d = {"B200|fp32|rs|gaussian|e-e-g|2^28": {"best": [[2, 3], [3, 3]], "ms": {"m2_b3": 0.9, "p3_b3": 5.0}}}
    autotune._store(d)
    assert autotune._load() == d
    assert not [f for f in os.listdir(tmp_path) if f.endswith(".tmp")]
