"""The material parameters the element loop is fed, against golden values
the reference produced itself (tests/golden/materials.json, written by
tests/golden/make_golden.py from python/precomp/materials.py and from the
material blocks of the reference's committed forming decks). The Swift and
Hollomon fits must give the same numbers, since every yield, every return
and so every yield flag follows from them."""
from __future__ import annotations

import importlib
import json
import os

import pytest

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "materials.json")))
KEYS = ("youngs_modulus", "poisson_ratio", "yield_stress", "hardening_modulus", "saturation_stress",
        "saturation_rate", "kinematic_hardening_modulus")


@pytest.fixture(scope="module")
def material():
    return importlib.import_module("springback-precomp_b200.material")


def close(a, b, rel=1e-12):
    return abs(a - b) <= rel * max(abs(b), 1e-300)


@pytest.mark.parametrize("name", sorted(GOLDEN["library"]))
def test_library_hollomon_fits(material, name):
    m = material.library_material(name)
    for k in KEYS:
        assert close(getattr(m, k), GOLDEN["library"][name][k]), (k, getattr(m, k), GOLDEN["library"][name][k])


@pytest.mark.parametrize("case", GOLDEN["swift"], ids=lambda c: f"K{c['K']:.0f}_n{c['n']}")
def test_swift_fits(material, case):
    m = material.Material.from_swift("swift", 70e9, 0.33, case["K"], case["eps0"], case["n"])
    for k in KEYS:
        assert close(getattr(m, k), case[k]), (k, getattr(m, k), case[k])


def test_the_forming_sheet_law(material):
    """The 40x40x2 forming sheet's Swift law (K = 425 MPa, eps0 = 0.003,
    n = 0.29), the isotropic hardening of the element microbenchmark."""
    m = material.aluminium_swift()
    g = [c for c in GOLDEN["swift"] if c["K"] == 425e6][0]
    assert close(m.yield_stress, g["yield_stress"]) and close(m.saturation_rate, g["saturation_rate"])
    hc = material.hill_chaboche_sheet()
    assert (hc.hardening_modulus, hc.saturation_stress) == (m.hardening_modulus, m.saturation_stress)


@pytest.mark.parametrize("deck", sorted(GOLDEN["decks"]))
def test_committed_decks_carry_the_library_fit(material, deck):
    d = GOLDEN["decks"][deck]
    m = material.library_material(d["name"])
    for k in KEYS:
        assert close(getattr(m, k), d[k]), (k, getattr(m, k), d[k])
