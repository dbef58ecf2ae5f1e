"""The part shapes of the forming workloads (springback-precomp_b200/parts.py)
against the reference's own part families (python/precomp/geometry/parts.py):
heights at seeded points and footprint radii, from the committed fixture
tests/golden/parts.json (written by tests/golden/make_golden.py)."""
from __future__ import annotations

import importlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "parts.json")
CASES = json.load(open(GOLDEN))


@pytest.mark.parametrize("case", CASES, ids=[f"{c['family']}-{i}" for i, c in enumerate(CASES)])
def test_heights_match_the_reference_families(case):
    parts = importlib.import_module("springback-precomp_b200.parts")
    part = parts.FAMILIES[case["family"]](**case["params"])
    xy = np.array(case["xy"])
    z = part.height(xy[:, 0], xy[:, 1])
    ref = np.array(case["z"])
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(z - ref).max() <= 1e-12 * scale, np.abs(z - ref).max() / scale
    assert abs(part.footprint_radius() - case["footprint_radius"]) <= 1e-12 * case["footprint_radius"]


def test_fine_mesh_cone_has_the_configured_footprint():
    """The fine-mesh configuration's cone: an 18 mm footprint, 3 mm deep, a
    50 degree wall (1 mm fillets)."""
    parts = importlib.import_module("springback-precomp_b200.parts")
    cone = parts.TruncatedCone.with_footprint(9.0e-3, 50.0, 3.0e-3, 1.0e-3, 1.0e-3)
    assert abs(cone.footprint_radius() - 9.0e-3) < 1e-15
    assert abs(cone.height(np.array([0.0]), np.array([0.0]))[0] + 3.0e-3) < 1e-15
    r = np.linspace(0.0, 12e-3, 2001)
    z = cone.height(r, 0 * r)
    assert np.all(np.diff(z) >= -1e-15)  # rising from the floor to the rim
    slope = np.diff(z) / np.diff(r)
    assert abs(slope.max() - np.tan(np.radians(50.0))) < 1e-3
    assert z[r >= 9.0e-3].max() == 0.0 and z[r < 9.0e-3 - 1e-6].max() < 0.0
