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


def test_sweep_parts_keep_a_floor():
    """The design sweep's 64 parts: four families, 16 each, within the
    footprint and wall-angle ranges, meshes of 20k-150k elements; every part
    leaves its floor clear of the footprint's medial axis (a sheet laid on
    a crease where two walls meet folds inside one element, which no
    forming run survives), the depth capped where the sampled one would
    not (the capped parts at the largest depth that does)."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    parts = wl.sweep_parts(64)
    families = [type(p).family for p, _ in parts]
    assert {f: families.count(f) for f in set(families)} == {f: 16 for f in wl.SWEEP_FAMILIES}
    capped = 0
    for p, m in parts:
        assert 20000 * 0.95 <= m.num_elements <= 150000 * 1.05
        if p.family == "dome":
            continue
        assert 30.0 <= p.wall_angle_deg <= 55.0
        r = p.footprint_radius()
        # A pyramid's rounded square is inscribed in the sampled footprint.
        lo = 0.0 if p.family == "pyramid" else 7.5e-3 * (1 - 1e-9)
        assert lo <= r <= 10.0e-3 * (1 + 1e-9), r
        if p.family == "truncated_cone":
            inner = p.top_radius
        elif p.family == "elliptic_cone":
            a, b = max(p.semi_axis_x, p.semi_axis_y), min(p.semi_axis_x, p.semi_axis_y)
            inner = b * b / a
        else:
            inner = min(p.half_width_x, p.half_width_y, p.corner_radius)
        room = inner - p.profile.w_last
        assert room >= wl.SWEEP_FLOOR_MARGIN * (1 - 1e-6), (p, room)
        if p.depth < 2.0e-3 - 1e-12 or room < wl.SWEEP_FLOOR_MARGIN * 1.01:
            capped += 1
        assert p.depth <= 4.0e-3
    assert capped < 32


def test_spiral_follows_the_dome_without_gouging():
    """The spiral tool path of the CPU-runnable forming run (the reference's
    spiral_toolpath restated for a target of revolution): it starts and
    ends in the air above the sheet, its height never rises on the part,
    each revolution drops one step-down until the deepest level, the ball
    never cuts into the target (its lowest point along the contact normal
    stays on or above the dome everywhere), and it reaches the dome's
    depth within a step-down."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    parts = importlib.import_module("springback-precomp_b200.parts")
    dome = parts.Dome(5e-3, 2e-3, 2e-3)
    R, step = 3e-3, 0.5e-3
    pts, t, t_form = wl.revolution_spiral(lambda r: dome.height(r, 0 * r), 10e-3, R, step, 1e-3)
    assert pts[0, 2] > R and pts[-1, 2] > R  # approach and retract in the air
    assert np.all(np.diff(t) > 0) and t[0] == 0.0 and t[-1] == 1.0 and 0.8 < t_form < 1.0
    body = pts[1:-1]
    assert np.all(np.diff(body[:, 2]) <= 1e-15)
    assert body[0, 2] == R  # the tip at the sheet plane
    # No gouge: the ball's centre is at least R from every point of the
    # target's surface of revolution (sampled densely in the meridian plane
    # through the centre).
    s = np.linspace(-10e-3, 10e-3, 20001)
    zs = dome.height(np.abs(s), 0 * s)
    for p in body[::3]:
        rho = np.hypot(p[0], p[1])
        d = np.sqrt((s - rho) ** 2 + (zs - p[2]) ** 2).min()
        assert d >= R * (1 - 1e-6), (p, d)
    # The deepest tip within a step-down of the dome's depth.
    assert -2e-3 <= body[:, 2].min() - R <= -2e-3 + step
