"""CPU checks of the end-to-end test harness (forming_harness.py) against
the reference runs it replays: its region selection (Selector::contains,
src/fem/Selector.cpp:49-56) picks the prescribed DOFs the reference's
output shows held, and its contact slaves carry the top surface's area."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from forming_harness import in_region, top_face_slaves

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["strip_h2_im_nz4", "strip_h1_im_nz4", "plate_h2_im_mu0.1_drag3", "strip_h2_std_mu0.1",
         "plate_h2_std_mu0.1_drag3", "strip_h2_nobbar_mu0.1"]


def load(case):
    fx = json.load(open(os.path.join(GOLDEN, case + ".json")))
    nodes = np.array(fx["nodes"])
    tol = 1e-9 * float(np.linalg.norm(nodes.max(0) - nodes.min(0)))
    return fx, nodes, tol


@pytest.mark.parametrize("case", CASES)
def test_held_dofs_are_the_ones_the_reference_held(case):
    """Every DOF a step's boundary conditions hold keeps, in the reference's
    own output, the value it had at the start of the step."""
    fx, nodes, tol = load(case)
    u_prev = np.zeros(3 * len(nodes))
    for step in fx["steps"]:
        u = np.array(step["u"]).reshape(-1)
        held = np.zeros(3 * len(nodes), dtype=bool)
        for bc in step["deck"]["boundary_conditions"]:
            sel = np.where(in_region(nodes, bc["region"], tol))[0]
            assert len(sel) > 0, bc["name"]
            for comp in bc["fix"]:
                held[3 * sel + "xyz".index(comp)] = True
        assert np.array_equal(u[held], u_prev[held]), step["deck"]["name"]
        assert np.abs(u[~held]).max() > 0.0
        u_prev = u


@pytest.mark.parametrize("case", CASES)
def test_slaves_carry_the_top_surface(case):
    fx, nodes, tol = load(case)
    elements = np.array(fx["elements"])
    for tool in fx["tools"]:
        ids, area = top_face_slaves(nodes, elements, tool["surface"], tol)
        top = nodes[:, 2].max()
        assert np.allclose(nodes[ids, 2], top)
        extent = nodes.max(0) - nodes.min(0)
        assert area.sum() == pytest.approx(extent[0] * extent[1], rel=1e-12)
        assert len(ids) == np.sum(np.isclose(nodes[:, 2], top))


def test_nearest_node_and_boxes():
    x = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.5]])
    assert in_region(x, {"nearest_node": [0.9, 0.1, 0.0]}, 1e-9).tolist() == [False, True, False]
    assert in_region(x, {"box": {"xmin": 1.0, "zmax": 0.0}}, 1e-9).tolist() == [False, True, False]
    assert in_region(x, {"any_of": [{"box": {"xmax": 0.0}}, {"box": {"zmin": 0.5}}]}, 1e-9).tolist() == [True, False,
                                                                                                    True]
    assert in_region(x, {"all": True}, 1e-9).all()
