"""End to end against a forming run the reference committed
(benchmarks/physics_audit/calculix/punch/strip_h2_im_nz4: a 20 x 1 x 4
incompatible-mode Hex8 strip, logarithmic strain, J2 with Voce hardening,
a cylindrical punch with Coulomb friction 0.1 pressed 4 mm into it, then
the tool taken away over 20 increments and the clamps released onto
supports). The element loop and the contact are this package's, on the
GPU; the Newton driver around them is the test harness in
forming_harness.py. The formed, unloaded and released nodal displacements
must agree with the reference's within 1e-5 mm (1e-8 m)."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from forming_harness import FormingRun

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "strip_h2_im_nz4.json")
HEIGHT_TOL = 1.0e-8  # [m]: 1e-5 mm


@pytest.fixture(scope="module")
def run(pkg, cuda):
    fx = json.load(open(FIXTURE))
    r = FormingRun(pkg, fx, cuda)
    results = [r.run_step(k) for k in range(len(fx["steps"]))]
    return fx, results


@pytest.mark.parametrize("k,name", [(0, "form"), (1, "unload"), (2, "release")])
def test_step_displacements_match_the_reference(run, k, name):
    fx, results = run
    ref = np.array(fx["steps"][k]["u"]).reshape(-1)
    got = results[k].u
    assert fx["steps"][k]["deck"]["name"] == name
    assert results[k].increments == fx["steps"][k]["increments"]
    err = np.abs(got - ref).reshape(-1, 3)
    assert err[:, 2].max() <= HEIGHT_TOL, f"{name}: heights differ by up to {err[:, 2].max():.3e} m"
    assert err.max() <= HEIGHT_TOL, f"{name}: displacements differ by up to {err.max():.3e} m"


def test_tool_force_history_matches_the_reference(run):
    """The punch force of every forming increment (tool_forces.csv), to the
    reference's residual tolerance (1e-6 of the force scale)."""
    fx, results = run
    ref = np.array([float(r["fz"]) for r in fx["tool_forces"] if r["step"] == "1"])
    got = np.array(results[0].tool_fz)
    assert len(got) == len(ref)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
