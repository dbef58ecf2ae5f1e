"""End to end against forming runs the reference committed
(benchmarks/physics_audit/calculix/punch/<case>/sparlab and
benchmarks/physics_audit/challenge/cases/<case>), under logarithmic strain
with Coulomb friction 0.1:

- strip_h2_im_nz4: a 20 x 1 x 4 strip under a cylindrical punch pressed
  4 mm into it, the tool taken away over 20 increments and the clamps
  released onto supports;
- strip_h1_im_nz4: the same strip at 40 x 1 x 4, whose forming step the
  reference's Newton iterations cut four times;
- plate_h2_im_mu0.1_drag3: a clamped 20 x 20 x 2 plate under a spherical
  punch pressed 3 mm in and dragged 3 mm sideways, released onto 3-2-1
  supports (two cuts);
- kin_h0833 (benchmarks/physics_audit/challenge/cases): a 48 x 48 x 1
  sheet with the 2 x 2 x 5 rule, Hill48 with two Chaboche backstresses and
  Voce hardening, a spherical tool on a 113-knot spiral path over 395
  increments (three cuts), released onto 3-2-1 supports - the element
  microbenchmark's law class; about three minutes on a B200;
- strip_h2_std_mu0.1: a 20 x 1 x 2 strip under the same punch, and
  plate_h2_std_mu0.1_drag3: the plate of the third run, both in the
  standard Hex8 with mean dilatation (the element of the reference's
  springback_2mm preset); strip_h2_nobbar_mu0.1 the strip without it.

The element loop and the contact are this package's, on the GPU; the
Newton driver around them is the test harness in forming_harness.py, which
takes the reference's accepted increments (their times in its
tool_forces.csv) through the forming step. The formed, unloaded and
released nodal displacements must agree with the reference's within 1e-5 mm
(1e-8 m), the bar set for formed and released heights."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from forming_harness import FormingRun

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["strip_h2_im_nz4", "strip_h1_im_nz4", "plate_h2_im_mu0.1_drag3", "kin_h0833", "strip_h2_std_mu0.1",
         "plate_h2_std_mu0.1_drag3", "strip_h2_nobbar_mu0.1"]
HEIGHT_TOL = 1.0e-8  # [m]: 1e-5 mm


def load_fixture(case):
    """A reference run's fixture; the larger ones keep their mesh and step
    displacements in an npz beside the JSON."""
    fx = json.load(open(os.path.join(GOLDEN, case + ".json")))
    if "arrays" in fx:
        a = np.load(os.path.join(GOLDEN, fx["arrays"]))
        fx["nodes"], fx["elements"] = a["nodes"], a["elements"]
        for k, st in enumerate(fx["steps"]):
            st["u"] = a["u"][k]
            st["elements"] = {"eq_plastic_strain": a["eq_plastic_strain"][k], "von_mises_Pa": a["von_mises"][k]}
    return fx


@pytest.fixture(scope="module", params=CASES)
def run(request, pkg, cuda):
    fx = load_fixture(request.param)
    r = FormingRun(pkg, fx, cuda)
    results = []
    for k in range(len(fx["steps"])):
        times = [float(f["t"]) for f in fx["tool_forces"] if int(f["step"]) == k + 1]
        results.append(r.run_step(k, times if times else None))
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


# Step-end element fields: the von Mises stress within 1e-10 of the largest
# in the step, the largest equivalent plastic strain within 1e-12 (absolute;
# the fields are O(0.1) at most). Measured on a B200 over the seven runs:
# 2.9e-12 and 2.2e-14.
VM_TOL = 1.0e-10
EQPS_TOL = 1.0e-12


@pytest.mark.parametrize("k,name", [(0, "form"), (1, "unload"), (2, "release")])
def test_step_element_fields_match_the_reference(run, k, name):
    """The step-end stress recovery (elastoplastic_stress of every element,
    IncompatibleModes.cpp:602-664 / Elastoplastic.cpp:342-430, called at
    Forming.cpp:1266-1281) against the element fields the reference wrote
    for the same step (step_<k>_<s>_elements.csv: eq_plastic_strain,
    von_mises_Pa)."""
    fx, results = run
    ref = fx["steps"][k]["elements"]
    vm_ref = np.asarray(ref["von_mises_Pa"], dtype=np.float64)
    ep_ref = np.asarray(ref["eq_plastic_strain"], dtype=np.float64)
    vm, ep = results[k].von_mises, results[k].eq_plastic_strain
    assert vm.shape == vm_ref.shape and ep.shape == ep_ref.shape
    vm_err = np.abs(vm - vm_ref).max() / np.abs(vm_ref).max()
    ep_err = np.abs(ep - ep_ref).max()
    print(f"{name}: von Mises rel. {vm_err:.2e} (largest {np.abs(vm_ref).max():.4e} Pa), eq. plastic strain "
          f"{ep_err:.2e} (largest {ep_ref.max():.4e})")
    assert vm_err <= VM_TOL, vm_err
    assert ep_err <= EQPS_TOL, ep_err
