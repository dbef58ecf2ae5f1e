"""Increment cuts driven by the element loop's failures, end to end: the
forming driver's rule (Forming.cpp:1149-1247 - a failed increment is halved
and retried from the last converged state, at most 10 times in a row; an
increment that converged in at most 4 Newton iterations lets the next grow
by 1.5) in the test harness around this package's element loop, contact and
solves. The failures are the element loop's SolverError (the C ABI's
SBK_ERR_SOLVER with the failing element and its code), raised by the GPU or,
in one test, injected on the host in its place."""
from __future__ import annotations

import numpy as np
import pytest

from forming_harness import FormingRun
from test_gpu_forming import HEIGHT_TOL, load_fixture

pytestmark = pytest.mark.gpu


def test_harness_schedule_is_the_references(pkg, cuda):
    """Without failures the harness's own increment schedule is the
    reference's (strip_h2_im_nz4: 40 increments, no cut), and so are the
    formed displacements."""
    fx = load_fixture("strip_h2_im_nz4")
    run = FormingRun(pkg, fx, cuda)
    res = run.run_step(0, None)
    ref_times = [float(f["t"]) for f in fx["tool_forces"] if int(f["step"]) == 1]
    assert res.cuts == 0 and res.increments == fx["steps"][0]["increments"]
    np.testing.assert_allclose(run.times, ref_times, rtol=0, atol=1e-12)
    assert np.abs(res.u - np.array(fx["steps"][0]["u"]).reshape(-1)).max() <= HEIGHT_TOL


def test_injected_local_failure_cuts_the_increment(pkg, cuda):
    """An element's LOCAL_NO_CONVERGE reported at the 10th increment (made on
    the host in place of the GPU's report) cuts that increment once; the
    step completes on the halved increments, and replaying the same
    increment times without the fault gives the same state to the bit."""
    fx = load_fixture("strip_h2_im_nz4")
    faulty = FormingRun(pkg, fx, cuda)
    faulty.inject_at = {10}
    res = faulty.run_step(0, None)
    assert res.cuts == 1
    assert res.increments > fx["steps"][0]["increments"]
    replay = FormingRun(pkg, fx, cuda)
    again = replay.run_step(0, faulty.times)
    assert np.array_equal(again.u, res.u)
    # Another increment path of a path-dependent material: the formed shape
    # stays within 1e-3 mm of the reference's (measured 3.6e-5 mm).
    err = np.abs(res.u - np.array(fx["steps"][0]["u"]).reshape(-1)).max()
    print(f"injected cut: {res.increments} increments, largest difference from the reference {err:.3e} m")
    assert err <= 1.0e-6


def test_gpu_failures_cut_the_strip_the_reference_cut(pkg, cuda):
    """strip_h1_im_nz4 (40 x 1 x 4), whose forming step the reference cut
    four times (inverted points and local iterations that did not converge),
    on the harness's own schedule: the GPU's element failures cut the same
    increments, so the run takes the reference's 92 increments and 4 cuts
    and ends at its formed shape (measured on a B200: 3.5e-18 m apart)."""
    fx = load_fixture("strip_h1_im_nz4")
    run = FormingRun(pkg, fx, cuda)
    res = run.run_step(0, None)
    err = np.abs(res.u - np.array(fx["steps"][0]["u"]).reshape(-1)).max()
    print(f"strip_h1_im_nz4: {res.increments} increments, {res.cuts} cuts (reference "
          f"{fx['steps'][0]['increments']}, {fx['steps'][0]['cuts']}); largest difference {err:.3e} m")
    assert res.cuts == fx["steps"][0]["cuts"] and res.increments == fx["steps"][0]["increments"]
    assert err <= HEIGHT_TOL
