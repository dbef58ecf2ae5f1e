"""The CPU-runnable forming run's deck through the forming harness on the
CPU (the oracle's system and contact, scipy's solves): a 20 x 20 x 2 copy of
the 40 x 40 x 2 sheet, the spiral's first revolution. The tool comes down
from the air, touches the sheet and presses it; every increment converges
or is cut and retried; the sheet under the tool moves down and pushes back.
The deck, the tool path and the harness's schedule are exercised together
without a GPU."""
from __future__ import annotations

import importlib

import numpy as np

from forming_harness import FormingRun
from oracle_backend import OracleBackend


def test_first_revolution_of_the_spiral(pkg, orc):
    wl = importlib.import_module("springback-precomp_b200.workload")
    deck = wl.cfg1_deck(nx=20)
    times = deck["tools"][0]["trajectory"]["times"]
    points = np.array(deck["tools"][0]["trajectory"]["points"])
    # The form step cut short after the path's fourth point on the part.
    t_end = times[5]
    deck["steps"][0]["deck"]["time"] = [0.0, t_end]
    run = FormingRun(OracleBackend(pkg, orc), deck, "cpu", solver="host", growth_test="reference",
                     tolerance="reference")
    res = run.run_step(0, None)
    assert res.increments >= 4
    assert res.tool_fz[-1] > 0.0  # the sheet pushes the tool up
    top = np.flatnonzero(np.isclose(run.nodes[:, 2], 0.0))
    dz = res.u.reshape(-1, 3)[top, 2]
    # The sheet under the tool pressed down by a fraction of the step-down.
    tip = points[5, 2] - deck["tools"][0]["radius"]
    assert -0.5e-3 < dz.min() < 0.0
    assert dz.min() >= tip - 1e-4
