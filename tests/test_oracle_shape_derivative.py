"""The oracle's shape derivative of the condensed IM residual,
lambda . d f* / d X (the building block of an adjoint with respect to the
reference geometry), pinned against central differences of the oracle's own
element routine - the restatement of the reference's CPU element - with the
modes re-solved to their local equilibrium at every perturbed geometry.
Central differences with h = 1e-9 m on a 1 mm element; the agreement is
limited by their rounding (about 1e-9 relative)."""
from __future__ import annotations

import numpy as np
import pytest


def element(rng):
    corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
                       dtype=float)
    X = (1e-3 * (corners + 0.08 * rng.standard_normal(corners.shape))).reshape(1, 24)
    F = np.array([[1.0, 0.3, 0.1], [0.05, 0.9, 0.2], [0.0, -0.1, 1.15]]) - np.eye(3)
    ue = (0.02 * (X.reshape(8, 3) @ F.T) + 4e-6 * rng.standard_normal((8, 3))).reshape(1, 24)
    return X, ue


@pytest.mark.parametrize("kin", ["finite", "logarithmic"])
@pytest.mark.parametrize("frozen", [True, False])
def test_shape_derivative_is_the_central_difference(pkg, orc, kin, frozen):
    rng = np.random.default_rng(3)
    m = pkg.material.hill_chaboche_sheet().as_dict()
    if frozen:
        m["yield_stress"] = 1e300  # the committed plastic state as it is, no return
    X, ue = element(rng)
    committed = np.zeros((1, 8, orc.NF))
    ep = 0.01 * rng.standard_normal((8, 6))
    ep[:, 0:3] -= ep[:, 0:3].mean(axis=1, keepdims=True)
    committed[0, :, 0:6] = ep
    committed[0, :, 36] = 0.02
    lam = rng.standard_normal((1, 24))
    g, st = orc.vjp_x(m, X, ue, lam, committed, kinematics=kin)
    assert st[0] == 0
    if not frozen:
        assert orc.elements(m, X, ue, committed, kinematics=kin)["yielding"][0] > 0
    h = 1e-9
    fd = np.zeros(24)
    for j in range(24):
        Xp, Xm = X.copy(), X.copy()
        Xp[0, j] += h
        Xm[0, j] -= h
        fp = orc.elements(m, Xp, ue, committed, kinematics=kin, want_tangent=False)["force"].reshape(24)
        fm = orc.elements(m, Xm, ue, committed, kinematics=kin, want_tangent=False)["force"].reshape(24)
        fd[j] = lam[0] @ (fp - fm) / (2 * h)
    assert np.abs(g[0] - fd).max() <= 1e-7 * np.abs(fd).max(), np.abs(g[0] - fd).max() / np.abs(fd).max()
