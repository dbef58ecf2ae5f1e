"""The oracle's standard Hex8 (elastoplastic_element for an element without
internal modes, src/fem/Elastoplastic.cpp:96-340), pinned by restatements
of the reference's own checks of it:

- the tangent is the derivative of the internal force, for every
  kinematics, with and without mean dilatation, for J2, Hill48 and
  Chaboche (tests/test_logarithmic.cpp:259-327, tests/test_plasticity.cpp:
  460-502 and 543-596, tests/test_anisotropy.cpp:1296-1357; central
  differences, h = 1e-10 m (1e-7 of the 1 mm element), 1e-8 of the tangent's
  largest entry in the reference);
- an elastic element is the linear element, and mean dilatation leaves a
  homogeneous dilatation alone (tests/test_plasticity.cpp:504-541)."""
from __future__ import annotations

import numpy as np
import pytest

KIN = ["small", "finite", "logarithmic"]


@pytest.fixture(scope="module")
def laws(pkg):
    mat = pkg.material
    elastic = mat.aluminium_swift()
    elastic_d = dict(elastic.as_dict(), yield_stress=1e15, saturation_stress=0.0, hardening_modulus=0.0)
    return {"elastic": elastic_d, "j2": mat.aluminium_swift().as_dict(),
            "hill48+chaboche": mat.hill_chaboche_sheet().as_dict()}


def element_x():
    """A distorted 1 mm hexahedron (node-major, VTK order)."""
    corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
                       dtype=float)
    rng = np.random.default_rng(3)
    return (1e-3 * (corners + 0.08 * rng.standard_normal(corners.shape))).reshape(1, 24)


def motion(x, scale, seed):
    """A homogeneous stretch and shear with a random part, scale x 1 mm."""
    X = x.reshape(8, 3)
    F = np.array([[1.0, 0.3, 0.1], [0.05, 0.9, 0.2], [0.0, -0.1, 1.15]]) - np.eye(3)
    rng = np.random.default_rng(seed)
    return (scale * (X @ F.T) + scale * 1e-3 * 0.2 * rng.standard_normal((8, 3))).reshape(1, 24)


def evaluate(orc, m, x, u, committed, kin, averaged, want_tangent):
    with orc.element(True, averaged):
        r = orc.elements(m, x, u, committed, kinematics=kin, want_tangent=want_tangent)
    assert int(r["status"][0]) == 0, r["status"]
    return r


@pytest.mark.parametrize("law", ["elastic", "j2", "hill48+chaboche"])
@pytest.mark.parametrize("kin", KIN)
@pytest.mark.parametrize("averaged", [False, True])
def test_tangent_is_the_derivative_of_the_force(orc, laws, law, kin, averaged):
    m = laws[law]
    x = element_x()
    scale = 0.02 if kin != "small" else 0.004
    first = evaluate(orc, m, x, motion(x, scale, 7), None, kin, averaged, False)
    u2 = motion(x, 1.1 * scale, 9)
    base = evaluate(orc, m, x, u2, first["states"], kin, averaged, True)
    if law != "elastic":
        assert first["yielding"][0] > 0 and base["yielding"][0] > 0
    K = base["tangent"].reshape(24, 24)
    h = 1e-10
    err = 0.0
    for j in range(24):
        up, um = u2.copy(), u2.copy()
        up[0, j] += h
        um[0, j] -= h
        fd = (evaluate(orc, m, x, up, first["states"], kin, averaged, False)["force"].reshape(24)
              - evaluate(orc, m, x, um, first["states"], kin, averaged, False)["force"].reshape(24)) / (2 * h)
        err = max(err, np.abs(fd - K[:, j]).max())
    assert err / np.abs(K).max() <= 1e-8, err / np.abs(K).max()
    sym = np.abs(K - K.T).max() / np.abs(K).max()
    if law == "hill48+chaboche":
        assert sym > 1e-10  # recovering backstresses: not symmetric, and kept so
    else:
        assert sym == 0.0


def test_elastic_element_is_linear_and_bbar_keeps_a_homogeneous_dilatation(orc, laws):
    m = laws["elastic"]
    x = element_x()
    ue = motion(x, 1e-3, 5)
    r = evaluate(orc, m, x, ue, None, "small", False, True)
    K = r["tangent"].reshape(24, 24)
    f = r["force"].reshape(24)
    assert np.abs(f - K @ ue[0]).max() <= 1e-12 * (np.abs(K) @ np.abs(ue[0])).max()
    assert r["energy"][0] == pytest.approx(0.5 * ue[0] @ K @ ue[0], rel=1e-12)
    X = x.reshape(8, 3)
    homogeneous = np.zeros((8, 3))
    homogeneous[:, 0] = 1e-3 * (X[:, 0] - 0.4 * X[:, 1])
    homogeneous[:, 1] = 1e-3 * 0.7 * X[:, 1]
    homogeneous[:, 2] = 1e-3 * 0.7 * X[:, 2]
    hom = homogeneous.reshape(1, 24)
    f_std = evaluate(orc, m, x, hom, None, "small", False, False)["force"].reshape(24)
    f_bar = evaluate(orc, m, x, hom, None, "small", True, False)["force"].reshape(24)
    assert np.abs(f_std - f_bar).max() <= 1e-10 * np.abs(f_std).max()
