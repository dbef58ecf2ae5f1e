"""The oracle pinned to the reference's own known-answer and derivative
tests (CPU only). The reference's C++ tests cannot be built here (they need
Eigen, Catch2 and CMake), so their closed-form solutions, invariants and
central-difference checks are restated against the oracle with the
reference's tolerances:

- tests/test_plasticity.cpp:156-199 (uniaxial J2 with linear hardening,
  exact), :323-351 (the J2 consistent tangent is the derivative of the
  return);
- tests/test_anisotropy.cpp:255-290 (Hill48 calibration), :390-436 (Hill48
  uniaxial yield stress and r-value in every direction, equibiaxial),
  :578-647 (Chaboche exact monotonic curve, backward Euler at first order),
  :789-877 (the general consistent tangent);
- tests/test_logarithmic.cpp:110-207 (the Hencky strain and its first and
  second derivatives);
- tests/test_incompatible_modes.cpp:112-136 (line rules), :281-319 (exact
  pure bending), :433-508 (the condensed tangent of every kinematics and
  law), :510-595 (local iteration through reversals), :597-632 (homogeneous
  deformation), :634-689 (objectivity, the tangent at rest);
- tests/test_forming.cpp:235-329 (the penalty contact tangent is the
  derivative of its forces, with friction).

The random strains are the reference's own mt19937 draws; the matrix logarithm the Hencky strain is
checked against is mpmath's in 40 digits (the reference takes Eigen's
Schur-Pade)."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.linalg

E_STEEL, NU = 200.0e9, 0.3
SY = 250.0e6


def steel(**kw) -> dict:
    m = dict(youngs_modulus=E_STEEL, poisson_ratio=NU, yield_stress=SY)
    m.update(kw)
    return m


def ret(orc, m, strain, committed=None, tangent=True):
    r = orc.plastic_return(m, np.asarray(strain, dtype=np.float64), committed, tangent)
    assert r["code"] == 0, r["code"]
    return r


def relative(a, b) -> float:
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def drive(orc, m, strain, free, a, committed=None):
    """The return at a strain whose `free` components Newton finds so that
    a . sigma = 0 (test_anisotropy.cpp:91-110)."""
    strain = np.array(strain, dtype=np.float64)
    a = np.atleast_2d(np.asarray(a, dtype=np.float64))
    for _ in range(60):
        r = ret(orc, m, strain, committed)
        res = a @ r["stress"]
        scale = max(np.abs(r["stress"]).max(), m.get("yield_stress", 0.0))
        if np.abs(res).max() <= 1e-13 * scale:
            return r
        j = np.stack([a @ r["tangent"][:, c] for c in free], axis=1)
        strain[free] -= np.linalg.solve(j, res)
    raise AssertionError("the stress-state iteration did not converge")


def uniaxial(orc, m, e11, committed=None):
    """sigma_11 at eps_11 = e11 with the other five stresses zero."""
    ep = np.zeros(6) if committed is None else committed[0:6]
    strain = ep.copy()
    strain[0] = e11
    strain[1:3] = ep[1:3] - m["poisson_ratio"] * (e11 - ep[0])
    free = [1, 2, 3, 4, 5]
    return drive(orc, m, strain, free, np.eye(6)[free], committed)


def mt19937_uniform(seed, n):
    """n draws of std::uniform_real_distribution<double>(-1, 1) from
    std::mt19937(seed), as the reference's tests take them: numpy's legacy
    RandomState seeds MT19937 as std::mt19937 does, and libstdc++'s
    generate_canonical makes each double from two 32-bit outputs."""
    raw = np.random.RandomState(seed).randint(0, 2 ** 32, size=2 * n, dtype=np.uint32).astype(np.float64)
    u = (raw[0::2] + raw[1::2] * 2.0 ** 32) / 2.0 ** 64
    u = np.where(u >= 1.0, np.nextafter(1.0, 0.0), u)
    return u * 2.0 - 1.0


def random_strain(amplitude, seed):
    """random_strain of the reference's tests (test_plasticity.cpp:86-92)."""
    return amplitude * mt19937_uniform(seed, 6)


def return_tangent_error(orc, m, strain, committed, h=1e-8):
    r = ret(orc, m, strain, committed)
    worst = 0.0
    for j in range(6):
        up, um = strain.copy(), strain.copy()
        up[j] += h
        um[j] -= h
        fd = (ret(orc, m, up, committed)["stress"] - ret(orc, m, um, committed)["stress"]) / (2 * h)
        worst = max(worst, np.abs(fd - r["tangent"][:, j]).max())
    return worst / np.abs(r["tangent"]).max()


# --------------------------------------------------------------------------
# The returns
# --------------------------------------------------------------------------

@pytest.mark.parametrize("h,hk", [(0.0, 0.0), (2.0e9, 0.0), (0.0, 5.0e9), (1.0e9, 3.0e9)])
def test_uniaxial_linear_hardening_is_exact(orc, h, hk):
    m = steel(hardening_modulus=h, kinematic_hardening_modulus=hk)
    hh = h + hk
    target = 0.01
    exact = E_STEEL * (SY + hh * target) / (E_STEEL + hh)
    one = uniaxial(orc, m, target)
    assert one["yielding"]
    assert one["stress"][0] == pytest.approx(exact, rel=1e-12)
    state = None
    for k in range(1, 41):
        r = uniaxial(orc, m, target * k / 40.0, state)
        state = r["state"]
    assert r["stress"][0] == pytest.approx(exact, rel=1e-12)
    eps_p = target - exact / E_STEEL
    assert state[0] == pytest.approx(eps_p, rel=1e-10)
    assert state[1] == pytest.approx(-0.5 * eps_p, rel=1e-10)
    assert state[36] == pytest.approx(eps_p, rel=1e-10)
    assert r["energy"] == pytest.approx(exact * exact / (2 * E_STEEL) + 0.5 * hh * eps_p * eps_p, rel=1e-10)


def test_j2_consistent_tangent_is_the_derivative(orc):
    m = steel(hardening_modulus=1.5e9, kinematic_hardening_modulus=4.0e9, saturation_stress=100.0e6,
              saturation_rate=20.0)
    first = random_strain(4.0e-3, 3)
    second = first + random_strain(3.0e-3, 5)
    r1 = ret(orc, m, first)
    assert r1["yielding"]
    r2 = ret(orc, m, second, r1["state"])
    assert r2["yielding"]
    assert return_tangent_error(orc, m, second, r1["state"]) <= 1e-6
    back = second - 0.1 * (second - first)
    assert not ret(orc, m, back, r2["state"])["yielding"]
    assert return_tangent_error(orc, m, back, r2["state"]) <= 1e-6
    t = r2["tangent"]
    assert np.abs(t - t.T).max() <= 1e-12 * np.abs(t).max()


def hill(theta_deg=0.0, r0=1.9, r45=1.5, r90=2.3, **kw):
    a = np.deg2rad(theta_deg)
    return steel(criterion="hill48", r0=r0, r45=r45, r90=r90, rolling_direction=(np.cos(a), np.sin(a), 0.0), **kw)


def hill_coefficients(r0=1.9, r45=1.5, r90=2.3):
    F = r0 / (r90 * (1 + r0))
    G = 1 / (1 + r0)
    H = r0 / (1 + r0)
    N = (r0 + r90) * (1 + 2 * r45) / (2 * r90 * (1 + r0))
    return F, G, H, N


def test_hill48_yield_matrix_follows_the_calibration(orc):
    F, G, H, N = hill_coefficients()
    assert F == pytest.approx(1.9 / (2.3 * 2.9), rel=1e-15)
    assert N == pytest.approx((1.9 + 2.3) * 4.0 / (2.0 * 2.3 * 2.9), rel=1e-15)
    P = orc.yield_matrix(hill(0.0))
    expect = np.array([[G + H, -H, -G], [-H, F + H, -F], [-G, -F, F + G]])
    assert relative(P[:3, :3], expect) <= 1e-15
    assert P[3, 3] == pytest.approx(2 * N, rel=1e-15)
    assert P[4, 4] == pytest.approx(3.0, rel=1e-15) and P[5, 5] == pytest.approx(3.0, rel=1e-15)
    # r = 1 is von Mises: sigma^T P sigma is the von Mises stress squared.
    iso = orc.yield_matrix(hill(0.0, 1.0, 1.0, 1.0))
    s = random_strain(3.0e8, 11)
    vm2 = 0.5 * ((s[0] - s[1]) ** 2 + (s[1] - s[2]) ** 2 + (s[2] - s[0]) ** 2) + 3 * (s[3] ** 2 + s[4] ** 2 + s[5] ** 2)
    assert s @ iso @ s == pytest.approx(vm2, rel=1e-14)
    # Pressure-insensitive and symmetric in a tilted frame.
    pt = orc.yield_matrix(steel(criterion="hill48", r0=1.9, r45=1.5, r90=2.3, rolling_direction=(1.0, 0.3, -0.2),
                                sheet_normal=(0.2, -0.4, 1.0)))
    assert np.abs(pt @ np.array([1, 1, 1, 0, 0, 0.0])).max() <= 1e-14 * np.abs(pt).max()
    assert relative(pt, pt.T) <= 1e-15


@pytest.mark.parametrize("theta", [0.0, 15.0, 30.0, 45.0, 60.0, 75.0, 90.0])
def test_hill48_uniaxial_yield_stress_and_r_value(orc, theta):
    F, G, H, N = hill_coefficients()
    t = np.deg2rad(theta)
    s, c = np.sin(t), np.cos(t)
    phi = F * s ** 4 + G * c ** 4 + H * np.cos(2 * t) ** 2 + 2 * N * s * s * c * c
    r_theta = (H + (2 * N - F - G - 4 * H) * s * s * c * c) / (F * s * s + G * c * c)
    m = hill(-theta)  # rolled at -theta from x: loaded along x at theta from RD
    r = uniaxial(orc, m, 0.01)
    assert r["yielding"]
    assert r["stress"][0] == pytest.approx(SY / np.sqrt(phi), rel=1e-12)
    ep = r["state"][0:6]
    thickness = -(ep[0] + ep[1])
    assert abs(ep[0] + ep[1] + ep[2]) <= 1e-15 * ep[0]
    assert ep[2] == pytest.approx(thickness, rel=1e-12)
    assert abs(ep[4]) + abs(ep[5]) <= 1e-12 * ep[0]
    assert ep[1] / thickness == pytest.approx(r_theta, rel=1e-12)
    assert r["state"][36] == pytest.approx(r["stress"][0] * ep[0] / SY, rel=1e-12)


def test_hill48_equibiaxial(orc):
    """sigma_b = sigma_y sqrt(r90 (1 + r0) / (r0 + r90)), eps_p22 / eps_p11 =
    r0 / r90 (in 3-D: sigma_33 and the shears free and zero)."""
    m = hill(0.0)
    a = np.zeros((5, 6))
    a[0, 0], a[0, 1] = -1.0, 1.0
    for i, k in enumerate([2, 3, 4, 5]):
        a[i + 1, k] = 1.0
    strain = np.array([0.01, 0.01, -0.02 * NU / (1 - NU), 0, 0, 0])
    b = drive(orc, m, strain, [1, 2, 3, 4, 5], a)
    assert b["yielding"]
    assert b["stress"][0] == pytest.approx(SY * np.sqrt(2.3 * 2.9 / 4.2), rel=1e-12)
    assert b["stress"][1] == pytest.approx(b["stress"][0], rel=1e-13)
    assert b["state"][1] / b["state"][0] == pytest.approx(1.9 / 2.3, rel=1e-12)


def chaboche_stress(law, p):
    s = law["yield_stress"] + law.get("hardening_modulus", 0.0) * p
    s += law.get("saturation_stress", 0.0) * -np.expm1(-law.get("saturation_rate", 0.0) * p)
    for C, g in law["backstresses"]:
        s += C / g * -np.expm1(-g * p) if g > 0 else C * p
    return s


def test_chaboche_exact_monotonic_curve_and_backward_euler_order(orc):
    law = steel(yield_stress=170.0e6, saturation_stress=90.0e6, saturation_rate=12.0,
                backstresses=[(60.0e9, 600.0), (8.0e9, 60.0), (1.0e9, 0.0)])

    def exact(strain):
        lo, hi = 0.0, strain
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if mid + chaboche_stress(law, mid) / E_STEEL - strain > 0:
                hi = mid
            else:
                lo = mid
        return chaboche_stress(law, 0.5 * (lo + hi))

    for target in (0.002, 0.02, 0.2):
        sigma = exact(target)
        one = uniaxial(orc, law, target)
        assert one["stress"][0] == pytest.approx(sigma, rel=1e-11)
        point = None
        for step in range(1, 26):
            r = uniaxial(orc, law, target * step / 25.0, point)
            point = r["state"]
        assert r["stress"][0] == pytest.approx(sigma, rel=1e-11)
        plastic = point[36]
        assert point[0] == pytest.approx(plastic, rel=1e-10)
        for i, (C, g) in enumerate(law["backstresses"]):
            x = C / g * -np.expm1(-g * plastic) if g > 0 else C * plastic
            assert 1.5 * point[12 + 6 * i] == pytest.approx(x, rel=1e-10)
        assert point[6] == pytest.approx(point[12] + point[18] + point[24], rel=1e-15)
    be = dict(law, kinematic_integration="backward_euler")
    sigma = exact(0.02)
    errors = []
    for steps in (10, 20, 40, 80):
        point = None
        for step in range(1, steps + 1):
            r = uniaxial(orc, be, 0.02 * step / steps, point)
            point = r["state"]
        errors.append(abs(r["stress"][0] - sigma) / sigma)
    assert errors[0] > 1e-4
    for a, b in zip(errors, errors[1:]):
        assert a / b == pytest.approx(2.0, rel=0.1)


def general_cases():
    chab = [(50.0e9, 500.0), (6.0e9, 50.0), (1.0e9, 0.0)]
    h = hill(25.0, hardening_modulus=1.0e9, saturation_stress=80.0e6, saturation_rate=20.0)
    both = dict(h, backstresses=chab, kinematic_hardening_modulus=2.0e9, rolling_direction=(1.0, 0.4, 0.3),
                sheet_normal=(-0.3, 0.1, 1.0))
    return [("hill_voce", h, True),
            ("chaboche_voce", steel(backstresses=chab, saturation_stress=60.0e6, saturation_rate=15.0), False),
            ("hill_chaboche_prager_voce", both, False),
            ("backward_euler", dict(both, kinematic_integration="backward_euler"), False),
            ("in_plane", dict(both, rolling_direction=(np.cos(np.deg2rad(25)), np.sin(np.deg2rad(25)), 0.0),
                              sheet_normal=(0.0, 0.0, 1.0)), False),
            ("hill_two_linear", dict(h, backstresses=[(6.0e9, 0.0)], kinematic_hardening_modulus=1.0e9), True)]


@pytest.mark.parametrize("name,m,symmetric", general_cases(), ids=[c[0] for c in general_cases()])
def test_general_consistent_tangent(orc, name, m, symmetric):
    first = random_strain(4.0e-3, 3)
    second = first + random_strain(3.0e-3, 5)
    r1 = ret(orc, m, first)
    assert r1["yielding"]
    r2 = ret(orc, m, second, r1["state"])
    assert r2["yielding"]
    assert return_tangent_error(orc, m, second, r1["state"]) <= 1e-8
    asym = relative(r2["tangent"], r2["tangent"].T)
    assert (asym <= 1e-12) if symmetric else (asym >= 1e-4)
    back = second - 0.1 * (second - first)
    assert not ret(orc, m, back, r2["state"])["yielding"]
    assert return_tangent_error(orc, m, back, r2["state"]) <= 1e-8
    again = ret(orc, m, second, r2["state"])
    assert not again["yielding"]
    assert relative(again["stress"], r2["stress"]) <= 1e-12
    lean = ret(orc, m, second, r1["state"], tangent=False)
    assert np.array_equal(lean["stress"], r2["stress"])
    bad = random_strain(4.0e-3, 3)
    bad[0] = np.nan
    assert orc.plastic_return(m, bad)["code"] != 0


# --------------------------------------------------------------------------
# The logarithmic strain
# --------------------------------------------------------------------------

def engineering(t):
    return np.array([t[0, 0], t[1, 1], t[2, 2], 2 * t[0, 1], 2 * t[1, 2], 2 * t[2, 0]])


def rotation(angle, axis):
    axis = np.asarray(axis, dtype=np.float64)
    return scipy.spatial.transform.Rotation.from_rotvec(angle * axis / np.linalg.norm(axis)).as_matrix()


def logm_exact(c):
    """ln C of the double matrix C in 40-digit arithmetic (mpmath), an
    independent matrix logarithm accurate to the last bit of the result."""
    import mpmath

    with mpmath.workdps(40):
        lm = mpmath.logm(mpmath.matrix([[mpmath.mpf(float(v)) for v in row] for row in c]))
        return np.array([[float(lm[i, j]) for j in range(3)] for i in range(3)])


def derivative4(f, x, h):
    d = np.zeros((6, 6))
    for j in range(6):
        def at(s):
            y = x.copy()
            y[j] += s
            return f(y)
        d[:, j] = (-at(2 * h) + 8 * at(h) - 8 * at(-h) + at(-2 * h)) / (12 * h)
    return d


A = 1.4
LOG_CASES = [("distinct", (2.3, 0.6, 1.1)), ("two_equal", (1.7, 1.7, 0.5)), ("identity", (1.0, 1.0, 1.0)),
             ("scaled_identity", (1.69, 1.69, 1.69)), ("two_1e-9", (A, A * (1 + 1e-9), 0.8)),
             ("two_1e-7", (A, A * (1 + 1e-7), 0.8)), ("two_1e-4", (A, A * (1 + 1e-4), 0.8)),
             ("three_1e-9", (A, A * (1 + 1e-9), A * (1 + 2e-9))), ("three_1e-7", (A, A * (1 + 0.4e-7), A * (1 + 1e-7))),
             ("three_1e-4", (A, A * (1 + 1e-4), A * (1 + 2.5e-4))),
             ("three_4e-3_series", (A, A * (1 + 2e-3), A * (1 + 4e-3))),
             ("three_6e-3_quotient", (A, A * (1 + 3e-3), A * (1 + 6e-3))),
             ("stretch2_nearly_equal", (4.0, 0.25, 0.25 * (1 + 1e-8)))]
T_LOG = np.array([3.0e8, -1.0e8, 0.5e8, 0.7e8, -0.4e8, 0.2e8])


@pytest.mark.parametrize("name,lam", LOG_CASES, ids=[c[0] for c in LOG_CASES])
def test_log_strain_and_derivatives(orc, name, lam):
    import scipy.spatial.transform  # noqa: F401  (rotation())

    q = rotation(0.7, (0.3, -1.0, 0.5))
    lam = np.array(lam)
    cg = q @ np.diag(lam) @ q.T
    green = engineering(0.5 * (cg - np.eye(3)))
    log = orc.log_strain(green, T_LOG)
    assert log["code"] == 0
    reference = engineering(0.5 * logm_exact(cg))
    assert relative(log["strain"], reference) <= 1e-14
    assert log["strain"][:3].sum() == pytest.approx(0.5 * np.log(np.linalg.det(cg)), abs=4e-15)
    h = 5e-4 * lam.min()
    p_fd = derivative4(lambda e: orc.log_strain(e)["strain"], green, h)
    l_fd = derivative4(lambda e: orc.log_strain(e, T_LOG)["stress"], green, h)
    assert relative(log["projection"], p_fd) <= 1e-11
    assert relative(log["curvature"], l_fd) <= 1e-11
    assert relative(log["curvature"], log["curvature"].T) <= 1e-15
    assert relative(log["stress"], log["projection"].T @ T_LOG) <= 1e-15


def test_log_strain_continuity_identity_small_and_refusals(orc):
    import scipy.spatial.transform  # noqa: F401

    q = rotation(0.7, (0.3, -1.0, 0.5))

    def green(l):
        return engineering(0.5 * (q @ np.diag(l) @ q.T - np.eye(3)))

    equal = orc.log_strain(green((A, A, 0.8)), T_LOG)
    near = orc.log_strain(green((A, A * (1 + 1e-9), 0.8)), T_LOG)
    assert relative(near["projection"], equal["projection"]) <= 2e-9
    assert relative(near["curvature"], equal["curvature"]) <= 2e-9
    ident = orc.log_strain(np.zeros(6))
    assert np.abs(ident["projection"] - np.eye(6)).max() <= 1e-15
    draws = iter(mt19937_uniform(5, 6))
    e = np.zeros((3, 3))
    for i in range(3):
        for j in range(i, 3):
            e[i, j] = e[j, i] = 1e-6 * next(draws)
    series = e - e @ e + 4.0 / 3.0 * e @ e @ e
    assert relative(orc.log_strain(engineering(e))["strain"], engineering(series)) <= 1e-15
    bad = np.zeros(6)
    bad[0] = -0.6
    assert orc.log_strain(bad)["code"] != 0
    bad[0] = np.nan
    assert orc.log_strain(bad)["code"] != 0


# --------------------------------------------------------------------------
# The incompatible-mode Hex8
# --------------------------------------------------------------------------

X_DISTORTED = np.array([[0.05, 0.00, 0.00], [1.10, 0.10, -0.05], [1.20, 1.15, 0.10], [-0.05, 0.90, 0.05],
                        [0.10, 0.05, 0.90], [0.95, -0.05, 1.05], [1.05, 1.05, 1.20], [0.00, 1.10, 1.00]])


def deformation(x, scale):
    ue = np.zeros(24)
    for a in range(8):
        p = x[a]
        ue[3 * a:3 * a + 3] = scale * np.array([0.8 * p[0] + 0.6 * p[0] * p[2] + 0.2 * p[1],
                                                -0.3 * p[1] + 0.5 * p[1] * p[2] - 0.4 * p[0] * p[1],
                                                -0.4 * p[2] - 0.5 * p[0] ** 2 + 0.3 * p[0] * p[1] * p[2]])
    return ue


def one(orc, m, ue, committed=None, alpha=None, kin="logarithmic", tp=0, X=X_DISTORTED, tangent=True):
    r = orc.elements(m, X.reshape(1, 24), np.asarray(ue).reshape(1, 24),
                     None if committed is None else committed[None], None if alpha is None else alpha[None], kin,
                     2, tp, 2, tangent)
    assert r["status"][0] == 0, r["status"][0]
    return {k: (v[0] if v is not None else None) for k, v in r.items()}


def batch_forces(orc, m, ues, committed, alpha, kin, tp, X=X_DISTORTED):
    n = len(ues)
    nq = orc.rule_size(2, tp, 2)
    r = orc.elements(m, np.repeat(X.reshape(1, 24), n, 0), np.asarray(ues),
                     np.repeat(committed[None], n, 0) if committed is not None else np.zeros((n, nq, orc.NF)),
                     np.repeat(alpha[None], n, 0) if alpha is not None else None, kin, 2, tp, 2, False)
    assert (r["status"] == 0).all()
    return r


def materials(pkg):
    mm = pkg.material
    return {"elastic": mm.elastic_steel().as_dict(), "j2": mm.j2_steel().as_dict(), "hill": mm.hill_sheet().as_dict(),
            "chaboche": mm.chaboche_steel().as_dict(), "perfect": mm.perfectly_plastic().as_dict()}


IM_CASES = [("small", "elastic", 1e-3, 0), ("small", "j2", 4e-3, 0), ("small", "hill", 4e-3, 3),
            ("small", "chaboche", 4e-3, 0), ("finite", "elastic", 0.05, 0), ("finite", "j2", 0.02, 0),
            ("finite", "hill", 0.02, 5), ("finite", "chaboche", 0.02, 0), ("logarithmic", "elastic", 0.05, 0),
            ("logarithmic", "j2", 0.1, 0), ("logarithmic", "hill", 0.1, 3), ("logarithmic", "chaboche", 0.1, 0)]


@pytest.mark.parametrize("kin,law,scale,tp", IM_CASES, ids=[f"{c[0]}-{c[1]}" for c in IM_CASES])
def test_condensed_tangent_is_the_derivative(orc, pkg, kin, law, scale, tp):
    m = materials(pkg)[law]
    plastic = m["yield_stress"] > 0
    x = X_DISTORTED
    first = one(orc, m, deformation(x, scale), kin=kin, tp=tp)
    committed = first["states"] if plastic else None
    alpha = first["alpha"]
    ue = deformation(x, 1.3 * scale)
    for a in range(8):
        ue[3 * a + 2] += 0.2 * scale * x[a, 0] * x[a, 1]
    el = one(orc, m, ue, committed, alpha, kin, tp)
    nq = orc.rule_size(2, tp, 2)
    if plastic:
        assert el["yielding"] == nq
    assert 1 <= el["iterations"] <= (1 if kin == "small" and not plastic else 5)
    K = el["tangent"]
    symmetric = all(g <= 0 for _, g in m["backstresses"])
    if symmetric:
        assert np.abs(K - K.T).max() == 0.0
    else:
        assert np.abs(K - K.T).max() > 1e-6 * np.abs(K).max()
    h = 1e-8
    ues = []
    for j in range(24):
        up, um = ue.copy(), ue.copy()
        up[j] += h
        um[j] -= h
        ues += [up, um]
    r = batch_forces(orc, m, ues, committed, alpha, kin, tp)
    fd = (r["force"][0::2] - r["force"][1::2]).T / (2 * h)
    assert np.abs(fd - K).max() / np.abs(K).max() <= 1e-6
    if not plastic:
        de = (r["energy"][0::2] - r["energy"][1::2]) / (2 * h)
        # (energies through the same perturbations at h = 1e-8, not 1e-7)
        assert np.abs(de - el["force"]).max() <= 1e-6 * np.abs(el["force"]).max()


@pytest.mark.parametrize("law", ["j2", "chaboche"])
@pytest.mark.parametrize("kin", ["small", "logarithmic"])
def test_local_iteration_through_a_reversal(orc, pkg, law, kin):
    m = materials(pkg)[law]
    x = X_DISTORTED
    scale = 4e-3 if kin == "small" else 0.02
    first = one(orc, m, deformation(x, scale), kin=kin, tp=5, tangent=False)
    assert first["yielding"] > 0
    ue = deformation(x, -6.0 * scale)
    for a in range(8):
        ue[3 * a] += 2.0 * scale * x[a, 2] ** 2
    el = one(orc, m, ue, first["states"], first["alpha"], kin, 5)
    assert el["yielding"] > 0
    assert el["iterations"] <= 15
    again = one(orc, m, ue, first["states"], el["alpha"], kin, 5, tangent=False)
    assert again["iterations"] <= 1
    assert np.abs(again["force"] - el["force"]).max() <= 1e-8 * np.abs(el["force"]).max()


@pytest.mark.parametrize("law", ["perfect", "j2", "chaboche", "hill"])
@pytest.mark.parametrize("tp", [5, 7])
@pytest.mark.parametrize("factor", [-6.0, -10.0, -15.0])
def test_local_iteration_through_large_reversals(orc, pkg, law, tp, factor):
    m = materials(pkg)[law]
    x = X_DISTORTED
    first = one(orc, m, deformation(x, 0.02), tp=tp, tangent=False)
    ue = deformation(x, factor * 0.02)
    el = one(orc, m, ue, first["states"], first["alpha"], "logarithmic", tp, tangent=False)
    assert el["yielding"] > 0
    assert el["iterations"] <= 20
    again = one(orc, m, ue, first["states"], el["alpha"], "logarithmic", tp, tangent=False)
    assert again["iterations"] <= 1
    assert np.abs(again["force"] - el["force"]).max() <= 1e-8 * np.abs(el["force"]).max()


def test_reversals_spread_under_round_off_below_the_parity_bar(orc, pkg):
    """How far the reference's algorithm itself moves under a round-off
    perturbation on the 36 reversal cases (test_incompatible_modes.cpp:510-595,
    the cases of the GPU parity tests): the oracle built twice - every
    product and sum rounded separately, and -O3 -march=native with fused
    multiply-adds - gives the same local iteration counts and tangents that
    differ by up to about 8e-12 relative Frobenius (measured here), under the
    1e-11 bar the GPU is held to on the same cases. The largest spread comes
    from perfect plasticity and Chaboche at 10-15 times the first strain."""
    from conftest import rel_frobenius

    worst = 0.0
    try:
        for tp in (0, 5, 7):
            for law in ("j2", "chaboche", "hill", "perfect"):
                m = materials(pkg)[law]
                for factor in (-6.0, -10.0, -15.0):
                    out = {}
                    for variant in ("strict", "fast"):
                        orc.use_variant(variant)
                        kw = dict(kinematics="logarithmic", in_plane=2, thickness=tp)
                        X = X_DISTORTED.reshape(1, 24)
                        first = orc.elements(m, X, deformation(X_DISTORTED, 0.02).reshape(1, 24), want_tangent=False,
                                             **kw)
                        out[variant] = orc.elements(m, X, deformation(X_DISTORTED, factor * 0.02).reshape(1, 24),
                                                    first["states"], first["alpha"], **kw)
                    a, b = out["strict"], out["fast"]
                    assert a["status"][0] == b["status"][0]
                    if a["status"][0] != 0:
                        continue
                    assert a["iterations"][0] == b["iterations"][0], (tp, law, factor)
                    np.testing.assert_array_equal(a["yield_flags"], b["yield_flags"])
                    worst = max(worst, float(rel_frobenius(b["tangent"], a["tangent"]).max()))
    finally:
        orc.use_variant("strict")
    assert 1e-13 < worst < 2e-11, worst


@pytest.mark.parametrize("law", ["elastic", "j2", "hill"])
@pytest.mark.parametrize("kin", ["small", "finite", "logarithmic"])
def test_homogeneous_deformation_leaves_the_modes_at_zero(orc, pkg, law, kin):
    F = np.array([[1.04, 0.03, -0.02], [0.01, 0.97, 0.05], [-0.03, 0.02, 1.02]])
    scale = 0.1 if kin == "small" else 1.0
    ue = np.concatenate([scale * (F - np.eye(3)) @ X_DISTORTED[a] for a in range(8)])
    el = one(orc, materials(pkg)[law], ue, kin=kin, tp=3, tangent=False)
    assert np.abs(el["alpha"]).max() <= 1e-12


def test_objectivity_and_the_tangent_at_rest(orc, pkg):
    import scipy.spatial.transform  # noqa: F401

    m = materials(pkg)["j2"]
    x = X_DISTORTED
    R = rotation(0.7, (1.0, 2.0, 3.0))
    for kin in ("finite", "logarithmic"):
        rigid = np.concatenate([(R - np.eye(3)) @ x[a] for a in range(8)])
        rest = one(orc, m, rigid, kin=kin, tangent=False)
        assert np.abs(rest["force"]).max() <= 1e-3
        assert np.abs(rest["alpha"]).max() <= 1e-14
        ue = deformation(x, 0.02)
        rotated = np.concatenate([R @ (x[a] + ue[3 * a:3 * a + 3]) - x[a] for a in range(8)])
        el = one(orc, m, ue, kin=kin, tangent=False)
        er = one(orc, m, rotated, kin=kin, tangent=False)
        assert el["yielding"] == 8
        fmax = np.abs(el["force"]).max()
        for a in range(8):
            assert np.abs(er["force"][3 * a:3 * a + 3] - R @ el["force"][3 * a:3 * a + 3]).max() <= 1e-9 * fmax
        amax = np.abs(el["alpha"]).max()
        for k in range(3):
            assert np.abs(er["alpha"][3 * k:3 * k + 3] - R @ el["alpha"][3 * k:3 * k + 3]).max() <= 1e-9 * amax
    elastic = materials(pkg)["elastic"]
    k = one(orc, elastic, np.zeros(24), kin="small")["tangent"]
    for kin in ("small", "finite", "logarithmic"):
        el = one(orc, elastic, np.zeros(24), kin=kin)
        assert np.abs(el["tangent"] - k).max() <= 1e-12 * np.abs(k).max()
        assert el["iterations"] == 0


def free_compliance(k, f):
    w, v = np.linalg.eigh(k)
    top = np.abs(w).max()
    keep = np.abs(w) > 1e-10 * top
    p = v[:, keep].T @ f
    return float((p * p / w[keep]).sum())


@pytest.mark.parametrize("slenderness", [1.0, 10.0, 100.0])
def test_exact_pure_bending(orc, slenderness):
    young, nu, kappa = 70.0e9, 0.3, 1.0e-3
    h, width = 0.01, 0.02
    length = slenderness * h
    X = np.array([[0, 0, 0], [length, 0, 0], [length, width, 0], [0, width, 0], [0, 0, h], [length, 0, h],
                  [length, width, h], [0, width, h]], dtype=np.float64)
    ue = np.zeros(24)
    f = np.zeros(24)
    for a in range(8):
        x, y, z = X[a]
        zp = z - 0.5 * h
        ue[3 * a:3 * a + 3] = [kappa * x * zp, -nu * kappa * y * zp, -0.5 * kappa * (x * x + nu * (zp * zp - y * y))]
        sx = 1.0 if x > 0 else -1.0
        sz = 1.0 if z > 0 else -1.0
        f[3 * a] = sx * sz * 0.5 * width * young * kappa * h * h / 12.0
    m = dict(youngs_modulus=young, poisson_ratio=nu)
    el = one(orc, m, ue, kin="small", X=X)
    K = el["tangent"]
    gross = (np.abs(K) @ np.abs(ue)).max()
    assert np.abs(K @ ue - f).max() <= 1e-13 * gross
    assert np.abs(el["force"] - f).max() <= 1e-13 * gross
    assert free_compliance(K, f) / f.dot(ue) == pytest.approx(1.0, rel=1e-9)


@pytest.mark.parametrize("n", range(1, 8))
def test_line_rules_integrate_degree_2n_minus_1(orc, n):
    """A box rule of 2 x 2 in-plane points and n thickness points: its
    thickness coordinates are the n-point Gauss-Legendre line rule."""
    r = orc.rule(2, n, 2)
    assert len(r) == 4 * n
    # xi fastest: each layer of four points shares one zeta, and the 2 x 2
    # in-plane weights are 1, so a layer's weight is the line weight.
    zeta, line_w = r[::4, 2], r[::4, 3]
    for i in range(n):
        assert (r[4 * i:4 * i + 4, 2] == zeta[i]).all() and (r[4 * i:4 * i + 4, 3] == line_w[i]).all()
    for k in range(2 * n):
        exact = 0.0 if k % 2 else 2.0 / (k + 1.0)
        assert abs((line_w * zeta ** k).sum() - exact) <= 2e-15, k
    assert (np.diff(zeta) > 0).all()
    assert r[:, 3].sum() == pytest.approx(8.0, abs=1e-14)


# --------------------------------------------------------------------------
# Penalty contact
# --------------------------------------------------------------------------

def block(nx=20, ny=20, lx=0.01, ly=0.01, lz=0.001, seed=7):
    """The nodes of an nx x ny x 1 block with its top at z = 0, moved off
    the grid by up to 0.1 mm in x and y."""
    xs, ys, zs = np.linspace(0, lx, nx + 1), np.linspace(0, ly, ny + 1), np.array([-lz, 0.0])
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    coords = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=1)
    rng = np.random.default_rng(seed)
    coords[:, :2] += rng.uniform(-1e-4, 1e-4, (len(coords), 2))
    top = np.where(coords[:, 2] == 0.0)[0].astype(np.int32)
    area = np.full(len(top), lx * ly / (nx * ny))
    kappa = 10.0 * 70e9 / np.sqrt(area)
    return coords, top, area, kappa


def contact_fd_error(c, u, t, n):
    ev = c.evaluate(u, t, True)
    assert ev["code"] == 0
    top = np.abs(ev["blocks"]).max()
    h = 1e-9
    worst = 0.0
    for b, node in enumerate(ev["nodes"]):
        for col in range(3):
            d = 3 * node + col
            up, dn = u.copy(), u.copy()
            up[d] += h
            dn[d] -= h
            fd = (c.evaluate(up, t, False)["residual"] - c.evaluate(dn, t, False)["residual"]) / (2 * h)
            fd[3 * node:3 * node + 3] -= ev["blocks"][b][:, col]
            worst = max(worst, np.abs(fd).max() / top)
    return worst, ev


@pytest.mark.parametrize("shape", ["sphere", "plane", "cylinder"])
@pytest.mark.parametrize("friction", [0.0, 0.1, 0.8])
def test_contact_tangent_is_the_derivative(orc, shape, friction):
    coords, top, area, kappa = block()
    n = coords.size
    centre = (0.005, 0.005, -2e-5) if shape == "plane" else (0.0052, 0.0047, 0.005 - 1e-4)
    tool = dict(shape=shape, radius=0.005, friction=friction, tangential_ratio=1.0, normal=(0.1, -0.2, 1.0),
                axis=(1.0, 0.3, 0.0), times=[0.0, 1.0], points=[centre, tuple(np.add(centre, (1e-3, 0, 0)))],
                nodes=top, area=area, kappa=kappa)
    rng = np.random.default_rng(11)
    u1 = 0.02 * rng.uniform(-1e-4, 1e-4, n)
    u2 = u1 + 0.005 * rng.uniform(-1e-4, 1e-4, n)
    for mode in ("exact", "symmetric"):
        c = orc.Contact(coords, [tool], friction_tangent=mode)
        # A committed increment makes the friction history the second one
        # starts from.
        c.begin_increment(np.zeros(n), 0.0, 0.2, [True], 1e-3)
        assert c.evaluate(u1, 0.2, False)["code"] == 0
        c.commit()
        c.begin_increment(u1, 0.2, 0.25, [True], 1e-3)
        err, ev = contact_fd_error(c, u2, 0.25, n)
        active, slipping = ev["tools"][0][6], ev["tools"][0][7]
        assert active >= 3
        if mode == "exact":
            assert err < 1e-6, (err, active, slipping)
            if friction == 0.0:
                assert ev["symmetric"]
        else:
            assert ev["symmetric"]
            for b in ev["blocks"]:
                assert np.abs(b - b.T).max() == 0.0
            exact = orc.Contact(coords, [tool])
            exact.begin_increment(np.zeros(n), 0.0, 0.2, [True], 1e-3)
            exact.evaluate(u1, 0.2, False)
            exact.commit()
            exact.begin_increment(u1, 0.2, 0.25, [True], 1e-3)
            assert np.array_equal(exact.evaluate(u2, 0.25, False)["residual"], ev["residual"])


def test_stress_recovery_is_objective_and_reproduces_the_state(orc, pkg):
    """Stress recovery (incompatible_elastoplastic_stress,
    IncompatibleModes.cpp:602-664) at the converged state of a plastic step:
    the recovered second Piola-Kirchhoff stress and log strain are unchanged
    by a superposed rotation, the Kirchhoff and Cauchy stresses rotate
    (tests/test_logarithmic.cpp:329-383), the largest accumulated plastic
    strain is the committed one (the return from it is an elastic check),
    and at rest every stress is zero."""
    import scipy.spatial.transform  # noqa: F401

    m = dict(materials(pkg)["hill"], backstresses=[(30.0e9, 300.0)])
    x = X_DISTORTED
    R = rotation(0.9, (0.2, 1.0, -0.4))
    ue = deformation(x, 0.08)
    turned = np.concatenate([R @ (x[a] + ue[3 * a:3 * a + 3]) - x[a] for a in range(8)])
    el = one(orc, m, ue, tangent=False)
    er = one(orc, m, turned, tangent=False)
    assert el["yielding"] > 0
    s1, st1 = orc.element_stress(m, x.reshape(1, 24), ue.reshape(1, 24), el["states"][None], el["alpha"][None])
    s2, st2 = orc.element_stress(m, x.reshape(1, 24), turned.reshape(1, 24), er["states"][None], er["alpha"][None])
    assert st1[0] == 0 and st2[0] == 0
    s1, s2 = s1[0], s2[0]

    def tens(v):
        return np.array([[v[0], v[3], v[5]], [v[3], v[1], v[4]], [v[5], v[4], v[2]]])

    def voigt(t):
        return np.array([t[0, 0], t[1, 1], t[2, 2], t[0, 1], t[1, 2], t[2, 0]])

    assert relative(s2[6:12], s1[6:12]) <= 1e-11  # second Piola-Kirchhoff
    assert relative(s2[22:28], s1[22:28]) <= 1e-12  # log strain
    assert relative(s2[16:22], voigt(R @ tens(s1[16:22]) @ R.T)) <= 1e-11  # Kirchhoff
    assert relative(s2[0:6], voigt(R @ tens(s1[0:6]) @ R.T)) <= 1e-11  # Cauchy
    assert s2[12] == pytest.approx(s1[12], rel=1e-11)  # von Mises
    assert s2[15] == pytest.approx(s1[15], rel=1e-13)  # min det F
    assert s1[13] == pytest.approx(el["states"][:, 36].max(), rel=1e-15)
    rest, st = orc.element_stress(m, x.reshape(1, 24), np.zeros((1, 24)))
    assert st[0] == 0 and np.abs(rest[0][:13]).max() == 0.0 and rest[0][15] == 1.0
