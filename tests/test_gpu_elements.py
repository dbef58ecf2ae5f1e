"""Parity of the CUDA element kernel (through the C ABI's sbk_element_batch)
with the oracle: per-element K_T and R within 1e-11 relative Frobenius,
per-point yield flags bit-exact, the modes, states, energies and local
iteration counts alike, on the reference's own test elements
(tests/test_incompatible_modes.cpp:433-595) and on seeded microbenchmark
elements."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

from conftest import X_DISTORTED, deformation, dense_from_blocks, device_to_oracle, oracle_to_device, rel_frobenius

pytestmark = pytest.mark.gpu

TOL_K = 1.0e-11  # relative Frobenius, per element
TOL_F = 1.0e-11

LAWS = ["elastic", "j2", "hill", "chaboche"]
KINEMATICS = ["small", "finite", "logarithmic"]
SCALES = {("small", False): 1e-3, ("small", True): 4e-3, ("finite", False): 0.05, ("finite", True): 0.02,
          ("logarithmic", False): 0.05, ("logarithmic", True): 0.1}


def material(pkg, law):
    m = pkg.material
    return {"elastic": m.elastic_steel, "j2": m.j2_steel, "hill": m.hill_sheet, "chaboche": m.chaboche_steel,
            "hill_chaboche": m.hill_chaboche_sheet, "perfect": m.perfectly_plastic}[law]()


def run_gpu(pkg, mat, X, ue, state_dev, alpha, kin, cuda, want_tangent=True, rule=(2, 0)):
    x = torch.tensor(np.asarray(X).reshape(-1, 24), device=cuda)
    u = torch.tensor(np.asarray(ue).reshape(-1, 24), device=cuda)
    st = torch.tensor(np.ascontiguousarray(state_dev), device=cuda) if state_dev is not None else None
    al = torch.tensor(np.asarray(alpha).reshape(-1, 9), device=cuda) if alpha is not None else None
    r = pkg.element_batch(mat, x, u, st, al, kinematics=kin, want_tangent=want_tangent, stiffness_points=rule[0],
                          thickness_points=rule[1])
    torch.cuda.synchronize()
    return r


def compare(ref, r, nterms, want_tangent=True, tol_k=TOL_K, tol_f=TOL_F):
    np.testing.assert_array_equal(r.code.cpu().numpy(), ref["status"])
    ok = ref["status"] == 0
    if not ok.any():
        return
    f = r.force.cpu().numpy()[ok]
    ef = rel_frobenius(f, ref["force"][ok])
    assert ef.max() <= tol_f, f"force error {ef.max():.3e}"
    if want_tangent:
        K = dense_from_blocks(r.tangent.cpu().numpy())[ok]
        ek = rel_frobenius(K, ref["tangent"][ok])
        assert ek.max() <= tol_k, f"tangent error {ek.max():.3e}"
    np.testing.assert_array_equal(r.yielding.cpu().numpy()[ok].astype(bool), ref["yield_flags"][ok])
    np.testing.assert_array_equal(r.iterations.cpu().numpy()[ok], ref["iterations"][ok])
    a, ra = r.alpha.cpu().numpy()[ok], ref["alpha"][ok]
    assert np.abs(a - ra).max() <= 1e-10 * (np.abs(ra).max() + 1e-300)
    st = device_to_oracle(r.states.cpu().numpy(), nterms)[ok]
    rs = ref["states"][ok]
    for lo, hi in [(0, 6), (6, 12), (12, 12 + 6 * nterms), (36, 37)]:
        if hi > lo:
            d = np.abs(st[..., lo:hi] - rs[..., lo:hi]).max()
            assert d <= 1e-10 * (np.abs(rs[..., lo:hi]).max() + 1e-30), (lo, hi, d)
    np.testing.assert_array_equal(st[..., 38], rs[..., 38])
    e, re_ = r.energy.cpu().numpy()[ok], ref["energy"][ok]
    assert np.abs(e - re_).max() <= 1e-11 * (np.abs(re_).max() + 1e-300)


@pytest.mark.parametrize("kin", KINEMATICS)
@pytest.mark.parametrize("law", LAWS)
def test_two_step_cases(pkg, orc, cuda, law, kin):
    """The reference's condensed-tangent cases: a committed first step, then
    the check at a second one (test_incompatible_modes.cpp:433-508, with the
    2 x 2 x 2 rule)."""
    mat = material(pkg, law)
    plastic = mat.yield_stress > 0
    s = SCALES[(kin, plastic)]
    X = X_DISTORTED.reshape(1, 24)
    first = orc.elements(mat.as_dict(), X, deformation(X_DISTORTED, s).reshape(1, 24), kinematics=kin,
                         want_tangent=False)
    committed = first["states"] if plastic else np.zeros_like(first["states"])
    ue = deformation(X_DISTORTED, 1.3 * s)
    for a in range(8):
        ue[3 * a + 2] += 0.2 * s * X_DISTORTED[a, 0] * X_DISTORTED[a, 1]
    ref = orc.elements(mat.as_dict(), X, ue.reshape(1, 24), committed, first["alpha"], kinematics=kin)
    nt = mat.kinematic_terms
    r = run_gpu(pkg, mat, X, ue, oracle_to_device(committed, nt), first["alpha"], kin, cuda)
    compare(ref, r, nt)
    if plastic:
        assert int(r.yielding.sum()) == 8


@pytest.mark.parametrize("law", ["j2", "chaboche", "hill", "perfect"])
@pytest.mark.parametrize("factor", [-6.0, -10.0, -15.0])
def test_reversal(pkg, orc, cuda, law, factor):
    """A committed plastic step, then a reversal of several times the strain
    in one increment under logarithmic kinematics
    (test_incompatible_modes.cpp:510-595): the line searches, the shifted
    direction and the Levenberg-Marquardt fallback of the local iteration."""
    mat = material(pkg, law)
    X = X_DISTORTED.reshape(1, 24)
    first = orc.elements(mat.as_dict(), X, deformation(X_DISTORTED, 0.02).reshape(1, 24), kinematics="logarithmic",
                         want_tangent=False)
    ue = deformation(X_DISTORTED, factor * 0.02)
    ref = orc.elements(mat.as_dict(), X, ue.reshape(1, 24), first["states"], first["alpha"],
                       kinematics="logarithmic")
    nt = mat.kinematic_terms
    r = run_gpu(pkg, mat, X, ue, oracle_to_device(first["states"], nt), first["alpha"], "logarithmic", cuda)
    # 9 to 18 local iterations: measured on a B200 up to 7.6e-12 (perfect
    # plasticity, -10); two builds of the oracle itself (with and without
    # fused multiply-adds) differ by up to 8.0e-12 on these cases.
    compare(ref, r, nt)


def test_random_batch(pkg, orc, cuda):
    """Seeded microbenchmark elements (Hill48 + two-term Chaboche,
    logarithmic strain, about 40 % of the points yielding)."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    prob = wl.make_problem(40, 20, 2, seed=3, sample=512)
    mesh, mat = prob.mesh, prob.material
    X = mesh.element_coordinates()
    ue = mesh.gather(prob.u)
    nt = mat.kinematic_terms
    committed = device_to_oracle(prob.state, nt)
    ref = orc.elements(mat.as_dict(), X, ue, committed, prob.alpha, kinematics="logarithmic")
    r = run_gpu(pkg, mat, X, ue, prob.state, prob.alpha, "logarithmic", cuda)
    frac = ref["yield_flags"].mean()
    assert 0.2 < frac < 0.6, frac
    compare(ref, r, nt)


def test_residual_only_matches(pkg, cuda):
    """want_tangent = false gives the same force, modes and states."""
    mat = pkg.material.hill_chaboche_sheet()
    X = np.tile(X_DISTORTED.reshape(1, 24) * 1e-3, (4, 1))
    ue = np.stack([deformation(X_DISTORTED * 1e-3, s) for s in (0.01, 0.02, -0.015, 0.03)])
    a = run_gpu(pkg, mat, X, ue, None, None, "logarithmic", cuda, want_tangent=True)
    b = run_gpu(pkg, mat, X, ue, None, None, "logarithmic", cuda, want_tangent=False)
    assert torch.equal(a.force, b.force)
    assert torch.equal(a.alpha, b.alpha)
    assert torch.equal(a.states, b.states)


def test_failure_codes(pkg, orc, cuda):
    """An element inverted at rest (MeshError) and one whose deformation
    inverts a point under logarithmic kinematics (SolverError) report the
    oracle's codes; the good element beside them is unaffected."""
    mat = pkg.material.j2_steel()
    good = X_DISTORTED.reshape(24)
    bad = X_DISTORTED[[4, 5, 6, 7, 0, 1, 2, 3]].reshape(24)  # top and bottom swapped: det J < 0
    X = np.stack([good, bad, good])
    ue = np.stack([deformation(X_DISTORTED, 0.01), np.zeros(24), np.zeros(24)])
    for a in range(4, 8):
        ue[2, 3 * a + 2] = -2.5 * X_DISTORTED[a, 2]  # crush the third through itself
    ref = orc.elements(mat.as_dict(), X, ue, kinematics="logarithmic")
    r = run_gpu(pkg, mat, X, ue, None, None, "logarithmic", cuda)
    assert ref["status"][1] == 6 and ref["status"][2] != 0 and ref["status"][0] == 0
    compare(ref, r, mat.kinematic_terms)


def test_deterministic(pkg, cuda):
    """Two launches give bit-identical results."""
    mat = pkg.material.hill_chaboche_sheet()
    rng = np.random.default_rng(0)
    X = np.tile(X_DISTORTED.reshape(1, 24) * 1e-3, (64, 1))
    ue = np.stack([deformation(X_DISTORTED * 1e-3, s) for s in rng.uniform(-0.03, 0.03, 64)])
    a = run_gpu(pkg, mat, X, ue, None, None, "logarithmic", cuda)
    b = run_gpu(pkg, mat, X, ue, None, None, "logarithmic", cuda)
    assert torch.equal(a.force, b.force) and torch.equal(a.tangent, b.tangent)


RULES = [(2, 3), (2, 5), (2, 7), (3, 0)]


@pytest.mark.parametrize("rule", RULES, ids=lambda r: f"{r[0]}x{r[0]}x{r[1] or r[0]}")
@pytest.mark.parametrize("law", ["j2", "hill", "chaboche"])
def test_rules_beyond_eight_points(pkg, orc, cuda, law, rule):
    """The sheet rules with thickness points (2 x 2 x 3, 5, 7: 12 to 28
    points, the production rule being 2 x 2 x 5) and the 3 x 3 x 3 cube, a
    warp per element: the reference's condensed-tangent case
    (test_incompatible_modes.cpp:433-508) under logarithmic strain."""
    mat = material(pkg, law)
    X = X_DISTORTED.reshape(1, 24)
    kw = dict(kinematics="logarithmic", in_plane=rule[0], thickness=rule[1])
    first = orc.elements(mat.as_dict(), X, deformation(X_DISTORTED, 0.1).reshape(1, 24), want_tangent=False, **kw)
    ue = deformation(X_DISTORTED, 0.13)
    for a in range(8):
        ue[3 * a + 2] += 0.02 * X_DISTORTED[a, 0] * X_DISTORTED[a, 1]
    ref = orc.elements(mat.as_dict(), X, ue.reshape(1, 24), first["states"], first["alpha"], **kw)
    nt = mat.kinematic_terms
    r = run_gpu(pkg, mat, X, ue, oracle_to_device(first["states"], nt), first["alpha"], "logarithmic", cuda,
                rule=rule)
    compare(ref, r, nt)
    assert int(r.yielding.sum()) == orc.rule_size(*rule, 2)


@pytest.mark.parametrize("law", ["perfect", "j2", "chaboche", "hill"])
@pytest.mark.parametrize("tp", [5, 7])
@pytest.mark.parametrize("factor", [-6.0, -10.0, -15.0])
def test_reversal_with_thickness_points(pkg, orc, cuda, law, tp, factor):
    """Reversals of 6 to 15 times a 2 % logarithmic strain with 5 and 7
    thickness points (test_incompatible_modes.cpp:549-595), where K_aa turns
    indefinite and the shifted and Levenberg-Marquardt steps act."""
    mat = material(pkg, law)
    X = X_DISTORTED.reshape(1, 24)
    kw = dict(kinematics="logarithmic", in_plane=2, thickness=tp)
    first = orc.elements(mat.as_dict(), X, deformation(X_DISTORTED, 0.02).reshape(1, 24), want_tangent=False, **kw)
    ue = deformation(X_DISTORTED, factor * 0.02)
    ref = orc.elements(mat.as_dict(), X, ue.reshape(1, 24), first["states"], first["alpha"], **kw)
    assert ref["status"][0] == 0
    nt = mat.kinematic_terms
    r = run_gpu(pkg, mat, X, ue, oracle_to_device(first["states"], nt), first["alpha"], "logarithmic", cuda,
                rule=(2, tp))
    compare(ref, r, nt)


def test_rules_beyond_thirty_two_points_are_refused(pkg, cuda):
    mat = pkg.material.j2_steel()
    X = torch.tensor(X_DISTORTED.reshape(1, 24), device=cuda)
    with pytest.raises(pkg.SbkError) as e:
        pkg.element_batch(mat, X, torch.zeros_like(X), stiffness_points=4)  # 64 points
    assert e.value.status == 6


def _batch_both_ways(pkg, mat, X, ue, state_dev, alpha, cuda, rule=(2, 0)):
    system = importlib.import_module("springback-precomp_b200.system")
    out = {}
    try:
        for mode in ("phases", "single"):
            system.set_local_iteration(mode)
            out[mode] = run_gpu(pkg, mat, X, ue, state_dev, alpha, "logarithmic", cuda, rule=rule)
    finally:
        system.set_local_iteration("phases")
    return out["phases"], out["single"]


# The phase kernels and the single kernel run the same functions on the same
# values, compiled into different kernels: the compiler may fuse a product
# into a sum across a function boundary in one and not in the other, so
# results may differ in the last bits. Every decision must be the same.
SAME_TOL = 1.0e-13


def _assert_same(a, b):
    for name in ("code", "iterations", "yielding"):
        assert torch.equal(getattr(a, name), getattr(b, name)), name
    ok = a.code == 0
    for name in ("force", "tangent", "energy", "alpha"):
        x, y = getattr(a, name)[ok], getattr(b, name)[ok]
        scale = y.abs().max().item() + 1e-300
        assert (x - y).abs().max().item() <= SAME_TOL * scale, (name, (x - y).abs().max().item() / scale)
    x, y = a.states[:, ok], b.states[:, ok]
    for f in range(x.shape[0]):
        scale = y[f].abs().max().item() + 1e-300
        assert (x[f] - y[f]).abs().max().item() <= SAME_TOL * scale, f


def test_phase_kernels_give_the_single_kernels_results(pkg, orc, cuda):
    """The local iteration as phase kernels over all elements takes every
    decision of the single kernel - status, local iteration count, yield
    flag of every point - and gives its outputs to 1e-13 of their scale:
    seeded microbenchmark elements (most on the full-Newton-step road, a few
    handed back to the single kernel) and the reference's reversal cases
    (line searches, shifted direction, Levenberg-Marquardt) side by side,
    plus a failing element."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    prob = wl.make_problem(40, 20, 2, seed=3, sample=512)
    mesh, mat = prob.mesh, prob.material
    X = mesh.element_coordinates()
    ue = mesh.gather(prob.u)
    a, b = _batch_both_ways(pkg, mat, X, ue, prob.state, prob.alpha, cuda)
    assert int((a.code == 0).sum()) == mesh.num_elements
    _assert_same(a, b)
    # Reversals of several times the first strain, one element each, with a
    # crushed element beside them.
    for law in ("perfect", "chaboche", "hill", "j2"):
        m = material(pkg, law)
        nt = m.kinematic_terms
        # The committed first step, from the CPU restatement.
        first = orc.elements(m.as_dict(), X_DISTORTED.reshape(1, 24), deformation(X_DISTORTED, 0.02).reshape(1, 24),
                             kinematics="logarithmic", want_tangent=False)
        Xs = np.tile(X_DISTORTED.reshape(1, 24), (4, 1))
        ues = np.stack([deformation(X_DISTORTED, f * 0.02) for f in (-6.0, -10.0, -15.0, 1.0)])
        for k in range(4, 8):
            ues[3, 3 * k + 2] = -2.5 * X_DISTORTED[k, 2]  # crush the last through itself
        st = np.repeat(oracle_to_device(first["states"], nt), 4, axis=1)
        al = np.repeat(first["alpha"].reshape(1, 9), 4, axis=0)
        a, b = _batch_both_ways(pkg, m, Xs, ues, st, al, cuda)
        assert int(a.code[3]) != 0
        _assert_same(a, b)
