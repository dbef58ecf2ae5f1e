"""The system (NonlinearSystem::evaluate / commit through the C ABI) against
the oracle's restatement of the reference's element loop, gather and
element-order scatter (src/fem/NonlinearSystem.hpp:192-268,
src/fem/Assembler.cpp:86-215)."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

from conftest import dense_from_blocks, device_to_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(pkg, cuda):
    wl = importlib.import_module("springback-precomp_b200.workload")
    return wl.make_problem(24, 12, 2, seed=11, sample=576)


def make_system(pkg, prob):
    sys_ = pkg.NonlinearSystem(prob.mesh, prob.material, kinematics="logarithmic")
    sys_.set_committed(prob.state)
    sys_.set_internal(prob.alpha)
    return sys_


def test_pattern_is_the_reference_pattern(pkg, orc, problem):
    sys_ = make_system(pkg, problem)
    pat = orc.pattern(problem.mesh.num_nodes, problem.mesh.connectivity)
    np.testing.assert_array_equal(sys_.outer.cpu().numpy(), pat["outer"])
    np.testing.assert_array_equal(sys_.inner.cpu().numpy(), pat["inner"])


def test_evaluate_matches_oracle(pkg, orc, problem, cuda):
    mesh, mat = problem.mesh, problem.material
    sys_ = make_system(pkg, problem)
    u = torch.tensor(problem.u, device=cuda)
    ev = sys_.evaluate(u, 0.0, True)
    nt = mat.kinematic_terms
    ref = orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, problem.u,
                              device_to_oracle(problem.state, nt), problem.alpha, kinematics="logarithmic")
    assert ref["code"] == 0
    f = ev.internal.cpu().numpy()
    scale = np.abs(ref["internal"]).max()
    assert np.abs(f - ref["internal"]).max() <= 1e-11 * ref["gross"]
    v = ev.tangent.cpu().numpy()
    assert np.linalg.norm(v - ref["values"]) <= 1e-11 * np.linalg.norm(ref["values"])
    assert ev.yielding_points == ref["yielding_points"]
    assert abs(ev.gross - ref["gross"]) <= 1e-12 * ref["gross"]
    assert abs(ev.energy - ref["energy"]) <= 1e-11 * abs(ref["energy"])
    st = device_to_oracle(sys_.trial_states(), nt)
    assert np.abs(st[..., 36] - ref["states"][..., 36]).max() <= 1e-10 * scale + 1e-12
    assert (sys_.trial_yield().sum() == ref["yielding_points"])


def test_assembly_is_the_element_order_sum(pkg, orc, problem, cuda):
    """Given the same element matrices, the gathered values equal the
    reference's element-by-element scatter bit for bit."""
    mesh, mat = problem.mesh, problem.material
    sys_ = make_system(pkg, problem)
    u = torch.tensor(problem.u, device=cuda)
    ev = sys_.evaluate(u, 0.0, True)
    values = ev.tangent.cpu().numpy().copy()
    x = torch.tensor(mesh.element_coordinates(), device=cuda)
    ue = torch.tensor(mesh.gather(problem.u), device=cuda)
    r = pkg.element_batch(mat, x, ue, torch.tensor(problem.state, device=cuda), torch.tensor(problem.alpha,
                                                                                                device=cuda))
    K = dense_from_blocks(r.tangent.cpu().numpy())
    pat = orc.pattern(mesh.num_nodes, mesh.connectivity)
    ref = orc.scatter(mesh.num_nodes, mesh.connectivity, pat, K)
    assert np.array_equal(values, ref)
    # f_int likewise, in element order per DOF.
    f = r.force.cpu().numpy()
    fi = np.zeros(mesh.num_dofs)
    for e in range(mesh.num_elements):
        for a in range(8):
            n = mesh.connectivity[e, a]
            fi[3 * n:3 * n + 3] += f[e, 3 * a:3 * a + 3]
    assert np.array_equal(ev.internal.cpu().numpy(), fi)


def test_commit_and_restart(pkg, problem, cuda):
    sys_ = make_system(pkg, problem)
    u = torch.tensor(problem.u, device=cuda)
    sys_.evaluate(u, 0.0, False)
    trial = sys_.trial_states()
    modes = sys_.trial_modes()
    sys_.commit()
    np.testing.assert_array_equal(sys_.committed_all(), trial)
    np.testing.assert_array_equal(sys_.internal_all(), modes)
    # A restart from the saved history evaluates alike.
    other = make_system(pkg, problem)
    other.set_committed(trial)
    other.set_internal(modes)
    a = sys_.evaluate(u, 0.0, True)
    fa, va = a.internal.clone(), a.tangent.clone()
    b = other.evaluate(u, 0.0, True)
    assert torch.equal(fa, b.internal) and torch.equal(va, b.tangent)


def test_solver_error_names_the_element(pkg, problem, cuda):
    sys_ = make_system(pkg, problem)
    u = torch.tensor(problem.u, device=cuda).clone()
    mesh = problem.mesh
    # Fold element 5 through itself: its top nodes below its bottom ones.
    top = mesh.connectivity[5, 4:]
    u.view(-1, 3)[torch.tensor(top, device=cuda), 2] -= 3.0 * 5e-4
    with pytest.raises(pkg.SolverError) as err:
        sys_.evaluate(u, 0.0, True)
    assert err.value.element >= 0


def test_stiffness_gross_is_the_reference_norm(pkg, orc, problem, cuda):
    """stiffness_gross (NonlinearSystem.hpp:49-67) of the assembled tangent
    over a free-DOF list that leaves out a clamped edge, after node blocks
    were added into it, against the oracle's column-ordered restatement."""
    mesh = problem.mesh
    sys_ = make_system(pkg, problem)
    u = torch.tensor(problem.u, device=cuda)
    ev = sys_.evaluate(u, 0.0, True)
    nodes = torch.arange(0, mesh.num_nodes, 7, dtype=torch.int32, device=cuda)
    blocks = torch.tensor(np.random.default_rng(3).uniform(-1e6, 1e6, (len(nodes), 3, 3)), device=cuda)
    sys_.add_node_blocks(nodes, blocks)
    x = mesh.coords[:, 0]
    clamped = np.where(x <= x.min() + 1e-12)[0]
    free = np.setdiff1d(np.arange(mesh.num_dofs), np.concatenate([3 * clamped, 3 * clamped + 1, 3 * clamped + 2]))
    u_host = problem.u.copy()
    u_host[3 * clamped] = 0.0  # columns of zero displacement are skipped
    got = sys_.stiffness_gross(torch.tensor(u_host, device=cuda), torch.tensor(free, device=cuda))
    pat = orc.pattern(mesh.num_nodes, mesh.connectivity)
    ref = orc.stiffness_gross(pat, ev.tangent.cpu().numpy(), u_host, free)
    assert abs(got - ref) <= 1e-14 * ref, (got, ref)
    with pytest.raises(pkg.SbkError):
        fresh = make_system(pkg, problem)
        fresh.stiffness_gross(u, torch.tensor(free, device=cuda))


def test_schedule_changes_no_result(pkg, problem, cuda):
    """The element schedule (elements grouped by the cost of their last
    evaluation) reorders only which warp evaluates which element: two
    evaluations with it equal, bit for bit, the same two in mesh order."""
    u = torch.tensor(problem.u, device=cuda)
    outs = []
    for by_cost in (False, True):
        sys_ = make_system(pkg, problem)
        sys_.set_schedule(by_cost)
        for _ in range(2):  # the second evaluation runs on the schedule of the first
            ev = sys_.evaluate(u, 0.0, True)
        outs.append((ev.internal.clone(), ev.tangent.clone(), ev.energy, ev.gross,
                     torch.tensor(sys_.trial_states()), torch.tensor(sys_.trial_modes())))
    for a, b in zip(*outs):
        if isinstance(a, torch.Tensor):
            assert torch.equal(a, b)
        else:
            assert a == b


def test_production_rule_system(pkg, orc, cuda):
    """A sheet with the production rule 2 x 2 x 5 (20 points per element;
    python/precomp/fea/setup.py:142-144), Hill48 + Chaboche, logarithmic
    strain, from virgin points: the system's f_int and assembled tangent
    against the oracle's."""
    mesh = pkg.structured_hex_mesh(8, 4, 1, 4e-3, 2e-3, 1e-3)
    mat = pkg.material.hill_chaboche_sheet()
    x = mesh.coords
    u = np.zeros_like(x)
    u[:, 2] = -0.005 * (x[:, 0] - x[:, 0].mean()) ** 2 / 4e-3  # bending: the outer points of the rule yield
    u[:, 0] = 0.0005 * (x[:, 2] - x[:, 2].mean()) * (x[:, 0] - x[:, 0].mean()) / 4e-3
    u = u.reshape(-1)
    sys_ = pkg.NonlinearSystem(mesh, mat, kinematics="logarithmic", thickness_points=5)
    assert sys_.nq == 20
    ev = sys_.evaluate(torch.tensor(u, device=cuda), 0.0, True)
    ref = orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, u, kinematics="logarithmic",
                              in_plane=2, thickness=5)
    assert ref["code"] == 0
    assert 0 < ref["yielding_points"] < 20 * mesh.num_elements
    assert ev.yielding_points == ref["yielding_points"]
    f = ev.internal.cpu().numpy()
    assert np.abs(f - ref["internal"]).max() <= 1e-11 * ref["gross"]
    v = ev.tangent.cpu().numpy()
    assert np.linalg.norm(v - ref["values"]) <= 1e-11 * np.linalg.norm(ref["values"])


@pytest.mark.parametrize("kin", ["logarithmic", "finite", "small"])
def test_stress_recovery_matches_oracle(pkg, orc, problem, cuda, kin):
    """Step-end stress recovery (elastoplastic_stress, IncompatibleModes.cpp
    :602-664) after a commit: every element's averages against the oracle's
    restatement at the committed points and modes."""
    mesh, mat = problem.mesh, problem.material
    sys_ = pkg.NonlinearSystem(mesh, mat, kinematics=kin)
    if kin == "logarithmic":
        sys_.set_committed(problem.state)
        sys_.set_internal(problem.alpha)
    u = torch.tensor(problem.u if kin == "logarithmic" else 0.5 * problem.u, device=cuda)
    sys_.evaluate(u, 0.0, False)
    sys_.commit()
    st, al = sys_.committed_views()
    committed = device_to_oracle(st.cpu().numpy(), mat.kinematic_terms)
    alpha = al.cpu().numpy()
    got = sys_.stress(u)
    X = mesh.element_coordinates()
    ue = mesh.gather(u.cpu().numpy())
    ref, status = orc.element_stress(mat.as_dict(), X, ue, committed, alpha, kinematics=kin)
    assert (status == 0).all()
    packed = torch.cat([got.cauchy, got.piola_kirchhoff, got.von_mises[:, None], got.max_plastic_strain[:, None],
                        got.max_strain[:, None], got.min_jacobian[:, None], got.kirchhoff, got.log_strain],
                       dim=1).cpu().numpy()
    for lo, hi in [(0, 6), (6, 12), (12, 13), (13, 14), (14, 15), (15, 16), (16, 22), (22, 28)]:
        scale = max(np.abs(ref[:, lo:hi]).max(), 1e-300)
        assert np.abs(packed[:, lo:hi] - ref[:, lo:hi]).max() <= 1e-11 * scale, (lo, hi)
    if kin == "logarithmic":
        assert ref[:, 13].max() > 0.0


def test_out_of_range_indices_are_refused(pkg, problem, cuda):
    """Node blocks naming a node outside the mesh and free DOFs outside the
    model are refused: the kernels check each index before using it."""
    mesh = problem.mesh
    sys_ = make_system(pkg, problem)
    u = torch.tensor(problem.u, device=cuda)
    sys_.evaluate(u, 0.0, True)
    nodes = torch.tensor([0, mesh.num_nodes], dtype=torch.int32, device=cuda)
    blocks = torch.zeros((2, 3, 3), dtype=torch.float64, device=cuda)
    with pytest.raises(pkg.SbkError):
        sys_.add_node_blocks(nodes, blocks)
    free = torch.tensor([0, 1, mesh.num_dofs], dtype=torch.int32, device=cuda)
    with pytest.raises(pkg.SbkError):
        sys_.stiffness_gross(u, free)


def test_system_phase_kernels_match_the_single_kernel(pkg, cuda):
    """NonlinearSystem.evaluate through the phase kernels (the default) and
    through the single kernel: the same yielding points, and the assembled
    tangent, f_int, energy, trial states and modes within 1e-13 of their
    scale (the compiled arithmetic may differ in the last bits), on the
    microbenchmark construction, for a first evaluation and for one under
    the element schedule."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    prob = wl.make_problem(30, 16, 2, seed=11, sample=480)
    out = {}
    for mode in ("phases", "single"):
        sysm = pkg.NonlinearSystem(prob.mesh, prob.material, kinematics="logarithmic")
        sysm.set_local_iteration(mode)
        sysm.set_committed(prob.state)
        sysm.set_internal(prob.alpha)
        u = torch.tensor(prob.u, device=cuda)
        evs = []
        for _ in range(2):  # the second walks the schedule
            ev = sysm.evaluate(u, 0.0, True)
            evs.append((ev.tangent.clone(), ev.internal.clone(), ev.energy, ev.yielding_points))
        out[mode] = (evs, sysm.trial_states(), sysm.trial_modes())
    (ea, sa, ma), (eb, sb, mb) = out["phases"], out["single"]
    tol = 1.0e-13
    for (ka, fa, ena, ya), (kb, fb, enb, yb) in zip(ea, eb):
        assert (ka - kb).abs().max().item() <= tol * kb.abs().max().item()
        assert (fa - fb).abs().max().item() <= tol * fb.abs().max().item()
        assert abs(ena - enb) <= tol * abs(enb) and ya == yb
    assert np.abs(sa - sb).max() <= tol * np.abs(sb).max()
    assert np.abs(ma - mb).max() <= tol * np.abs(mb).max()


def test_values_buffer_of_the_caller(pkg, cuda):
    """sbk_system_set_values_buffer: evaluations with the tangent assemble
    into the caller's buffer - alternating two, as a driver that reads one
    back while the next evaluation fills the other - with the values of the
    system's own buffer; node blocks go into the current buffer; None
    returns to the own buffer."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    prob = wl.make_problem(12, 8, 2, seed=4, sample=192)
    sysm = pkg.NonlinearSystem(prob.mesh, prob.material, kinematics="logarithmic")
    sysm.set_committed(prob.state)
    sysm.set_internal(prob.alpha)
    u = torch.tensor(prob.u, device=cuda)
    own = sysm.evaluate(u, 0.0, True).tangent.clone()
    bufs = [torch.full((sysm.nnz,), float("nan"), dtype=torch.float64, device=cuda) for _ in range(2)]
    for k in range(4):
        sysm.set_values_buffer(bufs[k % 2])
        ev = sysm.evaluate(u, 0.0, True)
        assert ev.tangent.data_ptr() == bufs[k % 2].data_ptr()
        assert torch.equal(bufs[k % 2], own)
    nodes = torch.tensor([0, 3], dtype=torch.int32, device=cuda)
    blocks = torch.ones((2, 3, 3), dtype=torch.float64, device=cuda)
    sysm.add_node_blocks(nodes, blocks)  # into bufs[1], the current one
    assert not torch.equal(bufs[1], own) and torch.equal(bufs[0], own)
    sysm.set_values_buffer(None)
    ev = sysm.evaluate(u, 0.0, True)
    assert ev.tangent.data_ptr() not in (bufs[0].data_ptr(), bufs[1].data_ptr())
    assert torch.equal(ev.tangent, own)
