"""The allocation-free evaluation (sbk_evaluate_noalloc) for callers that
cannot allocate device memory - a solver confined to a device arena its host
application hands it, or code that must not call cudaMalloc while it runs.
Through the C ABI it must give what the allocating path
(sbk_system_evaluate) gives on the same small mesh, on two calls in a row:
the second call reuses the library's fixed scratch array and must not see
the first call's sums.

This file is collected last, so that a run stopping at the first failure
has run every other test before it; it also passes alone in a fresh
process."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1.0e-11  # relative, as the parity tests


def test_noalloc_matches_system_evaluate_twice(pkg, cuda):
    wl = importlib.import_module("springback-precomp_b200.workload")
    system = importlib.import_module("springback-precomp_b200.system")
    prob = wl.make_problem(12, 6, 2, seed=21, sample=144)
    mesh, mat = prob.mesh, prob.material
    assert mesh.num_elements <= system.NOALLOC_MAX_ELEMENTS

    sysm = pkg.NonlinearSystem(mesh, mat, kinematics="logarithmic")
    sysm.set_committed(prob.state)
    sysm.set_internal(prob.alpha)
    u = torch.tensor(prob.u, device=cuda)
    ev = sysm.evaluate(u, 0.0, True)
    ref_internal = ev.internal.clone()
    ref_values = ev.tangent.clone()
    ref_energy, ref_gross, ref_yield = ev.energy, ev.gross, ev.yielding_points
    ref_trial = torch.tensor(sysm.trial_states(), device=cuda)
    ref_modes = torch.tensor(sysm.trial_modes(), device=cuda)

    # The caller's own buffers (here allocated by the test, as the caller would).
    coords = torch.tensor(mesh.coords, device=cuda)
    conn = torch.tensor(mesh.connectivity, device=cuda)
    state = torch.tensor(prob.state, device=cuda)
    alpha = torch.tensor(prob.alpha, device=cuda)
    internal = torch.empty(mesh.num_dofs, dtype=torch.float64, device=cuda)
    values = torch.empty(sysm.nnz, dtype=torch.float64, device=cuda)
    trial = torch.empty_like(state)
    alpha_out = torch.empty_like(alpha)
    yielding = torch.empty((mesh.num_elements, 8), dtype=torch.uint8, device=cuda)
    summary = torch.empty(5, dtype=torch.float64, device=cuda)
    outer, inner = sysm.outer.clone(), sysm.inner.clone()

    for call in range(2):
        internal.fill_(np.nan)
        values.fill_(np.nan)
        system.evaluate_noalloc(mat, coords, conn, u, state, alpha, outer, inner, internal, values, trial,
                                alpha_out, yielding, summary)
        torch.cuda.synchronize()
        s = summary.cpu().numpy()
        assert s[3] == -1.0, f"call {call}: element {s[3]} failed (code {s[4]})"
        assert torch.linalg.norm(internal - ref_internal) <= TOL * ref_gross, call
        assert torch.linalg.norm(values - ref_values) <= TOL * torch.linalg.norm(ref_values), call
        assert abs(s[0] - ref_energy) <= TOL * abs(ref_energy), call
        assert abs(s[1] - ref_gross) <= TOL * ref_gross, call
        assert int(s[2]) == ref_yield, call
        assert torch.allclose(trial, ref_trial, rtol=TOL, atol=0.0), call
        assert torch.allclose(alpha_out, ref_modes, rtol=TOL, atol=1e-300), call


def test_noalloc_refuses_a_mesh_beyond_its_maximum(pkg, cuda):
    system = importlib.import_module("springback-precomp_b200.system")
    n = system.NOALLOC_MAX_ELEMENTS + 1
    mat = pkg.material.j2_steel()
    coords = torch.zeros((8 * n, 3), dtype=torch.float64, device=cuda)
    conn = torch.arange(8 * n, dtype=torch.int32, device=cuda).view(n, 8)
    buf = torch.zeros(24 * n, dtype=torch.float64, device=cuda)
    with pytest.raises(pkg.SbkError) as err:
        system.evaluate_noalloc(mat, coords, conn, buf, buf, None, conn.view(-1), conn.view(-1), buf, None, buf,
                                buf, torch.zeros(8 * n, dtype=torch.uint8, device=cuda),
                                torch.zeros(5, dtype=torch.float64, device=cuda))
    assert err.value.status == 6 and "2048" in str(err.value)


def _buffers(mesh, state, alpha, nnz, cuda):
    internal = torch.empty(mesh.num_dofs, dtype=torch.float64, device=cuda)
    values = torch.empty(nnz, dtype=torch.float64, device=cuda)
    trial = torch.empty_like(state)
    alpha_out = torch.empty_like(alpha)
    summary = torch.empty(5, dtype=torch.float64, device=cuda)
    return internal, values, trial, alpha_out, summary


def _dense(values, outer, inner, n):
    import scipy.sparse as sp
    return sp.csc_matrix((values, inner, outer), shape=(n, n)).toarray()


@pytest.mark.parametrize("bad", ["node_out_of_range", "inverted"])
def test_noalloc_leaves_a_failed_element_out_of_the_sums(pkg, cuda, bad):
    """A failed element is left out of every sum even though the shared
    scratch still holds an earlier call's values in its slots: a good call
    first fills the scratch, then element 5 fails - by naming a node out of
    range (SBK_EL_BAD_NODE before anything of it is read), or by listing its
    top face before its bottom face, which inverts it (SBK_EL_MESH_INVERTED,
    after its nodes were read) - and the sums must equal the allocating
    path's on the mesh without element 5. The caller's yield bytes of the
    failed element are garbage and must not count."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    system = importlib.import_module("springback-precomp_b200.system")
    mesh_mod = importlib.import_module("springback-precomp_b200.mesh")
    prob = wl.make_problem(6, 4, 1, seed=3, sample=24)
    mesh, mat = prob.mesh, prob.material
    sysm = pkg.NonlinearSystem(mesh, mat, kinematics="logarithmic")
    u = torch.tensor(prob.u, device=cuda)
    coords = torch.tensor(mesh.coords, device=cuda)
    conn = torch.tensor(mesh.connectivity, device=cuda)
    state = torch.tensor(prob.state, device=cuda)
    alpha = torch.tensor(prob.alpha, device=cuda)
    outer, inner = sysm.outer.clone(), sysm.inner.clone()
    internal, values, trial, alpha_out, summary = _buffers(mesh, state, alpha, sysm.nnz, cuda)
    yielding = torch.zeros((mesh.num_elements, 8), dtype=torch.uint8, device=cuda)
    system.evaluate_noalloc(mat, coords, conn, u, state, alpha, outer, inner, internal, values, trial, alpha_out,
                            yielding, summary)
    torch.cuda.synchronize()
    assert summary[3].item() == -1.0

    if bad == "node_out_of_range":
        conn[5, 3] = mesh.num_nodes  # one past the last node
        expected_code = 9  # SBK_EL_BAD_NODE
    else:
        conn[5] = conn[5][[4, 5, 6, 7, 0, 1, 2, 3]]
        expected_code = 6  # SBK_EL_MESH_INVERTED
    yielding.fill_(1)  # what the caller's buffer held before: must not be counted for element 5
    system.evaluate_noalloc(mat, coords, conn, u, state, alpha, outer, inner, internal, values, trial, alpha_out,
                            yielding, summary)
    torch.cuda.synchronize()
    s = summary.cpu().numpy()
    assert s[3] == 5.0, s
    assert int(s[4]) == expected_code, s

    # The allocating path on the mesh without element 5.
    keep = np.array([e for e in range(mesh.num_elements) if e != 5])
    sub = mesh_mod.HexMesh(mesh.coords, np.ascontiguousarray(mesh.connectivity[keep]))
    ref = pkg.NonlinearSystem(sub, mat, kinematics="logarithmic")
    ref.set_committed(np.ascontiguousarray(prob.state[:, keep, :]))
    ref.set_internal(np.ascontiguousarray(prob.alpha[keep]))
    ev = ref.evaluate(u, 0.0, True)
    torch.cuda.synchronize()
    tol = 1e-11
    assert abs(s[0] - ev.energy) <= tol * abs(ev.energy), (s[0], ev.energy)
    assert abs(s[1] - ev.gross) <= tol * ev.gross, (s[1], ev.gross)
    assert int(s[2]) == ev.yielding_points + 0, (s[2], ev.yielding_points)
    assert torch.linalg.norm(internal - ev.internal) <= tol * ev.gross
    n = mesh.num_dofs
    got = _dense(values.cpu().numpy(), outer.cpu().numpy(), inner.cpu().numpy(), n)
    want = _dense(ev.tangent.cpu().numpy(), ref.outer.cpu().numpy(), ref.inner.cpu().numpy(), n)
    assert np.linalg.norm(got - want) <= tol * np.linalg.norm(want)


def test_noalloc_adds_both_blocks_of_an_element_naming_a_node_twice(pkg, cuda):
    """An element whose connectivity names a node twice - a hexahedron with
    one vertical edge collapsed into its neighbour, a wedge that still
    evaluates - sends two of its blocks to one CSC entry and two of its
    force rows to one DOF: both contributions must count, as in the
    allocating path on the same connectivity."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    system = importlib.import_module("springback-precomp_b200.system")
    mesh_mod = importlib.import_module("springback-precomp_b200.mesh")
    prob = wl.make_problem(4, 2, 1, seed=7, sample=8)
    conn = prob.mesh.connectivity.copy()
    conn[0, 3] = conn[0, 2]  # corner 3 onto corner 2 (bottom face)
    conn[0, 7] = conn[0, 6]  # and its top twin
    mesh = mesh_mod.HexMesh(prob.mesh.coords, conn)
    mat = prob.material
    sysm = pkg.NonlinearSystem(mesh, mat, kinematics="logarithmic")
    sysm.set_committed(prob.state)
    sysm.set_internal(prob.alpha)
    u = torch.tensor(prob.u, device=cuda)
    ev = sysm.evaluate(u, 0.0, True)
    torch.cuda.synchronize()
    state = torch.tensor(prob.state, device=cuda)
    alpha = torch.tensor(prob.alpha, device=cuda)
    internal, values, trial, alpha_out, summary = _buffers(mesh, state, alpha, sysm.nnz, cuda)
    yielding = torch.zeros((mesh.num_elements, 8), dtype=torch.uint8, device=cuda)
    outer, inner = sysm.outer.clone(), sysm.inner.clone()
    system.evaluate_noalloc(mat, torch.tensor(mesh.coords, device=cuda), torch.tensor(conn, device=cuda), u, state,
                            alpha, outer, inner, internal, values, trial, alpha_out, yielding, summary)
    torch.cuda.synchronize()
    s = summary.cpu().numpy()
    assert s[3] == -1.0, s
    tol = 1e-11
    assert torch.linalg.norm(internal - ev.internal) <= tol * ev.gross
    assert torch.linalg.norm(values - ev.tangent) <= tol * torch.linalg.norm(ev.tangent)
    assert abs(s[1] - ev.gross) <= tol * ev.gross
