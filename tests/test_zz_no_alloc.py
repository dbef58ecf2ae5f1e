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


def test_noalloc_fails_an_element_naming_a_node_out_of_range(pkg, cuda):
    """The caller's device connectivity is not checked on the host: an
    element naming a node out of range fails (SBK_EL_BAD_NODE) before
    anything of it is read, and the sums leave it out."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    system = importlib.import_module("springback-precomp_b200.system")
    prob = wl.make_problem(6, 4, 1, seed=3, sample=24)
    mesh, mat = prob.mesh, prob.material
    sysm = pkg.NonlinearSystem(mesh, mat, kinematics="logarithmic")
    u = torch.tensor(prob.u, device=cuda)
    coords = torch.tensor(mesh.coords, device=cuda)
    conn = torch.tensor(mesh.connectivity, device=cuda)
    conn[5, 3] = mesh.num_nodes  # one past the last node
    state = torch.tensor(prob.state, device=cuda)
    alpha = torch.tensor(prob.alpha, device=cuda)
    internal = torch.empty(mesh.num_dofs, dtype=torch.float64, device=cuda)
    values = torch.empty(sysm.nnz, dtype=torch.float64, device=cuda)
    trial = torch.empty_like(state)
    alpha_out = torch.empty_like(alpha)
    yielding = torch.zeros((mesh.num_elements, 8), dtype=torch.uint8, device=cuda)
    summary = torch.empty(5, dtype=torch.float64, device=cuda)
    system.evaluate_noalloc(mat, coords, conn, u, state, alpha, sysm.outer.clone(), sysm.inner.clone(), internal,
                            values, trial, alpha_out, yielding, summary)
    torch.cuda.synchronize()
    s = summary.cpu().numpy()
    assert s[3] == 5.0 and int(s[4]) == 9, s
