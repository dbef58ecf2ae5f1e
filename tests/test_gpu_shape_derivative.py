"""The shape derivative on the GPU (sbk_system_vjp_x: lambda^T d f_int / d X
for the IM Hex8, the modes through their local equilibrium) against the
oracle's restatement, element by element and assembled: within 1e-10 of
its largest entry, on a 24 x 12 x 2 sheet with a committed plastic history
(Hill48 + Chaboche), frozen (the committed plastic state as it is) and with
the returns, under finite and logarithmic strain. The oracle's own
derivative is pinned against central differences on the CPU."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

from conftest import device_to_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(pkg, cuda):
    wl = importlib.import_module("springback-precomp_b200.workload")
    return wl.make_problem(24, 12, 2, seed=11, sample=576)


@pytest.mark.parametrize("kin", ["logarithmic", "finite"])
@pytest.mark.parametrize("frozen", [True, False])
def test_shape_derivative_matches_oracle(pkg, orc, problem, cuda, kin, frozen):
    mesh, mat = problem.mesh, problem.material
    u_host = problem.u if kin == "logarithmic" else 0.5 * problem.u
    s = pkg.NonlinearSystem(mesh, mat, kinematics=kin)
    s.set_committed(problem.state)
    s.set_internal(problem.alpha)
    lam = np.random.default_rng(5).standard_normal(mesh.num_dofs)
    gx = s.vjp_x(torch.tensor(u_host, device=cuda), torch.tensor(lam, device=cuda), frozen=frozen).cpu().numpy()
    m = mat.as_dict()
    if frozen:
        m["yield_stress"] = 1e300
    conn = mesh.connectivity
    per, st = orc.vjp_x(m, mesh.element_coordinates(), mesh.gather(u_host), lam[(3 * conn[:, :, None] +
                                                                                 np.arange(3)).reshape(-1, 24)],
                        device_to_oracle(problem.state, mat.kinematic_terms), problem.alpha, kinematics=kin)
    assert (st == 0).all()
    ref = np.zeros(mesh.num_dofs)
    for e in range(mesh.num_elements):
        for a in range(8):
            ref[3 * conn[e, a]:3 * conn[e, a] + 3] += per[e, 3 * a:3 * a + 3]
    assert np.abs(gx - ref).max() <= 1e-10 * np.abs(ref).max(), np.abs(gx - ref).max() / np.abs(ref).max()


def test_shape_derivative_of_a_rigid_translation_is_zero(pkg, problem, cuda):
    """Translating the whole reference body leaves f_int unchanged, so the
    shape derivative summed over the nodes vanishes component by component."""
    mesh, mat = problem.mesh, problem.material
    s = pkg.NonlinearSystem(mesh, mat)
    s.set_committed(problem.state)
    s.set_internal(problem.alpha)
    lam = torch.tensor(np.random.default_rng(6).standard_normal(mesh.num_dofs), device=cuda)
    gx = s.vjp_x(torch.tensor(problem.u, device=cuda), lam, frozen=True).cpu().numpy().reshape(-1, 3)
    assert np.abs(gx.sum(axis=0)).max() <= 1e-9 * np.abs(gx).sum(axis=0).max()
