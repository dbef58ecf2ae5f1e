"""The standard Hex8 on the GPU (sbk_system_set_element, the standard
element of src/fem/Elastoplastic.cpp:226-340 with or without mean
dilatation) against the oracle's restatement of it, through the system:
the assembled tangent and f_int within 1e-11 (relative Frobenius / of the
gross norm), the yield count, every point's accumulated plastic strain and
the energy, for every kinematics, on a 24 x 12 x 2 sheet with a committed
plastic history (Hill48 + Chaboche, non-symmetric, and J2, symmetric)."""
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


@pytest.mark.parametrize("law", ["hill48+chaboche", "j2"])
@pytest.mark.parametrize("kin", ["small", "finite", "logarithmic"])
@pytest.mark.parametrize("mean_dilatation", ["auto", "none"])
def test_standard_element_matches_oracle(pkg, orc, problem, cuda, law, kin, mean_dilatation):
    mesh = problem.mesh
    mat = problem.material if law == "hill48+chaboche" else pkg.material.aluminium_swift()
    state = problem.state if law == "hill48+chaboche" else np.zeros((mat.state_fields,) + problem.state.shape[1:])
    scale = 1.0 if kin != "small" else 0.2
    u_host = scale * problem.u
    s = pkg.NonlinearSystem(mesh, mat, kinematics=kin, element="standard", mean_dilatation=mean_dilatation)
    assert s.averaged == (mean_dilatation == "auto")
    s.set_committed(state)
    ev = s.evaluate(torch.tensor(u_host, device=cuda), 0.0, True)
    nt = mat.kinematic_terms
    with orc.element(True, mean_dilatation == "auto"):
        ref = orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, u_host,
                                  device_to_oracle(state, nt), None, kinematics=kin)
    assert ref["code"] == 0
    assert ref["yielding_points"] > 0
    assert ev.yielding_points == ref["yielding_points"]
    f = ev.internal.cpu().numpy()
    assert np.abs(f - ref["internal"]).max() <= 1e-11 * ref["gross"]
    v = ev.tangent.cpu().numpy()
    assert np.linalg.norm(v - ref["values"]) <= 1e-11 * np.linalg.norm(ref["values"])
    assert abs(ev.energy - ref["energy"]) <= 1e-11 * abs(ref["energy"])
    st = device_to_oracle(s.trial_states(), nt)
    eq = ref["states"][..., 36]
    assert np.abs(st[..., 36] - eq).max() <= 1e-10 * max(eq.max(), 1e-12)
    assert int(s.trial_yield().sum()) == ref["yielding_points"]


def test_incompatible_modes_refuse_mean_dilatation_all(pkg, problem):
    with pytest.raises(pkg.SbkError):
        pkg.NonlinearSystem(problem.mesh, problem.material, element="incompatible_modes", mean_dilatation="all")
    s = pkg.NonlinearSystem(problem.mesh, problem.material)
    assert s.element == "incompatible_modes" and not s.averaged


@pytest.mark.parametrize("kin", ["small", "finite", "logarithmic"])
@pytest.mark.parametrize("mean_dilatation", ["auto", "none"])
def test_standard_stress_recovery_matches_oracle(pkg, orc, problem, cuda, kin, mean_dilatation):
    """Step-end stress recovery of the standard Hex8 (elastoplastic_stress,
    Elastoplastic.cpp:342-430) after a commit: the averages at the
    committed points, with mean dilatation at the averaged strain, against
    the oracle's restatement within 1e-11 of each field's scale."""
    mesh, mat = problem.mesh, problem.material
    s = pkg.NonlinearSystem(mesh, mat, kinematics=kin, element="standard", mean_dilatation=mean_dilatation)
    s.set_committed(problem.state)
    u = torch.tensor(problem.u if kin != "small" else 0.2 * problem.u, device=cuda)
    s.evaluate(u, 0.0, False)
    s.commit()
    st, _ = s.committed_views()
    committed = device_to_oracle(st.cpu().numpy(), mat.kinematic_terms)
    got = s.stress(u)
    with orc.element(True, mean_dilatation == "auto"):
        ref, status = orc.element_stress(mat.as_dict(), mesh.element_coordinates(), mesh.gather(u.cpu().numpy()),
                                         committed, None, kinematics=kin)
    assert (status == 0).all()
    packed = torch.cat([got.cauchy, got.piola_kirchhoff, got.von_mises[:, None], got.max_plastic_strain[:, None],
                        got.max_strain[:, None], got.min_jacobian[:, None], got.kirchhoff, got.log_strain],
                       dim=1).cpu().numpy()
    for lo, hi in [(0, 6), (6, 12), (12, 13), (13, 14), (14, 15), (15, 16), (16, 22), (22, 28)]:
        scale = max(np.abs(ref[:, lo:hi]).max(), 1e-300)
        assert np.abs(packed[:, lo:hi] - ref[:, lo:hi]).max() <= 1e-11 * scale, (lo, hi)
    assert ref[:, 13].max() > 0.0
