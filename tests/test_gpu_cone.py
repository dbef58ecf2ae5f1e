"""The fine-mesh configuration's workload at a small size: a truncated cone
(18 mm footprint, 3 mm deep, 50 degree wall) formed half way in a 4-layer
1 mm sheet, with the forming ball on its top face and the support ball under
its bottom face (double-sided forming). The evaluation of the IM Hex8 loop
on the GPU against the oracle on the same committed history, and both
tools' contact - the active sets bit-exact, in order - against the
oracle's, with the candidates found by the uniform-grid hash and by the
scan."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

from conftest import device_to_oracle

pytestmark = pytest.mark.gpu

TOL = 1.0e-11


@pytest.fixture(scope="module")
def cone(pkg, cuda):
    wl = importlib.import_module("springback-precomp_b200.workload")
    return wl.make_cone_problem(32, 4, device=cuda)


def test_cone_evaluation_matches_the_oracle(pkg, orc, cuda, cone):
    sysm, prob = cone
    mesh, mat = prob.mesh, prob.material
    ev = sysm.evaluate(torch.tensor(prob.u, device=cuda), 0.0, True)
    committed = device_to_oracle(sysm.committed_all(), mat.kinematic_terms)
    ref = orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, prob.u, committed, sysm.internal_all(),
                              kinematics="logarithmic")
    assert ref["code"] == 0
    v = ev.tangent.cpu().numpy()
    assert np.linalg.norm(v - ref["values"]) <= TOL * np.linalg.norm(ref["values"])
    assert np.abs(ev.internal.cpu().numpy() - ref["internal"]).max() <= TOL * ref["gross"]
    assert ev.yielding_points == ref["yielding_points"]
    assert 0.05 < ev.yielding_points / (8.0 * mesh.num_elements) < 0.95


@pytest.mark.parametrize("search", ["grid", "scan"])
def test_two_tool_contact_matches_the_oracle(pkg, orc, cuda, cone, search):
    sysm, prob = cone
    mesh = prob.mesh
    ref = orc.Contact(mesh.coords, prob.tools)
    gpu = pkg.ToolContact(mesh, [pkg.Tool(**t) for t in prob.tools])
    gpu.set_search(search)
    margin = 2.0e-3
    counts = ref.begin_increment(prob.u0, 0.0, 1.0, [True, True], margin)
    gpu.begin_increment(torch.tensor(prob.u0, device=cuda), 0.0, 1.0, [True, True], margin)
    assert [gpu.candidates(k) for k in range(2)] == list(counts)
    r = ref.evaluate(prob.u, 1.0, True)
    ev = gpu.evaluate(torch.tensor(prob.u, device=cuda), 1.0, True)
    assert r["code"] == 0
    np.testing.assert_array_equal(ev.nodes.cpu().numpy(), r["nodes"])
    assert len(r["nodes"]) > 0
    for k in range(2):
        np.testing.assert_array_equal(ev.tools[k][6:8], r["tools"][k][6:8])
        assert ev.tools[k][6] > 0, f"tool {k} not in contact"
    assert np.abs(ev.residual.cpu().numpy() - r["residual"]).max() <= 1e-12 * r["gross"]
    assert np.abs(ev.blocks.cpu().numpy() - r["blocks"]).max() <= 1e-12 * np.abs(r["blocks"]).max()
    gpu.close()


def test_cone_release_in_increments_is_the_oracles(pkg, orc, cuda):
    """The frozen release of a 16 x 16 x 4 cone part whose history was
    loaded by imposed displacements: its start is far from equilibrium, and
    full Newton steps from it reach another equilibrium of the supported
    sheet or invert elements, so the release takes the start's imbalance off
    in 8 increments. The device's u* against the oracle's release with the
    same increments (scipy solves of the oracle's tangents) within 1e-9; the
    springback is a fraction of a millimetre."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    sysm, prob = wl.make_cone_problem(16, 4, device=cuda)
    mesh, mat = prob.mesh, prob.material
    committed_dev, modes = sysm.committed_all(), sysm.internal_all()
    sysm.close()
    free = pkg.supports_321(mesh)
    release = pkg.Release(mesh, mat, committed_dev, modes, free, increments=8)
    x0 = torch.tensor(mesh.coords, device=cuda)
    u_star = release.solve(x0, torch.tensor(prob.u0, device=cuda)).cpu().numpy()
    release.close()
    m = mat.as_dict()
    m["yield_stress"] = 1e300  # frozen
    committed = device_to_oracle(committed_dev, mat.kinematic_terms)
    u_ref, iterations = orc.release_solve(m, mesh.coords, mesh.connectivity, committed, modes, free, prob.u0,
                                          increments=8)
    rel = np.linalg.norm(u_star - u_ref) / np.linalg.norm(u_ref)
    spring = np.abs(u_ref - prob.u0).max()
    print(f"cone release: {iterations} Newton iterations, springback {spring * 1e3:.3f} mm, device against "
          f"oracle {rel:.2e}")
    assert rel <= 1e-9
    assert 0.1e-3 < spring < 2.0e-3
