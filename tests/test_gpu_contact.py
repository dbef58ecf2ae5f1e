"""Penalty contact on the GPU (ToolContact through the C ABI) against the
oracle's restatement of src/fem/RigidTool.cpp: the candidate search of an
increment, the active set (bit-exact), the contact residual and node
blocks, the Coulomb friction with its transported history, the
anticipation of the semismooth step and the refusal of a node deep inside
a tool."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1.0e-12


def sheet(pkg, n=16, h=1.0e-3, nz=2, t=1.0e-3):
    return pkg.structured_hex_mesh(n, n, nz, n * h, n * h, t)


def top_slaves(mesh, young=70e9, penalty=10.0):
    """The top surface's nodes with their tributary areas and penalties
    (kappa = penalty E / sqrt(area), ToolContact's constructor,
    RigidTool.cpp:313-321)."""
    z = mesh.coords[:, 2]
    top = np.where(np.isclose(z, z.max()))[0]
    x, y = mesh.coords[top, 0], mesh.coords[top, 1]
    hx = np.diff(np.unique(x)).min()
    hy = np.diff(np.unique(y)).min()
    wx = np.where(np.isclose(x, x.min()) | np.isclose(x, x.max()), 0.5, 1.0)
    wy = np.where(np.isclose(y, y.min()) | np.isclose(y, y.max()), 0.5, 1.0)
    area = wx * wy * hx * hy
    kappa = penalty * young / np.sqrt(area)
    return top.astype(np.int32), area, kappa


def tools_for(mesh, shape, friction):
    nodes, area, kappa = top_slaves(mesh)
    L = mesh.coords[:, 0].max()
    ztop = mesh.coords[:, 2].max()
    if shape == "sphere":
        R = 3.0e-3
        pts = [(0.3 * L, 0.4 * L, ztop + R - 2.0e-4), (0.7 * L, 0.5 * L, ztop + R - 3.0e-4)]
        extra = dict(radius=R)
    elif shape == "cylinder":
        R = 2.0e-3
        pts = [(0.5 * L, 0.3 * L, ztop + R - 1.5e-4), (0.5 * L, 0.7 * L, ztop + R - 2.5e-4)]
        extra = dict(radius=R, axis=(1.0, 0.2, 0.0))
    else:
        pts = [(0.0, 0.0, ztop - 5.0e-5), (0.1 * L, 0.0, ztop - 8.0e-5)]
        extra = dict(normal=(0.1, 0.05, -1.0))
    return dict(shape=shape, times=[0.0, 1.0], points=pts, nodes=nodes, area=area, kappa=kappa,
                friction=friction, tangential_ratio=1.0, **extra)


def displacements(mesh, seed, scale=2.0e-5):
    rng = np.random.default_rng(seed)
    u = rng.uniform(-scale, scale, size=mesh.coords.shape)
    x, y = mesh.coords[:, 0], mesh.coords[:, 1]
    L = x.max()
    u[:, 2] -= 1.0e-4 * np.exp(-(((x - 0.5 * L) ** 2 + (y - 0.5 * L) ** 2) / (0.2 * L) ** 2))
    return u.reshape(-1)


def compare(ev, ref, ntools):
    assert ref["code"] == 0
    np.testing.assert_array_equal(ev.nodes.cpu().numpy(), ref["nodes"])  # the active set, in order
    r = ev.residual.cpu().numpy()
    assert np.abs(r - ref["residual"]).max() <= TOL * max(ref["gross"], 1e-300)
    if len(ref["nodes"]):
        b = ev.blocks.cpu().numpy()
        assert np.abs(b - ref["blocks"]).max() <= TOL * np.abs(ref["blocks"]).max()
    for k in range(ntools):
        np.testing.assert_array_equal(ev.tools[k][6:8], ref["tools"][k][6:8])  # active, slipping counts
        np.testing.assert_array_equal(ev.tools[k][0:3], ref["tools"][k][0:3])  # the tool's centre
        assert np.abs(ev.tools[k][3:6] - ref["tools"][k][3:6]).max() <= TOL * max(ref["gross"], 1e-300)
        assert ev.tools[k][8] == ref["tools"][k][8]
    assert abs(ev.gross - ref["gross"]) <= TOL * max(ref["gross"], 1e-300)
    assert abs(ev.round_off - ref["round_off"]) <= TOL * max(ref["round_off"], 1e-300)
    assert ev.symmetric == ref["symmetric"]


@pytest.mark.parametrize("shape", ["sphere", "cylinder", "plane"])
@pytest.mark.parametrize("friction", [0.0, 0.1])
@pytest.mark.parametrize("tangent", ["exact", "symmetric"])
def test_contact_increments(pkg, orc, cuda, shape, friction, tangent):
    mesh = sheet(pkg)
    tool = tools_for(mesh, shape, friction)
    ref = orc.Contact(mesh.coords, [tool], friction_tangent=tangent)
    gpu = pkg.ToolContact(mesh, [pkg.Tool(**tool)], friction_tangent=tangent)
    u0 = np.zeros(mesh.num_dofs)
    u1 = displacements(mesh, 1)
    u2 = u1 + displacements(mesh, 2, scale=5.0e-6)
    for (ua, ub, t0, t1) in [(u0, u1, 0.0, 0.5), (u1, u2, 0.5, 1.0)]:
        counts = ref.begin_increment(ua, t0, t1, [True], 5.0e-4)
        gpu.begin_increment(torch.tensor(ua, device=cuda), t0, t1, [True], 5.0e-4)
        r = ref.evaluate(ub, t1, True)
        ev = gpu.evaluate(torch.tensor(ub, device=cuda), t1, True)
        compare(ev, r, 1)
        assert counts[0] >= len(r["nodes"])
        # Anticipation of a correction that pushes the surface 0.2 mm down.
        du = np.zeros(mesh.num_dofs)
        du[2::3] = -2.0e-4
        res_ref, n_ref, b_ref = ref.anticipate(ub, du, t1, r["residual"])
        resid = ev.residual.clone()
        added, nodes, blocks = gpu.anticipate(torch.tensor(ub, device=cuda), torch.tensor(du, device=cuda), t1, resid)
        assert added == len(n_ref)
        np.testing.assert_array_equal(nodes.cpu().numpy()[len(r["nodes"]):], n_ref)
        assert np.abs(resid.cpu().numpy() - res_ref).max() <= TOL * max(r["gross"], np.abs(res_ref).max())
        if added:
            assert np.abs(blocks.cpu().numpy()[len(r["nodes"]):] - b_ref).max() <= TOL * np.abs(b_ref).max()
        ref.commit()
        gpu.commit()
        h_ref, h_gpu = ref.history(0), gpu.history(0)
        np.testing.assert_array_equal(h_gpu[:, 0], h_ref[:, 0])
        if len(h_ref):
            assert np.abs(h_gpu[:, 1:] - h_ref[:, 1:]).max() <= TOL * np.abs(h_ref[:, 1:]).max()
        if friction > 0:
            assert len(h_ref) == len(r["nodes"])


def test_two_tools_sum_in_tool_order(pkg, orc, cuda):
    mesh = sheet(pkg)
    tools = [tools_for(mesh, "sphere", 0.1), tools_for(mesh, "cylinder", 0.1)]
    ref = orc.Contact(mesh.coords, tools)
    gpu = pkg.ToolContact(mesh, [pkg.Tool(**t) for t in tools])
    u = displacements(mesh, 3)
    ref.begin_increment(np.zeros(mesh.num_dofs), 0.0, 0.6, [True, True], 1.0e-3)
    gpu.begin_increment(torch.zeros(mesh.num_dofs, dtype=torch.float64, device=cuda), 0.0, 0.6, [True, True], 1.0e-3)
    compare(gpu.evaluate(torch.tensor(u, device=cuda), 0.6, True), ref.evaluate(u, 0.6, True), 2)
    # An inactive tool takes no part.
    ref.begin_increment(u, 0.6, 0.8, [True, False], 1.0e-3)
    gpu.begin_increment(torch.tensor(u, device=cuda), 0.6, 0.8, [True, False], 1.0e-3)
    compare(gpu.evaluate(torch.tensor(u, device=cuda), 0.8, True), ref.evaluate(u, 0.8, True), 2)


def test_moved_beyond_margin_checks_every_slave(pkg, orc, cuda):
    """A node that moved farther than the margin makes the evaluation scan
    all slave nodes, not the candidates (RigidTool.cpp:417-433)."""
    mesh = sheet(pkg)
    tool = tools_for(mesh, "sphere", 0.0)
    ref = orc.Contact(mesh.coords, [tool])
    gpu = pkg.ToolContact(mesh, [pkg.Tool(**tool)])
    u = np.zeros(mesh.num_dofs)
    ref.begin_increment(u, 0.0, 0.0, [True], 1.0e-6)  # tiny margin: few candidates
    gpu.begin_increment(torch.tensor(u, device=cuda), 0.0, 0.0, [True], 1.0e-6)
    ub = displacements(mesh, 4)
    r = ref.evaluate(ub, 0.9, True)
    compare(gpu.evaluate(torch.tensor(ub, device=cuda), 0.9, True), r, 1)
    assert len(r["nodes"]) > 0


def test_node_through_the_tool_is_refused(pkg, orc, cuda):
    mesh = sheet(pkg)
    tool = tools_for(mesh, "sphere", 0.0)
    ref = orc.Contact(mesh.coords, [tool])
    gpu = pkg.ToolContact(mesh, [pkg.Tool(**tool)])
    u = np.zeros(mesh.num_dofs)
    # Pull the node nearest the sphere's start onto its centre.
    c = np.array(tool["points"][0])
    n = tool["nodes"][np.argmin(np.linalg.norm(mesh.coords[tool["nodes"]] - c, axis=1))]
    u[3 * n:3 * n + 3] = c - mesh.coords[n]
    assert ref.evaluate(u, 0.0, True)["code"] == -1
    with pytest.raises(pkg.SolverError):
        gpu.evaluate(torch.tensor(u, device=cuda), 0.0, True)


def test_slave_nodes_outside_the_mesh_are_refused(pkg, cuda):
    """A tool whose slave list names a node outside the mesh, or repeats
    one, is refused when the contact is made (the kernels index by it)."""
    mesh = sheet(pkg)
    for bad in ("out_of_range", "repeated"):
        tool = tools_for(mesh, "sphere", 0.0)
        nodes = np.array(tool["nodes"])
        if bad == "out_of_range":
            nodes[-1] = mesh.num_nodes
        else:
            nodes[1] = nodes[0]
        tool["nodes"] = nodes
        # (the Python wrapper already refuses a list that does not ascend)
        with pytest.raises((ValueError, pkg.SbkError)):
            pkg.ToolContact(mesh, [pkg.Tool(**tool)])


def test_contact_blocks_into_the_system_tangent(pkg, orc, cuda):
    """add_node_block of the contact blocks into the assembled tangent
    (src/fem/Forming.cpp:280-297) equals the oracle's."""
    mesh = sheet(pkg, n=8)
    mat = pkg.material.j2_steel()
    sysm = pkg.NonlinearSystem(mesh, mat, kinematics="logarithmic")
    u = displacements(mesh, 5, scale=1e-6)
    ev = sysm.evaluate(torch.tensor(u, device=cuda), 0.0, True)
    values = ev.tangent.clone()
    tool = tools_for(mesh, "sphere", 0.1)
    gpu = pkg.ToolContact(mesh, [pkg.Tool(**tool)])
    cev = gpu.evaluate(torch.tensor(u, device=cuda), 0.5, True)
    assert len(cev.nodes) > 0
    sysm.add_node_blocks(cev.nodes, cev.blocks)  # ev.tangent views the system's values
    pat = orc.pattern(mesh.num_nodes, mesh.connectivity)
    ref = orc.add_node_blocks(pat, values.cpu().numpy(), cev.nodes.cpu().numpy(), cev.blocks.cpu().numpy())
    assert np.array_equal(ev.tangent.cpu().numpy(), ref)


@pytest.mark.parametrize("margin", [1.0e-6, 5.0e-4, 3.0e-3])
def test_grid_search_finds_the_scans_candidates(pkg, orc, cuda, margin):
    """The uniform-grid hash of the slave nodes (spherical tools) gives the
    candidates of the reference's linear scan (RigidTool.cpp:345-393) - the
    same count, and then the same active set, residual and blocks - over
    increments whose swept segments are short, long, on cell boundaries and
    far from the sheet, on a 60 x 60 x 2 sheet (3,721 top nodes) with a
    deflected surface; and both equal the oracle's."""
    mesh = sheet(pkg, n=60, h=0.25e-3)
    nodes, area, kappa = top_slaves(mesh)
    L = mesh.coords[:, 0].max()
    ztop = mesh.coords[:, 2].max()
    R = 2.0e-3
    # Knots: a pass across the sheet, a jump along a cell boundary (x =
    # k (R + margin)), a long diagonal and a leg high above the sheet.
    h = R + margin
    pts = [(0.2 * L, 0.3 * L, ztop + R - 1.0e-4), (0.8 * L, 0.35 * L, ztop + R - 1.5e-4),
           (3 * h, 0.6 * L, ztop + R - 1.0e-4), (3 * h, 0.9 * L, ztop + R - 1.2e-4),
           (0.9 * L, 0.1 * L, ztop + R - 0.8e-4), (0.9 * L, 0.1 * L, ztop + 0.05)]
    times = [0.0, 0.2, 0.4, 0.6, 0.8, 1.0]
    tool = dict(shape="sphere", times=times, points=pts, nodes=nodes, area=area, kappa=kappa, friction=0.1,
                tangential_ratio=1.0, radius=R)
    ref = orc.Contact(mesh.coords, [tool])
    grid = pkg.ToolContact(mesh, [pkg.Tool(**tool)])
    scan = pkg.ToolContact(mesh, [pkg.Tool(**tool)])
    scan.set_search("scan")
    u = displacements(mesh, 7, scale=1.0e-5)
    steps = [(0.0, 0.1), (0.1, 0.3), (0.3, 0.45), (0.45, 0.7), (0.7, 0.9), (0.9, 1.0), (0.0, 1.0)]
    seen = 0
    for t0, t1 in steps:
        counts = ref.begin_increment(u, t0, t1, [True], margin)
        ud = torch.tensor(u, device=cuda)
        grid.begin_increment(ud, t0, t1, [True], margin)
        scan.begin_increment(ud, t0, t1, [True], margin)
        assert grid.candidates(0) == scan.candidates(0) == counts[0], (t0, t1)
        seen += counts[0]
        r = ref.evaluate(u, t1, True)
        eg = grid.evaluate(ud, t1, True)
        es = scan.evaluate(ud, t1, True)
        compare(eg, r, 1)
        assert torch.equal(eg.nodes, es.nodes) and torch.equal(eg.residual, es.residual)
        assert torch.equal(eg.blocks, es.blocks)
    assert seen > 0
