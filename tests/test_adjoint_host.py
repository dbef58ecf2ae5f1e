"""The host side of the release adjoint: the clamped cubic B-spline basis
(a partition of unity, non-negative, reproducing linear functions from
controls at the Greville abscissae, C1 across knots), the bicubic height
grid and its gradient (the stencil's transpose), and the 3-2-1 supports."""
from __future__ import annotations

import numpy as np
import pytest
import torch


@pytest.fixture(scope="module")
def adj(pkg):
    return pkg.adjoint


@pytest.mark.parametrize("n", [4, 5, 20])
def test_basis_is_a_nonnegative_partition_of_unity(adj, n):
    t = np.concatenate([np.linspace(0.0, 1.0, 1001), [0.0, 1.0, 1.0 / (n - 3)]])
    first, w = adj.cubic_bspline_basis(t, n)
    assert (w >= -1e-15).all()
    np.testing.assert_allclose(w.sum(axis=1), 1.0, rtol=0, atol=1e-14)
    assert first.min() == 0 and first.max() == n - 4


@pytest.mark.parametrize("n", [4, 7, 20])
def test_basis_reproduces_linear_functions(adj, n):
    """Controls at the Greville abscissae (the means of three consecutive
    inner knots) reproduce f(t) = t exactly."""
    knots = np.concatenate([np.zeros(3), np.linspace(0.0, 1.0, n - 2), np.ones(3)])
    greville = np.array([knots[i + 1:i + 4].mean() for i in range(n)])
    t = np.linspace(0.0, 1.0, 777)
    first, w = adj.cubic_bspline_basis(t, n)
    f = (w * greville[first[:, None] + np.arange(4)]).sum(axis=1)
    np.testing.assert_allclose(f, t, rtol=0, atol=1e-14)


def test_basis_is_continuous_with_its_slope_across_knots(adj):
    n = 9
    rng = np.random.default_rng(0)
    c = rng.standard_normal(n)
    for knot in np.linspace(0.0, 1.0, n - 2)[1:-1]:
        vals = []
        for t in (knot - 1e-7, knot, knot + 1e-7):
            first, w = adj.cubic_bspline_basis(np.array([t]), n)
            vals.append(float((w[0] * c[first[0] + np.arange(4)]).sum()))
        left, mid, right = vals
        assert abs(mid - 0.5 * (left + right)) < 1e-10
        assert abs((mid - left) - (right - mid)) < 1e-9


def test_bicubic_heights_and_their_gradient(pkg):
    grid = pkg.BicubicHeights(0.0, 2.0, -1.0, 1.0, n=6)
    rng = np.random.default_rng(1)
    xy = np.column_stack([rng.uniform(0.0, 2.0, 50), rng.uniform(-1.0, 1.0, 50)])
    st = grid.stencil(xy)
    # A constant control grid is a constant surface.
    np.testing.assert_allclose(grid.heights(torch.full((6, 6), 0.25, dtype=torch.float64), st).numpy(), 0.25,
                               rtol=0, atol=1e-15)
    # The heights are linear in p; their gradient is the stencil's transpose.
    p = torch.tensor(rng.standard_normal((6, 6)), requires_grad=True)
    g = torch.tensor(rng.standard_normal(50))
    (grid.heights(p, st) * g).sum().backward()
    dense = np.zeros((50, 36))
    idx, w = st
    for m in range(50):
        for k in range(16):
            dense[m, idx[m, k]] += w[m, k]
    np.testing.assert_allclose(p.grad.numpy().reshape(-1), dense.T @ g.numpy(), rtol=1e-13, atol=1e-14)
    assert grid.num_parameters == 36


def test_supports_hold_six_dofs(pkg):
    mesh = pkg.structured_hex_mesh(4, 3, 2, 0.4, 0.3, 0.02)
    free = pkg.supports_321(mesh)
    assert len(free) == mesh.num_dofs - 6
    held = np.setdiff1d(np.arange(mesh.num_dofs), free)
    nodes = held // 3
    corners = mesh.coords[np.unique(nodes)]
    assert np.allclose(corners[:, 2], 0.0)
    assert sorted(np.bincount(nodes)[np.unique(nodes)].tolist()) == [1, 2, 3]


def test_bad_inputs_are_refused(pkg, adj):
    with pytest.raises(ValueError):
        adj.cubic_bspline_basis(np.array([0.5]), 3)
    with pytest.raises(ValueError):
        pkg.BicubicHeights(1.0, 1.0, 0.0, 1.0)
    # A mesh with no node at a support corner (its corner element removed).
    mesh = pkg.structured_hex_mesh(3, 3, 1, 0.3, 0.3, 0.01)
    keep = np.ones(mesh.num_elements, dtype=bool)
    keep[0] = False
    conn = mesh.connectivity[keep]
    used = np.unique(conn)
    remap = -np.ones(mesh.num_nodes, dtype=np.int64)
    remap[used] = np.arange(len(used))
    holed = pkg.HexMesh(mesh.coords[used], remap[conn].astype(np.int32))
    with pytest.raises(ValueError):
        pkg.supports_321(holed)


def test_heights_clamp_outside_the_footprint(pkg):
    """Points outside the footprint take the edge's heights (the parameter
    is clamped), so a mesh overhanging the grid stays defined."""
    grid = pkg.BicubicHeights(0.0, 1.0, 0.0, 1.0, n=5)
    p = torch.tensor(np.random.default_rng(3).standard_normal((5, 5)))
    inside = grid.heights(p, grid.stencil(np.array([[0.0, 0.3], [1.0, 0.7]])))
    outside = grid.heights(p, grid.stencil(np.array([[-0.2, 0.3], [1.4, 0.7]])))
    np.testing.assert_array_equal(inside.numpy(), outside.numpy())
