"""The adjoint shape gradient of a springback measure, end to end on the
device, against central differences of the released equilibrium.

A 12 x 6 x 2 sheet carries the committed plastic history of a bending
load (Hill48 + Chaboche). Released onto 3-2-1 supports (the support DOFs
held where the loaded sheet left them) it springs back to u*(X), the root
of the free rows of f_int(u, X) that the device Newton iteration finds
(PartitionedFactor factorisations of the device tangent). The measure is
J = 1/2 sum u_z^2 over the top face. Its gradient with respect to the
nodal reference coordinates is

    dJ/dX = -lambda^T d f_int / d X,    K_ff^T lambda_f = dJ/du_f,

the adjoint solved with the same factorisation (transposed) and the shape
derivative taken by sbk_system_vjp_x. Two cases: the committed plastic
state frozen (the release elastic; symmetric tangent, the Cholesky) and
the release as one increment with the returns (the consistent tangent,
the dense LU solved transposed). Directional derivatives along seeded
random perturbations of every node and along the coordinate of the
largest gradient entry agree with central differences of J to 1e-6
relative."""
from __future__ import annotations

import dataclasses
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GRADIENT_TOL = 1e-6


@pytest.fixture(scope="module")
def sheet(pkg, cuda):
    wl = importlib.import_module("springback-precomp_b200.workload")
    return wl.make_problem(12, 6, 2, seed=11, sample=144)


def supports(mesh):
    """3-2-1: the corner at the origin in x, y and z, the corner along x in
    y and z, the corner along y in z."""
    x = mesh.coords
    lo, hi = x.min(axis=0), x.max(axis=0)
    a = int(np.flatnonzero(np.all(np.isclose(x, lo), axis=1))[0])
    b = int(np.flatnonzero(np.all(np.isclose(x, [hi[0], lo[1], lo[2]]), axis=1))[0])
    c = int(np.flatnonzero(np.all(np.isclose(x, [lo[0], hi[1], lo[2]]), axis=1))[0])
    held = np.zeros(mesh.num_dofs, dtype=bool)
    held[[3 * a, 3 * a + 1, 3 * a + 2, 3 * b + 1, 3 * b + 2, 3 * c + 2]] = True
    return np.flatnonzero(~held).astype(np.int32)


class Release:
    """The released equilibrium of one reference geometry X."""

    def __init__(self, pkg, mesh, material, state, alpha, free, top_z, cuda):
        self.pkg, self.free, self.top_z, self.cuda = pkg, free, top_z, cuda
        self.system = pkg.NonlinearSystem(mesh, material, kinematics="logarithmic")
        self.system.set_committed(state)
        self.system.set_internal(alpha)
        self.part = pkg.PartitionedFactor.for_system(self.system, free)

    def solve(self, u0: torch.Tensor) -> torch.Tensor:
        """Newton from u0 (its support DOFs kept), a step halved while an
        element refuses it, until a full step falls below 1e-10 of u, and
        one step more: the root to rounding."""
        u = u0.clone()
        ev = self.system.evaluate(u, 0.0, True)
        r = self.part.restrict(ev.internal)
        r0, converged = float(torch.linalg.norm(r)), False
        for _ in range(40):
            self.part.factorize(ev.tangent, self.system.symmetric())
            du = self.part.solve(-r)
            step = 1.0
            while True:
                trial = self.part.add_to(u.clone(), du, step)
                try:
                    ev = self.system.evaluate(trial, 0.0, True)
                    break
                except self.pkg.SolverError:
                    step *= 0.5
                    assert step > 1e-3
            u = trial
            r = self.part.restrict(ev.internal)
            if converged:
                break
            converged = step == 1.0 and float(torch.linalg.norm(du)) <= 1e-10 * float(torch.linalg.norm(u))
        assert converged
        floor = self.system.stiffness_gross(u, torch.tensor(self.free))
        assert float(torch.linalg.norm(r)) <= max(1e-9 * r0, 1e-12 * floor)
        self.tangent = ev.tangent
        self.yielding = ev.yielding_points
        return u

    def measure(self, u: torch.Tensor) -> float:
        return 0.5 * float((u[self.top_z] ** 2).sum())

    def gradient(self, u: torch.Tensor, frozen: bool) -> np.ndarray:
        c = torch.zeros_like(u)
        c[self.top_z] = u[self.top_z]
        self.part.factorize(self.tangent, self.system.symmetric())
        lam_f = self.part.solve(self.part.restrict(c), transpose=True)
        lam = self.part.add_to(torch.zeros_like(u), lam_f, 1.0)
        return -self.system.vjp_x(u, lam, frozen=frozen).cpu().numpy()


@pytest.mark.parametrize("frozen", [True, False])
def test_adjoint_shape_gradient_matches_central_differences(pkg, sheet, cuda, frozen):
    mesh, state, alpha = sheet.mesh, sheet.state, sheet.alpha
    material = dataclasses.replace(sheet.material, yield_stress=1e30) if frozen else sheet.material
    free = supports(mesh)
    top = np.flatnonzero(np.isclose(mesh.coords[:, 2], mesh.coords[:, 2].max()))
    top_z = torch.tensor(3 * top + 2, device=cuda)
    elastic = Release(pkg, mesh, dataclasses.replace(sheet.material, yield_stress=1e30), state, alpha, free, top_z,
                      cuda)
    u_star = elastic.solve(torch.tensor(sheet.u, device=cuda))
    base = elastic
    if not frozen:
        base = Release(pkg, mesh, material, state, alpha, free, top_z, cuda)
        u_star = base.solve(u_star)
    print(f"frozen={frozen} yielding points at the release {base.yielding}")
    assert frozen or base.yielding > 0
    grad = base.gradient(u_star, frozen)
    assert np.isfinite(grad).all() and np.abs(grad).max() > 0.0

    cell = float(np.min(np.ptp(mesh.coords, axis=0) / np.array([12, 6, 2])))
    rng = np.random.default_rng(21)
    directions = [rng.uniform(-1.0, 1.0, size=mesh.coords.shape), np.zeros(mesh.coords.shape)]
    directions[1].reshape(-1)[int(np.abs(grad).argmax())] = 1.0
    for d in directions:
        h = 1e-4 * cell
        jd = []
        for sign in (1.0, -1.0):
            moved = pkg.HexMesh(mesh.coords + sign * h * d, mesh.connectivity)
            rel = Release(pkg, moved, material, state, alpha, free, top_z, cuda)
            jd.append(rel.measure(rel.solve(u_star)))
        fd = (jd[0] - jd[1]) / (2.0 * h)
        adj = float(grad @ d.reshape(-1))
        print(f"frozen={frozen} adjoint {adj:.12e} central difference {fd:.12e} "
              f"relative {abs(adj - fd) / abs(fd):.2e}")
        assert abs(adj - fd) <= GRADIENT_TOL * abs(fd), (adj, fd, abs(adj - fd) / abs(fd))


def test_frozen_system_is_the_elastic_release(pkg, sheet, cuda):
    """sbk_system_set_frozen: the committed plastic state taken as it is -
    the response of the same history under a yield stress no point reaches,
    with no yielding point and a symmetric tangent (the Cholesky)."""
    mesh = sheet.mesh
    u = torch.tensor(sheet.u, device=cuda)
    frozen = pkg.NonlinearSystem(mesh, sheet.material)
    elastic = pkg.NonlinearSystem(mesh, dataclasses.replace(sheet.material, yield_stress=1e30))
    for s in (frozen, elastic):
        s.set_committed(sheet.state)
        s.set_internal(sheet.alpha)
    assert frozen.plastic() and not frozen.symmetric()
    frozen.set_frozen(True)
    assert frozen.symmetric()
    a, b = frozen.evaluate(u), elastic.evaluate(u)
    assert a.yielding_points == 0 and b.yielding_points == 0
    for x, y in ((a.internal, b.internal), (a.tangent, b.tangent)):
        assert float(torch.linalg.norm(x - y)) <= 1e-12 * float(torch.linalg.norm(y))
    frozen.set_frozen(False)
    assert frozen.evaluate(u).yielding_points > 0 and not frozen.symmetric()


def test_moved_nodes_are_a_new_mesh(pkg, sheet, cuda):
    """sbk_system_set_coordinates: a system whose nodes moved evaluates as a
    system built on the moved mesh, to the bit."""
    mesh = sheet.mesh
    moved = mesh.coords + 1e-6 * np.random.default_rng(3).standard_normal(mesh.coords.shape)
    a = pkg.NonlinearSystem(mesh, sheet.material)
    b = pkg.NonlinearSystem(pkg.HexMesh(moved, mesh.connectivity), sheet.material)
    for s in (a, b):
        s.set_committed(sheet.state)
        s.set_internal(sheet.alpha)
    a.set_coordinates(torch.tensor(moved, device=cuda))
    u = torch.tensor(sheet.u, device=cuda)
    ea, eb = a.evaluate(u), b.evaluate(u)
    assert torch.equal(ea.internal, eb.internal) and torch.equal(ea.tangent, eb.tangent)


@pytest.fixture(scope="module")
def part(pkg, cuda):
    wl = importlib.import_module("springback-precomp_b200.workload")
    return wl.make_problem(32, 32, 2, seed=5, sample=512)


def test_height_gradient_matches_central_differences(pkg, part, cuda):
    """The commanded-shape gradient through torch.autograd: a 32 x 32 x 2
    part, its end-of-forming history frozen, released onto 3-2-1 supports;
    J = the RMS vertical deviation of its top face from the formed heights
    (the springback); p the 20 x 20 bicubic grid of height offsets over the
    footprint. dJ/dp from backward() (one adjoint solve and one shape
    derivative) against central differences of J with h = 1e-6 mm along 32
    seeded random directions: within 1e-6 relative each."""
    mesh = part.mesh
    x0 = torch.tensor(mesh.coords, device=cuda)
    lo, hi = mesh.coords.min(axis=0), mesh.coords.max(axis=0)
    grid = pkg.BicubicHeights(lo[0], hi[0], lo[1], hi[1], n=20)
    stencil = grid.stencil(mesh.coords[:, :2], device=cuda)
    top = torch.tensor(np.flatnonzero(np.isclose(mesh.coords[:, 2], hi[2])), device=cuda)
    u_formed = torch.tensor(part.u, device=cuda)
    target = x0[top, 2] + u_formed.reshape(-1, 3)[top, 2]
    release = pkg.Release(mesh, part.material, part.state, part.alpha, pkg.supports_321(mesh))

    def coords_of(p):
        lift = torch.zeros_like(x0)
        lift[:, 2] = grid.heights(p, stencil)
        return x0 + lift

    p = torch.zeros((20, 20), dtype=torch.float64, device=cuda, requires_grad=True)
    coords = coords_of(p)
    u_star = pkg.released(coords, release, u_formed)
    j = pkg.springback_rms(coords, u_star, top, target)
    j.backward()
    grad = p.grad.detach().cpu().numpy()
    assert float(j.detach()) > 0.0 and np.abs(grad).max() > 0.0
    u_star = u_star.detach()

    h = 1e-9  # m: 1e-6 mm
    rng = np.random.default_rng(32)
    worst = 0.0
    for _ in range(32):
        d = rng.uniform(-1.0, 1.0, size=(20, 20))
        jd = []
        for sign in (1.0, -1.0):
            c = coords_of(torch.tensor(sign * h * d, device=cuda))
            jd.append(float(pkg.springback_rms(c, release.solve(c, u_star), top, target)))
        fd = (jd[0] - jd[1]) / (2.0 * h)
        adj = float((grad * d).sum())
        worst = max(worst, abs(adj - fd) / abs(fd))
        assert abs(adj - fd) <= GRADIENT_TOL * abs(fd), (adj, fd, abs(adj - fd) / abs(fd))
    print(f"heights: J {float(j.detach()):.6e} m, worst relative difference over 32 directions {worst:.2e}")


def test_height_gradient_is_the_oracles(pkg, orc, part, cuda):
    """The device's release and its 400-height gradient against the same
    built from the oracle's CPU element routines (the oracle's release
    Newton with scipy solves, the oracle's adjoint and per-element shape
    derivative): u* within 1e-10 and dJ/dp within 1e-8 relative."""
    import test_oracle_adjoint as toa

    j_ref, grad_ref, u_ref, _ = toa.oracle_gradient(pkg, orc, part)
    mesh = part.mesh
    x0 = torch.tensor(mesh.coords, device=cuda)
    lo, hi = mesh.coords.min(axis=0), mesh.coords.max(axis=0)
    grid = pkg.BicubicHeights(lo[0], hi[0], lo[1], hi[1], n=20)
    stencil = grid.stencil(mesh.coords[:, :2], device=cuda)
    top = torch.tensor(np.flatnonzero(np.isclose(mesh.coords[:, 2], hi[2])), device=cuda)
    u_formed = torch.tensor(part.u, device=cuda)
    target = x0[top, 2] + u_formed.reshape(-1, 3)[top, 2]
    release = pkg.Release(mesh, part.material, part.state, part.alpha, pkg.supports_321(mesh))
    p = torch.zeros((20, 20), dtype=torch.float64, device=cuda, requires_grad=True)
    lift = torch.zeros_like(x0)
    lift[:, 2] = grid.heights(p, stencil)
    coords = x0 + lift
    u_star = pkg.released(coords, release, u_formed)
    j = pkg.springback_rms(coords, u_star, top, target)
    j.backward()
    u_np, grad = u_star.detach().cpu().numpy(), p.grad.cpu().numpy()
    assert np.linalg.norm(u_np - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
    assert abs(float(j.detach()) - j_ref) <= 1e-10 * j_ref
    rel = np.linalg.norm(grad - grad_ref) / np.linalg.norm(grad_ref)
    print(f"heights: device against oracle gradient {rel:.2e}")
    assert rel <= 1e-8


def test_adjoint_reuses_the_factorisation_at_the_root(pkg, part, cuda):
    """The adjoint after a release reuses the factorisation its last Newton
    evaluate left at u*: the same gradient as one that re-evaluates and
    factorises again, one factorisation fewer; a u it was not factorised at
    is factorised anew."""
    mesh = part.mesh
    x0 = torch.tensor(mesh.coords, device=cuda)
    release = pkg.Release(mesh, part.material, part.state, part.alpha, pkg.supports_321(mesh))
    u_star = release.solve(x0, torch.tensor(part.u, device=cuda))
    c = torch.tensor(np.random.default_rng(2).standard_normal(mesh.num_dofs), device=cuda)
    n0 = release.factorizations
    warm = release.adjoint(x0, u_star, c)
    assert release.factorizations == n0
    release.forget_factorization()
    cold = release.adjoint(x0, u_star, c)
    assert release.factorizations == n0 + 1
    assert float(torch.linalg.norm(warm - cold)) <= 1e-12 * float(torch.linalg.norm(cold))
    other = release.adjoint(x0, u_star * (1.0 + 1e-9), c)
    assert release.factorizations == n0 + 2 and torch.isfinite(other).all()


def test_compensation_reduces_the_springback(pkg, part, cuda):
    """Adjoint-driven compensation on the 32 x 32 x 2 part: L-BFGS over the
    20 x 20 control heights, every step one release solve and one adjoint,
    pre-distorts the part so that its released top face comes back towards
    the formed heights - the RMS deviation falls to at most half its
    uncompensated value within 10 iterations and the best point found is the
    one returned."""
    mesh = part.mesh
    x0 = torch.tensor(mesh.coords, device=cuda)
    lo, hi = mesh.coords.min(axis=0), mesh.coords.max(axis=0)
    grid = pkg.BicubicHeights(lo[0], hi[0], lo[1], hi[1], n=20)
    stencil = grid.stencil(mesh.coords[:, :2], device=cuda)
    top = torch.tensor(np.flatnonzero(np.isclose(mesh.coords[:, 2], hi[2])), device=cuda)
    u_formed = torch.tensor(part.u, device=cuda)
    target = x0[top, 2] + u_formed.reshape(-1, 3)[top, 2]
    release = pkg.Release(mesh, part.material, part.state, part.alpha, pkg.supports_321(mesh))
    p, history, solves = pkg.compensate(release, grid, stencil, x0, top, target, u_formed, iterations=10)
    print(f"compensation: RMS {history[0]:.4e} m -> {min(history):.4e} m in {solves} release solves; "
          f"history {[f'{h:.3e}' for h in history]}")
    assert min(history) <= 0.5 * history[0]
    lift = torch.zeros_like(x0)
    lift[:, 2] = grid.heights(p, stencil)
    with torch.no_grad():
        j = float(pkg.springback_rms(x0 + lift, release.solve(x0 + lift, u_formed), top, target))
    assert j <= 0.5 * history[0]
