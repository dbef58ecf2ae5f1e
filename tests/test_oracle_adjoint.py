"""The oracle's release adjoint on the CPU, pinned by central differences:
an 8 x 8 x 2 part whose committed Hill48 + Chaboche history the oracle
loaded, frozen and released onto 3-2-1 supports; J = the RMS springback of
its top face; dJ/dp for the 20 x 20 bicubic grid of commanded heights from
the oracle's adjoint (scipy solve of the transposed block, the oracle's
per-element shape derivative) agrees with central differences of the
oracle's own release (h = 1e-6 mm) to 1e-6 relative. The GPU's gradient is
checked against this one in test_gpu_adjoint.py."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

GRADIENT_TOL = 1e-6


@pytest.fixture(scope="module")
def problem(pkg, orc):
    wl = importlib.import_module("springback-precomp_b200.workload")

    def evaluate(mesh, mat, u, state, alpha, want_yield=False):
        nt = mat.kinematic_terms
        r = orc.elements(mat.as_dict(), mesh.element_coordinates(), mesh.gather(u),
                         orc.device_to_oracle(state, nt), alpha, want_tangent=False)
        out = (orc.oracle_to_device(r["states"], nt), r["alpha"], r["status"])
        return out + ((r["yield_flags"],) if want_yield else ())

    return wl.make_problem(8, 8, 2, seed=5, evaluate=evaluate, sample=128)


def oracle_gradient(pkg, orc, prob):
    """(J, dJ/dp, release) from the oracle for the springback RMS of the top
    face at p = 0, and a function J(p) by a fresh release."""
    mesh, mat = prob.mesh, prob.material
    m = mat.as_dict()
    m["yield_stress"] = 1e300  # frozen: no point returns
    committed = orc.device_to_oracle(prob.state, mat.kinematic_terms)
    free = pkg.supports_321(mesh)
    lo, hi = mesh.coords.min(axis=0), mesh.coords.max(axis=0)
    grid = pkg.BicubicHeights(lo[0], hi[0], lo[1], hi[1], n=20)
    stencil = grid.stencil(mesh.coords[:, :2])
    top = np.flatnonzero(np.isclose(mesh.coords[:, 2], hi[2]))
    target = mesh.coords[top, 2] + prob.u.reshape(-1, 3)[top, 2]

    def coords_of(p):
        x = mesh.coords.copy()
        x[:, 2] += grid.heights(torch.as_tensor(p), stencil).numpy()
        return x

    def rms(x, u):
        d = x[top, 2] + u.reshape(-1, 3)[top, 2] - target
        return float(np.sqrt(np.mean(d * d))), d

    u_star, _ = orc.release_solve(m, mesh.coords, mesh.connectivity, committed, prob.alpha, free, prob.u)
    j, d = rms(mesh.coords, u_star)
    dj_dz = d / (len(top) * j)
    dj_du = np.zeros(mesh.num_dofs)
    dj_du[3 * top + 2] = dj_dz
    gx = orc.release_adjoint(m, mesh.coords, mesh.connectivity, committed, prob.alpha, free, u_star, dj_du)
    gx[top, 2] += dj_dz  # z = X_z + u_z: the explicit share
    p = torch.zeros((20, 20), dtype=torch.float64, requires_grad=True)
    grid.heights(p, stencil).backward(torch.as_tensor(gx[:, 2]))

    def j_of(p_np):
        x = coords_of(p_np)
        u, _ = orc.release_solve(m, x, mesh.connectivity, committed, prob.alpha, free, u_star)
        return rms(x, u)[0]

    return j, p.grad.numpy(), u_star, j_of


def test_oracle_height_gradient_matches_central_differences(pkg, orc, problem):
    j, grad, _, j_of = oracle_gradient(pkg, orc, problem)
    assert j > 0.0 and np.abs(grad).max() > 0.0
    h = 1e-9
    rng = np.random.default_rng(8)
    for _ in range(4):
        d = rng.uniform(-1.0, 1.0, size=(20, 20))
        fd = (j_of(h * d) - j_of(-h * d)) / (2.0 * h)
        adj = float((grad * d).sum())
        assert abs(adj - fd) <= GRADIENT_TOL * abs(fd), (adj, fd, abs(adj - fd) / abs(fd))


def test_incremental_release_reaches_equilibrium(pkg, orc):
    """The oracle's release in increments (the start's imbalance r0 taken
    off in equal steps) on a 16 x 16 x 4 cone part whose history was loaded
    by imposed displacements: the end state is an equilibrium of the free
    rows (f_int(u*) within 1e-8 of r0), every increment's equilibrium was
    reached, and the sheet sprang back by a fraction of a millimetre."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    mesh = wl.cone_sheet(16, 4)
    mat = pkg.material.hill_chaboche_sheet()
    cone = wl.cone_part()
    X = mesh.element_coordinates()
    committed = np.zeros((mesh.num_elements, 8, orc.NF))
    alpha = np.zeros((mesh.num_elements, 9))
    for k in range(1, 8):
        uk = (wl.formed_positions(mesh, cone, k * 0.35 / 7) - mesh.coords).reshape(-1)
        r = orc.elements(mat.as_dict(), X, mesh.gather(uk), committed, alpha, want_tangent=False)
        assert (r["status"] == 0).all()
        committed, alpha = r["states"], r["alpha"]
    u0 = (wl.formed_positions(mesh, cone, 0.35) - mesh.coords).reshape(-1)
    m = mat.as_dict()
    m["yield_stress"] = 1e300  # frozen
    free = pkg.supports_321(mesh)
    r0 = orc.system_evaluate(m, mesh.coords, mesh.connectivity, u0, committed, alpha)["internal"][free]
    u, iterations = orc.release_solve(m, mesh.coords, mesh.connectivity, committed, alpha, free, u0, increments=8)
    r = orc.system_evaluate(m, mesh.coords, mesh.connectivity, u, committed, alpha)["internal"][free]
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(r0)
    assert iterations >= 8 * 2
    assert 0.05e-3 < np.abs(u - u0).max() < 2.0e-3
