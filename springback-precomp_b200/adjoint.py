"""The release step made differentiable: the springback of a part released
onto its supports with the end-of-forming plastic state frozen, as a
function of the nodal reference coordinates X, behind torch.autograd.

The reference has no gradient. Its compensation is displacement
adjustment, c_{k+1} = c_k - alpha (f(c_k) - t), one full forming and
release simulation per step (python/precomp/compensation.py:273-366, the
FEAPredictor of :382-410), scored by the RMS of the vertical deviation of
the formed surface from the target (vertical_deviation and metrics,
python/precomp/metrology.py:448-486). This module gives that score a
gradient:

- Release.solve: Newton on the free rows of f_int(u, X) = 0 (the device
  element loop, the device PartitionedFactor), the support DOFs held where
  the formed part left them, the committed points and modes frozen
  (sbk_system_set_frozen) - the release step of the forming driver
  (Forming.cpp release handling) without its tool and clamp bookkeeping.
- Release.adjoint: K_ff^T lambda_f = dJ/du_f solved with the factorisation
  of the tangent at u* transposed (the one the release's last Newton
  evaluate left, or a new one), and dJ/dX = -lambda^T d f_int / d X by the
  shape-derivative kernel (sbk_system_vjp_x, the modes through their local
  equilibrium), which recomputes the points from the committed state rather
  than reading them from the forward solve.
- ReleaseFunction: both as a torch.autograd.Function of X.
- BicubicHeights: the commanded-shape parametrisation, a clamped uniform
  cubic B-spline surface over the footprint whose n x n control heights move
  every node vertically: X(p) = X0 + h(x0, y0; p) e_z. The reference's
  commanded shape reaches the model only through the tool path
  (python/precomp/fea/deck.py:99-104); here it moves the release step's
  reference geometry, the formed part following its commanded surface.
- springback_rms: metrics(vertical_deviation(...))["rms"] over the nodes of
  the measured surface, z = X_z + u_z against the target heights.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import _capi
from .mesh import HexMesh
from .partition import PartitionedFactor
from .system import NonlinearSystem


def cubic_bspline_basis(t: np.ndarray, n: int):
    """The four non-zero clamped uniform cubic B-spline basis functions of n
    control points at the parameters t in [0, 1] (Cox-de Boor recursion,
    Piegl and Tiller, The NURBS Book, algorithm A2.2): the index of the first
    of the four control points and their weights (len(t), 4)."""
    if n < 4:
        raise ValueError("a cubic B-spline needs at least four control points")
    t = np.clip(np.asarray(t, dtype=np.float64), 0.0, 1.0)
    spans = n - 3
    knots = np.concatenate([np.zeros(3), np.linspace(0.0, 1.0, spans + 1), np.ones(3)])
    k = np.minimum(np.floor(t * spans).astype(np.int64), spans - 1) + 3
    basis = np.zeros((t.size, 4))
    basis[:, 0] = 1.0
    left = np.zeros((t.size, 4))
    right = np.zeros((t.size, 4))
    for j in range(1, 4):
        left[:, j] = t - knots[k + 1 - j]
        right[:, j] = knots[k + j] - t
        saved = np.zeros(t.size)
        for r in range(j):
            temp = basis[:, r] / (right[:, r + 1] + left[:, j - r])
            basis[:, r] = saved + right[:, r + 1] * temp
            saved = left[:, j - r] * temp
        basis[:, j] = saved
    return k - 3, basis


class BicubicHeights:
    """Heights over the footprint [x0, x1] x [y0, y1] from an n x n grid of
    control heights p (p[i, j]: i along x, j along y): the tensor product of
    clamped uniform cubic B-splines, C2, each point weighted by 16 controls."""

    def __init__(self, x0: float, x1: float, y0: float, y1: float, n: int = 20):
        if not (x1 > x0 and y1 > y0):
            raise ValueError("an empty footprint")
        self.x0, self.x1, self.y0, self.y1, self.n = x0, x1, y0, y1, n

    @property
    def num_parameters(self) -> int:
        return self.n * self.n

    def stencil(self, xy: np.ndarray, device=None):
        """For points xy (m, 2): the flat indices of their 16 controls and
        the weights (m, 16), as device tensors."""
        xy = np.asarray(xy, dtype=np.float64)
        ix, wx = cubic_bspline_basis((xy[:, 0] - self.x0) / (self.x1 - self.x0), self.n)
        iy, wy = cubic_bspline_basis((xy[:, 1] - self.y0) / (self.y1 - self.y0), self.n)
        a = np.arange(4)
        idx = (ix[:, None, None] + a[None, :, None]) * self.n + (iy[:, None, None] + a[None, None, :])
        w = wx[:, :, None] * wy[:, None, :]
        return (torch.tensor(idx.reshape(-1, 16), device=device),
                torch.tensor(w.reshape(-1, 16), device=device))

    @staticmethod
    def heights(p: torch.Tensor, stencil) -> torch.Tensor:
        idx, w = stencil
        return (p.reshape(-1)[idx] * w).sum(dim=1)


class Release:
    """The release step of one part on one device: the system of its mesh
    with the committed points and modes of the end of forming, frozen, and
    the partition of its supports (`free`: the DOFs not held)."""

    def __init__(self, mesh: HexMesh, material, committed: np.ndarray, modes: np.ndarray, free: Sequence[int],
                 kinematics: str = "logarithmic", tolerance: float = 1e-10, max_iterations: int = 40,
                 increments: int = 1):
        self.mesh = mesh
        self.system = NonlinearSystem(mesh, material, kinematics=kinematics)
        self.system.set_committed(committed)
        self.system.set_internal(modes)
        self.system.set_frozen(True)
        self.free = np.ascontiguousarray(np.asarray(free, dtype=np.int32))
        self.part = PartitionedFactor.for_system(self.system, self.free)
        self.tolerance = tolerance
        self.max_iterations = max_iterations
        self.increments = increments
        self.iterations = 0
        self.factorizations = 0
        self._factored = None

    def close(self):
        self.part.close()
        self.system.close()

    def _tangent(self, u: torch.Tensor, coords: torch.Tensor):
        """Evaluate and factorise at (u, coords), remembering where: the last
        Newton evaluate is at the root, and the adjoint reuses it."""
        self._factored = None
        ev = self.system.evaluate(u, 0.0, True)
        self.part.factorize(ev.tangent, self.system.symmetric())
        self.factorizations += 1
        self._factored = (u.detach().clone(), coords.detach().reshape(-1, 3).clone())
        return ev

    def forget_factorization(self):
        """Make the next adjoint re-evaluate and factorise at its u."""
        self._factored = None

    def _factored_at(self, u: torch.Tensor, coords: torch.Tensor) -> bool:
        f = getattr(self, "_factored", None)
        return f is not None and torch.equal(f[0], u) and torch.equal(f[1], coords.reshape(-1, 3))

    def solve(self, coords: torch.Tensor, u0: torch.Tensor, increments: Optional[int] = None) -> torch.Tensor:
        """The released displacement u* at the reference coordinates coords
        (num_nodes x 3, device) from u0 (its held DOFs kept): Newton, a step
        halved while an element refuses it, until a full step is below
        `tolerance` of u, then one step more. SolverError when it does not
        converge.

        `increments` > 1 takes the imbalance of the start, r0 = f_int(u0) on
        the free rows, off in that many equal steps - Newton to equilibrium
        of f_int(u) = (1 - k / increments) r0 at each k - for a start far
        from equilibrium (a history loaded by imposed displacements), where
        full Newton steps from u0 overshoot. The material is frozen, so the
        end state solves f_int(u*) = 0 whatever the path that reached it.
        None: the release's own `increments`."""
        increments = self.increments if increments is None else int(increments)
        self.system.set_coordinates(coords.reshape(-1, 3))
        u = u0.detach().clone()
        ev = self._tangent(u, coords)
        r_start = self.part.restrict(ev.internal)
        total = 0
        for k in range(1, increments + 1):
            left = 1.0 - k / increments
            last = k == increments
            r = self.part.restrict(ev.internal) - left * r_start
            converged = False
            for it in range(self.max_iterations):
                du = self.part.solve(-r)
                step = 1.0
                while True:
                    trial = self.part.add_to(u.clone(), du, step)
                    try:
                        ev = self._tangent(trial, coords)
                        break
                    except _capi.SolverError:
                        step *= 0.5
                        if step < 1.0 / 1024:
                            raise
                u = trial
                total += 1
                r = self.part.restrict(ev.internal) - left * r_start
                if converged:
                    break
                converged = step == 1.0 and float(torch.linalg.norm(du)) <= self.tolerance * float(torch.linalg.norm(u))
                if converged and not last:
                    break
            else:
                raise _capi.SolverError(4, f"the release did not converge in {self.max_iterations} Newton "
                                           f"iterations (increment {k} of {increments})")
        self.iterations = total
        return u

    def adjoint(self, coords: torch.Tensor, u: torch.Tensor, grad_u: torch.Tensor) -> torch.Tensor:
        """dJ/dX (num_nodes x 3) from dJ/du at the released u: K_ff^T
        lambda_f = (dJ/du)_f with the factorisation of the tangent at u (the
        one the release's last Newton evaluate left, when it was at this u
        and these coordinates; else the points re-evaluated at u and the
        tangent factorised again), then -lambda^T d f_int / d X, whose kernel
        recomputes the points from the committed state. The held DOFs of u do
        not depend on X; their share of dJ/du stays with the caller."""
        self.system.set_coordinates(coords.reshape(-1, 3))
        if not self._factored_at(u, coords):
            self._tangent(u, coords)
        lam_f = self.part.solve(self.part.restrict(grad_u.detach().to(torch.float64)), transpose=True)
        lam = self.part.add_to(torch.zeros_like(u), lam_f, 1.0)
        return -self.system.vjp_x(u, lam, frozen=True).reshape(-1, 3)


class ReleaseFunction(torch.autograd.Function):
    """u* = ReleaseFunction.apply(coords, release, u0): the released
    displacement as a differentiable function of the reference coordinates;
    its backward is Release.adjoint."""

    @staticmethod
    def forward(ctx, coords: torch.Tensor, release: Release, u0: torch.Tensor) -> torch.Tensor:
        u = release.solve(coords.detach(), u0)
        ctx.release = release
        ctx.save_for_backward(coords.detach(), u)
        return u

    @staticmethod
    def backward(ctx, grad_u: torch.Tensor):
        coords, u = ctx.saved_tensors
        return ctx.release.adjoint(coords, u, grad_u).reshape(coords.shape), None, None


def released(coords: torch.Tensor, release: Release, u0: torch.Tensor) -> torch.Tensor:
    return ReleaseFunction.apply(coords, release, u0)


def springback_rms(coords: torch.Tensor, u: torch.Tensor, nodes: torch.Tensor, target_z: torch.Tensor) -> torch.Tensor:
    """The RMS of z - z_target over `nodes`, z = X_z + u_z (the reference's
    metrics(vertical_deviation(formed, target))["rms"] at the nodes of the
    measured surface)."""
    z = coords.reshape(-1, 3)[nodes, 2] + u.reshape(-1, 3)[nodes, 2]
    return torch.sqrt(torch.mean((z - target_z) ** 2))


def supports_321(mesh: HexMesh, tol: Optional[float] = None) -> np.ndarray:
    """The free DOFs of a sheet on 3-2-1 supports at its bottom corners: the
    corner at (x_min, y_min) held in x, y and z, the corner at (x_max, y_min)
    in y and z, the corner at (x_min, y_max) in z (the reference's release
    onto 3-2-1 supports)."""
    x = mesh.coords
    lo, hi = x.min(axis=0), x.max(axis=0)
    tol = tol if tol is not None else 1e-9 * float(np.max(hi - lo))

    def corner(cx, cy):
        d = np.abs(x - np.array([cx, cy, lo[2]])).max(axis=1)
        i = int(np.argmin(d))
        if d[i] > tol:
            raise ValueError("the sheet has no node at a support corner")
        return i

    a, b, c = corner(lo[0], lo[1]), corner(hi[0], lo[1]), corner(lo[0], hi[1])
    held = np.zeros(mesh.num_dofs, dtype=bool)
    held[[3 * a, 3 * a + 1, 3 * a + 2, 3 * b + 1, 3 * b + 2, 3 * c + 2]] = True
    return np.flatnonzero(~held).astype(np.int32)


def compensate(release: Release, grid: BicubicHeights, stencil, coords0: torch.Tensor, nodes: torch.Tensor,
               target_z: torch.Tensor, u0: torch.Tensor, iterations: int = 10, history_size: int = 10):
    """Adjoint-driven compensation: the control heights p that minimise the
    RMS vertical deviation of the released part from the target, by L-BFGS
    with a strong-Wolfe line search (torch.optim.LBFGS), every objective one
    release solve (warm-started from the last) and every gradient one
    adjoint. It takes the place of the reference's displacement adjustment,
    c_{k+1} = c_k - alpha (f(c_k) - t) (compensation.py:273-366), which
    needs one forming and release simulation per step and no gradient.

    p is optimised in units of the initial deviation (q = p / J0, the
    objective J / J0), so that the first step is of the springback's size.
    Returns (p, the objective after each evaluation in metres, the number of
    release solves)."""
    device = coords0.device
    warm = [u0.detach()]
    history = []

    def objective(q: torch.Tensor, scale: float) -> torch.Tensor:
        lift = torch.zeros_like(coords0)
        lift[:, 2] = grid.heights(q * scale, stencil)
        coords = coords0 + lift
        u = released(coords, release, warm[0])
        warm[0] = u.detach()
        return springback_rms(coords, u, nodes, target_z)

    zero = torch.zeros((grid.n, grid.n), dtype=torch.float64, device=device)
    with torch.no_grad():
        j0 = float(objective(zero, 1.0))
    history.append(j0)
    if j0 == 0.0:
        return zero, history, 1
    q = zero.clone().requires_grad_(True)
    opt = torch.optim.LBFGS([q], lr=1.0, max_iter=iterations, history_size=history_size,
                            tolerance_grad=0.0, tolerance_change=0.0, line_search_fn="strong_wolfe")

    def closure():
        opt.zero_grad()
        j = objective(q, j0)
        history.append(float(j.detach()))
        (j / j0).backward()
        return j / j0

    opt.step(closure)
    return (q.detach() * j0), history, len(history)
