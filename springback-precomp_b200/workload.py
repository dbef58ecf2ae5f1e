"""Synthetic inputs of the element-kernel microbenchmark: a regular
nx x ny x nz Hex8 sheet of 0.04 x 0.04 x 0.5 mm cells (1000 x 500 x 2 =
1,000,000 elements at full size), the Hill48 + two-term Chaboche law, and
nodal displacements u_ref of uniform noise (+-2 % of the mesh size h = 0.04 mm
on every component) plus a smooth bending field. Every point starts from a seeded history
(accumulated plastic strain U[0, 0.15], deviatoric backstresses of tensor
norm <= 20 MPa); loading to u_ref in four committed increments gives a
converged plastic history; the evaluated state is then u_ref + s du, du
reversing u_ref with a little noise, `s` found by bisection so that about
40 % of the points yield (reverse yielding after elastic unloading).

The inputs are seeded numpy; the history and the yield fraction come from
the element kernel itself (the GPU by default).
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional

import numpy as np

from .material import Material, hill_chaboche_sheet
from .mesh import HexMesh, structured_hex_mesh

CELL = (4.0e-5, 4.0e-5, 5.0e-4)  # m
# The noise of every displacement component: 2 % of the mesh size h of the
# sheet (its in-plane cell edge); 2 % of the 0.5 mm thickness cell would shear
# the 0.04 mm wide columns by about 25 %.
NOISE = 0.02 * CELL[0]


@dataclasses.dataclass
class Problem:
    mesh: HexMesh
    material: Material
    u: np.ndarray          # (3 nn,) the evaluated displacement
    state: np.ndarray      # (nfields, ne, nq) committed points, device layout
    alpha: np.ndarray      # (ne, 9) committed modes (zero)
    s: float               # the increment fraction
    kinematics: str = "logarithmic"


def displacement(mesh: HexMesh, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x, y, z = mesh.coords[:, 0], mesh.coords[:, 1], mesh.coords[:, 2]
    xc, yc, zc = 0.5 * (x.max() + x.min()), 0.5 * (y.max() + y.min()), 0.5 * (z.max() + z.min())
    kx, ky = 20.0, 10.0  # 1/m: 1 % and 0.5 % bending strain at the surfaces of the 1 mm sheet
    u = np.zeros_like(mesh.coords)
    u[:, 0] = -kx * (x - xc) * (z - zc)
    u[:, 1] = -ky * (y - yc) * (z - zc)
    u[:, 2] = 0.5 * kx * (x - xc) ** 2 + 0.5 * ky * (y - yc) ** 2
    u += rng.uniform(-NOISE, NOISE, size=u.shape)
    return u.reshape(-1)


def seeded_state(mesh: HexMesh, material: Material, seed: int, nq: int = 8) -> np.ndarray:
    """The seeded start of the loading: accumulated plastic strain
    U[0, 0.15], deviatoric backstresses of tensor norm <= 20 MPa, no plastic
    strain; (nfields, ne, nq)."""
    rng = np.random.default_rng(seed + 1)
    n = mesh.num_elements
    nterms = material.kinematic_terms

    def deviators(size, norm_max):
        d = rng.normal(size=size + (6,))
        d[..., :3] -= d[..., :3].mean(axis=-1, keepdims=True)
        tn = np.sqrt((d[..., :3] ** 2).sum(-1) + 2 * (d[..., 3:] ** 2).sum(-1))
        return d / tn[..., None] * rng.uniform(0.0, norm_max, size=size)[..., None]

    st = np.zeros((material.state_fields, n, nq))
    back = [deviators((n, nq), 20.0e6) for _ in range(nterms)]
    for t in range(nterms):
        st[12 + 6 * t:18 + 6 * t] = np.moveaxis(back[t], -1, 0)
    if nterms:
        st[6:12] = np.moveaxis(sum(back), -1, 0)
    st[12 + 6 * nterms] = rng.uniform(0.0, 0.15, size=(n, nq))
    return st


def load_history(mesh: HexMesh, material: Material, u_ref: np.ndarray, state: np.ndarray, evaluate: Callable,
                 steps: int = 4):
    """The committed history at u_ref: `steps` equal increments from the
    seeded state, each converged by `evaluate(mesh, material, u, state,
    alpha) -> (trial state, alpha, codes)` and committed. Elements whose
    local iteration fails keep their last committed history."""
    alpha = np.zeros((mesh.num_elements, 9))
    for k in range(1, steps + 1):
        trial, a, codes = evaluate(mesh, material, (k / steps) * u_ref, state, alpha)
        ok = codes == 0
        state = np.where(ok[None, :, None], trial, state)
        alpha = np.where(ok[:, None], a, alpha)
    return state, alpha


def make_problem(nx: int = 1000, ny: int = 500, nz: int = 2, seed: int = 7, s: Optional[float] = None,
                 target: float = 0.4, evaluate: Optional[Callable] = None, sample: int = 4096,
                 material: Optional[Material] = None, steps: int = 4) -> Problem:
    """The microbenchmark problem: the history of loading to u_ref (bending
    plus noise), then the increment u = u_ref + s du with du mostly
    reversing u_ref, `s` bisected so that a fraction `target` of the points
    yield. `evaluate` runs the element kernel (default: the GPU)."""
    mesh = structured_hex_mesh(nx, ny, nz, nx * CELL[0], ny * CELL[1], nz * CELL[2])
    material = material or hill_chaboche_sheet()
    evaluate = evaluate or gpu_evaluate
    u_ref, du = increment(mesh, seed)
    state, alpha = load_history(mesh, material, u_ref, seeded_state(mesh, material, seed), evaluate, steps)
    if s is None:
        els = np.sort(np.random.default_rng(seed + 2).choice(mesh.num_elements,
                                                             size=min(sample, mesh.num_elements), replace=False))
        sub = HexMesh(mesh.coords, mesh.connectivity[els])
        st_s, al_s = state[:, els], alpha[els]
        lo, hi = 0.0, 1.0
        for _ in range(16):
            mid = 0.5 * (lo + hi)
            _, _, codes, y = evaluate(sub, material, u_ref + mid * du, st_s, al_s, want_yield=True)
            f = float(y[codes == 0].mean()) if (codes == 0).any() else 1.0
            if f < target:
                lo = mid
            else:
                hi = mid
        s = 0.5 * (lo + hi)
    return Problem(mesh=mesh, material=material, u=u_ref + s * du, state=state, alpha=alpha, s=s)


def increment(mesh: HexMesh, seed: int):
    """u_ref and the mostly reversing direction du of the increment."""
    u_ref = displacement(mesh, seed)
    rng = np.random.default_rng(seed + 3)
    du = -u_ref + 0.25 * rng.uniform(-NOISE, NOISE, size=3 * mesh.num_nodes)
    return u_ref, du


def make_system_problem(nx: int = 1000, ny: int = 500, nz: int = 2, seed: int = 7, target: float = 0.4,
                        sample: int = 4096, steps: int = 4, material: Optional[Material] = None, device=None):
    """The same problem, built on the GPU without host round trips: the
    history is loaded by the element kernel straight into the committed
    buffers of a NonlinearSystem; the bisection runs the kernel on a sample.
    Returns (system, u on the device, s, mesh)."""
    import torch

    from .system import NonlinearSystem, element_batch

    dev = torch.device(device or "cuda")
    mesh = structured_hex_mesh(nx, ny, nz, nx * CELL[0], ny * CELL[1], nz * CELL[2])
    material = material or hill_chaboche_sheet()
    u_ref, du = increment(mesh, seed)
    sysm = NonlinearSystem(mesh, material, kinematics="logarithmic")
    u_ref_d = torch.tensor(u_ref, device=dev)
    du_d = torch.tensor(du, device=dev)
    cs, ca = sysm.committed_views()
    cs.copy_(torch.tensor(seeded_state(mesh, material, seed), device=dev))
    ca.zero_()
    conn_all = torch.tensor(mesh.connectivity, device=dev).long()
    coords = torch.tensor(mesh.coords, device=dev)
    # The history: `steps` committed increments to u_ref, element by element
    # (an element whose local iteration fails keeps its last history).
    chunk = 262144
    for k in range(1, steps + 1):
        uk = ((k / steps) * u_ref_d).view(-1, 3)
        for lo in range(0, mesh.num_elements, chunk):
            hi = min(mesh.num_elements, lo + chunk)
            cc = conn_all[lo:hi]
            r = element_batch(material, coords[cc].reshape(-1, 24).contiguous(), uk[cc].reshape(-1, 24).contiguous(),
                              cs[:, lo:hi].contiguous(), ca[lo:hi].contiguous(), want_tangent=False)
            ok = r.code == 0
            cs[:, lo:hi] = torch.where(ok[None, :, None], r.states, cs[:, lo:hi])
            ca[lo:hi] = torch.where(ok[:, None], r.alpha, ca[lo:hi])
    cs, ca = sysm.committed_views()
    els = torch.tensor(np.sort(np.random.default_rng(seed + 2).choice(mesh.num_elements,
                                                                      size=min(sample, mesh.num_elements),
                                                                      replace=False)), device=dev)
    conn = conn_all.index_select(0, els)
    x_s = coords[conn].reshape(-1, 24).contiguous()
    st_s = cs.index_select(1, els).contiguous()
    al_s = ca.index_select(0, els).contiguous()
    lo, hi = 0.0, 1.0
    for _ in range(16):
        mid = 0.5 * (lo + hi)
        u = (u_ref_d + mid * du_d).view(-1, 3)
        r = element_batch(material, x_s, u[conn].reshape(-1, 24).contiguous(), st_s, al_s, want_tangent=False)
        ok = r.code == 0
        f = float(r.yielding[ok].float().mean().item()) if bool(ok.any()) else 1.0
        if f < target:
            lo = mid
        else:
            hi = mid
    s = 0.5 * (lo + hi)
    # Every element must converge at the evaluated state (the reference would
    # cut the increment): shorten it until they do.
    for _ in range(20):
        u = (u_ref_d + s * du_d).contiguous()
        try:
            sysm.evaluate(u, 0.0, False)
            break
        except Exception as err:
            if not hasattr(err, "element"):
                raise
            s *= 0.9
    return sysm, u, s, mesh


def gpu_evaluate(mesh, material, u, state, alpha, want_yield=False):
    """The element kernel on the GPU (no tangent), batched."""
    import torch
    from .system import element_batch

    dev = torch.device("cuda")
    ne = mesh.num_elements
    out_st = np.empty_like(state)
    out_a = np.empty((ne, 9))
    codes = np.empty(ne, dtype=np.int32)
    ys = []
    chunk = 262144
    for lo in range(0, ne, chunk):
        hi = min(ne, lo + chunk)
        conn = mesh.connectivity[lo:hi]
        x = torch.tensor(mesh.coords[conn].reshape(-1, 24), device=dev)
        ue = torch.tensor(u.reshape(-1, 3)[conn].reshape(-1, 24), device=dev)
        st = torch.tensor(np.ascontiguousarray(state[:, lo:hi]), device=dev)
        al = torch.tensor(np.ascontiguousarray(alpha[lo:hi]), device=dev)
        r = element_batch(material, x, ue, st, al, want_tangent=False)
        out_st[:, lo:hi] = r.states.cpu().numpy()
        out_a[lo:hi] = r.alpha.cpu().numpy()
        codes[lo:hi] = r.code.cpu().numpy()
        ys.append(r.yielding.cpu().numpy())
    if want_yield:
        return out_st, out_a, codes, np.concatenate(ys).astype(bool)
    return out_st, out_a, codes


