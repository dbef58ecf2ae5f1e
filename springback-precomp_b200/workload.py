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
import math
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




# ---- the fine-mesh part: a truncated cone formed in a 4-layer sheet ---------

# The cone of the fine-mesh configuration: an 18 mm footprint, 3 mm deep, a
# 50 degree wall (2 mm fillets at rim and floor), in a 1 mm sheet.
CONE = dict(footprint_radius=9.0e-3, wall_angle_deg=50.0, depth=3.0e-3, top_fillet=2.0e-3, bottom_fillet=2.0e-3)
CONE_BLANK = 24.0e-3    # m, the square blank the cone is formed in
CONE_THICKNESS = 1.0e-3
TOOL_RADIUS = 2.0e-3    # both tools: the forming ball above, the support ball below
TOOL_TRAVEL = 5.0e-5    # m, the tools' travel in one increment (half the in-plane cell)


@dataclasses.dataclass
class ConeProblem:
    mesh: HexMesh
    material: Material
    cone: object
    s: float                 # the fraction of the cone's depth formed
    u0: np.ndarray           # committed displacement (start of the increment)
    u: np.ndarray            # evaluated displacement (end of the increment)
    tools: list              # two dicts of Tool arguments: forming (top), support (bottom)
    contact_radius: float    # m, where the tools act on the wall


def cone_part():
    from .parts import TruncatedCone

    return TruncatedCone.with_footprint(**CONE)


def cone_sheet(n: int = 224, layers: int = 4) -> HexMesh:
    """The blank: n x n x layers Hex8 over CONE_BLANK square, 1 mm thick, its
    top face at z = 0, centred on the cone's axis."""
    return structured_hex_mesh(n, n, layers, CONE_BLANK, CONE_BLANK, CONE_THICKNESS, x0=-0.5 * CONE_BLANK,
                               y0=-0.5 * CONE_BLANK, z0=-CONE_THICKNESS)


def formed_positions(mesh: HexMesh, cone, s: float) -> np.ndarray:
    """The sheet laid onto the surface z = s h(x, y) (s of the cone's depth):
    each mid-surface point moves to the surface, each through-thickness
    fibre follows the surface normal, shortened by the sine law (t cos of the
    local wall angle), so that the wall thins as in incremental forming."""
    x, y, z = mesh.coords[:, 0], mesh.coords[:, 1], mesh.coords[:, 2]
    zm = -0.5 * CONE_THICKNESS
    eps = 1.0e-7
    h = s * cone.height(x, y)
    hx = s * (cone.height(x + eps, y) - cone.height(x - eps, y)) / (2 * eps)
    hy = s * (cone.height(x, y + eps) - cone.height(x, y - eps)) / (2 * eps)
    norm = np.sqrt(1.0 + hx * hx + hy * hy)
    n = np.stack([-hx, -hy, np.ones_like(hx)], axis=1) / norm[:, None]
    off = (z - zm) / norm  # the fibre, thinned by cos = 1 / norm
    return np.stack([x, y, zm + h], axis=1) + off[:, None] * n


def slave_faces(mesh: HexMesh, top: bool, penalty: float = 10.0, young: float = 70.0e9):
    """The nodes of the sheet's top (or bottom) face with their tributary
    areas (a quarter of each adjacent cell) and penalties kappa = penalty E /
    sqrt(area) (ToolContact's constructor, RigidTool.cpp:292-321)."""
    z = mesh.coords[:, 2]
    nodes = np.flatnonzero(np.isclose(z, z.max() if top else z.min()))
    x, y = mesh.coords[nodes, 0], mesh.coords[nodes, 1]
    hx = np.diff(np.unique(x)).min()
    hy = np.diff(np.unique(y)).min()
    wx = np.where(np.isclose(x, x.min()) | np.isclose(x, x.max()), 0.5, 1.0)
    wy = np.where(np.isclose(y, y.min()) | np.isclose(y, y.max()), 0.5, 1.0)
    area = wx * wy * hx * hy
    return nodes.astype(np.int32), area, penalty * young / np.sqrt(area)


def place_ball(faces: np.ndarray, point: np.ndarray, normal: np.ndarray, radius: float, penetration: float):
    """The centre c = point + d normal of a ball of `radius` whose deepest
    face node lies `penetration` inside it (min |x - c| = radius -
    penetration), d found by bisection."""
    near = faces[np.linalg.norm(faces - point, axis=1) < 3.0 * radius]

    def gap(d):
        return np.linalg.norm(near - (point + d * normal), axis=1).min() - (radius - penetration)

    lo, hi = 0.0, 2.0 * radius
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if gap(mid) < 0.0:
            lo = mid
        else:
            hi = mid
    return point + 0.5 * (lo + hi) * normal


def make_cone_problem(n: int = 224, layers: int = 4, s: float = 0.35, steps: int = 7, device=None,
                      material: Optional[Material] = None, penetration: float = 5.0e-5, friction: float = 0.1):
    """The fine-mesh configuration a third of the way through forming: the
    cone formed to s of its depth in `steps` committed increments (the
    element kernel loading every element's history), the evaluated
    increment a quarter step further, and the two tools of double-sided
    forming - the forming ball on the top face and the support ball under
    the bottom face, on the wall, moving along the spiral by TOOL_TRAVEL in
    the increment, each `penetration` into its face at both ends of the
    increment. Returns (system, ConeProblem)."""
    import torch

    from .system import NonlinearSystem, element_batch

    dev = torch.device(device or "cuda")
    mesh = cone_sheet(n, layers)
    material = material or hill_chaboche_sheet()
    cone = cone_part()
    ds = s / steps
    sysm = NonlinearSystem(mesh, material, kinematics="logarithmic")
    cs, ca = sysm.committed_views()
    cs.zero_()
    ca.zero_()
    conn_all = torch.tensor(mesh.connectivity, device=dev).long()
    coords = torch.tensor(mesh.coords, device=dev)
    chunk = 262144
    for k in range(1, steps + 1):
        uk = torch.tensor((formed_positions(mesh, cone, k * ds) - mesh.coords), device=dev)
        for lo in range(0, mesh.num_elements, chunk):
            hi = min(mesh.num_elements, lo + chunk)
            cc = conn_all[lo:hi]
            r = element_batch(material, coords[cc].reshape(-1, 24).contiguous(), uk[cc].reshape(-1, 24).contiguous(),
                              cs[:, lo:hi].contiguous(), ca[lo:hi].contiguous(), want_tangent=False)
            ok = r.code == 0
            cs[:, lo:hi] = torch.where(ok[None, :, None], r.states, cs[:, lo:hi])
            ca[lo:hi] = torch.where(ok[:, None], r.alpha, ca[lo:hi])
    fracs = (s, s + 0.25 * ds)
    pos = [formed_positions(mesh, cone, f) for f in fracs]
    u0 = (pos[0] - mesh.coords).reshape(-1)
    u1 = (pos[1] - mesh.coords).reshape(-1)
    # The tools on the wall, where its slope is steepest.
    prof_r = np.linspace(0.0, CONE["footprint_radius"], 4001)
    hr = cone.height(prof_r, 0 * prof_r)
    rc = float(prof_r[np.argmax(np.abs(np.gradient(hr, prof_r)))])
    tools = []
    for top in (True, False):
        nodes, area, kappa = slave_faces(mesh, top)
        pts = []
        for t, frac, x_t in zip((0.0, 1.0), fracs, pos):
            th = t * TOOL_TRAVEL / rc
            x, y = rc * np.cos(th), rc * np.sin(th)
            eps = 1.0e-7
            hx = frac * (cone.height(np.array([x + eps]), np.array([y]))[0] -
                         cone.height(np.array([x - eps]), np.array([y]))[0]) / (2 * eps)
            hy = frac * (cone.height(np.array([x]), np.array([y + eps]))[0] -
                         cone.height(np.array([x]), np.array([y - eps]))[0]) / (2 * eps)
            nrm = np.array([-hx, -hy, 1.0]) / np.sqrt(1.0 + hx * hx + hy * hy)
            mid = np.array([x, y, -0.5 * CONE_THICKNESS + frac * cone.height(np.array([x]), np.array([y]))[0]])
            sign = 1.0 if top else -1.0
            pts.append(tuple(place_ball(x_t[nodes], mid, sign * nrm, TOOL_RADIUS, penetration)))
        tools.append(dict(shape="sphere", times=[0.0, 1.0], points=pts, nodes=nodes, area=area, kappa=kappa,
                          radius=TOOL_RADIUS, friction=friction, tangential_ratio=1.0,
                          name="forming" if top else "support"))
    return sysm, ConeProblem(mesh=mesh, material=material, cone=cone, s=s, u0=u0, u=u1, tools=tools,
                             contact_radius=rc)


# ---- the design sweep: parts of four families from a Sobol sequence ----------

SWEEP_BOUNDS = dict(footprint_radius=(7.5e-3, 10.0e-3), depth=(2.0e-3, 4.0e-3), wall_angle_deg=(30.0, 55.0),
                    axis_ratio=(1.0, 1.6), elements=(20000, 150000))
SWEEP_FAMILIES = ("dome", "truncated_cone", "elliptic_cone", "pyramid")


SWEEP_FLOOR_MARGIN = 0.5e-3


def sweep_part(family: str, r: float, d: float, ang: float, ratio: float, f: float = 2.0e-3):
    """One part of the sweep and the room its walls leave: (part, inner - w),
    with w the inward distance from the rim at which the floor fillet ends
    and inner the least inward distance of the footprint's medial axis (the
    truncated cone's top radius; the ellipse's b^2 / a, where the axis'
    ridge ends; the rounded rectangle's smaller half-width or corner
    radius). Where that room is negative the walls meet in a crease instead
    of a floor; a dome has none."""
    from .parts import Dome, EllipticCone, Pyramid, TruncatedCone

    if family == "dome":
        return Dome(r, min(d, 0.9 * r), f, 1.0 / ratio), math.inf
    cone = TruncatedCone.with_footprint(r, ang, d, f, f)
    w = cone.profile.w_last
    if family == "truncated_cone":
        return cone, cone.top_radius - w
    t = -cone.profile.w_first
    if family == "elliptic_cone":
        a, b = r - t, (r - t) / ratio
        return EllipticCone(a, b, ang, d, f, f), b * b / a - w
    half = (r - t) / math.sqrt(2.0)
    hy = half / ratio ** 0.5
    rc = min(hy, max(w + SWEEP_FLOOR_MARGIN, 0.5 * half))
    return Pyramid(half, hy, ang, d, rc, f, f), min(hy, rc) - w


def sweep_parts(count: int = 64, seed: int = 20260, layers: int = 2):
    """The design sweep's parts: a scrambled Sobol sequence (scipy's, seeded)
    over the family, footprint radius 7.5-10 mm, depth 2-4 mm, wall angle
    30-55 degrees, elliptic axis ratio 1.0-1.6 and the mesh size, 20k-150k
    Hex8 in `layers` layers over a square blank 2.6 footprint radii wide, 1
    mm thick. Fillets are 2 mm at rim and floor. A shallow wall does not fit
    a narrow footprint at full depth (a 30 degree wall 4 mm deep runs 6.9
    mm): where the walls would meet in a crease, the part takes the largest
    depth that leaves its floor SWEEP_FLOOR_MARGIN clear of the medial axis
    (a sheet laid on a crease folds within one element). Returns a list of
    (part, mesh)."""
    from scipy.stats import qmc

    pts = qmc.Sobol(d=6, scramble=True, seed=seed).random(count)
    b = SWEEP_BOUNDS

    def lerp(u, k):
        lo, hi = b[k]
        return lo + u * (hi - lo)

    out = []
    for u in pts:
        family = SWEEP_FAMILIES[min(int(u[0] * 4), 3)]
        r, d, ang = lerp(u[1], "footprint_radius"), lerp(u[2], "depth"), lerp(u[3], "wall_angle_deg")
        ratio = lerp(u[4], "axis_ratio")
        part, room = sweep_part(family, r, d, ang, ratio)
        if room < SWEEP_FLOOR_MARGIN:
            # The shallowest depth whose fillets fit the wall (below it they
            # overlap), then the deepest above it with a clear floor.
            lo, hi = 0.0, d
            for _ in range(50):
                mid = 0.5 * (lo + hi)
                try:
                    sweep_part(family, r, mid, ang, ratio)
                    hi = mid
                except ValueError:
                    lo = mid
            lo, hi = hi, d
            for _ in range(50):
                mid = 0.5 * (lo + hi)
                if sweep_part(family, r, mid, ang, ratio)[1] >= SWEEP_FLOOR_MARGIN:
                    lo = mid
                else:
                    hi = mid
            part, room = sweep_part(family, r, lo, ang, ratio)
        ne = int(lerp(u[5], "elements"))
        n = max(8, int(round(math.sqrt(ne / layers))))
        blank = 2.6 * r
        mesh = structured_hex_mesh(n, n, layers, blank, blank, CONE_THICKNESS, x0=-0.5 * blank, y0=-0.5 * blank,
                                   z0=-CONE_THICKNESS)
        out.append((part, mesh))
    return out


# ---- the CPU-runnable forming run: a dome by a spiral ------------------------

def revolution_spiral(height: Callable, r_max: float, tool_radius: float, step_down: float,
                      spacing: float = 1.0e-3, clearance: float = 2.0e-3, samples: int = 4001):
    """The reference's continuous spiral tool path (spiral_toolpath,
    python/precomp/toolpath.py:395-470) restated for a target of revolution
    z = height(r) (the reference extracts its loops with contourpy, which
    this image lacks; for a surface of revolution every loop is a circle):

    - the drop-cutter centre height c(r) = max over |s - r| <= R of
      height(|s|) + sqrt(R^2 - (s - r)^2), in the meridian plane (a ball
      touches a surface of revolution in the plane through the axis and its
      centre);
    - the levels R - k step_down above the deepest centre height, then one
      step_down / 1000 above it (toolpath.py:288-303), the deepest raised
      until its loop is at least two point spacings long;
    - revolution k falls linearly with its arc length from level k - 1 to
      level k (level 0 is level 1's loop at the sheet plane, where the tip
      touches z = 0), at the radius where c equals the height, starting at
      angle 0 counter-clockwise; a last revolution at the deepest level
      closes the path; approach and retract `clearance` above R.

    Returns (points (n, 3), pseudo-times t = s / total (n,), the pseudo-time
    of the last point on the part)."""
    R = float(tool_radius)
    r = np.linspace(0.0, r_max, samples)
    h = r[1] - r[0]
    offsets = np.arange(-int(R / h), int(R / h) + 1) * h
    cap = np.sqrt(np.maximum(R * R - offsets ** 2, 0.0))
    c = np.empty_like(r)
    for i in range(0, samples, 512):
        s = r[i:i + 512, None] + offsets[None, :]
        c[i:i + 512] = (np.asarray(height(np.abs(s))) + cap[None, :]).max(axis=1)
    c = np.maximum.accumulate(c)  # a bowl: the centre rises outward
    cmin, delta = float(c[0]), 1.0e-3 * step_down
    levels, k = [], 1
    while R - k * step_down > cmin + delta:
        levels.append(R - k * step_down)
        k += 1
    if not levels or levels[-1] - (cmin + delta) > delta:
        levels.append(cmin + delta)

    def radius_at(z):
        return np.interp(z, c, r)

    # A loop shorter than two point spacings cannot be followed; the deepest
    # levels whose loops are that short give way to the lowest height with
    # a followable loop, searched in 64 steps up to the deepest followable
    # level (toolpath.py:306-336, 389-392).
    def followable(z):
        return 2.0 * math.pi * float(radius_at(z)) >= 2.0 * spacing

    j = len(levels) - 1
    while j >= 0 and not followable(levels[j]):
        j -= 1
    if j < len(levels) - 1:
        last = levels[-1]
        above = levels[j] if j >= 0 else R
        dz = (above - last) / 64
        for q in range(64):
            if followable(last + q * dz):
                levels = levels[:j + 1] + [last + q * dz]
                break
        else:
            levels = levels[:j + 1]

    heights = [R] + levels
    radii = [float(radius_at(levels[0]))] + [float(radius_at(z)) for z in levels]
    pts = []
    for k in range(1, len(heights)):
        n = max(3, int(math.ceil(2.0 * math.pi * max(radii[k - 1], radii[k]) / spacing)))
        lam = np.arange(n) / n
        z = heights[k - 1] + lam * (heights[k] - heights[k - 1])
        rad = np.full(n, radii[1]) if k == 1 else radius_at(z)
        pts.append(np.column_stack([rad * np.cos(2 * np.pi * lam), rad * np.sin(2 * np.pi * lam), z]))
    n = max(3, int(math.ceil(2.0 * math.pi * radii[-1] / spacing)))
    lam = np.arange(n + 1) / n
    pts.append(np.column_stack([radii[-1] * np.cos(2 * np.pi * lam), radii[-1] * np.sin(2 * np.pi * lam),
                                np.full(n + 1, heights[-1])]))
    body = np.vstack(pts)
    safe = R + clearance
    points = np.vstack([[body[0, 0], body[0, 1], safe], body, [body[-1, 0], body[-1, 1], safe]])
    step = np.linalg.norm(np.diff(points, axis=0), axis=1)
    keep = np.concatenate([[True], step > 1e-15])
    points = points[keep]
    s = np.concatenate([[0.0], np.cumsum(np.linalg.norm(np.diff(points, axis=0), axis=1))])
    t = s / s[-1]
    return points, t, float(t[-2])


CFG1 = dict(blank=20.0e-3, thickness=1.0e-3, nx=40, nz=2, clamp=1.0e-3, tool_radius=3.0e-3, friction=0.1,
            dome_radius=5.0e-3, dome_depth=2.0e-3, dome_fillet=2.0e-3, step_down=0.5e-3, spacing=1.0e-3,
            max_tool_travel=1.0e-3, swift=(70.0e9, 0.33, 425.0e6, 0.003, 0.29))


def cfg1_deck(**overrides) -> dict:
    """The CPU-runnable forming run as a forming deck (the form the test
    harness's forming driver reads): a 20 x 20 x 1 mm sheet of 40 x 40 x 2
    IM Hex8, its top face at z = 0, clamped in its outer 1 mm band; J2 with
    the Swift law (E 70 GPa, nu 0.33, K 425 MPa, eps0 0.003, n 0.29) through
    from_swift; logarithmic strain; one sphere of radius 3 mm, penalty 10,
    Coulomb 0.1, on the spiral (revolution_spiral, 0.5 mm step-downs, 1 mm
    spacing) to a 10 mm, 2 mm deep dome with a 2 mm rim fillet; then the
    unload in the clamp and the release onto 3-2-1 supports, as the
    reference's deck writer builds them (python/precomp/fea/deck.py:107-179:
    the tool surface inside the clamp, the supports half the clamp margin
    from the blank's corners). No reference output exists for this run."""
    from .material import Material
    from .parts import Dome

    p = dict(CFG1, **overrides)
    b, th, nx, nz, e = p["blank"], p["thickness"], p["nx"], p["nz"], p["clamp"]
    mesh = structured_hex_mesh(nx, nx, nz, b, b, th, x0=-0.5 * b, y0=-0.5 * b, z0=-th)
    E, nu, K, eps0, n = p["swift"]
    mat = Material.from_swift("swift-j2", E, nu, K, eps0, n)
    dome = Dome(p["dome_radius"], p["dome_depth"], p["dome_fillet"])
    points, t, t_form = revolution_spiral(lambda r: dome.height(r, 0 * r), 0.5 * b, p["tool_radius"],
                                          p["step_down"], p["spacing"])
    half = 0.5 * b - e
    clamp = {"name": "clamp", "fix": ["x", "y", "z"], "mode": "hold",
             "region": {"any_of": [{"box": {"xmax": -half}}, {"box": {"xmin": half}}, {"box": {"ymax": -half}},
                                   {"box": {"ymin": half}}]}}
    a = 0.5 * b - 0.5 * e
    supports = [{"name": "support_xyz", "fix": ["x", "y", "z"], "mode": "hold",
                 "region": {"nearest_node": [-a, -a, 0.0]}},
                {"name": "support_yz", "fix": ["y", "z"], "mode": "hold", "region": {"nearest_node": [a, -a, 0.0]}},
                {"name": "support_z", "fix": ["z"], "mode": "hold", "region": {"nearest_node": [-a, a, 0.0]}}]
    return {
        "nodes": mesh.coords.tolist(), "elements": mesh.connectivity.tolist(),
        "material": {"name": mat.name, "youngs_modulus": mat.youngs_modulus, "poisson_ratio": mat.poisson_ratio,
                     "plasticity": {"yield_stress": mat.yield_stress, "hardening_modulus": mat.hardening_modulus,
                                    "saturation_stress": mat.saturation_stress,
                                    "saturation_rate": mat.saturation_rate}},
        "model": {"element_formulation": "incompatible_modes"}, "kinematics": "finite_logarithmic",
        "tools": [{"name": "tool", "shape": "sphere", "radius": p["tool_radius"], "friction": p["friction"],
                   "penalty": 10.0,
                   "surface": {"box": {"zmin": 0.0, "xmin": -half, "xmax": half, "ymin": -half, "ymax": half}},
                   "trajectory": {"times": t.tolist(), "points": points.tolist()}}],
        "steps": [
            {"deck": {"name": "form", "type": "form", "tools": ["tool"], "time": [0.0, t_form],
                      "max_tool_travel": p["max_tool_travel"], "boundary_conditions": [clamp]}},
            {"deck": {"name": "unload", "type": "release", "tools": [], "boundary_conditions": [clamp]}},
            {"deck": {"name": "release", "type": "release", "tools": [], "boundary_conditions": supports}},
        ],
        "dome": dome,
    }
