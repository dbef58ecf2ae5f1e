"""A forming driver for the end-to-end tests - test infrastructure, not part
of the product. It stands in for the reference's FormingAnalysis::run
(src/fem/Forming.cpp:686-1262), which calls the element loop and the contact
every Newton iteration: it runs a committed forming deck of the reference
through this package's NonlinearSystem, ToolContact and PartitionedFactor on
the GPU - the free-free block gathered and factorised on the device (or,
with solver="host", scipy's sparse LU on the host).

What it restates of the driver, because the converged states depend on it:
the step partition (prescribed DOFs held at their values, Forming.cpp:804-821),
the start imbalance r0 ramped out over the step (:829-846, :890-897), the
increment schedule (the tool travel per increment and the stations,
:1149-1163), the cut of an increment whose Newton iteration fails - an
element's SolverError from the GPU or no convergence - halved and retried,
with the growth after a quick one (:1165-1247), and the commit of every
converged increment (:1208-1215). What
it does not restate, because it only changes the path to the same converged
state: the predictor, the energy line search (a residual backtracking here),
and the tolerances (the iteration here runs to a correction of 1e-13 m,
1e-11 m after 40 iterations, well inside the reference's relative 1e-6). Its
Newton iteration follows the reference's: the semismooth anticipation of
contact and the line search on du . R, which keep the iterates where every
element's local iteration converges.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.sparse
import scipy.sparse.linalg
import torch


def in_region(x: np.ndarray, region: dict, tol: float) -> np.ndarray:
    """Selector::contains (src/fem/Selector.cpp:49-56) of a deck region:
    boxes inclusive with the tolerance, `all`, `any_of`."""
    if region.get("all"):
        return np.ones(len(x), dtype=bool)
    if "nearest_node" in region:  # the node nearest a point (the first of equals)
        out = np.zeros(len(x), dtype=bool)
        out[int(np.argmin(np.linalg.norm(x - np.asarray(region["nearest_node"], float), axis=1)))] = True
        return out
    if "any_of" in region:
        out = np.zeros(len(x), dtype=bool)
        for r in region["any_of"]:
            out |= in_region(x, r, tol)
        return out
    box = region["box"]
    inf = np.inf
    lo = [box.get("xmin", -inf), box.get("ymin", -inf), box.get("zmin", -inf)]
    hi = [box.get("xmax", inf), box.get("ymax", inf), box.get("zmax", inf)]
    ok = np.ones(len(x), dtype=bool)
    for k in range(3):
        ok &= (x[:, k] >= lo[k] - tol) & (x[:, k] <= hi[k] + tol)
    return ok


def top_face_slaves(nodes: np.ndarray, elements: np.ndarray, region: dict, tol: float):
    """The slave nodes of a tool and their tributary areas: the boundary
    faces whose every node lies in the tool's surface region, each face's
    shape-function integrals added to its nodes (ToolContact's constructor,
    src/fem/RigidTool.cpp:292-321). For the flat quadrilateral faces of a
    structured sheet every node of a face takes a quarter of its area."""
    faces = {}
    local = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
    for e, conn in enumerate(elements):
        for f in local:
            key = tuple(sorted(conn[list(f)]))
            faces.setdefault(key, []).append((e, [conn[i] for i in f]))
    inside = in_region(nodes, region, tol)
    area = {}
    for key, owners in sorted(faces.items()):
        if len(owners) != 1:
            continue  # an interior face
        quad = owners[0][1]
        if not all(inside[n] for n in quad):
            continue
        p = nodes[quad]
        a = 0.5 * np.linalg.norm(np.cross(p[2] - p[0], p[3] - p[1]))  # a planar quadrilateral
        for n in quad:
            area[n] = area.get(n, 0.0) + 0.25 * a
    ids = np.array(sorted(area), dtype=np.int32)
    return ids, np.array([area[i] for i in ids])


@dataclasses.dataclass
class StepResult:
    u: np.ndarray
    increments: int
    tool_fz: list
    # The step-end element fields the reference writes
    # (step_<k>_<s>_elements.csv): the largest equivalent plastic strain of
    # each element's points and the von Mises stress of its point-averaged
    # Cauchy stress, from the package's stress recovery at the end of the step
    # (Forming.cpp:1266-1281).
    eq_plastic_strain: np.ndarray = None
    von_mises: np.ndarray = None
    cuts: int = 0


class NewtonFailure(RuntimeError):
    """An increment's Newton iteration that did not converge."""


# The increment control of the forming driver (Forming.cpp:37-39, 1149-1247):
# a failed increment is halved, at most MAX_CUTS times in a row; an increment
# that converged in at most QUICK_ITERATIONS lets the next grow by GROWTH, up
# to the step's cap.
MAX_CUTS = 10
QUICK_ITERATIONS = 4
GROWTH = 1.5


class FormingRun:
    def __init__(self, pkg, fixture: dict, device, solver: str = "device", growth_test: str = "own",
                 tolerance: str = "own"):
        """growth_test: which Newton iteration count decides the growth of
        the next increment after a quick one - "own", the iterations to this
        harness's correction of 1e-13 m (the replays of the reference's runs
        use it), or "reference", the iterations until a full step's
        correction is within the reference's displacement tolerance, 1e-6 of
        the increment (Forming.cpp:914-921, 1112; displacement_tolerance,
        include/sparlab/fem/Forming.hpp:184): the iterations the reference
        counts, so that a run on the harness's own schedule grows back
        after a cut as the reference's does.

        tolerance: where an increment's Newton iteration stops - "own", a
        full step's correction of 1e-13 m (1e-11 m after 40 iterations),
        which the replays of the reference's committed runs need to meet its
        states to 1e-8 m; or "reference", the first full step whose
        correction is within the reference's displacement tolerance (1e-6 of
        the increment), for a run that no reference output is compared with
        and whose cost should be the reference driver's."""
        self.pkg = pkg
        self.solver = solver
        if growth_test not in ("own", "reference"):
            raise ValueError("growth_test must be 'own' or 'reference'")
        self.growth_test = growth_test
        if tolerance not in ("own", "reference"):
            raise ValueError("tolerance must be 'own' or 'reference'")
        self.tolerance = tolerance
        self.reference_iterations = 0
        self.part = None
        self.contact_symmetric = True
        self.fx = fixture
        self.dev = device
        self.nodes = np.array(fixture["nodes"], dtype=np.float64)
        self.elements = np.array(fixture["elements"], dtype=np.int32)
        self.mesh = pkg.HexMesh(self.nodes, self.elements)
        m = fixture["material"]
        pl = m["plasticity"]
        extra = {}
        if pl.get("yield_criterion") == "hill48":
            an = pl["anisotropy"]
            extra.update(criterion="hill48", r0=an["r0"], r45=an["r45"], r90=an["r90"],
                         rolling_direction=tuple(an.get("rolling_direction", (1.0, 0.0, 0.0))),
                         sheet_normal=tuple(an.get("sheet_normal", (0.0, 0.0, 1.0))))
        if pl.get("backstresses"):
            extra["backstresses"] = tuple((b["modulus"], b["recovery"]) for b in pl["backstresses"])
        self.material = pkg.Material(m["youngs_modulus"], m["poisson_ratio"], yield_stress=pl["yield_stress"],
                                     hardening_modulus=pl["hardening_modulus"],
                                     kinematic_hardening_modulus=pl.get("kinematic_hardening_modulus", 0.0),
                                     saturation_stress=pl["saturation_stress"],
                                     saturation_rate=pl["saturation_rate"], name=m["name"], **extra)
        kin = {"finite_logarithmic": "logarithmic", "finite": "finite", "small_strain": "small"}[fixture["kinematics"]]
        integ = fixture.get("model", {}).get("integration", {})
        tp = int(integ.get("thickness_points", 0))
        axis = "xyz".index(integ.get("thickness_direction", "z"))
        # The model's element formulation (the standard Hex8 unless it names
        # incompatible modes) and the forming block's mean dilatation.
        element = ("incompatible_modes" if fixture.get("model", {}).get("element_formulation") == "incompatible_modes"
                   else "standard")
        self.system = pkg.NonlinearSystem(self.mesh, self.material, kinematics=kin, thickness_points=tp,
                                          thickness_axis=axis, element=element,
                                          mean_dilatation=fixture.get("mean_dilatation", "auto"))
        extent = self.nodes.max(0) - self.nodes.min(0)
        self.tol = 1e-9 * float(np.linalg.norm(extent))
        self.tools = []
        self.paths = []
        for t in fixture["tools"]:
            ids, area = top_face_slaves(self.nodes, self.elements, t["surface"], self.tol)
            kappa = t.get("penalty", 10.0) * self.material.youngs_modulus / np.sqrt(area)
            tr = t["trajectory"]
            self.paths.append((np.array(tr["times"], float), np.array(tr["points"], float)))
            self.tools.append(pkg.Tool(shape=t["shape"], times=tr["times"], points=tr["points"], nodes=ids,
                                       area=area, kappa=kappa, radius=t.get("radius", 0.0),
                                       friction=t.get("friction", 0.0), axis=t.get("axis", (0.0, 0.0, 1.0)),
                                       normal=t.get("normal", (0.0, 0.0, 1.0)), name=t["name"]))
        self.min_size = float(np.sqrt(min(tl.area.min() for tl in self.tools))) if self.tools else 1.0
        self.contact = pkg.ToolContact(self.mesh, self.tools, friction_tangent="exact") if self.tools else None
        self.u = np.zeros(self.mesh.num_dofs)
        self.t = 0.0
        self.last_du = 0.0
        # Host-side fault injection for tests: the numbers (1-based, counted
        # over the run) of the increment attempts whose first evaluation
        # raises the SolverError of an element's local iteration, as the GPU
        # reports it.
        self.inject_at = set()
        self.attempts = 0
        self.times = []

    # -- pieces of one Newton iteration -------------------------------------
    def _residual(self, u, t, active, tangent):
        """f_int + the contact residual, with the contact node blocks added
        into the system tangent (Forming.cpp:986-990)."""
        ev = self.system.evaluate(torch.tensor(u, device=self.dev), 0.0, tangent)
        r = ev.residual.double().cpu().numpy().copy()
        fz = 0.0
        if tangent:
            self.contact_symmetric = True
        if self.contact is not None and any(active):
            cev = self.contact.evaluate(torch.tensor(u, device=self.dev), t, tangent)
            r += cev.residual.cpu().numpy()
            fz = float(sum(cev.tools[k][5] for k in range(len(active)) if active[k]))
            if tangent:
                self.contact_symmetric = cev.symmetric
            if tangent and len(cev.nodes):
                self.system.add_node_blocks(cev.nodes, cev.blocks)
        return ev, r, fz

    def _solve(self, ev, free, rhs):
        """K_ff x = rhs as Forming.cpp:1000-1016 and :1043-1050 solve it:
        the free-free block of the current tangent (node blocks included)
        assembled and factorised - on the device by the package's
        PartitionedFactor, symmetric when the system and the contact are -
        or with scipy's sparse LU on the host."""
        if self.solver == "host":
            n = self.mesh.num_dofs
            k = scipy.sparse.csc_matrix((ev.tangent.cpu().numpy(), self.system.inner.cpu().numpy(),
                                         self.system.outer.cpu().numpy()), shape=(n, n))
            return scipy.sparse.linalg.spsolve(k[free][:, free].tocsc(), rhs)
        if self.part is None or not self.part.same_partition(free):
            self.part = self.pkg.PartitionedFactor.for_system(self.system, free)
        self.part.factorize(ev.tangent, self.system.symmetric() and self.contact_symmetric)
        return self.part.solve(torch.as_tensor(np.ascontiguousarray(rhs), device=self.dev)).cpu().numpy()

    def _speed(self, t, active):
        v = 0.0
        for k, (times, pts) in enumerate(self.paths):
            if not active[k]:
                continue
            i = min(max(np.searchsorted(times, t, side="right") - 1, 0), len(times) - 2)
            v = max(v, np.linalg.norm(pts[i + 1] - pts[i]) / (times[i + 1] - times[i]))
        return v

    def run_step(self, k: int, times=None) -> StepResult:
        """Step k of the deck. `times`: the end times of the increments the
        reference accepted (its tool_forces.csv), to follow its increment
        sequence through the cuts its own Newton iterations made; else the
        schedule of Forming.cpp:1149-1163 without cuts."""
        st = self.fx["steps"][k]["deck"]
        names = [t["name"] for t in self.fx["tools"]]
        active = [n in st.get("tools", []) for n in names]
        release = st["type"] == "release"
        tb, te = (st["time"] if "time" in st else (self.t, self.t + 1.0))
        duration = te - tb
        fixed = np.zeros(self.mesh.num_dofs, dtype=bool)
        for bc in st["boundary_conditions"]:
            sel = in_region(self.nodes, bc["region"], self.tol)
            for comp in bc["fix"]:
                fixed[3 * np.where(sel)[0] + "xyz".index(comp)] = True
        free = np.where(~fixed)[0]
        # The start imbalance on the step's free DOFs.
        if self.contact is not None:
            self.contact.begin_increment(torch.tensor(self.u, device=self.dev), tb, tb, active, np.inf)
        _, r, _ = self._residual(self.u, tb, active, False)
        r0 = r[free]
        stations = sorted({tt for kk, (times, _) in enumerate(self.paths) if active[kk]
                           for tt in times if tb < tt <= te} | {te})
        parts = st.get("increments", 0) or (10 if release else 1)
        dt_max = duration / parts
        travel = st.get("max_tool_travel", 0.0) or 0.5 * self.min_size
        t, dt, count, fz_list = tb, dt_max, 0, []
        if times is not None:
            for t1 in times:
                s1 = 1.0 if t1 == te else (t1 - tb) / duration
                fz_list.append(self._newton(t, t1, s1, free, r0, active)[0])
                t = t1
            assert t == te, (t, te)
            self.t = te
            return self._step_end(StepResult(u=self.u.copy(), increments=len(times), tool_fz=fz_list))
        cuts = cuts_in_a_row = 0
        self.times = []
        while True:
            station = next(s for s in stations if s > t)
            h = min(dt, dt_max)
            speed = self._speed(t, active)
            if speed > 0:
                h = min(h, travel / speed)
            reach = station - t <= h * (1.0 + 1.0e-6)
            t1 = station if reach else t + h
            s1 = 1.0 if (reach and station == te) else (t1 - tb) / duration
            try:
                fz, iterations = self._newton(t, t1, s1, free, r0, active)
            except (self.pkg.SolverError, NewtonFailure) as err:
                # The increment is cut: halved and retried from the last
                # converged state (Forming.cpp:1173-1194).
                cuts += 1
                cuts_in_a_row += 1
                if cuts_in_a_row > MAX_CUTS:
                    raise NewtonFailure(f"an increment from t = {t} failed after {MAX_CUTS} halvings: {err}")
                dt = 0.5 * (t1 - t)
                continue
            fz_list.append(fz)
            self.times.append(t1)
            count += 1
            t = t1
            counted = iterations if self.growth_test == "own" else self.reference_iterations
            if counted <= QUICK_ITERATIONS:
                dt = min(GROWTH * dt, dt_max)
            cuts_in_a_row = 0
            if s1 >= 1.0:
                break
        self.t = te
        return self._step_end(StepResult(u=self.u.copy(), increments=count, tool_fz=fz_list, cuts=cuts))

    def _step_end(self, res: StepResult) -> StepResult:
        """The step-end stress recovery of every element at the converged
        displacement and the committed history."""
        st = self.system.stress(torch.tensor(self.u, device=self.dev))
        res.eq_plastic_strain = st.max_plastic_strain.cpu().numpy()
        res.von_mises = st.von_mises.cpu().numpy()
        return res

    def _newton(self, t0, t1, s1, free, r0, active):
        """One increment: Newton's method as Forming.cpp:900-1135 runs it -
        the semismooth anticipation of nodes the correction drives into a
        tool (:1017-1046), the line search on the energy du . R(a) with the
        full step's evaluation kept (:916-960, :1057-1075) - iterated here to
        a correction of 1e-13 m."""
        ramp = 1.0 - s1
        trial = self.u.copy()
        self.attempts += 1
        if self.attempts in self.inject_at:
            # The GPU's report of an element whose local iteration did not
            # converge (sbk_system_evaluate's SBK_ERR_SOLVER with the element
            # and code 3), made on the host.
            raise self.pkg.SolverError(4, "Hex8 element 0: SolverError (code 3), injected", 0, 3)
        any_tool = self.contact is not None and any(active)
        if self.contact is not None:
            self.contact.begin_increment(torch.tensor(self.u, device=self.dev), t0, t1, active,
                                         2.0 * 1e-3 + 2.0 * self.last_du + self.min_size)

        def g_at(x, du, tangent):
            try:
                ev, r, _ = self._residual(x, t1, active, tangent)
            except self.pkg.SolverError:
                return None, None, np.nan
            return ev, r, float(du @ (r[free] - ramp * r0))

        history = []
        self.reference_iterations = 0
        have = None  # the full step's evaluation with its tangent, when kept
        for it in range(300):
            if have is None:
                ev, r, _ = self._residual(trial, t1, active, True)
            else:
                ev, r = have
            have = None
            rf = r[free] - ramp * r0
            du = self._solve(ev, free, -rf)
            if any_tool:
                du_full = np.zeros(self.mesh.num_dofs)
                du_full[free] = du
                extra = torch.zeros(self.mesh.num_dofs, dtype=torch.float64, device=self.dev)
                added, nodes, blocks = self.contact.anticipate(torch.tensor(trial, device=self.dev),
                                                               torch.tensor(du_full, device=self.dev), t1, extra)
                if added > 0:
                    n0 = len(nodes) - added
                    self.system.add_node_blocks(nodes[n0:], blocks[n0:])
                    again = self._solve(ev, free, -(rf + extra.cpu().numpy()[free]))
                    if np.all(np.isfinite(again)):
                        du = again
            g0 = float(du @ rf)
            alpha = 1.0
            if g0 < 0.0:
                probe = trial.copy()
                probe[free] += du
                nxt, r_next, g1 = g_at(probe, du, True)
                a_hi, g_hi = 1.0, g1
                for _ in range(6):
                    if np.isfinite(g_hi):
                        break
                    a_hi *= 0.5
                    probe = trial.copy()
                    probe[free] += a_hi * du
                    nxt, r_next, g_hi = None, None, g_at(probe, du, False)[2]
                if not np.isfinite(g_hi) or abs(g_hi) <= 0.8 * abs(g0) or g_hi < 0.0:
                    alpha = a_hi
                else:
                    a_lo, g_lo, best = 0.0, g0, a_hi
                    for _ in range(5):
                        a = min(max(a_lo - g_lo * (a_hi - a_lo) / (g_hi - g_lo), 0.1 * a_hi), a_hi)
                        probe = trial.copy()
                        probe[free] += a * du
                        nxt, ga = None, g_at(probe, du, False)[2]
                        if not np.isfinite(ga):
                            a_hi, g_hi = a, abs(g0)
                            continue
                        best = a
                        if abs(ga) <= 0.8 * abs(g0):
                            break
                        if ga < 0.0:
                            a_lo, g_lo = a, ga
                        else:
                            a_hi, g_hi = a, ga
                    alpha = best
                if alpha == 1.0 and nxt is not None:
                    have = (nxt, r_next)  # the full step's evaluation, with its tangent: the next iteration's
            trial[free] += alpha * du
            step = alpha * np.abs(du).max()
            history.append((float(np.linalg.norm(rf)), float(step), alpha))
            if not self.reference_iterations and alpha == 1.0 and \
                    np.linalg.norm(du) <= 1.0e-6 * np.linalg.norm(trial[free] - self.u[free]):
                self.reference_iterations = it + 1
                if self.tolerance == "reference":
                    break
            if (alpha == 1.0 and step <= 1e-13) or (it >= 40 and step <= 1e-11):
                break
        else:
            raise NewtonFailure(f"the increment to t = {t1} did not converge: (|R|, step, alpha) {history[-8:]}")
        if not self.reference_iterations:
            self.reference_iterations = it + 1
        # The accepted state's own evaluation makes its trial history the one committed.
        _, _, fz = self._residual(trial, t1, active, False)
        self.system.commit()
        if self.contact is not None:
            self.contact.commit()
        self.last_du = float(np.abs((trial - self.u).reshape(-1, 3)).max())
        self.u = trial
        return fz, it + 1
