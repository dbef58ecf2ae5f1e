"""An oracle-backed stand-in for the package's NonlinearSystem and
ToolContact - test infrastructure, not part of the product. It lets the
forming harness (forming_harness.FormingRun) run a deck on the CPU: every
element evaluation, assembly and contact evaluation is the oracle's
restatement of the reference's (oracle_system.cpp), the solves scipy's (the
harness's solver="host"). A deck's run on the CPU this way shows how its
increments converge without a GPU; the numbers are the oracle's, so they
stand for what the GPU run computes to round-off.

Only the members the harness calls are provided: evaluate, add_node_blocks,
commit, stress, inner / outer and symmetric of the system; begin_increment,
evaluate, anticipate and commit of the contact.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch


@dataclasses.dataclass
class _Evaluation:
    internal: torch.Tensor
    residual: torch.Tensor
    tangent: torch.Tensor
    energy: float
    gross: float
    yielding_points: int


@dataclasses.dataclass
class _Stress:
    von_mises: torch.Tensor
    max_plastic_strain: torch.Tensor


@dataclasses.dataclass
class _ContactEvaluation:
    residual: torch.Tensor
    nodes: np.ndarray
    blocks: np.ndarray
    tools: np.ndarray
    symmetric: bool


class _System:
    def __init__(self, backend, mesh, material, kinematics, thickness_points, thickness_axis):
        self.b = backend
        self.orc = backend.orc
        self.mesh = mesh
        self.m = material.as_dict()
        self.kin = kinematics
        self.tp, self.axis = thickness_points, thickness_axis
        self.coords = mesh.coords
        self.conn = mesh.connectivity
        self.pat = self.orc.pattern(mesh.num_nodes, mesh.connectivity)
        self.inner = torch.from_numpy(np.asarray(self.pat["inner"]))
        self.outer = torch.from_numpy(np.asarray(self.pat["outer"]))
        nq = self.orc.rule_size(2, thickness_points, thickness_axis)
        self.committed = np.zeros((mesh.num_elements, nq, self.orc.NF))
        self.alpha = np.zeros((mesh.num_elements, 9))
        self.trial = None
        self.values = np.zeros(self.pat["nnz"])
        self.evaluations = 0

    def evaluate(self, u, t, want_tangent=True):
        r = self.orc.system_evaluate(self.m, self.coords, self.conn, np.asarray(u.cpu(), dtype=np.float64),
                                     self.committed, self.alpha, kinematics=self.kin, thickness=self.tp,
                                     axis=self.axis, want_tangent=bool(want_tangent), threads=self.b.threads,
                                     pat=self.pat)
        self.evaluations += 1
        if r["code"] != 0:
            raise self.b.SolverError(4, f"Hex8 element {r['failed_element']}: SolverError (code {r['code']})",
                                     r["failed_element"], r["code"])
        self.trial = (r["states"], r["alpha"])
        if want_tangent:  # as the package: no tangent asked, the last one stays
            self.values[:] = r["values"]
        internal = torch.from_numpy(r["internal"])
        return _Evaluation(internal=internal, residual=internal, tangent=torch.from_numpy(self.values),
                           energy=r["energy"], gross=r["gross"], yielding_points=r["yielding_points"])

    def add_node_blocks(self, nodes, blocks):
        self.values[:] = self.orc.add_node_blocks(self.pat, self.values, np.asarray(nodes), np.asarray(blocks))

    def commit(self):
        self.committed, self.alpha = self.trial

    def symmetric(self):
        return False

    def stress(self, u):
        ue = self.mesh.gather(np.asarray(u.cpu(), dtype=np.float64))
        out, st = self.orc.element_stress(self.m, self.mesh.element_coordinates(), ue, self.committed, self.alpha,
                                          kinematics=self.kin, thickness=self.tp, axis=self.axis,
                                          threads=self.b.threads)
        return _Stress(von_mises=torch.from_numpy(out[:, 12].copy()),
                       max_plastic_strain=torch.from_numpy(out[:, 13].copy()))


class _Contact:
    def __init__(self, backend, mesh, tools, friction_tangent):
        recs = [dict(shape=t.shape, radius=t.radius, friction=t.friction, tangential_ratio=t.tangential_ratio,
                     normal=tuple(t.normal), axis=tuple(t.axis), times=list(t.times),
                     points=[list(p) for p in t.points], nodes=list(t.nodes), area=list(t.area),
                     kappa=list(t.kappa)) for t in tools]
        self.c = backend.orc.Contact(mesh.coords, recs, friction_tangent=friction_tangent)

    def begin_increment(self, u0, t0, t1, active, margin):
        return self.c.begin_increment(np.asarray(u0.cpu(), dtype=np.float64), t0, t1, list(active), margin)

    def evaluate(self, u, t, want_tangent=True):
        r = self.c.evaluate(np.asarray(u.cpu(), dtype=np.float64), t, want_tangent)
        if r["code"] != 0:
            raise RuntimeError("the oracle's contact failed (a node deep inside a tool)")
        return _ContactEvaluation(residual=torch.from_numpy(r["residual"]), nodes=r["nodes"], blocks=r["blocks"],
                                  tools=r["tools"], symmetric=r["symmetric"])

    def anticipate(self, u, du, t, residual):
        res, nodes, blocks = self.c.anticipate(np.asarray(u.cpu(), dtype=np.float64),
                                               np.asarray(du.cpu(), dtype=np.float64), t,
                                               np.asarray(residual.cpu(), dtype=np.float64))
        residual.copy_(torch.from_numpy(res))
        return len(nodes), nodes, blocks

    def commit(self):
        self.c.commit()


class OracleBackend:
    """What FormingRun takes as its package: the package's own mesh,
    material, tool and error types, the oracle's system and contact."""

    def __init__(self, pkg, orc, threads: int = 0):
        self.orc = orc
        self.threads = threads
        self.HexMesh = pkg.HexMesh
        self.Material = pkg.Material
        self.Tool = pkg.Tool
        self.SolverError = pkg.SolverError

    def NonlinearSystem(self, mesh, material, kinematics="logarithmic", thickness_points=0, thickness_axis=2,
                        element="incompatible_modes", mean_dilatation="auto"):
        if element != "incompatible_modes":
            raise NotImplementedError("the oracle backend runs the incompatible-mode Hex8")
        return _System(self, mesh, material, kinematics, thickness_points, thickness_axis)

    def ToolContact(self, mesh, tools, friction_tangent="exact"):
        return _Contact(self, mesh, tools, friction_tangent)
