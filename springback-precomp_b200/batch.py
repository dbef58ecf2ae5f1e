"""Many parts in one element launch: the batched engine of the design-sweep
data generation.

The reference generates its training data by running one forming analysis
per part, each in its own process (python/precomp/fea/runner.py:305-335,
python/precomp/ml/generate.py:144-170), so every Newton iteration of every
part launches its own element loop. Here the parts of a sweep - meshes of
uneven size - form one system over their concatenated element lists: one
element launch per Newton iteration for all of them, with an offset table
that maps every part to its nodes, elements, DOFs and tangent values. The
parts share no node, so the union's node-block pattern is block diagonal
and every part's CSC slice is its own pattern. An evaluation of the batch
can be captured once as a CUDA graph and replayed every iteration, and a
small autotuner picks the element kernel's launch shape for the batch.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence

import numpy as np
import torch

from .material import Material
from .mesh import HexMesh
from .system import Evaluation, NonlinearSystem


@dataclasses.dataclass
class PartView:
    """One part's slices of a batch evaluation (views, no copies)."""

    internal: torch.Tensor  # (3 n_p,) f_int of the part's nodes
    values: Optional[torch.Tensor]  # the part's CSC values
    outer: torch.Tensor  # its column pointers, from 0
    inner: torch.Tensor  # its row indices, from 0


class PartBatch:
    """A batch of parts as one NonlinearSystem. offsets[p] = (first node,
    first element, first DOF, first tangent value) of part p; offsets[P] the
    totals."""

    def __init__(self, meshes: Sequence[HexMesh], material: Material, kinematics: str = "logarithmic",
                 stiffness_points: int = 2, thickness_points: int = 0, thickness_axis: int = 2, stream=None,
                 element: str = "incompatible_modes", mean_dilatation: str = "auto"):
        nodes = np.cumsum([0] + [m.num_nodes for m in meshes])
        elems = np.cumsum([0] + [m.num_elements for m in meshes])
        coords = np.concatenate([m.coords for m in meshes])
        conn = np.concatenate([m.connectivity + int(nodes[p]) for p, m in enumerate(meshes)]).astype(np.int32)
        self.meshes = list(meshes)
        self.mesh = HexMesh(coords, conn)
        self.system = NonlinearSystem(self.mesh, material, kinematics, stiffness_points, thickness_points,
                                      thickness_axis, stream, element=element, mean_dilatation=mean_dilatation)
        outer = self.system.outer.cpu().numpy()
        dofs = 3 * nodes
        self.offsets = np.stack([nodes, elems, dofs, outer[dofs].astype(np.int64)], axis=1)

    @property
    def num_parts(self) -> int:
        return len(self.meshes)

    def evaluate(self, u: torch.Tensor, want_tangent: bool = True) -> Evaluation:
        """All parts at once (NonlinearSystem.evaluate of the union)."""
        return self.system.evaluate(u, 0.0, want_tangent)

    def part(self, p: int, internal: torch.Tensor, values: Optional[torch.Tensor] = None) -> PartView:
        n0, _, d0, v0 = self.offsets[p]
        n1, _, d1, v1 = self.offsets[p + 1]
        outer = self.system.outer[d0:d1 + 1] - int(v0)
        return PartView(internal=internal[d0:d1], values=None if values is None else values[v0:v1], outer=outer,
                        inner=self.system.inner[v0:v1] - int(d0))

    def gather(self, parts_u: Sequence[torch.Tensor]) -> torch.Tensor:
        """The batch's displacement from the parts' ones."""
        return torch.cat([u.reshape(-1) for u in parts_u])

    def autotune(self, u: torch.Tensor, candidates=(("phases", 0), ("phases", 8), ("single", 16), ("single", 8)),
                 repeats: int = 2, want_tangent: bool = True):
        """Time the element loop at each candidate mapping on this batch -
        (local iteration, elements per block): the phase kernels (a thread
        per point in the point kernels, an 8-lane group per element in the
        others) or the single kernel (an 8-lane group per element, a point
        per lane, start to finish), each at a block shape - with CUDA events
        on the system's stream after one warm-up; keep the fastest and
        return {candidate: ms}. No result depends on the choice. A bare
        integer candidate is an elements-per-block of the current mode."""
        self.system.set_timing(True)
        times = {}
        for cand in candidates:
            mode, epb = cand if isinstance(cand, tuple) else (None, cand)
            if mode is not None:
                self.system.set_local_iteration(mode)
            self.system.set_elements_per_block(epb)
            self.system.evaluate(u, 0.0, want_tangent)
            best = float("inf")
            for _ in range(repeats):
                self.system.evaluate(u, 0.0, want_tangent)
                best = min(best, self.system.last_timings()["element"])
            times[cand] = best
        choice = min(times, key=times.get)
        mode, epb = choice if isinstance(choice, tuple) else (None, choice)
        if mode is not None:
            self.system.set_local_iteration(mode)
        self.system.set_elements_per_block(epb)
        self.chosen = choice
        self.chosen_elements_per_block = epb
        return times


class GraphedEvaluation:
    """One evaluation of a system captured as a CUDA graph and replayed each
    Newton iteration: the element kernel, the gathers, the schedule and the
    summary with no host work between them. The displacement is read from
    `u`, a device buffer the caller updates in place; the results are the
    system's internal_view() / values_view() and `summary` (energy, gross,
    yielding points, lowest failing element or -1, its code). The system
    commits by copying (stable buffers), so the graph stays valid across
    commits."""

    def __init__(self, system: NonlinearSystem, u: torch.Tensor, want_tangent: bool = True):
        self.system = system
        self.u = u
        system.set_stable_buffers(True)
        system.evaluate(u, 0.0, want_tangent)  # the schedule and the launch attributes, before capture
        self.summary = torch.zeros(5, dtype=torch.float64, device=u.device)
        stream = torch.cuda.Stream(device=u.device)
        stream.wait_stream(torch.cuda.current_stream(u.device))
        self.graph = torch.cuda.CUDAGraph()
        system.set_stream(stream)
        try:
            with torch.cuda.stream(stream):
                system.enqueue(u, want_tangent, self.summary)  # warm-up on the capture stream
                stream.synchronize()
                with torch.cuda.graph(self.graph, stream=stream):
                    system.enqueue(u, want_tangent, self.summary)
        finally:
            system.set_stream(None)
        torch.cuda.current_stream(u.device).wait_stream(stream)

    def replay(self) -> torch.Tensor:
        self.graph.replay()
        return self.summary
