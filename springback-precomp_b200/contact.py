"""Penalty contact with rigid tools behind the reference's ToolContact
interface (include/sparlab/fem/RigidTool.hpp:248-320): begin_increment,
evaluate, anticipate, commit, history. The slave nodes of each tool, their
tributary areas and penalty stiffnesses are inputs, as ToolContact's
constructor computes them once from the face geometry
(src/fem/RigidTool.cpp:275-333)."""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _capi
from .mesh import HexMesh
from .system import _ptr, _stream_ptr, device_view

SHAPES = {"sphere": 0, "plane": 1, "cylinder": 2}


@dataclasses.dataclass
class Tool:
    shape: str
    times: Sequence[float]
    points: Sequence[Sequence[float]]
    nodes: Sequence[int]
    area: Sequence[float]
    kappa: Sequence[float]
    radius: float = 0.0
    friction: float = 0.0
    tangential_ratio: float = 1.0
    normal: Sequence[float] = (0.0, 0.0, 1.0)
    axis: Sequence[float] = (0.0, 0.0, 1.0)
    name: str = "tool"


@dataclasses.dataclass
class ContactEvaluation:
    residual: torch.Tensor  # full length: minus the contact forces
    nodes: torch.Tensor     # block nodes, tool then slave order
    blocks: torch.Tensor    # (n, 3, 3): d(residual)/du of the node's own components
    tools: np.ndarray       # per tool: centre xyz, force xyz, active, slipping, max penetration
    gross: float
    round_off: float
    force_norm: float
    symmetric: bool


class ToolContact:
    def __init__(self, mesh: HexMesh, tools: List[Tool], friction_tangent: str = "exact", stream=None):
        self.mesh = mesh
        self.tools = tools
        self._coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
        self._conn = np.ascontiguousarray(mesh.connectivity, dtype=np.int32)
        m = _capi.sbk_mesh()
        m.num_nodes = mesh.num_nodes
        m.num_elements = mesh.num_elements
        m.coords = self._coords.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        m.connectivity = self._conn.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        arr = (_capi.sbk_tool * max(1, len(tools)))()
        self._keep = []
        for k, t in enumerate(tools):
            times = np.ascontiguousarray(t.times, dtype=np.float64)
            pts = np.ascontiguousarray(np.asarray(t.points, dtype=np.float64).reshape(-1, 3))
            nodes = np.ascontiguousarray(t.nodes, dtype=np.int32)
            area = np.ascontiguousarray(t.area, dtype=np.float64)
            kappa = np.ascontiguousarray(t.kappa, dtype=np.float64)
            if not (len(nodes) == len(area) == len(kappa)) or len(times) != len(pts):
                raise ValueError(f"tool {t.name}: inconsistent sizes")
            if len(nodes) > 1 and np.any(np.diff(nodes) <= 0):
                raise ValueError(f"tool {t.name}: slave nodes must ascend")
            self._keep += [times, pts, nodes, area, kappa]
            c = arr[k]
            c.shape = SHAPES[t.shape]
            c.num_knots = len(times)
            c.num_slaves = len(nodes)
            c.radius, c.friction, c.tangential_ratio = t.radius, t.friction, t.tangential_ratio
            for i in range(3):
                c.normal[i] = t.normal[i]
                c.axis[i] = t.axis[i]
            c.times = times.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            c.points = pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            c.nodes = nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            c.area = area.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            c.kappa = kappa.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        h = ctypes.c_void_p()
        _capi.check(_capi.lib().sbk_contact_create(ctypes.byref(m), len(tools), arr,
                                                   1 if friction_tangent == "symmetric" else 0, ctypes.byref(h)))
        self._h = h
        self.set_stream(stream)

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().sbk_contact_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream=None):
        _capi.check(_capi.lib().sbk_contact_set_stream(self._h, _stream_ptr(stream)))

    def set_search(self, mode: str = "grid"):
        """How begin_increment finds the candidates: "grid" (the default: a
        uniform-grid hash of the slave nodes for spherical tools) or "scan"
        (every slave node tested). The same candidates either way."""
        _capi.check(_capi.lib().sbk_contact_set_search(self._h, {"grid": 0, "scan": 1}[mode]))

    def candidates(self, k: int) -> int:
        """Tool k's candidate count from the last begin_increment."""
        n = ctypes.c_int32(0)
        _capi.check(_capi.lib().sbk_contact_candidates(self._h, int(k), ctypes.byref(n)))
        return int(n.value)

    def begin_increment(self, u0: torch.Tensor, t0: float, t1: float, active: Sequence[bool], margin: float):
        act = (ctypes.c_uint8 * max(1, len(self.tools)))(*[1 if a else 0 for a in active])
        _capi.check(_capi.lib().sbk_contact_begin(self._h, _ptr(u0.contiguous()), float(t0), float(t1), act,
                                                  float(margin)))

    def evaluate(self, u: torch.Tensor, t: float, want_tangent: bool = True) -> ContactEvaluation:
        r = _capi.sbk_contact_result()
        st = _capi.lib().sbk_contact_evaluate(self._h, _ptr(u.contiguous()), float(t), int(want_tangent),
                                              ctypes.byref(r))
        if st == 4:
            raise _capi.SolverError(st, _capi.last_error())
        _capi.check(st)
        return self._result(r)

    def _result(self, r) -> ContactEvaluation:
        nd = 3 * self.mesh.num_nodes
        res = (ctypes.c_double * (9 * max(1, len(self.tools))))()
        _capi.check(_capi.lib().sbk_contact_resultants(self._h, res))
        tools = np.array(list(res)).reshape(-1, 9)[: len(self.tools)]
        n = int(r.num_blocks)
        return ContactEvaluation(residual=device_view(r.residual_dev, (nd,)),
                                 nodes=device_view(r.block_nodes_dev, (n,), torch.int32),
                                 blocks=device_view(r.blocks_dev, (n * 9,)).view(n, 3, 3),
                                 tools=tools, gross=float(r.gross), round_off=float(r.round_off),
                                 force_norm=float(r.force_norm), symmetric=bool(r.symmetric))

    def anticipate(self, u: torch.Tensor, du: torch.Tensor, t: float, residual: torch.Tensor):
        """Adds the anticipated forces to `residual` (in place) and returns
        (count, all block nodes, all blocks) with the new ones appended."""
        added = ctypes.c_int32(0)
        r = _capi.sbk_contact_result()
        _capi.check(_capi.lib().sbk_contact_anticipate(self._h, _ptr(u.contiguous()), _ptr(du.contiguous()), float(t),
                                                       _ptr(residual), ctypes.byref(added), ctypes.byref(r)))
        n = int(r.num_blocks)
        return (int(added.value), device_view(r.block_nodes_dev, (n,), torch.int32),
                device_view(r.blocks_dev, (n * 9,)).view(n, 3, 3))

    def commit(self):
        _capi.check(_capi.lib().sbk_contact_commit(self._h))

    def history(self, k: int) -> np.ndarray:
        """(n, 7): node, committed tangential force xyz, relative position xyz."""
        count = ctypes.c_int32(0)
        _capi.check(_capi.lib().sbk_contact_history(self._h, k, 0, None, ctypes.byref(count)))
        n = int(count.value)
        out = (ctypes.c_double * max(1, 7 * n))()
        _capi.check(_capi.lib().sbk_contact_history(self._h, k, n, out, ctypes.byref(count)))
        return np.array(list(out))[: 7 * n].reshape(n, 7)
