"""The element loop behind the reference's own interfaces.

`NonlinearSystem` mirrors detail::NonlinearSystem
(src/fem/NonlinearSystem.hpp:85-334): evaluate(u, lambda, want_tangent)
returns an `Evaluation` (f_int, residual, the tangent in the Assembler's CSC
pattern, energy, gross, yield count, trial states and modes), commit() makes
the trial history the committed one, committed_all / set_committed and
internal_all / set_internal carry a restart. A failing element raises
`SolverError`, as the reference's SolverError does.

`element_batch` is incompatible_elastoplastic_element
(src/fem/IncompatibleModes.cpp:577-600) over a batch of independent
elements.

Everything runs in libsbk.so on the GPU; device buffers are torch tensors.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional

import numpy as np
import torch

from . import _capi
from .material import Material, rule_c, rule_size
from .mesh import HexMesh


class _DeviceView:
    """A zero-copy torch view of library-owned device memory."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": None, "stream": None}


def device_view(ptr: int, shape, dtype=torch.float64) -> torch.Tensor:
    typestr = {torch.float64: "<f8", torch.int32: "<i4", torch.uint8: "|u1"}[dtype]
    if int(np.prod(shape)) == 0 or not ptr:
        return torch.empty(shape, dtype=dtype, device="cuda")
    return torch.as_tensor(_DeviceView(ptr, shape, typestr), device="cuda")


def _ptr(t: Optional[torch.Tensor]):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("device buffers must be contiguous CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream) -> ctypes.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


@dataclasses.dataclass
class ElementBatchResult:
    force: torch.Tensor       # (ne, 24)
    tangent: Optional[torch.Tensor]  # (ne, 64, 3, 3) node blocks (a, b)
    energy: torch.Tensor      # (ne,)
    states: torch.Tensor      # (nfields, ne, nq)
    alpha: torch.Tensor       # (ne, 9)
    yielding: torch.Tensor    # (ne, nq) uint8
    iterations: torch.Tensor  # (ne,) int32
    code: torch.Tensor        # (ne,) int32

    def dense_tangent(self) -> torch.Tensor:
        """(ne, 24, 24) from the node-block layout."""
        t = self.tangent.view(-1, 8, 8, 3, 3).permute(0, 1, 3, 2, 4)
        return t.reshape(-1, 24, 24)


def element_batch(material: Material, x: torch.Tensor, u: torch.Tensor, state: Optional[torch.Tensor] = None,
                  alpha: Optional[torch.Tensor] = None, kinematics: str = "logarithmic", stiffness_points: int = 2,
                  thickness_points: int = 0, thickness_axis: int = 2, want_tangent: bool = True,
                  stream=None) -> ElementBatchResult:
    """Evaluate independent IM Hex8 elements on the GPU. x, u: (ne, 24)
    float64 CUDA tensors; state: (nfields, ne, nq) committed points (None:
    virgin); alpha: (ne, 9) committed modes (None: zero)."""
    ne = int(x.shape[0])
    nq = rule_size(stiffness_points, thickness_points, thickness_axis)
    if nq == 0:
        raise _capi.SbkError(2, "invalid integration rule")
    nf = material.state_fields
    dev = x.device
    f64 = dict(dtype=torch.float64, device=dev)
    if state is None:
        state = torch.zeros((nf, ne, nq), **f64)
    out = ElementBatchResult(
        force=torch.empty((ne, 24), **f64),
        tangent=torch.empty((ne, 64, 3, 3), **f64) if want_tangent else None,
        energy=torch.empty((ne,), **f64),
        states=torch.empty((nf, ne, nq), **f64),
        alpha=torch.empty((ne, 9), **f64),
        yielding=torch.zeros((ne, nq), dtype=torch.uint8, device=dev),
        iterations=torch.zeros((ne,), dtype=torch.int32, device=dev),
        code=torch.zeros((ne,), dtype=torch.int32, device=dev),
    )
    mat = material.to_c()
    rule = rule_c(stiffness_points, thickness_points, thickness_axis)
    st = _capi.lib().sbk_element_batch(ctypes.byref(mat), ctypes.byref(rule), _capi.KINEMATICS[kinematics], ne,
                                       _ptr(x.contiguous()), _ptr(u.contiguous()), _ptr(state.contiguous()),
                                       _ptr(alpha.contiguous()) if alpha is not None else None, _ptr(out.force),
                                       _ptr(out.tangent) if want_tangent else None, _ptr(out.energy),
                                       _ptr(out.states), _ptr(out.alpha), _ptr(out.yielding), _ptr(out.iterations),
                                       _ptr(out.code), _stream_ptr(stream))
    _capi.check(st)
    return out


LOCAL_ITERATION = {"phases": 0, "single": 1}


def set_local_iteration(mode: str = "phases"):
    """The local iteration of element_batch and of systems made from now on:
    "phases" (the default) or "single" (see NonlinearSystem.set_local_iteration)."""
    _capi.check(_capi.lib().sbk_set_local_iteration(LOCAL_ITERATION[mode]))


NOALLOC_MAX_ELEMENTS = 2048
NOALLOC_MAX_NODES = 16384


def evaluate_noalloc(material: Material, coords: torch.Tensor, connectivity: torch.Tensor, u: torch.Tensor,
                     state: torch.Tensor, alpha: Optional[torch.Tensor], outer: torch.Tensor, inner: torch.Tensor,
                     internal: torch.Tensor, values: Optional[torch.Tensor], trial: torch.Tensor,
                     alpha_out: torch.Tensor, yielding: torch.Tensor, summary: torch.Tensor,
                     kinematics: str = "logarithmic", stiffness_points: int = 2, thickness_points: int = 0,
                     thickness_axis: int = 2, stream=None):
    """sbk_evaluate_noalloc: the element loop of a small mesh (at most
    2048 elements, 16384 nodes) for callers that cannot allocate device
    memory; every buffer is the caller's (device tensors), the library
    allocates nothing. Results land in the given tensors on `stream`;
    summary (5 doubles): energy, gross, yielding points, lowest failing
    element (-1: none), its code. The tensors must all live on one CUDA
    device (the call runs with it current), be contiguous and have the C
    ABI's types: float64 for the coordinates, displacements, states, modes
    and outputs, int32 for the connectivity and the pattern, uint8 for the
    yield flags."""
    f64 = {"coords": coords, "u": u, "state": state, "alpha": alpha, "internal": internal, "values": values,
           "trial": trial, "alpha_out": alpha_out, "summary": summary}
    i32 = {"connectivity": connectivity, "outer": outer, "inner": inner}
    dev = coords.device
    for group, dtype in ((f64, torch.float64), (i32, torch.int32), ({"yielding": yielding}, torch.uint8)):
        for name, t in group.items():
            if t is None:
                continue
            if t.dtype != dtype:
                raise TypeError(f"evaluate_noalloc: {name} is {t.dtype}, expected {dtype}")
            if t.device != dev or t.device.type != "cuda":
                raise ValueError(f"evaluate_noalloc: {name} is on {t.device}, expected the CUDA device {dev}")
            if not t.is_contiguous():
                raise ValueError(f"evaluate_noalloc: {name} is not contiguous")
    mat = material.to_c()
    rule = rule_c(stiffness_points, thickness_points, thickness_axis)
    with torch.cuda.device(dev):
        st = _capi.lib().sbk_evaluate_noalloc(
            ctypes.byref(mat), ctypes.byref(rule), _capi.KINEMATICS[kinematics], int(coords.numel() // 3),
            int(connectivity.numel() // 8), _ptr(coords), _ptr(connectivity), _ptr(u), _ptr(state),
            _ptr(alpha) if alpha is not None else None, _ptr(outer), _ptr(inner), int(inner.numel()),
            _ptr(internal), _ptr(values) if values is not None else None, _ptr(trial), _ptr(alpha_out),
            _ptr(yielding), _ptr(summary), _stream_ptr(stream))
    _capi.check(st)


@dataclasses.dataclass
class ElementStresses:
    """ElastoplasticStress (include/sparlab/fem/Elastoplastic.hpp:206-221)
    of every element: point averages, [Pa] and [-]."""

    cauchy: torch.Tensor            # (ne, 6) tensorial Voigt
    piola_kirchhoff: torch.Tensor   # (ne, 6)
    von_mises: torch.Tensor         # (ne,) of the average Cauchy stress
    max_plastic_strain: torch.Tensor  # (ne,) largest accumulated plastic strain
    max_strain: torch.Tensor        # (ne,) largest strain component
    min_jacobian: torch.Tensor      # (ne,) smallest det F
    kirchhoff: torch.Tensor         # (ne, 6) logarithmic kinematics, else 0
    log_strain: torch.Tensor        # (ne, 6) tensor components, logarithmic, else 0

    @classmethod
    def from_packed(cls, t: torch.Tensor) -> "ElementStresses":
        return cls(t[:, 0:6], t[:, 6:12], t[:, 12], t[:, 13], t[:, 14], t[:, 15], t[:, 16:22], t[:, 22:28])


@dataclasses.dataclass
class Evaluation:
    """NonlinearSystem.hpp:27-47. Tensors are views of the system's buffers,
    valid until its next evaluate (clone to keep them)."""

    internal: torch.Tensor
    residual: torch.Tensor
    tangent: Optional[torch.Tensor]  # CSC values in the pattern
    energy: float
    gross: float
    yielding_points: int
    system: "NonlinearSystem"

    @property
    def states(self) -> np.ndarray:
        return self.system.trial_states()

    @property
    def modes(self) -> np.ndarray:
        return self.system.trial_modes()


ELEMENTS = {"incompatible_modes": 0, "standard": 1}
MEAN_DILATATION = {"auto": 0, "all": 1, "none": 2}


class NonlinearSystem:
    """element: "incompatible_modes" (the default) or "standard" (the
    standard Hex8, Elastoplastic.cpp:226-340); mean_dilatation: "auto",
    "all" or "none" (B-bar for the standard Hex8 under "auto" / "all"; the
    incompatible-mode Hex8 refuses "all", NonlinearSystem.hpp:283-309)."""

    def __init__(self, mesh: HexMesh, material: Material, kinematics: str = "logarithmic", stiffness_points: int = 2,
                 thickness_points: int = 0, thickness_axis: int = 2, stream=None, element: str = "incompatible_modes",
                 mean_dilatation: str = "auto"):
        self.mesh = mesh
        self.material = material
        self.kinematics = kinematics
        self.nq = rule_size(stiffness_points, thickness_points, thickness_axis)
        self.nfields = material.state_fields
        self._coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
        self._conn = np.ascontiguousarray(mesh.connectivity, dtype=np.int32)
        m = _capi.sbk_mesh()
        m.num_nodes = mesh.num_nodes
        m.num_elements = mesh.num_elements
        m.coords = self._coords.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        m.connectivity = self._conn.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        self._mat = material.to_c()
        self._rule = rule_c(stiffness_points, thickness_points, thickness_axis)
        h = ctypes.c_void_p()
        _capi.check(_capi.lib().sbk_system_create(ctypes.byref(m), ctypes.byref(self._mat), ctypes.byref(self._rule),
                                                  _capi.KINEMATICS[kinematics], ctypes.byref(h)))
        self._h = h
        self.set_stream(stream)
        self.set_element(element, mean_dilatation)
        self.frozen = False
        pat = _capi.sbk_pattern()
        _capi.check(_capi.lib().sbk_system_pattern(self._h, ctypes.byref(pat)))
        self.num_dofs = int(pat.num_dofs)
        self.nnz = int(pat.nnz)
        self.outer = device_view(pat.outer_dev, (self.num_dofs + 1,), torch.int32)
        self.inner = device_view(pat.inner_dev, (self.nnz,), torch.int32)

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().sbk_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream=None):
        _capi.check(_capi.lib().sbk_system_set_stream(self._h, _stream_ptr(stream)))

    def set_element(self, element: str = "incompatible_modes", mean_dilatation: str = "auto"):
        """The element formulation of the evaluations that follow (the
        committed point states carry over; the standard Hex8 has no modes)."""
        if element not in ELEMENTS or mean_dilatation not in MEAN_DILATATION:
            raise ValueError(f"unknown element {element!r} or mean_dilatation {mean_dilatation!r}")
        _capi.check(_capi.lib().sbk_system_set_element(self._h, ELEMENTS[element], MEAN_DILATATION[mean_dilatation]))
        self.element = element
        av = ctypes.c_int(0)
        _capi.check(_capi.lib().sbk_system_element(self._h, None, ctypes.byref(av)))
        self.averaged = bool(av.value)

    def set_stable_buffers(self, stable: bool = True):
        """Commit by copying on the device instead of exchanging buffers, so
        that a captured graph of evaluate stays valid across commits."""
        _capi.check(_capi.lib().sbk_system_set_stable_buffers(self._h, 1 if stable else 0))

    def enqueue(self, u: torch.Tensor, want_tangent: bool, summary: torch.Tensor):
        """evaluate without a host synchronisation (capturable in a CUDA
        graph): results in internal_view() / values_view(), and summary (5
        doubles on the device): energy, gross, yielding points, lowest
        failing element (-1: none), its code."""
        _capi.check(_capi.lib().sbk_system_enqueue(self._h, _ptr(u), int(want_tangent), _ptr(summary)))

    def internal_view(self) -> torch.Tensor:
        """The f_int buffer (num_dofs) every evaluation writes (known after
        the first evaluate)."""
        return self._internal_view

    def values_view(self) -> torch.Tensor:
        """The tangent value buffer (nnz, CSC) every evaluation with the
        tangent writes (known after the first evaluate with the tangent)."""
        return self._values_view

    def set_schedule(self, by_cost: bool = True):
        """Walk the elements grouped by the cost of their last evaluation (the
        default) or in mesh order; no result depends on it."""
        _capi.check(_capi.lib().sbk_system_set_schedule(self._h, 1 if by_cost else 0))

    def set_local_iteration(self, mode: str = "phases"):
        """How the incompatible-mode Hex8's local iteration runs: "phases"
        (the default: phase kernels over the whole mesh, the elements that
        need a line search or a fallback handed to the single kernel) or
        "single" (one kernel per element from start to finish). No result
        depends on it."""
        _capi.check(_capi.lib().sbk_system_set_local_iteration(self._h, LOCAL_ITERATION[mode]))

    def set_values_buffer(self, values: Optional[torch.Tensor] = None):
        """Assemble the tangent of the next evaluations into `values` (nnz
        float64 on the device, kept alive by the system meanwhile), or back
        into the system's own buffer (None): a driver alternating two
        buffers reads one back while the next evaluation fills the other."""
        if values is not None and (values.dtype != torch.float64 or values.numel() != self.nnz or not values.is_cuda
                                   or not values.is_contiguous()):
            raise ValueError("values must be a contiguous CUDA float64 tensor of nnz entries")
        self._values_buffer = values
        _capi.check(_capi.lib().sbk_system_set_values_buffer(self._h, _ptr(values) if values is not None else None))

    def set_elements_per_block(self, epb: int):
        _capi.check(_capi.lib().sbk_system_set_elements_per_block(self._h, int(epb)))

    def set_timing(self, enable: bool = True):
        _capi.check(_capi.lib().sbk_system_set_timing(self._h, int(enable)))

    def last_timings(self) -> dict:
        """Device ms of the last evaluate: element kernel, force gather, value gather."""
        out = (ctypes.c_double * 3)()
        _capi.check(_capi.lib().sbk_system_last_timings(self._h, out))
        return {"element": out[0], "forces": out[1], "values": out[2]}

    def symmetric(self) -> bool:
        return bool(_capi.lib().sbk_system_symmetric(self._h))

    def plastic(self) -> bool:
        return bool(_capi.lib().sbk_system_plastic(self._h))

    def evaluate(self, u: torch.Tensor, lam: float = 0.0, want_tangent: bool = True) -> Evaluation:
        if u.dtype != torch.float64 or u.numel() != self.num_dofs:
            raise ValueError("u must hold num_dofs float64 values")
        ev = _capi.sbk_evaluation()
        st = _capi.lib().sbk_system_evaluate(self._h, _ptr(u.contiguous()), float(lam), int(want_tangent),
                                             ctypes.byref(ev))
        if st == 4:
            raise _capi.SolverError(st, _capi.last_error(), ev.failed_element, ev.failure_code)
        _capi.check(st)
        internal = device_view(ev.internal_dev, (self.num_dofs,))
        values = device_view(ev.values_dev, (self.nnz,)) if want_tangent else None
        self._internal_view = internal
        if values is not None:
            self._values_view = values
        return Evaluation(internal=internal, residual=internal, tangent=values, energy=float(ev.energy),
                          gross=float(ev.gross), yielding_points=int(ev.yielding_points), system=self)

    def commit(self, ev: Optional[Evaluation] = None):
        _capi.check(_capi.lib().sbk_system_commit(self._h))

    def _state_shape(self):
        return (self.nfields, self.mesh.num_elements, self.nq)

    def committed_all(self) -> np.ndarray:
        out = np.empty(self._state_shape())
        _capi.check(_capi.lib().sbk_system_get_committed(self._h, out.ctypes.data_as(ctypes.c_void_p), None))
        return out

    def internal_all(self) -> np.ndarray:
        out = np.empty((self.mesh.num_elements, 9))
        _capi.check(_capi.lib().sbk_system_get_committed(self._h, None, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def set_committed(self, states: np.ndarray):
        states = np.ascontiguousarray(states, dtype=np.float64)
        if states.shape != self._state_shape():
            raise _capi.SbkError(2, f"the saved plastic history has shape {states.shape}; the system keeps "
                                    f"{self._state_shape()}")
        _capi.check(_capi.lib().sbk_system_set_committed(self._h, states.ctypes.data_as(ctypes.c_void_p), None))

    def set_internal(self, alpha: np.ndarray):
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        if alpha.shape != (self.mesh.num_elements, 9):
            raise _capi.SbkError(2, "the saved internal-mode history does not match the mesh")
        _capi.check(_capi.lib().sbk_system_set_committed(self._h, None, alpha.ctypes.data_as(ctypes.c_void_p)))

    def committed_views(self):
        """Zero-copy device views of the committed points (nfields, ne, nq)
        and modes (ne, 9); valid until the next commit."""
        c_st, c_al, t_st, t_al = (ctypes.c_void_p() for _ in range(4))
        _capi.check(_capi.lib().sbk_system_buffers(self._h, ctypes.byref(c_st), ctypes.byref(c_al),
                                                   ctypes.byref(t_st), ctypes.byref(t_al)))
        return (device_view(c_st.value, self._state_shape()), device_view(c_al.value, (self.mesh.num_elements, 9)))

    def trial_states(self) -> np.ndarray:
        out = np.empty(self._state_shape())
        _capi.check(_capi.lib().sbk_system_get_trial(self._h, out.ctypes.data_as(ctypes.c_void_p), None, None))
        return out

    def trial_modes(self) -> np.ndarray:
        out = np.empty((self.mesh.num_elements, 9))
        _capi.check(_capi.lib().sbk_system_get_trial(self._h, None, out.ctypes.data_as(ctypes.c_void_p), None))
        return out

    def trial_yield(self) -> np.ndarray:
        out = np.empty((self.mesh.num_elements, self.nq), dtype=np.uint8)
        _capi.check(_capi.lib().sbk_system_get_trial(self._h, None, None, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def max_plastic_strain(self) -> float:
        st = self.committed_all()
        return float(st[12 + 6 * self.material.kinematic_terms].max()) if st.size else 0.0

    def add_node_blocks(self, nodes: torch.Tensor, blocks: torch.Tensor):
        """add_node_block (src/fem/Forming.cpp:280-297) into the tangent of
        the last evaluate; nodes distinct within one call."""
        n = int(nodes.numel())
        _capi.check(_capi.lib().sbk_system_add_node_blocks(self._h, n, _ptr(nodes.to(torch.int32).contiguous()),
                                                           _ptr(blocks.to(torch.float64).contiguous())))

    def stress(self, u: torch.Tensor) -> ElementStresses:
        """elastoplastic_stress of every element at u from the committed
        points and modes (IncompatibleModes.cpp:602-664), the step-end stress
        recovery of the forming driver (Forming.cpp:1266-1281): call after
        commit(). Overwrites the trial state of the last evaluate."""
        u = u.to(torch.float64).contiguous()
        if u.numel() != self.num_dofs:
            raise ValueError(f"u has {u.numel()} values, the system {self.num_dofs} DOFs")
        out = torch.empty((self.mesh.num_elements, 28), dtype=torch.float64, device=u.device)
        st = _capi.lib().sbk_system_stress(self._h, _ptr(u), _ptr(out))
        if st == 4:
            raise _capi.SolverError(st, _capi.last_error())
        _capi.check(st)
        return ElementStresses.from_packed(out)

    def vjp_x(self, u: torch.Tensor, lam: torch.Tensor, frozen: bool = True) -> torch.Tensor:
        """lambda^T d f_int / d X (num_dofs) at u: the shape derivative of the
        internal force with respect to the nodal reference coordinates, the
        modes through their local equilibrium, the committed history as the
        history (frozen: its plastic state taken as it is, no return). The
        trial state of the last evaluate is overwritten."""
        out = torch.empty(self.num_dofs, dtype=torch.float64, device="cuda")
        st = _capi.lib().sbk_system_vjp_x(self._h, _ptr(u.contiguous()), _ptr(lam.contiguous()), int(bool(frozen)),
                                          _ptr(out))
        if st == 4:
            raise _capi.SolverError(st, _capi.last_error())
        _capi.check(st)
        return out

    def set_frozen(self, frozen: bool = True):
        """Take the committed plastic state as it is in the evaluations that
        follow (no return; the elastic, symmetric tangent): the release step
        with the end-of-forming state frozen."""
        _capi.check(_capi.lib().sbk_system_set_frozen(self._h, int(bool(frozen))))
        self.frozen = bool(frozen)

    def set_coordinates(self, coords: torch.Tensor):
        """Move the nodes: the reference coordinates (num_nodes x 3, float64,
        on the device) replace the mesh's; connectivity, pattern and history
        stay."""
        if coords.dtype != torch.float64 or coords.numel() != 3 * self.mesh.num_nodes or not coords.is_cuda:
            raise ValueError("coords must hold num_nodes x 3 float64 values on the device")
        self._coords_dev = coords.detach().contiguous()
        _capi.check(_capi.lib().sbk_system_set_coordinates(self._h, _ptr(self._coords_dev)))

    def stiffness_gross(self, u: torch.Tensor, free: torch.Tensor) -> float:
        """stiffness_gross (src/fem/NonlinearSystem.hpp:49-67): the norm over
        the DOFs in `free` of |K| |u|, K the tangent of the last evaluate (with
        any node blocks added since): the round-off floor the forming
        driver's convergence test takes from the displacement's rounding."""
        u = u.to(torch.float64).contiguous()
        if u.numel() != self.num_dofs:
            raise ValueError(f"u has {u.numel()} values, the system {self.num_dofs} DOFs")
        free = free.to(device=u.device, dtype=torch.int32).contiguous()
        out = ctypes.c_double(0.0)
        _capi.check(_capi.lib().sbk_system_stiffness_gross(self._h, _ptr(u), int(free.numel()), _ptr(free),
                                                           ctypes.byref(out)))
        return out.value
