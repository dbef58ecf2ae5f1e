"""The free-free tangent of a Dirichlet partition, on the device.

`PartitionedFactor` mirrors the forming driver's PartitionedFactor
(src/fem/Forming.cpp:59-241): built for one partition (its free DOFs,
ascending) of a system's CSC pattern, `assemble` gathers the free-free
values of the full tangent, `factorize` factorises them and `solve` solves
K_ff x = b; `restrict` and `add_to` are the driver's vector helpers
(src/fem/NonlinearSystem.hpp:336-347). The pattern of the block, its
fill-reducing order and the gather maps are built once per partition; every
iteration then reads the full tangent once. The factorisations are
cuSOLVER's device sparse Cholesky for a symmetric block; for a
non-symmetric one (Chaboche recovery, exact friction tangent) or one that is
not positive definite, a dense LU on the device up to the dense limit
(20000 rows by default), beyond it restarted GMRES preconditioned by the
Cholesky of the symmetric part and the device sparse QR where that fails -
where the reference takes CHOLMOD's supernodal Cholesky, then LDL^T, then LU
(UMFPACK).

Everything runs in libsbk.so on the GPU; device buffers are torch tensors.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _capi
from ._capi import SbkError, SolverError
from .system import _ptr, _stream_ptr

CHOLESKY = 1
QR = 2
GMRES = 3
LU = 4


class PartitionedFactor:
    """A partition's free-free block and its factorisation (device).

    outer, inner: the full tangent's CSC pattern (int32 CUDA tensors, as
    NonlinearSystem.outer / .inner); free: the free DOFs, strictly
    ascending. A partition that keeps its free DOFs keeps its pattern and
    its analyses, as the reference's reset does for an unchanged partition."""

    def __init__(self, outer: torch.Tensor, inner: torch.Tensor, free: Sequence[int]):
        free_np = np.ascontiguousarray(np.asarray(free, dtype=np.int32))
        self.num_dofs = int(outer.numel()) - 1
        self.free = free_np
        h = ctypes.c_void_p()
        _capi.check(_capi.lib().sbk_partition_create(self.num_dofs, _ptr(outer), _ptr(inner), int(inner.numel()),
                                                     int(free_np.size), free_np.ctypes.data_as(ctypes.c_void_p),
                                                     ctypes.byref(h)))
        self._h = h
        nf, nnz = ctypes.c_int32(), ctypes.c_int64()
        _capi.check(_capi.lib().sbk_partition_info(self._h, ctypes.byref(nf), ctypes.byref(nnz)))
        self.num_free, self.nnz = int(nf.value), int(nnz.value)
        self.free_dev = torch.as_tensor(free_np, device="cuda")
        self.kind = 0
        self.set_stream()

    @classmethod
    def for_system(cls, system, free: Sequence[int]) -> "PartitionedFactor":
        return cls(system.outer, system.inner, free)

    def close(self):
        if getattr(self, "_h", None) and _capi is not None and _capi.lib is not None:
            _capi.lib().sbk_partition_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def same_partition(self, free: Sequence[int]) -> bool:
        f = np.asarray(free)
        return f.shape == self.free.shape and bool(np.array_equal(f, self.free))

    def set_stream(self, stream=None):
        _capi.check(_capi.lib().sbk_partition_set_stream(self._h, _stream_ptr(stream)))

    def pattern(self):
        """The block's CSC pattern (outer: num_free + 1, inner: nnz)."""
        outer = torch.empty(self.num_free + 1, dtype=torch.int32, device="cuda")
        inner = torch.empty(self.nnz, dtype=torch.int32, device="cuda")
        _capi.check(_capi.lib().sbk_partition_pattern(self._h, _ptr(outer), _ptr(inner)))
        return outer, inner

    def assemble(self, values: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """The block's values, in its CSC order (PartitionedFactor::assemble)."""
        if out is None:
            out = torch.empty(self.nnz, dtype=torch.float64, device="cuda")
        _capi.check(_capi.lib().sbk_partition_assemble(self._h, _ptr(values), _ptr(out)))
        return out

    def restrict(self, full: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if out is None:
            out = torch.empty(self.num_free, dtype=torch.float64, device="cuda")
        _capi.check(_capi.lib().sbk_partition_restrict(self._h, _ptr(full.contiguous()), _ptr(out)))
        return out

    def add_to(self, full: torch.Tensor, part: torch.Tensor, factor: float) -> torch.Tensor:
        """full[free[i]] += factor * part[i], in place."""
        _capi.check(_capi.lib().sbk_partition_add_to(self._h, _ptr(full), _ptr(part.contiguous()), float(factor)))
        return full

    def set_dense_limit(self, max_rows: int):
        """Blocks of at most max_rows rows take the dense LU (0: never)."""
        _capi.check(_capi.lib().sbk_partition_set_dense_limit(self._h, int(max_rows)))

    def factorize(self, values: torch.Tensor, symmetric: bool) -> int:
        """Factorise the free-free block of the full tangent `values`;
        returns CHOLESKY, LU, GMRES (a large non-symmetric block: the
        Cholesky of its symmetric part preconditions GMRES) or QR.
        SolverError when the block is singular."""
        kind = ctypes.c_int(0)
        st = _capi.lib().sbk_partition_factorize(self._h, _ptr(values), int(bool(symmetric)), ctypes.byref(kind))
        if st == 4:
            raise SolverError(st, _capi.last_error())
        _capi.check(st)
        self.kind = int(kind.value)
        return self.kind

    def solve(self, b: torch.Tensor, out: Optional[torch.Tensor] = None, transpose: bool = False) -> torch.Tensor:
        """x = K_ff^-1 b on the free DOFs (transpose: K_ff^-T b, the adjoint
        system; Cholesky or dense LU); SolverError when the block is singular
        (a rigid-body motion or a mechanism left free)."""
        if out is None:
            out = torch.empty(self.num_free, dtype=torch.float64, device="cuda")
        fn = _capi.lib().sbk_partition_solve_transpose if transpose else _capi.lib().sbk_partition_solve
        st = fn(self._h, _ptr(b.contiguous()), _ptr(out))
        if st == 4:
            raise SolverError(st, _capi.last_error())
        if st != 0:
            raise SbkError(st, _capi.last_error())
        return out

    def counts(self) -> dict:
        """Factorisations by kind and fallbacks (names() and failures())."""
        c = (ctypes.c_int64 * 9)()
        _capi.check(_capi.lib().sbk_partition_counts(self._h, ctypes.byref(c)))
        return dict(zip(("cholesky", "gmres", "lu", "qr", "cholesky_fell_back", "gmres_fell_back", "singular",
                         "gmres_steps", "solves"), (int(v) for v in c)))
