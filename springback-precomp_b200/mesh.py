"""Structured Hex8 meshes (the reference's make_structured_hex_mesh,
src/mesh/StructuredMesh.cpp:61-113): nodes numbered x fastest, then y, then
z; elements likewise, each in VTK order (bottom face counter-clockwise seen
from +z, then the top face)."""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class HexMesh:
    coords: np.ndarray  # (nn, 3) float64
    connectivity: np.ndarray  # (ne, 8) int32

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def num_elements(self) -> int:
        return int(self.connectivity.shape[0])

    @property
    def num_dofs(self) -> int:
        return 3 * self.num_nodes

    def element_coordinates(self) -> np.ndarray:
        """(ne, 24): node-major coordinates of every element."""
        return self.coords[self.connectivity].reshape(-1, 24)

    def gather(self, u: np.ndarray) -> np.ndarray:
        """(ne, 24) element displacements of a nodal vector u (3 per node)."""
        return np.asarray(u).reshape(-1, 3)[self.connectivity].reshape(-1, 24)


def structured_hex_mesh(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float,
                        x0: float = 0.0, y0: float = 0.0, z0: float = 0.0) -> HexMesh:
    if min(nx, ny, nz) < 1:
        raise ValueError("every direction needs at least one cell")
    nnx, nny, nnz = nx + 1, ny + 1, nz + 1
    i = np.arange(nnx, dtype=np.float64)
    j = np.arange(nny, dtype=np.float64)
    k = np.arange(nnz, dtype=np.float64)
    zz, yy, xx = np.meshgrid(k, j, i, indexing="ij")
    coords = np.stack([x0 + xx * (lx / nx), y0 + yy * (ly / ny), z0 + zz * (lz / nz)], axis=-1).reshape(-1, 3)
    layer = nnx * nny
    ek, ej, ei = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (ek * layer + ej * nnx + ei).reshape(-1).astype(np.int64)
    conn = np.stack([n0, n0 + 1, n0 + nnx + 1, n0 + nnx, n0 + layer, n0 + layer + 1, n0 + layer + nnx + 1,
                     n0 + layer + nnx], axis=1)
    if conn.max() >= 2 ** 31:
        raise ValueError("node indices exceed int32")
    return HexMesh(np.ascontiguousarray(coords), np.ascontiguousarray(conn.astype(np.int32)))


def distorted_hex_coords() -> np.ndarray:
    """A distorted but valid hexahedron (the reference's test fixture,
    tests/TestSupport.hpp:104-112), (8, 3)."""
    return np.array([[0.05, 0.00, 0.00], [1.10, 0.10, -0.05], [1.20, 1.15, 0.10], [-0.05, 0.90, 0.05],
                     [0.10, 0.05, 0.90], [0.95, -0.05, 1.05], [1.05, 1.05, 1.20], [0.00, 1.10, 1.00]])
