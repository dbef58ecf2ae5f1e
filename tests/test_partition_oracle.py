"""The oracle's restatement of the free-free block (PartitionedFactor::build
and ::assemble, src/fem/Forming.cpp:89-98, 213-241; the same map as
Assembler::reduce_free_free, src/fem/Assembler.cpp:294-320) and of the
driver's restrict / add_to (src/fem/NonlinearSystem.hpp:336-347), pinned
against scipy's own submatrix of the same CSC tangent: the block keeps the
entries whose row and column are free, columns ascending, rows sorted."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp


@pytest.fixture(scope="module")
def tangent(orc, pkg):
    mesh = pkg.structured_hex_mesh(6, 4, 2, 0.06, 0.04, 0.002)
    nn = mesh.num_nodes
    pat = orc.pattern(nn, mesh.connectivity)
    rng = np.random.default_rng(5)
    values = rng.standard_normal(pat["nnz"])
    return nn, pat, values


def free_set(n, seed, fraction):
    rng = np.random.default_rng(seed)
    return np.flatnonzero(rng.random(n) < fraction).astype(np.int32)


@pytest.mark.parametrize("seed,fraction", [(0, 1.0), (1, 0.9), (2, 0.5), (3, 0.05)])
def test_block_is_scipys_submatrix(orc, tangent, seed, fraction):
    nn, pat, values = tangent
    n = 3 * nn
    free = free_set(n, seed, fraction)
    outer, inner, source, kff = orc.free_free_block(pat, values, free)
    full = sp.csc_matrix((values, pat["inner"], pat["outer"]), shape=(n, n))
    ref = full[free][:, free].tocsc()
    ref.sort_indices()
    np.testing.assert_array_equal(outer, ref.indptr)
    np.testing.assert_array_equal(inner, ref.indices)
    assert np.array_equal(kff, ref.data)  # copied, not summed
    assert np.all(np.diff(source) > 0)  # the full pattern's order


def test_all_free_is_the_full_tangent(orc, tangent):
    nn, pat, values = tangent
    outer, inner, source, kff = orc.free_free_block(pat, values, np.arange(3 * nn))
    np.testing.assert_array_equal(outer, pat["outer"])
    np.testing.assert_array_equal(inner, pat["inner"])
    assert np.array_equal(kff, values)


def test_restrict_and_add_to(orc):
    full = np.arange(10.0)
    free = np.array([1, 4, 7])
    np.testing.assert_array_equal(orc.restrict(full, free), [1.0, 4.0, 7.0])
    out = orc.add_to(full, free, np.array([1.0, 2.0, 3.0]), 0.5)
    np.testing.assert_array_equal(out, [0, 1.5, 2, 3, 5, 5, 6, 8.5, 8, 9])
