"""The free-free block on the device (sbk_partition_*, the forming driver's
PartitionedFactor, src/fem/Forming.cpp:59-241) against the oracle's
restatement: the block's pattern and values to the bit, restrict and add_to
to the bit, and the device factorisations' solutions against a dense solve
of the same block (1e-9 relative: the sparse and the dense factorisations
round differently, the blocks' condition numbers reach about 1e6)."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import scipy.sparse as sp
import torch

pytestmark = pytest.mark.gpu
SOLVE_TOL = 1e-9


@pytest.fixture(scope="module")
def plastic(pkg, cuda):
    """A bent 24 x 12 x 2 sheet with yielding points (its tangent)."""
    wl = importlib.import_module("springback-precomp_b200.workload")
    prob = wl.make_problem(24, 12, 2, seed=11, sample=576)
    s = pkg.NonlinearSystem(prob.mesh, prob.material, kinematics="logarithmic")
    s.set_committed(prob.state)
    s.set_internal(prob.alpha)
    ev = s.evaluate(torch.tensor(prob.u, device=cuda), 0.0, True)
    return s, ev.tangent.clone()


@pytest.fixture(scope="module")
def elastic(pkg, cuda):
    """A 6 x 4 x 2 block at rest (the elastic tangent) and its bottom face."""
    mat = pkg.material.aluminium_swift()
    mesh = pkg.structured_hex_mesh(6, 4, 2, 0.06, 0.04, 0.004)
    s = pkg.NonlinearSystem(mesh, mat, kinematics="logarithmic")
    ev = s.evaluate(torch.zeros(mesh.num_dofs, dtype=torch.float64, device=cuda), 0.0, True)
    bottom = np.flatnonzero(np.isclose(mesh.coords[:, 2], 0.0))
    held = np.zeros(mesh.num_dofs, dtype=bool)
    for c in range(3):
        held[3 * bottom + c] = True
    return s, ev.tangent.clone(), np.flatnonzero(~held).astype(np.int32)


def oracle_pattern(s):
    return dict(outer=s.outer.cpu().numpy(), inner=s.inner.cpu().numpy())


def dense_block(s, values, free):
    n = s.num_dofs
    full = sp.csc_matrix((values, s.inner.cpu().numpy(), s.outer.cpu().numpy()), shape=(n, n))
    return full[free][:, free].toarray()


@pytest.mark.parametrize("seed,fraction", [(0, 1.0), (1, 0.9), (2, 0.3)])
def test_block_is_the_oracles(pkg, orc, plastic, seed, fraction):
    s, values = plastic
    free = np.flatnonzero(np.random.default_rng(seed).random(s.num_dofs) < fraction).astype(np.int32)
    part = pkg.PartitionedFactor.for_system(s, free)
    outer, inner, source, kff = orc.free_free_block(oracle_pattern(s), values.cpu().numpy(), free)
    o, i = part.pattern()
    np.testing.assert_array_equal(o.cpu().numpy(), outer)
    np.testing.assert_array_equal(i.cpu().numpy(), inner)
    assert part.nnz == len(kff) and part.num_free == len(free)
    assert np.array_equal(part.assemble(values).cpu().numpy(), kff)


def test_restrict_and_add_to_are_the_oracles(pkg, orc, plastic, cuda):
    s, _ = plastic
    rng = np.random.default_rng(3)
    free = np.flatnonzero(rng.random(s.num_dofs) < 0.7).astype(np.int32)
    part = pkg.PartitionedFactor.for_system(s, free)
    full = rng.standard_normal(s.num_dofs)
    v = rng.standard_normal(len(free))
    assert np.array_equal(part.restrict(torch.tensor(full, device=cuda)).cpu().numpy(), orc.restrict(full, free))
    got = part.add_to(torch.tensor(full, device=cuda), torch.tensor(v, device=cuda), -0.37).cpu().numpy()
    assert np.array_equal(got, orc.add_to(full, free, v, -0.37))


def test_constrained_elastic_block_takes_the_cholesky(pkg, elastic, cuda):
    """As the reference's 'reduced stiffness matrix is positive definite once
    constrained' (tests/test_assembly_solver.cpp:136-148): held on its bottom
    face, the block is positive definite and the Cholesky takes it."""
    s, values, free = elastic
    part = pkg.PartitionedFactor.for_system(s, free)
    assert part.factorize(values, symmetric=True) == 1
    rng = np.random.default_rng(7)
    b = rng.standard_normal(len(free))
    x = part.solve(torch.tensor(b, device=cuda)).cpu().numpy()
    ref = np.linalg.solve(dense_block(s, values.cpu().numpy(), free), b)
    assert np.linalg.norm(x - ref) <= SOLVE_TOL * np.linalg.norm(ref)
    assert part.counts() == {"cholesky": 1, "gmres": 0, "lu": 0, "qr": 0, "cholesky_fell_back": 0,
                             "gmres_fell_back": 0, "singular": 0, "gmres_steps": 0, "solves": 1}
    # A second right-hand side reuses the factorisation.
    x2 = part.solve(torch.tensor(2.0 * b, device=cuda)).cpu().numpy()
    assert np.linalg.norm(x2 - 2.0 * ref) <= SOLVE_TOL * np.linalg.norm(2.0 * ref)


def shifted(s, values, free):
    """The elastic values shifted between two eigenvalues of the block: a
    symmetric block that is not positive definite, and the shift."""
    v = values.cpu().numpy().copy()
    lam = np.linalg.eigvalsh(dense_block(s, v, free))
    shift = 0.5 * (lam[len(lam) // 2] + lam[len(lam) // 2 + 1])
    outer, inner = s.outer.cpu().numpy(), s.inner.cpu().numpy()
    for col in range(s.num_dofs):
        for q in range(outer[col], outer[col + 1]):
            if inner[q] == col:
                v[q] -= shift
    return v


@pytest.mark.parametrize("dense_limit,kind", [(20000, 4), (0, 2)])
def test_indefinite_block_falls_back(pkg, elastic, cuda, dense_limit, kind):
    """A symmetric block that is not positive definite leaves the Cholesky
    for the dense LU (or, above the dense limit, the QR), as the reference's
    CHOLMOD leaves for LDL^T and LU."""
    s, values, free = elastic
    v = shifted(s, values, free)
    part = pkg.PartitionedFactor.for_system(s, free)
    part.set_dense_limit(dense_limit)
    part.factorize(torch.tensor(v, device=cuda), symmetric=True)
    b = np.random.default_rng(8).standard_normal(len(free))
    x = part.solve(torch.tensor(b, device=cuda)).cpu().numpy()
    assert part.kind == kind
    c = part.counts()
    assert c["cholesky_fell_back"] == 1 and c["cholesky"] == 0 and c["gmres"] == 0
    assert c["lu" if kind == 4 else "qr"] == 1
    ref = np.linalg.solve(dense_block(s, v, free), b)
    assert np.linalg.norm(x - ref) <= SOLVE_TOL * np.linalg.norm(ref)


@pytest.mark.parametrize("skew,dense_limit,kinds", [(1e-3, 20000, (4,)), (1e-3, 0, (3,)), (1e-1, 0, (2, 3))])
def test_nonsymmetric_block(pkg, plastic, cuda, skew, dense_limit, kinds):
    """A non-symmetric block (every value perturbed independently, so the
    block and its transpose differ by `skew` of their size): the dense LU
    below the dense limit; above it GMRES preconditioned by the Cholesky of
    the symmetric part - or, where the larger perturbation leaves the
    symmetric part indefinite, the QR."""
    s, values = plastic
    rng = np.random.default_rng(9)
    free = np.flatnonzero(rng.random(s.num_dofs) < 0.8).astype(np.int32)
    v = values.cpu().numpy() * (1.0 + skew * rng.standard_normal(s.nnz))
    part = pkg.PartitionedFactor.for_system(s, free)
    part.set_dense_limit(dense_limit)
    assert part.factorize(torch.tensor(v, device=cuda), symmetric=False) in kinds
    b = rng.standard_normal(len(free))
    x = part.solve(torch.tensor(b, device=cuda)).cpu().numpy()
    ref = np.linalg.solve(dense_block(s, v, free), b)
    assert np.linalg.norm(x - ref) <= SOLVE_TOL * np.linalg.norm(ref)
    c = part.counts()
    assert c["gmres"] + c["qr"] + c["lu"] == 1 and part.kind in kinds


@pytest.mark.parametrize("dense_limit", [20000, 0])
def test_nonsymmetric_block_with_an_indefinite_symmetric_part_is_solved(pkg, elastic, cuda, dense_limit):
    """GMRES's preconditioner (the symmetric part) is indefinite: the solve
    still reaches the block's solution, by whichever method."""
    s, values, free = elastic
    v = shifted(s, values, free) * (1.0 + 1e-3 * np.random.default_rng(4).standard_normal(s.nnz))
    part = pkg.PartitionedFactor.for_system(s, free)
    part.set_dense_limit(dense_limit)
    part.factorize(torch.tensor(v, device=cuda), symmetric=False)
    b = np.random.default_rng(5).standard_normal(len(free))
    x = part.solve(torch.tensor(b, device=cuda)).cpu().numpy()
    ref = np.linalg.solve(dense_block(s, v, free), b)
    assert np.linalg.norm(x - ref) <= SOLVE_TOL * np.linalg.norm(ref)
    c = part.counts()
    assert c["cholesky"] + c["gmres"] + c["qr"] + c["lu"] == 1


@pytest.mark.parametrize("dense_limit", [20000, 0])
def test_unconstrained_block_is_singular(pkg, elastic, cuda, dense_limit):
    """Every DOF free: the rigid-body motions make the block singular, and
    the factorisation (LU) or the solve (QR) says so, as the reference's
    factorize returns false."""
    s, values, _ = elastic
    part = pkg.PartitionedFactor.for_system(s, np.arange(s.num_dofs, dtype=np.int32))
    part.set_dense_limit(dense_limit)
    with pytest.raises(pkg.SolverError):
        part.factorize(values, symmetric=False)
        part.solve(torch.ones(s.num_dofs, dtype=torch.float64, device=cuda))
    assert part.counts()["singular"] == 1


def test_bad_partitions_are_refused(pkg, elastic):
    s, _, free = elastic
    with pytest.raises(pkg.SbkError):
        pkg.PartitionedFactor.for_system(s, free[::-1].copy())
    with pytest.raises(pkg.SbkError):
        pkg.PartitionedFactor.for_system(s, np.array([0, s.num_dofs], dtype=np.int32))


@pytest.mark.parametrize("case", ["cholesky", "lu"])
def test_transposed_solve(pkg, elastic, plastic, cuda, case):
    """K_ff^-T b with the factorisation K_ff^-1 b uses (the adjoint system):
    the Cholesky of the held elastic block solves it as it stands; the dense
    LU of a non-symmetric block solves with its transpose - against a dense
    solve of the transposed block."""
    rng = np.random.default_rng(12)
    if case == "cholesky":
        s, values, free = elastic
        v = values.cpu().numpy()
    else:
        s, values = plastic
        free = np.flatnonzero(rng.random(s.num_dofs) < 0.8).astype(np.int32)
        v = values.cpu().numpy() * (1.0 + 1e-3 * rng.standard_normal(s.nnz))
    part = pkg.PartitionedFactor.for_system(s, free)
    kind = part.factorize(torch.tensor(v, device=cuda), symmetric=case == "cholesky")
    assert kind == (1 if case == "cholesky" else 4)
    b = rng.standard_normal(len(free))
    x = part.solve(torch.tensor(b, device=cuda), transpose=True).cpu().numpy()
    ref = np.linalg.solve(dense_block(s, v, free).T, b)
    assert np.linalg.norm(x - ref) <= SOLVE_TOL * np.linalg.norm(ref)
    if case == "lu":
        fwd = np.linalg.solve(dense_block(s, v, free), b)
        assert np.linalg.norm(fwd - ref) > 1e3 * SOLVE_TOL * np.linalg.norm(ref)


def test_transposed_solve_is_refused_by_gmres(pkg, plastic, cuda):
    """GMRES keeps no factorisation of the block to transpose."""
    s, values = plastic
    rng = np.random.default_rng(13)
    free = np.flatnonzero(rng.random(s.num_dofs) < 0.8).astype(np.int32)
    v = values.cpu().numpy() * (1.0 + 1e-3 * rng.standard_normal(s.nnz))
    part = pkg.PartitionedFactor.for_system(s, free)
    part.set_dense_limit(0)
    if part.factorize(torch.tensor(v, device=cuda), symmetric=False) != 3:
        pytest.skip("the block left GMRES")
    with pytest.raises(pkg.SbkError):
        part.solve(torch.ones(len(free), dtype=torch.float64, device=cuda), transpose=True)
