"""The batched engine (springback-precomp_b200/batch.py): parts of uneven
size in one element launch, per-part views of the result through the
offset table, an evaluation captured as a CUDA graph and replayed across
commits, and the launch-shape autotuner. The batch must give every part
what the part's own system gives, bit for bit: each element is evaluated
alone, and each tangent value sums the part's own elements in element
order."""
from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def part_meshes(pkg):
    return [pkg.structured_hex_mesh(6, 4, 2, 6e-3, 4e-3, 1e-3), pkg.structured_hex_mesh(10, 3, 2, 10e-3, 3e-3, 1e-3),
            pkg.structured_hex_mesh(5, 5, 1, 5e-3, 5e-3, 1e-3)]


def bend(mesh, c):
    x = mesh.coords
    u = np.zeros_like(x)
    xc = x[:, 0].mean()
    u[:, 2] = -c * (x[:, 0] - xc) ** 2 / (x[:, 0].max() - x[:, 0].min())
    u[:, 0] = 0.1 * c * (x[:, 2] - x[:, 2].mean()) * (x[:, 0] - xc) / (x[:, 0].max() - x[:, 0].min())
    return u.reshape(-1)


@pytest.fixture(scope="module")
def batch_setup(pkg, cuda):
    batch_mod = importlib.import_module("springback-precomp_b200.batch")
    meshes = part_meshes(pkg)
    mat = pkg.material.hill_chaboche_sheet()
    us = [bend(m, c) for m, c in zip(meshes, (0.004, 0.006, 0.003))]
    return batch_mod, meshes, mat, us


def test_batch_gives_every_part_its_own_result(pkg, cuda, batch_setup):
    batch_mod, meshes, mat, us = batch_setup
    batch = batch_mod.PartBatch(meshes, mat)
    assert batch.offsets.shape == (4, 4)
    u = torch.tensor(np.concatenate(us), device=cuda)
    ev = batch.evaluate(u)
    assert ev.yielding_points > 0
    internal, values = ev.internal.clone(), ev.tangent.clone()
    for p, (m, up) in enumerate(zip(meshes, us)):
        own = pkg.NonlinearSystem(m, mat)
        oe = own.evaluate(torch.tensor(up, device=cuda), 0.0, True)
        view = batch.part(p, internal, values)
        assert torch.equal(view.internal, oe.internal)
        assert torch.equal(view.outer, own.outer)
        assert torch.equal(view.inner, own.inner)
        assert torch.equal(view.values, oe.tangent)


def test_standard_element_batch_gives_every_part_its_own_result(pkg, cuda, batch_setup):
    """The same for the standard Hex8 with mean dilatation (the element of
    the reference's springback_2mm preset): each element's averaged
    dilatation is its own, so the batch changes no bit."""
    batch_mod, meshes, mat, us = batch_setup
    batch = batch_mod.PartBatch(meshes, mat, element="standard", mean_dilatation="auto")
    assert batch.system.averaged
    u = torch.tensor(np.concatenate(us), device=cuda)
    ev = batch.evaluate(u)
    assert ev.yielding_points > 0
    internal, values = ev.internal.clone(), ev.tangent.clone()
    for p, (m, up) in enumerate(zip(meshes, us)):
        own = pkg.NonlinearSystem(m, mat, element="standard", mean_dilatation="auto")
        oe = own.evaluate(torch.tensor(up, device=cuda), 0.0, True)
        view = batch.part(p, internal, values)
        assert torch.equal(view.internal, oe.internal)
        assert torch.equal(view.values, oe.tangent)


def test_graph_replay_across_commits(pkg, cuda, batch_setup):
    """A captured evaluation replayed at two displacements with a commit
    between equals the same sequence through plain evaluate calls."""
    batch_mod, meshes, mat, us = batch_setup
    u1 = np.concatenate(us)
    u2 = 1.3 * u1
    batch = batch_mod.PartBatch(meshes, mat)
    ubuf = torch.tensor(u1, device=cuda)
    g = batch_mod.GraphedEvaluation(batch.system, ubuf)
    ref = batch_mod.PartBatch(meshes, mat)
    got, want = [], []
    for k, uk in enumerate((u1, u2)):
        ubuf.copy_(torch.tensor(uk, device=cuda))
        summary = g.replay()
        torch.cuda.synchronize()
        s = summary.cpu().numpy()
        assert s[3] == -1.0
        got.append((batch.system.internal_view().clone(), batch.system.values_view().clone(), s[0], s[1], int(s[2])))
        batch.system.commit()
        ev = ref.evaluate(torch.tensor(uk, device=cuda))
        want.append((ev.internal.clone(), ev.tangent.clone(), ev.energy, ev.gross, ev.yielding_points))
        ref.system.commit()
    for (gi, gv, ge, gg, gy), (wi, wv, we, wg, wy) in zip(got, want):
        assert torch.equal(gi, wi) and torch.equal(gv, wv)
        assert ge == we and gy == wy
        assert abs(gg - wg) <= 1e-15 * wg


def test_autotune_picks_a_shape_and_changes_no_result(pkg, cuda, batch_setup):
    batch_mod, meshes, mat, us = batch_setup
    batch = batch_mod.PartBatch(meshes, mat)
    u = torch.tensor(np.concatenate(us), device=cuda)
    before = batch.evaluate(u).internal.clone()
    times = batch.autotune(u, candidates=(1, 2, 4, 8))
    assert set(times) == {1, 2, 4, 8} and all(t > 0 for t in times.values())
    assert batch.chosen_elements_per_block == min(times, key=times.get)
    assert torch.equal(batch.evaluate(u).internal, before)


def test_autotune_over_the_thread_mappings(pkg, cuda, batch_setup):
    """The autotuner's search over the mapping of points to threads - the
    phase kernels or the single kernel, at two block shapes each - keeps the
    fastest; the results stay those of the default mapping (to the last bits
    the two compiled paths may differ in)."""
    batch_mod, meshes, mat, us = batch_setup
    batch = batch_mod.PartBatch(meshes, mat)
    u = torch.tensor(np.concatenate(us), device=cuda)
    before = batch.evaluate(u)
    f0, k0 = before.internal.clone(), before.tangent.clone()
    cands = (("phases", 0), ("phases", 8), ("single", 16), ("single", 8))
    times = batch.autotune(u, candidates=cands)
    assert set(times) == set(cands) and batch.chosen == min(times, key=times.get)
    after = batch.evaluate(u)
    assert (after.internal - f0).abs().max().item() <= 1e-13 * f0.abs().max().item()
    assert (after.tangent - k0).abs().max().item() <= 1e-13 * k0.abs().max().item()
