"""Batches: many independent cases packed into one mesh and advanced by the
same kernels (needs a B200)."""
import numpy as np
import pytest

from axisim import batch, cases
import axisim.abi as abi
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _batch(n, seed, scale, **settings):
    cs = batch.random_cases(n, seed=seed, scale=scale)
    for c in cs:
        c.settings.update(settings)
    meshes = [abi.multiblock(c.blocks) for c in cs]
    union, start, bcs = batch.pack_union(meshes, [c.groups for c in cs])
    return cs, meshes, union, start, bcs


def test_batch_without_multigrid_is_bitexact_per_case():
    # without multigrid every kernel is per cell / per face, so each case of the
    # batch must evolve exactly as it does alone
    cs, meshes, union, start, bcs = _batch(4, 3, 0.02, useMultigrid=0, maxIter=6, resTol=[1e-30] * 3)
    g = abi.Solver(union, bcs, cs[0].settings)
    g.set_batch(start)
    r = g.solve()
    assert r["iterations"] == 6
    for i, c in enumerate(cs):
        alone = abi.Solver(meshes[i], c.bc_fields(), c.settings)
        alone.solve()
        for f in ("u", "v", "p"):
            np.testing.assert_array_equal(batch.split_fields(g.get(f), start)[i], alone.get(f), err_msg=f"{i} {f}")


def test_batch_with_multigrid_converges_to_standalone_fields():
    # The batch builds ONE agglomeration hierarchy over all cases, and its
    # global stop (<= 64 cells in total) coarsens each case deeper than a
    # standalone solve would, so iteration counts differ; every case that
    # converges alone must converge in the batch to the same fields. (Seed 7
    # holds one expansion that stalls under the reference algorithm even alone.)
    cs, meshes, union, start, bcs = _batch(5, 7, 0.02, maxIter=12000, resTol=[1e-8] * 3)
    g = abi.Solver(union, bcs, cs[0].settings)
    g.set_batch(start)
    g.solve()
    conv_at, res = g.batch_status()
    n_conv = 0
    for i, c in enumerate(cs):
        alone = abi.Solver(meshes[i], c.bc_fields(), c.settings)
        ra = alone.solve()
        if not ra["converged"]:
            continue
        n_conv += 1
        assert conv_at[i] >= 0, (i, ra)
        for f in ("u", "p"):
            assert rel_l2(batch.split_fields(g.get(f), start)[i], alone.get(f)) <= 1e-5, (i, f)
    assert n_conv >= 3


def test_batch_layout_is_validated():
    cs, meshes, union, start, bcs = _batch(2, 1, 0.02)
    g = abi.Solver(union, bcs, cs[0].settings)
    with pytest.raises(abi.AxisimError):
        g.set_batch([0, 10, union["nCells"]])   # a face crosses the boundary at cell 10
    with pytest.raises(abi.AxisimError):
        g.set_batch([0, union["nCells"] - 1])   # does not cover the mesh


def test_batched_solve_matches_reference_solver_on_the_union():
    # the reference solves the packed union of four cases as one mesh; batch
    # mode only adds per-case monitoring, so with the tolerance out of reach the
    # batched fields equal the reference's to rounding (its atomicAdd order)
    import os
    import make_golden
    case, start = make_golden.batch_union()
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", case.name + "_5it.npz"))
    s = abi.Solver(case.mesh, case.bc_fields(), case.settings)
    s.set_batch(start)
    r = s.solve()
    assert r["iterations"] == int(g["iterations"]) == 5
    for f in ("u", "v", "p"):
        assert rel_l2(s.get(f), g[f]) <= 1e-10, (f, rel_l2(s.get(f), g[f]))
