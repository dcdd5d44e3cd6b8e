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


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_batch_with_multigrid_is_bitexact_per_case(precision):
    # every case is coarsened on its own (its standalone hierarchy), and the
    # cases whose hierarchy ends above the deepest batch level get their
    # coarsest-level sweeps there, so each case evolves exactly as it does alone
    cs, meshes, union, start, bcs = _batch(6, 5, 0.05, maxIter=5, resTol=[1e-30] * 3)
    cells, term = abi.mg_batch_levels_host(union, start)
    assert term.sum() > 0, "the draw should hold cases of different depths"
    g = abi.Solver(union, bcs, cs[0].settings, precision=precision)
    g.set_batch(start)
    r = g.solve()
    assert r["iterations"] == 5
    np.testing.assert_array_equal(g.mg_levels(), cells)
    for i, c in enumerate(cs):
        alone = abi.Solver(meshes[i], c.bc_fields(), c.settings, precision=precision)
        alone.solve()
        for f in ("u", "v", "p", "pp"):
            np.testing.assert_array_equal(batch.split_fields(g.get(f), start)[i], alone.get(f), err_msg=f"{i} {f}")
        np.testing.assert_array_equal(_split_faces(g.get("mDot"), meshes, i), alone.get("mDot"), err_msg=f"{i} mDot")
        alone.close()
    g.close()


def _split_faces(a, meshes, i):
    off = sum(int(m["nFaces"]) for m in meshes[:i])
    return a[off:off + int(meshes[i]["nFaces"])]


def test_batch_converges_each_case_where_it_converges_alone():
    # per-case hierarchies and per-case monitoring: every case that converges
    # alone converges in the batch, at the same iteration
    cs, meshes, union, start, bcs = _batch(5, 7, 0.02, maxIter=12000, resTol=[1e-8] * 3)
    g = abi.Solver(union, bcs, cs[0].settings)
    g.set_batch(start)
    g.solve()
    conv_at, res = g.batch_status()
    g.close()
    n_conv = 0
    for i, c in enumerate(cs):
        alone = abi.Solver(meshes[i], c.bc_fields(), c.settings)
        ra = alone.solve()
        alone.close()
        assert (conv_at[i] >= 0) == ra["converged"], (i, conv_at[i], ra)
        if ra["converged"]:
            n_conv += 1
            # convergedAt is the index of the converging iteration; total counts iterations
            assert conv_at[i] + 1 == ra["total"], (i, conv_at[i], ra["total"])
    assert n_conv >= 3


def test_batch_layout_is_validated():
    cs, meshes, union, start, bcs = _batch(2, 1, 0.02)
    g = abi.Solver(union, bcs, cs[0].settings)
    with pytest.raises(abi.AxisimError):
        g.set_batch([0, 10, union["nCells"]])   # a face crosses the boundary at cell 10
    with pytest.raises(abi.AxisimError):
        g.set_batch([0, union["nCells"] - 1])   # does not cover the mesh


def test_batched_solve_matches_reference_solver_per_case():
    # the reference solves each of the four cases alone (fixtures
    # batch4_case*); the batched solve of their packed union must give each
    # case's fields to rounding (the reference's atomicAdd order). Unbatched,
    # the union is one mesh with one hierarchy, as the reference solves it.
    import os
    import make_golden
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    case, start = make_golden.batch_union()
    s = abi.Solver(case.mesh, case.bc_fields(), case.settings)
    s.set_batch(start)
    r = s.solve()
    assert r["iterations"] == 5
    names = [n for n, _ in make_golden.fixture_cases() if n.startswith("batch4_case")]
    assert len(names) == len(start) - 1
    for i, name in enumerate(names):
        g = np.load(os.path.join(here, name + ".npz"))
        assert int(g["iterations"]) == 5
        for f in ("u", "v", "p"):
            mine = batch.split_fields(s.get(f), start)[i]
            assert rel_l2(mine, g[f]) <= 1e-10, (name, f, rel_l2(mine, g[f]))
    s.close()
    u = abi.Solver(case.mesh, case.bc_fields(), case.settings)
    u.solve()
    g = np.load(os.path.join(here, case.name + "_5it.npz"))
    for f in ("u", "v", "p"):
        assert rel_l2(u.get(f), g[f]) <= 1e-10, (f, rel_l2(u.get(f), g[f]))
    u.close()
