"""Multigrid launch-shape autotuner (needs a B200): a tuned solve computes the
same fields bit for bit as an untuned one, because a level's block size changes
no cell's arithmetic; the report gives a candidate size for every level the
V-cycle launches kernels on, 0 for the levels solved inside the one-CTA tail,
and positive sweep times."""
import numpy as np
import pytest

from axisim import batch, cases
import axisim.abi as abi

pytestmark = pytest.mark.gpu


def _check_report(s):
    blocks, us = s.autotune_report()
    assert len(blocks) == len(s.mg_levels())
    tuned = blocks > 0
    k = int(tuned.sum())
    assert k >= 1 and tuned[:k].all() and not tuned[k:].any()
    assert set(blocks[:k].tolist()) <= {64, 128, 256}
    assert (us[:k] > 0).all()
    return blocks


@pytest.mark.parametrize("prec,psolve", [(abi.PREC_FP64, abi.PSOLVE_VCYCLES), (abi.PREC_MIXED, abi.PSOLVE_VCYCLES),
                                         (abi.PREC_MIXED, abi.PSOLVE_FCG)], ids=["fp64", "mixed", "mixed_fcg"])
def test_tuned_solve_is_bitexact_with_untuned(prec, psolve):
    case = cases.expansion(scale=1 / 4, max_iter=8, tol=0.0)
    mesh = abi.multiblock(case.blocks)
    plain = abi.Solver(mesh, case.bc_fields(), case.settings, precision=prec, pressure_solver=psolve)
    tuned = abi.Solver(mesh, case.bc_fields(), case.settings, precision=prec, pressure_solver=psolve, autotune=True)
    ra, rb = plain.solve(), tuned.solve()
    assert ra["iterations"] == rb["iterations"] == 8
    for f in ("u", "v", "p"):
        np.testing.assert_array_equal(plain.get(f), tuned.get(f), err_msg=f)
    _check_report(tuned)
    assert (plain.autotune_report()[0] == 0).all()
    tuned.set_autotune(False)
    assert (tuned.autotune_report()[0] == 0).all()


def test_tuned_batch_is_bitexact_with_untuned():
    cs = batch.random_cases(6, seed=5, scale=0.05)
    for c in cs:
        c.settings.update(maxIter=6, resTol=[1e-30] * 3)
    meshes = [abi.multiblock(c.blocks) for c in cs]
    union, start, bcs = batch.pack_union(meshes, [c.groups for c in cs])
    runs = []
    for tune in (False, True):
        g = abi.Solver(union, bcs, cs[0].settings, precision=abi.PREC_MIXED, autotune=tune)
        g.set_batch(start)
        assert g.solve()["iterations"] == 6
        runs.append({f: g.get(f) for f in ("u", "v", "p")})
        if tune:
            _check_report(g)
    for f in ("u", "v", "p"):
        np.testing.assert_array_equal(runs[0][f], runs[1][f], err_msg=f)
