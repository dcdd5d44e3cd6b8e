"""The resident V-cycle (needs a B200): every multigrid phase below the finest
level run by one cooperative kernel with grid-wide barriers between phases.

Each phase keeps the per-cell arithmetic of its separate kernel, so a solve
with the resident kernel must equal the same solve with one launch per phase
bit for bit: FP64, mixed precision, the flexible-CG p' solve (the V-cycle as
its preconditioner, inside the graph's conditional loop) and a batch with
per-case hierarchies (terminal cases solved inside the resident kernel). The
give-up path of its barrier is tested by making a wait run out on purpose: the
solve returns AXISIM_E_TIMEOUT after about a second and the handle is usable
again.
"""
import time

import numpy as np
import pytest

from axisim import batch, cases
import axisim.abi as abi

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "p", "pp", "mDot")


def _pair(mesh, bcs, settings, **kw):
    out = []
    for mode in (abi.VCYCLE_PER_PHASE, abi.VCYCLE_RESIDENT):
        s = abi.Solver(mesh, bcs, settings, **kw)
        s.set_vcycle_kernel(mode)
        r = s.solve()
        out.append((s, r))
    return out


@pytest.mark.parametrize("precision,psolve", [(abi.PREC_FP64, abi.PSOLVE_VCYCLES), (abi.PREC_MIXED, abi.PSOLVE_VCYCLES),
                                              (abi.PREC_MIXED, abi.PSOLVE_FCG)], ids=["fp64", "mixed", "mixed_fcg"])
def test_resident_vcycle_is_bitexact_with_per_phase_launches(precision, psolve):
    case = cases.expansion(scale=1 / 4, max_iter=4, tol=1e-30)  # 54k cells, 7 levels, tail below 1024 cells
    mesh = abi.multiblock(case.blocks)
    st = dict(case.settings)
    kw = {"precision": precision}
    if psolve == abi.PSOLVE_FCG:
        st["mgMaxIter"] = 12
        kw.update(pressure_solver=abi.PSOLVE_FCG, pressure_tol=1e-3, prolong_scale=2.0)
    (a, ra), (b, rb) = _pair(mesh, case.bc_fields(), st, **kw)
    assert ra["iterations"] == rb["iterations"] == 4
    for f in FIELDS:
        np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)
    names = {k["name"] for k in b.profile(1)}
    assert any(n.startswith("mg_resident") for n in names), names
    assert not any(n.startswith("mg_resident") for n in {k["name"] for k in a.profile(1)})
    a.close()
    b.close()


def test_resident_vcycle_runs_terminal_cases_of_a_batch():
    cs = batch.random_cases(6, seed=5, scale=0.05, max_iter=4, tol=1e-30)
    meshes = [abi.multiblock(c.blocks) for c in cs]
    union, start, bcs = batch.pack_union(meshes, [c.groups for c in cs])
    _, term = abi.mg_batch_levels_host(union, start)
    assert term.sum() > 0
    out = []
    for mode in (abi.VCYCLE_PER_PHASE, abi.VCYCLE_RESIDENT):
        s = abi.Solver(union, bcs, cs[0].settings)
        s.set_batch(start)
        s.set_vcycle_kernel(mode)
        assert s.solve()["iterations"] == 4
        out.append({f: s.get(f) for f in FIELDS})
        s.close()
    for f in FIELDS:
        np.testing.assert_array_equal(out[0][f], out[1][f], err_msg=f)


def test_resident_barrier_gives_up_and_the_handle_recovers():
    case = cases.expansion(scale=1 / 8, max_iter=50, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    s = abi.Solver(mesh, case.bc_fields(), case.settings)
    s.set_vcycle_kernel(abi.VCYCLE_RESIDENT)
    assert abi.lib().axisim_test_barrier_timeout(s.h, 1) == abi.OK
    t0 = time.perf_counter()
    r = s.solve(allow=(abi.E_TIMEOUT,))
    assert r["status"] == abi.E_TIMEOUT, r
    assert time.perf_counter() - t0 < 60
    assert r["iterations"] <= 1, r
    ok, why = s.can_continue()
    assert not ok and "barrier" in why
    assert abi.lib().axisim_test_barrier_timeout(s.h, 0) == abi.OK
    s.set_max_iter(5)
    r = s.solve()
    assert r["status"] == abi.OK and r["iterations"] == 5
    g = abi.Solver(mesh, case.bc_fields(), dict(case.settings, maxIter=5))
    g.set_vcycle_kernel(abi.VCYCLE_RESIDENT)
    g.solve()
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f), g.get(f), err_msg=f)
    s.close()
    g.close()
