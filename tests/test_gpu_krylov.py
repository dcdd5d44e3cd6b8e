"""Flexible CG with the FP32 V-cycle preconditioner for the p' solve.

The Krylov solve changes how accurately each pressure correction is computed,
not the discrete equations, so a converged run reaches the FP64 oracle's
converged fields; what it changes is the number of SIMPLE iterations needed.
"""
import pytest

from axisim import cases
import axisim.abi as abi
import oracle
from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("case", [cases.pipe(nr=10, nz=50, max_iter=20000, tol=1e-8, fully_developed=True),
                                  cases.expansion(scale=1 / 16, max_iter=40000, tol=1e-8)],
                         ids=["pipe", "expansion"])
def test_fcg_converges_to_fp64_solution(case, precision):
    mesh = oracle.multiblock(case.blocks)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it_o, conv_o = orc.run()
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings, precision=precision, pressure_solver=abi.PSOLVE_FCG)
    r = gpu.solve()
    assert conv_o and r["converged"]
    # A more exact p' does not always mean fewer SIMPLE iterations: on the
    # 1/16-scale expansion the fixed three V-cycles damp the pressure update
    # the way the under-relaxation needs and FCG takes about twice as many.
    assert r["iterations"] < 3 * it_o, (r["iterations"], it_o)
    for f in ("u", "v", "p"):
        assert rel_l2(gpu.get(f), orc.get(f)) <= 1e-6, (f, rel_l2(gpu.get(f), orc.get(f)))


def test_fcg_runs_krylov_kernels_and_rejects_unknown_mode():
    case = cases.expansion(scale=1 / 8, max_iter=3, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings, pressure_solver=abi.PSOLVE_FCG)
    gpu.solve()
    names = {k["name"] for k in gpu.profile(1)}
    assert {"fcg_init", "fcg_dots", "fcg_spmv", "fcg_update"} <= names
    # the coarser levels' sweeps: their own launches, or inside the resident kernel
    assert any(n.startswith(("mg_smooth", "mg_prolong_smooth", "mg_resident")) and n.endswith("32") for n in names)
    assert "ir_update_pp" not in names
    st = abi.lib().axisim_set_pressure_solver(gpu.h, 7, 0.0, 1.0)
    assert st == abi.E_ARG


def test_fcg_reaches_lower_continuity_than_vcycles_in_same_iterations():
    case = cases.expansion(scale=1 / 8, max_iter=400, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    a = abi.Solver(mesh, case.bc_fields(), case.settings)
    b = abi.Solver(mesh, case.bc_fields(), case.settings, pressure_solver=abi.PSOLVE_FCG)
    ra, rb = a.solve(), b.solve()
    assert ra["iterations"] == rb["iterations"] == 400
    assert rb["residual"][2] < ra["residual"][2], (rb["residual"], ra["residual"])


def test_fcg_relative_tolerance_stops_early_and_keeps_the_solution():
    case = cases.expansion(scale=1 / 16, max_iter=40000, tol=1e-8)
    mesh = abi.multiblock(case.blocks)
    st = dict(case.settings)
    st["mgMaxIter"] = 40
    full = abi.Solver(mesh, case.bc_fields(), case.settings, pressure_solver=abi.PSOLVE_FCG)
    early = abi.Solver(mesh, case.bc_fields(), st, pressure_solver=abi.PSOLVE_FCG, pressure_tol=1e-2)
    rf, re = full.solve(), early.solve()
    assert rf["converged"] and re["converged"]
    solves, iters = early.pressure_stats()
    assert solves == re["iterations"] and 0 < iters < 40 * solves
    for f in ("u", "v", "p"):
        assert rel_l2(early.get(f), full.get(f)) <= 1e-6, f
    assert abi.lib().axisim_set_pressure_solver(early.h, abi.PSOLVE_FCG, 1.5, 1.0) == abi.E_ARG
    assert abi.lib().axisim_set_pressure_solver(early.h, abi.PSOLVE_FCG, 0.1, 0.0) == abi.E_ARG


@pytest.mark.parametrize("cap", [9, 10])
def test_fcg_conditional_loop_matches_unrolled_iterations_and_keeps_the_cap(cap):
    """With a tolerance the captured solve repeats its Krylov iterations in a
    conditional WHILE node (two per body); without one they are unrolled. A
    tolerance no solve reaches runs every solve to the cap either way, so both
    graphs compute the same iterations: same fields bit for bit, and exactly
    cap iterations per solve for an odd and an even number of loop iterations."""
    import numpy as np
    case = cases.expansion(scale=1 / 8, max_iter=6, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    st = dict(case.settings, mgMaxIter=cap)
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        loop = abi.Solver(mesh, case.bc_fields(), st, precision=prec, pressure_solver=abi.PSOLVE_FCG,
                          pressure_tol=1e-300)
        unrolled = abi.Solver(mesh, case.bc_fields(), st, precision=prec, pressure_solver=abi.PSOLVE_FCG)
        ra, rb = loop.solve(), unrolled.solve()
        assert ra["iterations"] == rb["iterations"] == 6
        assert loop.pressure_stats() == unrolled.pressure_stats() == (6, 6 * cap)
        for f in ("u", "v", "p"):
            assert np.array_equal(loop.get(f), unrolled.get(f)), (prec, f)


def test_fcg_over_corrected_preconditioner_converges_to_the_same_solution():
    case = cases.expansion(scale=1 / 16, max_iter=40000, tol=1e-8)
    mesh = abi.multiblock(case.blocks)
    a = abi.Solver(mesh, case.bc_fields(), case.settings, pressure_solver=abi.PSOLVE_FCG)
    b = abi.Solver(mesh, case.bc_fields(), case.settings, pressure_solver=abi.PSOLVE_FCG, prolong_scale=2.0)
    ra, rb = a.solve(), b.solve()
    assert ra["converged"] and rb["converged"]
    for f in ("u", "v", "p"):
        assert rel_l2(b.get(f), a.get(f)) <= 1e-6, f
