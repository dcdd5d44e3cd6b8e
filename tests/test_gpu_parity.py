"""CUDA path vs the CPU oracle, through the C ABI (needs a B200).

The FP64 path is built to reproduce the oracle bit for bit (same operation
order, no FMA contraction, deterministic multigrid gathers), so intermediate
state after a fixed number of SIMPLE iterations is compared with exact
equality. Residual norms come from a different reduction order and are compared
to 1e-12 relative.
"""
import numpy as np
import pytest

from axisim import cases
import axisim.abi as abi
import oracle
from helpers import FIELDS, GEOM, rel_l2

pytestmark = pytest.mark.gpu


def _variants():
    v = []
    c = cases.pipe(nr=10, nz=50, max_iter=5, tol=1e-30)
    v.append(("pipe_gg_gsrb_upwind", c))
    c = cases.expansion(scale=1 / 32, max_iter=5, tol=1e-30)
    v.append(("expansion_lsq_jacobi_sou", c))
    c = cases.expansion(scale=1 / 32, max_iter=4, tol=1e-30)
    c.settings.update(convectionScheme=cases.CONV_CENTRAL, gradientScheme=cases.GRAD_GREEN_GAUSS)
    v.append(("expansion_gg_central", c))
    c = cases.expansion(scale=1 / 32, max_iter=3, tol=1e-30)
    c.settings.update(useNonOrthCorrector=1)
    v.append(("expansion_nonortho", c))
    c = cases.pipe(nr=8, nz=40, max_iter=4, tol=1e-30)
    c.settings.update(useMultigrid=0, linearType=cases.LINEAR_JACOBI, linearMaxIter=7)
    v.append(("pipe_no_mg_jacobi_odd", c))
    c = cases.pipe(nr=8, nz=40, max_iter=4, tol=1e-30)
    c.settings.update(useMultigrid=0, linearType=cases.LINEAR_GS_RB)
    v.append(("pipe_no_mg_gs", c))
    c = cases.pipe(nr=8, nz=40, max_iter=4, tol=1e-30, fully_developed=True)
    c.settings.update(convectionScheme=cases.CONV_QUICK, mgPreSweep=2, mgPostSweep=1, mgMaxIter=2,
                      resNorm=[1, 2, 0], resScale=[1, 2, 0], checkConv=2)
    v.append(("pipe_quick_norms", c))
    c = cases.expansion(scale=1 / 4, max_iter=2, tol=1e-30)
    v.append(("expansion_54k_deep_multigrid", c))
    c = cases.expansion(scale=1 / 4, max_iter=2, tol=1e-30)
    c.settings.update(mgPreSweep=0, mgPostSweep=2, mgLinearSweep=7, mgMaxIter=1)
    v.append(("expansion_54k_mg_sweeps", c))
    c = cases.bullet(scale=0.1, max_iter=4, tol=1e-30)
    v.append(("bullet_triangles_lsq_nonortho", c))
    c = cases.bullet(scale=0.25, max_iter=2, tol=1e-30)
    c.settings.update(gradientScheme=cases.GRAD_GREEN_GAUSS, convectionScheme=cases.CONV_SOU)
    v.append(("bullet_triangles_gg_sou_deep_mg", c))
    c = cases.pulsatile_expansion(scale=1 / 32, dt=1e-3, steps=3, max_iter=3, tol=1e-30)
    v.append(("pulsatile_bdf2", c))
    c = cases.pulsatile_expansion(scale=1 / 32, dt=1e-3, steps=2, max_iter=3, tol=1e-30)
    c.settings.update(timeScheme=cases.TIME_FIRST_ORDER)
    v.append(("transient_bdf1", c))
    return v


VARIANTS = _variants()


@pytest.mark.parametrize("name,case", VARIANTS, ids=[n for n, _ in VARIANTS])
def test_bitexact_after_iterations(name, case):
    mesh = case.packed(oracle.multiblock)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    it_o, conv_o = orc.run()
    r = gpu.solve()
    assert r["iterations"] == it_o
    for g in GEOM:
        np.testing.assert_array_equal(gpu.get(g), orc.get(g), err_msg=g)
    for f in FIELDS:
        a, b = gpu.get(f), orc.get(f)
        assert a.shape == b.shape, f
        if f.startswith("res_") and name == "pipe_quick_norms":
            continue  # residual arrays are only written on check iterations (checkConv=2)
        np.testing.assert_array_equal(a, b, err_msg=f"{name}: {f}")
    np.testing.assert_allclose(r["residual"], orc.residuals(), rtol=1e-12, atol=0)


def test_continue_matches_single_run():
    case = cases.expansion(scale=1 / 32, max_iter=3, tol=1e-30)
    mesh = oracle.multiblock(case.blocks)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    orc.run()
    orc.run(cont=True)
    gpu.solve()
    ok, why = gpu.can_continue()
    assert ok, why
    r = gpu.solve(cont=True)
    assert r["total"] == orc.iterations() == 6
    for f in ("u", "v", "p", "mDot"):
        np.testing.assert_array_equal(gpu.get(f), orc.get(f), err_msg=f)


def test_converged_pipe_matches_oracle_and_poiseuille():
    case = cases.pipe(nr=10, nz=50, max_iter=5000, tol=1e-6, fully_developed=True)
    mesh = oracle.multiblock(case.blocks)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    it_o, conv_o = orc.run()
    r = gpu.solve()
    assert conv_o and r["converged"]
    assert r["iterations"] == it_o
    for f in ("u", "v", "p"):
        assert rel_l2(gpu.get(f), orc.get(f)) <= 1e-12, f
    u = gpu.get("u")
    rr, zz = mesh["cellCenterR"], mesh["cellCenterZ"]
    ua = 0.1 * (1 - (rr / 0.01) ** 2)
    assert rel_l2(u, ua) < 5e-3


def test_multigrid_hierarchy_and_coloring_match_oracle():
    case = cases.expansion(scale=1 / 16, max_iter=1)
    case.settings.update(linearType=cases.LINEAR_GS_RB)
    mesh = oracle.multiblock(case.blocks)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    np.testing.assert_array_equal(gpu.mg_levels(), orc.mg_levels())
    for lvl in range(len(orc.mg_levels()) - 1):
        for a, b in zip(gpu.mg_level_maps(lvl), orc.mg_level_maps(lvl)):
            np.testing.assert_array_equal(a, b)
    ca, na = gpu.coloring()
    cb, nb = orc.coloring()
    assert na == nb
    np.testing.assert_array_equal(ca, cb)


def test_errors_are_status_codes():
    case = cases.pipe(nr=4, nz=8, max_iter=2)
    mesh = oracle.multiblock(case.blocks)
    s = dict(case.settings)
    s["mu"] = -1.0
    gpu = abi.Solver(mesh, case.bc_fields(), s)
    r = gpu.solve(allow=(abi.E_CONFIG,))
    assert r["status"] == abi.E_CONFIG
    s = dict(case.settings)
    s.update(transient=1, dt=0.0)
    gpu = abi.Solver(mesh, case.bc_fields(), s)
    assert gpu.solve(allow=(abi.E_CONFIG,))["status"] == abi.E_CONFIG
    with pytest.raises(abi.AxisimError):
        gpu.get("no_such_field")
    bad = dict(mesh)
    bad["faceOwner"] = mesh["faceOwner"].copy()
    bad["faceOwner"][0] = mesh["nCells"] + 5
    with pytest.raises(abi.AxisimError) as e:
        abi.Solver(bad, case.bc_fields(), case.settings)
    assert e.value.status == abi.E_MESH


@pytest.mark.parametrize("name", [n for n, _ in __import__("make_golden").fixture_cases()])
def test_cuda_path_matches_reference_solver(name):
    """The CUDA path against the reference's own solver (golden vectors)."""
    import os
    import make_golden
    case = dict(make_golden.fixture_cases())[name]
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
    mesh = case.packed(abi.multiblock)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    r = gpu.solve()
    assert r["iterations"] == int(g["iterations"]) and r["converged"] == bool(g["converged"])
    for k in ("u", "v", "p", "gradPZ", "gradPR"):
        if k in g:
            assert rel_l2(gpu.get(k), g[k]) <= 1e-10, (name, k)
