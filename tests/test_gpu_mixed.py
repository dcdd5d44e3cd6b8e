"""Mixed precision (FP32 inner solves inside FP64 refinement) against the FP64 oracle.

The FP32 path changes only how accurately each inner solve is done, not the
discrete equations, so a converged mixed run reaches the FP64 solution: the
check is relative L2 of u, v, p against the FP64 oracle run to the same
tolerance, plus the iteration count staying close to the FP64 one.
"""
import numpy as np
import pytest

from axisim import cases
import axisim.abi as abi
import oracle
from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [cases.pipe(nr=10, nz=50, max_iter=20000, tol=1e-8, fully_developed=True),
                                  cases.expansion(scale=1 / 16, max_iter=40000, tol=1e-8)],
                         ids=["pipe", "expansion"])
def test_mixed_converges_to_fp64_solution(case):
    mesh = oracle.multiblock(case.blocks)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it_o, conv_o = orc.run()
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings, precision=abi.PREC_MIXED)
    r = gpu.solve()
    assert conv_o and r["converged"]
    assert abs(r["iterations"] - it_o) <= 0.05 * it_o + 20
    for f in ("u", "v", "p"):
        assert rel_l2(gpu.get(f), orc.get(f)) <= 1e-6, (f, rel_l2(gpu.get(f), orc.get(f)))


def test_mixed_path_runs_fp32_inner_kernels():
    case = cases.expansion(scale=1 / 8, max_iter=3, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings, precision=abi.PREC_MIXED)
    gpu.solve()
    names = {k["name"] for k in gpu.profile(1)}
    assert {"ir_residual_uv", "ir_residual_pp"} <= names
    # the refinement update: its own launch, or inside the last finest-level pass of the cycle
    assert names & {"ir_update_pp", "mg_prolong_smooth_ir32"}
    assert names & {"jacobi_uv32", "jacobi_uv32_tiles"}
    # the coarser levels' sweeps: their own launches, or inside the resident kernel
    assert any(n.startswith(("mg_smooth", "mg_prolong_smooth", "mg_resident")) and n.endswith("32") for n in names)
    assert not names & {"jacobi_uv", "jacobi_uv_tiles"}


def test_mixed_few_iterations_close_to_fp64():
    case = cases.expansion(scale=1 / 8, max_iter=20, tol=1e-30)
    mesh = abi.multiblock(case.blocks)
    a = abi.Solver(mesh, case.bc_fields(), case.settings)
    b = abi.Solver(mesh, case.bc_fields(), case.settings, precision=abi.PREC_MIXED)
    a.solve()
    b.solve()
    for f in ("u", "v", "p"):
        assert rel_l2(b.get(f), a.get(f)) <= 1e-4, f
