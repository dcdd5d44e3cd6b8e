"""Energy and concentration transport on the CUDA path, through the C ABI (needs a B200).

The scalar kernels are FP64 with the oracle's operation order, so for
Michaelis-Menten walls without inhibition (no pow in the arithmetic) every
field matches the oracle bit for bit. Hill laws and substrate inhibition call
pow, which is CUDA's on the device and the C library's in the oracle; those
fields agree to 1e-12 relative. The flow fields never depend on the scalars
and stay bit-exact in every case. Against the reference's own solver
(tests/golden, generated by tests/golden/make_golden.py) the match is to
rounding, 1e-10 relative L2, as for the flow.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

from axisim import cases
import axisim.abi as abi
import oracle
from helpers import rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

FLOW = ["u", "v", "p", "mDot", "pp"]
SCALAR_FIELDS = {"T": ["T", "gradTZ", "gradTR", "AC_T", "b_T", "AF_T", "invAC_T", "TOld", "TOld2"],
                 "C": ["C", "gradCZ", "gradCR", "AC_C", "b_C", "AF_C", "invAC_C", "COld", "COld2", "cw", "ocrWall"]}


def _uses_pow(case):
    f = case.bc_fields().get("C")
    if f is None:
        return False
    kinetic = np.isin(f["type"], (cases.MICHAELIS_MENTEN, cases.HILL))
    return bool(np.any(kinetic & ((f["type"] == cases.HILL) | (f["v2"] != 0.0))))


def _variants():
    v = [(name, c) for name, c in make_golden.scalar_fixture_cases() if not name.endswith("converged")]
    c = cases.with_scalars(cases.pipe(nr=8, nz=30, max_iter=4, tol=1e-30), energy=False,
                           wall_c=cases.michaelis_menten(5e-4, 0.3), D=1e-6)
    c.settings.update(scalarResEnabled=[0, 1], scalarResNorm=[0, 2], scalarResScale=[3, 1])
    v.append(("pipe_concentration_only_linf", c))
    c = cases.with_scalars(cases.pipe(nr=8, nz=30, max_iter=4, tol=1e-30), concentration=False, k=6.0)
    c.settings.update(scalarResEnabled=[1, 0], scalarResNorm=[1, 0], useMultigrid=0, linearType=cases.LINEAR_JACOBI,
                      linearMaxIter=7)
    v.append(("pipe_energy_only_jacobi_odd", c))
    c = cases.with_scalars(cases.bullet(scale=0.1, max_iter=4, tol=1e-30),
                           wall_c=cases.michaelis_menten(1e-3, 0.2), wall_layers=[(2e-6, 5e-5), (1e-6, 1e-4)], D=1e-6)
    v.append(("bullet_triangles_lsq_nonortho_scalars", c))
    c = cases.with_scalars(cases.expansion(scale=1 / 32, max_iter=3, tol=1e-30),
                           wall_c=cases.michaelis_menten(2e-3, 0.4, inhibition=(1.5, 0.3, 0.6)), D=2e-6)
    c.settings.update(convectionScheme=cases.CONV_CENTRAL, gradientScheme=cases.GRAD_GREEN_GAUSS)
    v.append(("expansion_central_gg_mm_inhibition", c))
    c = cases.with_scalars(cases.pulsatile_expansion(scale=1 / 32, dt=1e-3, steps=5, max_iter=2, tol=1e-30),
                           wall_c=cases.hill(1e-3, 0.3, 2.0), D=1e-6)
    v.append(("pulsatile_bdf2_five_steps_hill", c))
    return v


VARIANTS = _variants()


@pytest.mark.parametrize("name,case", VARIANTS, ids=[n for n, _ in VARIANTS])
def test_scalars_match_oracle(name, case):
    mesh = abi.multiblock(case.blocks) if case.mesh is None else case.mesh
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    r = gpu.solve()
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it, conv = orc.run()
    assert r["iterations"] == it and r["converged"] == conv
    for f in FLOW:
        assert np.array_equal(gpu.get(f), orc.get(f)), (name, f)
    exact = not _uses_pow(case)
    s = case.settings
    for key, on in (("T", s["solveEnergy"]), ("C", s["solveConcentration"])):
        if not on:
            continue
        for f in SCALAR_FIELDS[key]:
            if f in ("TOld", "TOld2", "COld", "COld2") and not s["transient"]:
                continue
            a, b = gpu.get(f), orc.get(f)
            if exact or key == "T":
                assert np.array_equal(a, b), (name, f, np.max(np.abs(a - b)))
            else:
                assert rel_l2(a, b) <= 1e-12, (name, f, rel_l2(a, b))
    sr_gpu, sr_orc = gpu.scalar_residuals(), orc.scalar_residuals()
    for e in range(2):
        if s["scalarResEnabled"][e]:
            np.testing.assert_allclose(sr_gpu[e], sr_orc[e], rtol=1e-9, atol=1e-300)
    gpu.close()
    orc.close()


GOLDEN = make_golden.scalar_fixture_cases()


@pytest.mark.parametrize("name,case", GOLDEN, ids=[n for n, _ in GOLDEN])
def test_scalars_match_reference_solver(name, case):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    mesh = abi.multiblock(case.blocks)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    r = gpu.solve()
    assert r["iterations"] == int(g["iterations"]) and r["converged"] == bool(g["converged"])
    for k in ("T", "C", "gradTZ", "gradTR", "gradCZ", "gradCR", "u", "v", "p"):
        if k in g:
            assert rel_l2(gpu.get(k), g[k]) <= 1e-10, (name, k, rel_l2(gpu.get(k), g[k]))
    hist = g["residual_history"]
    s = case.settings
    for e, on in enumerate((s["solveEnergy"], s["solveConcentration"])):
        if on and s["scalarResEnabled"][e]:
            # scaled residuals at rounding level (1e-16) carry no digits to compare
            np.testing.assert_allclose(gpu.scalar_residuals()[e], hist[-1, 4 + e], rtol=1e-6, atol=1e-12)
    gpu.close()


def test_residual_callback_reports_scalar_entries():
    case = make_golden.scalar_fixture_cases()[0][1]
    mesh = abi.multiblock(case.blocks)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    rows = []

    def cb(ctx, it, res):
        rows.append([res[i] for i in range(5)])
    fn = abi.RESIDUAL_FN(cb)
    abi.lib().axisim_set_log(gpu.h, abi.LOG_FN(0), fn, None)
    gpu.solve()
    assert len(rows) == case.settings["maxIter"]
    np.testing.assert_allclose(rows[-1][3:], gpu.scalar_residuals(), rtol=0, atol=0)
    gpu.close()


def test_scalar_state_errors_and_continue():
    case = cases.with_scalars(cases.pipe(nr=6, nz=20, max_iter=3, tol=1e-30),
                              wall_c=cases.michaelis_menten(1e-3, 0.2), D=1e-6)
    mesh = abi.multiblock(case.blocks)
    plain = abi.Solver(mesh, cases.pipe(nr=6, nz=20).bc_fields(), cases.pipe(nr=6, nz=20, max_iter=2).settings)
    plain.solve()
    with pytest.raises(abi.AxisimError) as e:
        plain.get("T")
    assert e.value.status == abi.E_STATE
    # kinetics laws apply to the scalars only
    bad = dict(case.bc_fields()["u"])
    bad["type"] = bad["type"].copy()
    bad["type"][2] = cases.MICHAELIS_MENTEN
    b, keep = abi.bc_struct(bad)
    assert abi.lib().axisim_set_bc(plain.h, abi.VAR_U, b) == abi.E_CONFIG
    plain.close()
    # continuing the same selection resumes from the fields; a changed selection cannot
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    gpu.solve()
    T3 = gpu.get("T")
    gpu.solve(cont=True)
    orc = oracle.Oracle(mesh, case.bc_fields(), dict(case.settings, maxIter=6))
    orc.run()
    assert np.array_equal(gpu.get("T"), orc.get("T")) and np.array_equal(gpu.get("C"), orc.get("C"))
    assert not np.array_equal(T3, gpu.get("T"))
    abi.lib().axisim_set_scalars(gpu.h, 1, 0, None)
    buf = ctypes.create_string_buffer(256)
    assert abi.lib().axisim_can_continue(gpu.h, buf, 256) == 0
    assert b"Concentration field selection changed." in buf.value
    gpu.close()


def test_batch_rejects_scalar_monitoring():
    case = cases.with_scalars(cases.pipe(nr=6, nz=20, max_iter=2, tol=1e-30), D=1e-6)
    case.settings.update(scalarResEnabled=[1, 0])
    mesh = abi.multiblock(case.blocks)
    gpu = abi.Solver(mesh, case.bc_fields(), case.settings)
    gpu.set_batch([0, mesh["nCells"]])
    with pytest.raises(abi.AxisimError) as e:
        gpu.solve()
    assert e.value.status == abi.E_CONFIG
    gpu.close()
