"""Energy and concentration transport in the CPU oracle (no GPU needed).

The oracle restates the reference's scalar step (solver.cpp:1218-1238), the
reactive-wall branch of addTransportCoefficients (solver_util.cu:388-411) and
the wall Newton solves (concentration_equation.cu:90-160); its values are
pinned against the reference's own solver in test_oracle_golden.py. These
tests check properties the discretisation has whatever the pin: the scalars
are passive, each reactive wall face satisfies its flux balance, and a
converged concentration field conserves the species between inlet, outlet and
wall.
"""
import numpy as np

from axisim import cases, export
import oracle


def _pipe_mm(max_iter=10, tol=1e-30, **kw):
    return cases.with_scalars(cases.pipe(nr=10, nz=50, max_iter=max_iter, tol=tol),
                              wall_c=cases.michaelis_menten(1e-3, 0.2), wall_layers=[(1e-6, 1e-4)], D=1e-6, **kw)


def _run(case):
    mesh = oracle.multiblock(case.blocks)
    o = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it, conv = o.run()
    return mesh, o, it, conv


def _dpf(mesh, fc, n):
    return abs((mesh["faceCenterZ"][fc] - mesh["cellCenterZ"][n]) * mesh["faceNormalZ"][fc]
               + (mesh["faceCenterR"][fc] - mesh["cellCenterR"][n]) * mesh["faceNormalR"][fc])


def test_scalars_are_passive():
    base = cases.pipe(nr=10, nz=50, max_iter=8, tol=1e-30)
    _, o0, _, _ = _run(base)
    _, o1, _, _ = _run(_pipe_mm(max_iter=8))
    for f in ("u", "v", "p", "mDot", "pp"):
        assert np.array_equal(o0.get(f), o1.get(f)), f
    assert np.all(np.isfinite(o1.get("T"))) and np.all(np.isfinite(o1.get("C")))


def _wall_faces(mesh, case, var="C"):
    f = case.bc_fields()[var]
    g = mesh["faceBoundaryGroupID"]
    nb = mesh["faceNeighbor"]
    reactive = [k for k in range(len(f["type"])) if f["type"][k] in (cases.MICHAELIS_MENTEN, cases.HILL)]
    return np.flatnonzero((nb < 0) & np.isin(g, reactive)), f


def _rate(f, gid, c):
    t = f["type"][gid]
    vmax, km, n, m, k2, v2 = (f[k][gid] for k in ("vmax", "km", "n", "m", "k2", "v2"))
    r = vmax * c ** n / (km ** n + c ** n) if t == cases.HILL else vmax * c / (km + c)
    if v2 != 0.0:
        r = r * (1.0 - v2 * c ** m / (k2 ** m + c ** m))
    return r


def test_reactive_wall_faces_balance_diffusion_and_consumption():
    for case in (_pipe_mm(max_iter=1),
                 cases.with_scalars(cases.expansion(scale=1 / 32, max_iter=1, tol=1e-30),
                                    wall_c=cases.hill(2e-3, 0.4, 2.5, inhibition=(2.0, 0.5, 0.3)), D=2e-6)):
        mesh, o, _, _ = _run(case)
        for _ in range(6):  # one SIMPLE iteration per continued run
            o.run(cont=True)
        C = o.get("C")  # the wall solve of the next iteration starts from this field
        o.run(cont=True)
        faces, f = _wall_faces(mesh, case)
        assert len(faces) > 0
        cw, ocr = o.get("cw"), o.get("ocrWall")
        D = case.settings["D"]
        own, grp = mesh["faceOwner"], mesh["faceBoundaryGroupID"]
        for fc in faces:
            n, gid = own[fc], grp[fc]
            h = 1.0 / (_dpf(mesh, fc, n) / D + f["Rtot"][gid])
            J = _rate(f, gid, cw[fc])
            assert cw[fc] >= 0.0
            if cw[fc] > 0.0:  # interior root: the Newton residual h (c_P - c_w) - J(c_w) vanishes
                assert abs(h * (C[n] - cw[fc]) - J) <= 1e-8 * max(h * abs(C[n]), 1e-300)
            assert abs(ocr[fc] - mesh["faceArea"][fc] * J) <= 1e-12 * max(abs(ocr[fc]), 1e-300)


def test_converged_concentration_conserves_species():
    case = _pipe_mm(max_iter=5000, tol=1e-6)
    case.settings.update(scalarResEnabled=[1, 1], scalarResTol=[1e-8, 1e-8])
    mesh, o, it, conv = _run(case)
    assert conv
    C, mdot, ocr = o.get("C"), o.get("mDot"), o.get("ocrWall")
    rho, D = case.settings["rho"], case.settings["D"]
    f = case.bc_fields()["C"]
    own, nb, grp = mesh["faceOwner"], mesh["faceNeighbor"], mesh["faceBoundaryGroupID"]
    inflow = outflow = 0.0
    for fc in np.flatnonzero(nb < 0):
        n, gid = own[fc], grp[fc]
        F = mdot[fc] / rho
        if f["type"][gid] == cases.DIRICHLET:
            K = D * mesh["faceArea"][fc] / _dpf(mesh, fc, n)
            inflow += (-F if F < 0 else 0.0) * f["value"][gid] + K * (f["value"][gid] - C[n])
            outflow += (F * C[n] if F > 0 else 0.0)
        elif F > 0:
            outflow += F * C[n]
    consumed = ocr.sum()
    assert consumed > 0.01 * inflow  # the wall takes a visible share
    assert abs(inflow - outflow - consumed) <= 1e-4 * inflow


def test_unsolved_scalar_residual_entry_reads_zero():
    # the reference keeps an unsolved scalar's system all zero, so an enabled
    # entry reports 0 and passes (residualAllHost, residuals.cu:37-100)
    case = cases.with_scalars(cases.pipe(nr=6, nz=20, max_iter=3, tol=1e-30), concentration=False)
    case.settings.update(scalarResEnabled=[0, 1])
    _, o, it, _ = _run(case)
    assert it == 3 and o.scalar_residuals()[1] == 0.0


def test_structured_mesh_drops_the_nonorthogonal_corrector():
    # Solver::runCheck clears useNonOrthCorrector on a structured mesh (solver.cpp:548-555)
    case = cases.expansion(scale=1 / 32, max_iter=3, tol=1e-30)
    mesh, o0, _, _ = _run(case)
    case.settings.update(useNonOrthCorrector=1)
    o1 = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    o1.run()
    assert np.array_equal(o0.get("u"), o1.get("u"))
    o2 = oracle.Oracle(dict(mesh, meshType=1), case.bc_fields(), case.settings)
    o2.run()
    assert not np.array_equal(o0.get("u"), o2.get("u"))


def test_solution_table_carries_scalar_columns(tmp_path):
    case = _pipe_mm(max_iter=5)
    mesh, o, _, _ = _run(case)
    fluid = {k: case.settings[k] for k in ("rho", "mu", "cp", "k", "D")}
    sols = export.solutions_from(o.get, mesh, fluid, energy=True, concentration=True)
    cols = export.save_solution_npy(str(tmp_path), mesh, sols, fluid, quads=export.quad_corners(mesh))
    assert cols[:10] == ["Axial Velocity", "Radial Velocity", "Velocity Magnitude", "Pressure", "Temperature",
                         "dT/dz", "dT/dr", "Concentration", "dC/dz", "dC/dr"]
    t = np.load(tmp_path / "solution.npy")
    np.testing.assert_array_equal(t[:, 4 + cols.index("Temperature")], o.get("T"))
    np.testing.assert_array_equal(t[:, 4 + cols.index("dC/dr")], o.get("gradCR"))
