"""NumPy solution export (axisim.export) in the reference's on-disk format
(saveSolutionNpy, manager/source/file_manager.cpp:2074-2309), on oracle fields."""
import json
import os

import numpy as np
import pytest

from axisim import cases, export, trimesh
import oracle


def _solve(case, iters=20):
    mesh = oracle.multiblock(case.blocks)
    st = dict(case.settings)
    st["maxIter"] = iters
    orc = oracle.Oracle(mesh, case.bc_fields(), st)
    orc.run()
    return mesh, orc


def _shoelace(pts):
    z, r = pts[:, 0], pts[:, 1]
    return 0.5 * abs(np.dot(z, np.roll(r, -1)) - np.dot(r, np.roll(z, -1)))


def test_solution_table_container_and_columns(tmp_path):
    case = cases.pipe(nr=4, nz=6)
    mesh, orc = _solve(case)
    fluid = {"rho": case.settings["rho"], "mu": case.settings["mu"], "cp": 4180.0, "k": 0.6, "D": 3.0277e-9}
    sols = export.solutions_from(orc.get, mesh, fluid)
    cols = export.save_solution_npy(str(tmp_path), mesh, sols, fluid, quads=export.quad_corners(mesh))
    assert cols == ["Axial Velocity", "Radial Velocity", "Velocity Magnitude", "Pressure", "Continuity",
                    "Cell Reynolds Number", "dU/dz", "dU/dr", "dV/dz", "dV/dr", "dP/dz", "dP/dr"]
    raw = open(tmp_path / "solution.npy", "rb").read()
    hl = raw[8] | (raw[9] << 8)
    assert raw[:8] == b"\x93NUMPY\x01\x00" and (10 + hl) % 64 == 0 and raw[10 + hl - 1:10 + hl] == b"\n"
    assert b"{'descr': '<f8', 'fortran_order': False, 'shape': (24, 16), }" in raw[:10 + hl]
    t = np.load(tmp_path / "solution.npy")
    assert t.shape == (24, 16) and t.dtype == np.dtype("<f8")
    np.testing.assert_array_equal(t[:, 0], mesh["cellCenterZ"])
    np.testing.assert_array_equal(t[:, 3], mesh["cellArea2D"])
    np.testing.assert_array_equal(t[:, 4], orc.get("u"))
    np.testing.assert_array_equal(t[:, 7], orc.get("p"))
    u, v = orc.get("u"), orc.get("v")
    np.testing.assert_allclose(t[:, 6], np.sqrt(u * u + v * v), rtol=0, atol=0)
    # continuity: net outflow per cell, which sums to the net boundary outflow
    bnd = mesh["faceNeighbor"] < 0
    assert abs(t[:, 8].sum() - orc.get("mDot")[bnd].sum()) < 1e-12 * max(1.0, abs(t[:, 8]).sum())
    meta = json.load(open(tmp_path / "meta.json"))
    assert list(meta) == ["app", "format", "note", "cells", "meshType", "multiBlock", "structured", "points",
                          "cellCorners", "fluid", "transient", "dt", "columns", "frameColumns", "frames"]
    assert meta["columns"] == export.GEOM_COLUMNS + cols and meta["frameColumns"] == cols
    assert meta["fluid"]["mu"] == case.settings["mu"] and meta["frames"] == []


def test_quad_corners_weld_to_the_mesh_polygons(tmp_path):
    case = cases.expansion(scale=1 / 64)
    mesh, orc = _solve(case, iters=2)
    q = export.quad_corners(mesh)
    pts, cells = export.weld(q)
    N = int(mesh["nCells"])
    assert cells.shape == (N, 4) and cells.dtype == np.int32
    area = np.array([_shoelace(pts[cells[c]]) for c in range(N)])
    np.testing.assert_allclose(area, mesh["cellArea2D"], rtol=1e-12)
    cz = pts[cells][:, :, 0].mean(1)
    cr = pts[cells][:, :, 1].mean(1)
    np.testing.assert_allclose(cz, mesh["cellCenterZ"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(cr, mesh["cellCenterR"], rtol=1e-12, atol=1e-15)
    # every interior face is shared: its two cells have two corner points in common
    own, nb = mesh["faceOwner"], mesh["faceNeighbor"]
    for f in np.flatnonzero(nb >= 0)[:500]:
        assert len(set(cells[own[f]]) & set(cells[nb[f]])) == 2
    # welded points are unique
    assert len({(round(z, 12), round(r, 12)) for z, r in pts}) == len(pts)


def test_triangles_and_transient_frames(tmp_path):
    pts, tris, classify = trimesh.bullet_in_pipe(nz=24, nr=6, seed=0)
    mesh = trimesh.pack_triangles(pts, tris, classify)
    N = int(mesh["nCells"])
    rng = np.random.default_rng(0)
    sols = {"Axial Velocity": rng.standard_normal(N), "Pressure": rng.standard_normal(N)}
    frames = [(0.001, {"Axial Velocity": np.ones(N), "Pressure": np.zeros(N)}),
              (0.002, {"Axial Velocity": 2 * np.ones(N), "Pressure": np.ones(N)})]
    fluid = {"rho": 1000.0, "mu": 1e-3, "cp": 4180.0, "k": 0.6, "D": 3e-9}
    cols = export.save_solution_npy(str(tmp_path), mesh, sols, fluid, transient=True, dt=1e-3,
                                    mesh_type="Unstructured", multi_block=False,
                                    triangles=(pts, tris), frames=frames)
    assert cols == ["Axial Velocity", "Pressure"]
    c = np.load(tmp_path / "cells.npy")
    p = np.load(tmp_path / "points.npy")
    assert c.shape == (N, 3) and c.dtype == np.dtype("<i4") and p.shape == (len(pts), 2)
    area = np.array([_shoelace(p[c[k]]) for k in range(N)])
    np.testing.assert_allclose(area, mesh["cellArea2D"], rtol=1e-10)
    f1 = np.load(tmp_path / "frame_0001.npy")
    assert f1.shape == (N, 2) and (f1[:, 0] == 2).all() and (f1[:, 1] == 1).all()
    meta = json.load(open(tmp_path / "meta.json"))
    assert meta["cellCorners"] == 3 and meta["transient"] is True and meta["dt"] == 1e-3
    assert meta["frames"] == [{"file": "frame_0000.npy", "time": 0.001}, {"file": "frame_0001.npy", "time": 0.002}]
    assert "nr" not in meta and meta["structured"] is False
    assert os.path.getsize(tmp_path / "solution.npy") % 64 == (N * 6 * 8) % 64


def test_reference_reader_record_on_the_pipe_export(tmp_path):
    """The same export as tests/golden/make_npy_reader_golden.py, which ran the
    reference's own reader (tools/validation.py load_solution / load_cells) and
    Hagen-Poiseuille analysis (poiseuille_flow / poiseuille_report,
    validation.py:180-274) on it and recorded what they returned and printed.
    The folder is read back the way that reader reads it (meta.json columns
    name the solution.npy columns; points[cells] gives the cell polygons) and
    its analysis is repeated step by step against the record."""
    import sys
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "npy_reader_pipe10x50_fd.json")))
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_npy_reader_golden as mk
    cols, it, conv = mk.export_pipe(str(tmp_path))
    assert it == g["oracle_iterations"] and conv == g["oracle_converged"]
    meta = json.load(open(tmp_path / "meta.json"))
    sol = np.load(tmp_path / "solution.npy")
    col = {n: i for i, n in enumerate(meta["columns"])}
    assert meta["columns"] == g["columns"] and col == g["col"] and list(sol.shape) == g["solution_shape"]
    pts, cells = np.load(tmp_path / "points.npy"), np.load(tmp_path / "cells.npy")
    verts = pts[cells]
    assert [list(pts.shape), list(cells.shape), list(verts.shape)] == [g["points_shape"], g["cells_shape"],
                                                                      g["verts_shape"]]
    c = lambda n: sol[:, col[n]]  # noqa: E731
    z, r, u, vol = c("z"), c("r"), c("Axial Velocity"), c("volume")
    rho, mu = meta["fluid"]["rho"], meta["fluid"]["mu"]
    R = pts[:, 1].max()
    Umean = (u * vol).sum() / vol.sum()
    Re = rho * Umean * 2.0 * R / mu
    zDev = 2.0 * R * (0.619 ** 1.6 + (0.0567 * Re) ** 1.6) ** (1.0 / 1.6)
    dev = z >= zDev
    if not dev.any():
        dev = np.ones(len(z), bool)
    Umean = (u[dev] * vol[dev]).sum() / vol[dev].sum()
    UmaxDp = -c("dP/dz")[dev].mean() * R * R / (4.0 * mu)
    Umax = 2.0 * Umean
    prof = Umax * (1.0 - r * r / (R * R))
    want = g["poiseuille"]
    got = {"R": R, "Umean": Umean, "Umax": Umax, "UmaxFlux": Umax, "UmaxDp": UmaxDp, "Re": Re, "zDev": zDev,
           "u_sum": prof.sum()}
    for k, v in got.items():
        assert v == pytest.approx(want[k], rel=1e-12, abs=0), k
    assert int(dev.sum()) == want["dev_cells"]
    res = (u - prof)[dev] / Umax
    assert f"L2   error        = {100.0 * np.sqrt((res ** 2).mean()):.4f} % of Umax" in g["report"]
    assert f"Linf error        = {100.0 * np.abs(res).max():.4f} % of Umax" in g["report"]
