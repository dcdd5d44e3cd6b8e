"""Golden record of the reference's OWN solution reader on this project's export.

The reference's NumPy writer (saveSolutionNpy, manager/source/file_manager.cpp:
2074-2309) cannot be compiled here: file_manager.cpp includes mesh.h and
results.h, which include buffer_manager.h and through it the OpenGL loader
(glad/glad.h), and no stand-in for a graphics loader is used in this project.
Its reader can run: tools/validation.py loads an export folder (load_solution,
load_cells, validation.py:165-178) and derives the Hagen-Poiseuille check from
it (poiseuille_flow / poiseuille_report, :180-274).

This script solves the fully developed 10 x 50 pipe with the CPU oracle,
writes it with axisim.export, runs the reference's reader and Poiseuille
analysis on that folder, and stores what they return and print in
npy_reader_pipe10x50_fd.json. tests/test_export_cpu.py re-exports the same
case and checks the folder against that record.

validation.py imports matplotlib at module level for its plots; matplotlib is
not installed here, so empty modules stand in for it while the reader and the
analysis (which use only NumPy) run. Run from the repository root in this
container (the reference checkout is read at AXISIM_REFERENCE, default
/root/reference):

    python tests/golden/make_npy_reader_golden.py
"""
import contextlib
import importlib.util
import io
import json
import os
import sys
import tempfile
import types


HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "axisim-software_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

CASE = dict(nr=10, nz=50, max_iter=20000, tol=1e-8, fully_developed=True)
FLUID_EXTRA = {"cp": 4180.0, "k": 0.6, "D": 3.0277e-9}
OUT = os.path.join(HERE, "npy_reader_pipe10x50_fd.json")


def export_pipe(directory):
    """The case solved by the oracle and exported; returns the column names."""
    from axisim import cases, export
    import oracle
    case = cases.pipe(**CASE)
    mesh = oracle.multiblock(case.blocks)
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it, conv = orc.run()
    fluid = dict(rho=case.settings["rho"], mu=case.settings["mu"], **FLUID_EXTRA)
    sols = export.solutions_from(orc.get, mesh, fluid)
    cols = export.save_solution_npy(directory, mesh, sols, fluid, quads=export.quad_corners(mesh))
    orc.close()
    return cols, it, conv


def reference_reader():
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.tri", "matplotlib.collections"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["matplotlib.collections"].PolyCollection = object
    ref = os.environ.get("AXISIM_REFERENCE", "/root/reference")
    spec = importlib.util.spec_from_file_location("axisim_ref_validation", os.path.join(ref, "tools", "validation.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    val = reference_reader()
    with tempfile.TemporaryDirectory() as d:
        cols, it, conv = export_pipe(d)
        s = val.load_solution(d)  # an absolute folder replaces the reader's repo root
        c = val.load_cells(d)
        p = val.poiseuille_flow(s, c)
        text = io.StringIO()
        with contextlib.redirect_stdout(text):
            val.poiseuille_report(s, p)
    rec = {
        "case": CASE, "oracle_iterations": it, "oracle_converged": bool(conv),
        "columns": s.meta["columns"], "col": s.col, "solution_shape": list(s.sol.shape),
        "live_cells": int(s.live.sum()), "points_shape": list(c.pts.shape), "cells_shape": list(c.cells.shape),
        "verts_shape": list(c.verts.shape),
        "poiseuille": {"R": p.R, "Umean": p.Umean, "Umax": p.Umax, "refName": p.refName, "UmaxFlux": p.UmaxFlux,
                       "UmaxDp": p.UmaxDp, "Re": p.Re, "zDev": p.zDev, "dev_cells": int(p.dev.sum()),
                       "u_sum": float(p.u.sum())},
        "report": text.getvalue().splitlines(),
    }
    with open(OUT, "w") as f:
        json.dump(rec, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
