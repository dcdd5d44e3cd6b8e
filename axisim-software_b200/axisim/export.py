"""NumPy solution export in the reference's on-disk format.

Restates saveSolutionNpy (manager/source/file_manager.cpp:2074-2309) so the
reference's Python readers (tools/validation.py-style scripts) load this
solver's results unchanged:

* solution.npy: float64 little-endian, shape (nCells, 4 + nFields), row-major;
  columns z, r, volume, area2D, then the solution fields in the order of
  Solver::addFieldType (solver.cpp:333-362), each field present only if the
  run produced it with one value per cell (file_manager.cpp:2017-2044);
* points.npy (nPoints, 2) float64 and cells.npy (nCells, corners) int32: the
  cell polygons. Quads (multiblock meshes) are welded from their corners with
  the reference's tolerance, extent * 1e-9 with neighbouring buckets probed
  (file_manager.cpp:1908-1970); triangles (unstructured meshes) are written as
  given (:2162-2193);
* frame_%04d.npy: field columns only, for transient frames (:2199-2217);
* meta.json: the reference's keys in its order (:2219-2296), numbers printed
  with 17 significant digits and non-finite values as null.

The .npy container follows the reference's writer (file_manager.cpp:1800-1905):
format version 1.0, the shape always written as a 2-tuple, header padded with
spaces so the payload starts on a 64-byte boundary.
"""
import json
import math
import os

import numpy as np

# Solver::addFieldType (solver.cpp:333-362); energy and concentration fields
# are listed but only exported when present.
FIELD_TYPE = ["Axial Velocity", "Radial Velocity", "Velocity Magnitude", "Pressure",
              "Temperature", "dT/dz", "dT/dr", "Concentration", "dC/dz", "dC/dr",
              "Continuity", "Cell Reynolds Number", "dU/dz", "dU/dr", "dV/dz", "dV/dr", "dP/dz", "dP/dr"]
GEOM_COLUMNS = ["z", "r", "volume", "area2D"]


def write_npy(path, array, descr):
    """The reference's .npy container (v1.0, 2-tuple shape, 64-byte aligned)."""
    a = np.ascontiguousarray(array)
    if a.ndim != 2:
        raise ValueError("write_npy expects a 2-D array")
    dtype = {"<f8": np.dtype("<f8"), "<i4": np.dtype("<i4")}[descr]
    a = a.astype(dtype, copy=False)
    header = "{'descr': '%s', 'fortran_order': False, 'shape': (%d, %d), }" % (descr, a.shape[0], a.shape[1])
    unpadded = 6 + 2 + 2 + len(header) + 1
    total = (unpadded + 63) // 64 * 64
    header = header + " " * (total - unpadded) + "\n"
    with open(path, "wb") as f:
        f.write(b"\x93NUMPY\x01\x00")
        f.write(bytes([len(header) & 0xFF, (len(header) >> 8) & 0xFF]))
        f.write(header.encode("latin1"))
        f.write(a.tobytes(order="C"))


def solutions_from(get, mesh, fluid, energy=False, concentration=False):
    """Solver::createSolutions + createDerivedVelocitySolutions (solver.cpp:186-262)
    from a field getter (axisim.abi.Solver.get or oracle.Oracle.get): velocity
    magnitude |V| and the cell Reynolds number rho |V| sqrt(area2D) / mu are derived
    from the final u and v; the continuity field is the per-cell net outflow
    of the face mass fluxes (Solver::getMassImbalance, solver.cpp:298-331).
    energy / concentration add Temperature, dT/dz, dT/dr and Concentration,
    dC/dz, dC/dr (solver.cpp:199-209)."""
    N = int(mesh["nCells"])
    u, v, p = get("u")[:N], get("v")[:N], get("p")[:N]
    out = {"Axial Velocity": u, "Radial Velocity": v, "Pressure": p,
           "dU/dz": get("gradUZ")[:N], "dU/dr": get("gradUR")[:N], "dV/dz": get("gradVZ")[:N],
           "dV/dr": get("gradVR")[:N], "dP/dz": get("gradPZ")[:N], "dP/dr": get("gradPR")[:N]}
    if energy:
        out.update({"Temperature": get("T")[:N], "dT/dz": get("gradTZ")[:N], "dT/dr": get("gradTR")[:N]})
    if concentration:
        out.update({"Concentration": get("C")[:N], "dC/dz": get("gradCZ")[:N], "dC/dr": get("gradCR")[:N]})
    out["Continuity"] = mass_imbalance(mesh, get("mDot")[:int(mesh["nFaces"])])
    speed = np.sqrt(u * u + v * v)
    h = np.sqrt(np.maximum(np.asarray(mesh["cellArea2D"], np.float64), 0.0))
    mu, rho = float(fluid["mu"]), float(fluid["rho"])
    out["Velocity Magnitude"] = speed
    out["Cell Reynolds Number"] = rho * speed * h / mu if mu > 0 else np.zeros(N)
    return out


def mass_imbalance(mesh, mdot):
    N = int(mesh["nCells"])
    cfs, cfi = np.asarray(mesh["cellFaceStart"]), np.asarray(mesh["cellFaceIDs"])
    own, nb = np.asarray(mesh["faceOwner"]), np.asarray(mesh["faceNeighbor"])
    rows = np.repeat(np.arange(N), np.diff(cfs))
    sign = np.where(own[cfi] == rows, 1.0, np.where(nb[cfi] == rows, -1.0, 0.0))
    # the per-cell sum runs over the cell's faces in slot order, as the reference's loop
    out = np.zeros(N)
    for j in range(int(np.max(np.diff(cfs))) if N else 0):
        sel = np.diff(cfs) > j
        k = cfs[:-1][sel] + j
        out[sel] += sign[k] * np.asarray(mdot)[cfi[k]]
    return out


def quad_corners(mesh):
    """Corner quads (V(i,j), V(i,j+1), V(i+1,j+1), V(i+1,j)) of an axis-aligned
    structured mesh (Mesh::multiBlockCellCorners, mesh.cpp:2514-2538): each
    cell's z and r extents come from its faces (centre +- half the face's r-z
    length along the face's tangent). Returns (nCells, 4, 2) as (z, r)."""
    N = int(mesh["nCells"])
    cfs, cfi = np.asarray(mesh["cellFaceStart"]), np.asarray(mesh["cellFaceIDs"])
    fz, fr = np.asarray(mesh["faceCenterZ"]), np.asarray(mesh["faceCenterR"])
    nz, nr = np.asarray(mesh["faceNormalZ"]), np.asarray(mesh["faceNormalR"])
    area = np.asarray(mesh["faceArea"])
    # r-z length of a face: area = 2 pi r_f L, except on the axis (r_f = 0),
    # where the face is radial and has no length of its own
    with np.errstate(divide="ignore", invalid="ignore"):
        L = np.where(fr > 0, area / (2.0 * np.pi * fr), 0.0)
    rows = np.repeat(np.arange(N), np.diff(cfs))
    f = cfi
    z0 = np.full(N, np.inf); z1 = np.full(N, -np.inf); r0 = np.full(N, np.inf); r1 = np.full(N, -np.inf)
    # endpoints: centre -+ L/2 along the tangent (-n_r, n_z)
    ez = np.r_[fz[f] - 0.5 * L[f] * (-nr[f]), fz[f] + 0.5 * L[f] * (-nr[f])]
    er = np.r_[fr[f] - 0.5 * L[f] * nz[f], fr[f] + 0.5 * L[f] * nz[f]]
    rr = np.r_[rows, rows]
    np.minimum.at(z0, rr, ez); np.maximum.at(z1, rr, ez)
    np.minimum.at(r0, rr, er); np.maximum.at(r1, rr, er)
    q = np.empty((N, 4, 2))
    q[:, 0] = np.c_[z0, r0]; q[:, 1] = np.c_[z1, r0]; q[:, 2] = np.c_[z1, r1]; q[:, 3] = np.c_[z0, r1]
    return q


def weld(quads):
    """weldCellCorners (file_manager.cpp:1908-1970): unique points by rounding to
    tol = max(1, extent) * 1e-9 with the 3 x 3 neighbouring buckets probed, in
    first-seen order. Returns (points (P, 2), cells (nCells, 4) int32)."""
    extent = max(1.0, float(np.max(np.abs(quads)))) if quads.size else 1.0
    tol = extent * 1e-9
    seen = {}
    pts = []
    cells = np.empty(quads.shape[:2], np.int32)
    for c in range(quads.shape[0]):
        for k in range(quads.shape[1]):
            z, r = float(quads[c, k, 0]), float(quads[c, k, 1])
            key = (int(round(z / tol)), int(round(r / tol)))
            idx = -1
            for dz in (-1, 0, 1):
                for dr in (-1, 0, 1):
                    idx = seen.get((key[0] + dz, key[1] + dr), -1)
                    if idx >= 0:
                        break
                if idx >= 0:
                    break
            if idx < 0:
                idx = len(pts)
                pts.append((z, r))
                seen[key] = idx
            cells[c, k] = idx
    return np.asarray(pts, np.float64).reshape(-1, 2), cells


def _num(v):
    v = float(v)
    return "null" if not math.isfinite(v) else "%.17g" % v


def save_solution_npy(directory, mesh, solutions, fluid, transient=False, dt=0.0, mesh_type="Structured",
                      multi_block=True, nr=0, nz=0, quads=None, triangles=None, frames=()):
    """Writes solution.npy, the cell polygons and meta.json into `directory`.
    solutions: {field name: per-cell values}; quads: (nCells, 4, 2) corners or
    None; triangles: (points (P, 2), tris (nCells, 3)) or None; frames:
    [(time, solutions)] for a transient run."""
    N = int(mesh["nCells"])
    if N == 0:
        raise ValueError("no cells to export")
    os.makedirs(directory, exist_ok=True)
    cols = [n for n in FIELD_TYPE if n in solutions and len(solutions[n]) == N]
    table = np.empty((N, len(GEOM_COLUMNS) + len(cols)))
    table[:, 0] = mesh["cellCenterZ"]
    table[:, 1] = mesh["cellCenterR"]
    table[:, 2] = mesh["cellVolume"]
    table[:, 3] = mesh["cellArea2D"]
    for k, n in enumerate(cols):
        table[:, len(GEOM_COLUMNS) + k] = solutions[n]
    write_npy(os.path.join(directory, "solution.npy"), table, "<f8")
    n_points = corners = 0
    if quads is not None and len(quads) == N:
        pts, cells = weld(np.asarray(quads, np.float64))
        write_npy(os.path.join(directory, "points.npy"), pts, "<f8")
        write_npy(os.path.join(directory, "cells.npy"), cells, "<i4")
        n_points, corners = len(pts), 4
    elif triangles is not None and len(triangles[1]) == N:
        pts = np.asarray(triangles[0], np.float64).reshape(-1, 2)
        write_npy(os.path.join(directory, "points.npy"), pts, "<f8")
        write_npy(os.path.join(directory, "cells.npy"), np.asarray(triangles[1], np.int32).reshape(N, 3), "<i4")
        n_points, corners = len(pts), 3
    frame_index = []
    for i, (time, sols) in enumerate(frames):
        name = "frame_%04d.npy" % i
        ft = np.zeros((N, len(cols)))
        for k, n in enumerate(cols):
            if n in sols and len(sols[n]) == N:
                ft[:, k] = sols[n]
        write_npy(os.path.join(directory, name), ft, "<f8")
        frame_index.append((name, time))
    reshapable = nr > 0 and nz > 0
    lines = ["{", '  "app": "AxiSim",', '  "format": 1,', '  "note": "cell-centered values, base SI units",',
             '  "cells": %d,' % N, '  "meshType": "%s",' % mesh_type,
             '  "multiBlock": %s,' % ("true" if multi_block else "false"),
             '  "structured": %s,' % ("true" if reshapable else "false")]
    if reshapable:
        lines += ['  "nr": %d,' % nr, '  "nz": %d,' % nz]
    if corners:
        lines += ['  "points": %d,' % n_points, '  "cellCorners": %d,' % corners]
    lines.append('  "fluid": {"rho": %s, "mu": %s, "cp": %s, "k": %s, "D": %s},' % tuple(
        _num(fluid.get(k, 0.0)) for k in ("rho", "mu", "cp", "k", "D")))
    lines.append('  "transient": %s,' % ("true" if transient else "false"))
    lines.append('  "dt": %s,' % _num(dt))
    esc = lambda s: s.replace("\\", "\\\\").replace('"', '\\"')  # noqa: E731
    lines.append('  "columns": [%s],' % ", ".join('"%s"' % esc(c) for c in GEOM_COLUMNS + cols))
    lines.append('  "frameColumns": [%s],' % ", ".join('"%s"' % esc(c) for c in cols))
    if frame_index:
        items = ",\n    ".join('{"file": "%s", "time": %s}' % (f, _num(t)) for f, t in frame_index)
        lines.append('  "frames": [\n    ' + items + "\n  ]")
    else:
        lines.append('  "frames": []')
    lines.append("}")
    with open(os.path.join(directory, "meta.json"), "w") as f:
        f.write("\n".join(lines) + "\n")
    json.loads(open(os.path.join(directory, "meta.json")).read())  # the file must parse
    return cols
