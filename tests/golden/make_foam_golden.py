"""Generate OpenFOAM-case golden files from the REFERENCE's own exporter.

Runs oracle/_ref/foam_ref (the reference's manager/source/file_converter.cpp,
boundary_func.cpp and math_func.cpp compiled unchanged by
oracle/ref_build/Makefile, driven headless by oracle/ref_build/foam_driver.cpp)
on small cases and stores every file of each exported case in a JSON fixture
next to this script. Host code only: runs on any CPU.

    python tests/golden/make_foam_golden.py [outdir]
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "axisim-software_b200"))
from axisim import cases, foam, trimesh  # noqa: E402

FOAM_BIN = os.path.join(ROOT, "oracle", "_ref", "foam_ref")
VAR_NAMES = {cases.U: "u", cases.V: "v", cases.P: "p", cases.TEMP: "T", cases.CONC: "C"}
SETUP_KEYS = ("rho", "mu", "D", "cp", "k", "solveEnergy", "solveConcentration", "transient", "secondOrderTime", "dt",
              "tEnd", "steadyIterations", "convection", "leastSquaresGradient", "addConvection", "nonOrthCorrector",
              "momentumRelaxation", "pressureRelaxation", "concentrationRelaxation")


def foam_cases():
    """(name, dict(groups, settings, blocks + outline | points + tris + mesh))."""
    out = []
    c = cases.with_scalars(cases.expansion(scale=1 / 32), wall_c=cases.michaelis_menten(1e-3, 0.2), D=1e-6)
    names = ["Inlet (u = 2 Ubar)", "Outlet", "Outer wall", "Axis"]
    for g, n in zip(c.groups, names):
        g.name = n
    out.append(("expansion_scalars_sou", dict(groups=c.groups, settings=c.settings, blocks=c.blocks,
                                             outline=cases.expansion_outline())))
    c = cases.pulsatile_expansion(scale=1 / 32, dt=1e-3, steps=40)
    for g, n in zip(c.groups, ["inlet", "front", "3 walls!", "axis"]):
        g.name = n
    out.append(("pulsatile_bdf2_name_collisions", dict(groups=c.groups, settings=c.settings, blocks=c.blocks,
                                                       outline=cases.expansion_outline())))
    c = cases.with_scalars(cases.pipe(nr=6, nz=20, fully_developed=True), t_wall=None,
                           wall_c=cases.hill(2e-3, 0.4, 2.5, inhibition=(2.0, 0.5, 0.3)))
    c.groups[2].bcs[cases.TEMP] = (cases.NEUMANN, 250.0)
    for g, n in zip(c.groups, ["Inlet", "Outlet", "Wall", "Axis"]):
        g.name = n
    c.settings.update(convectionScheme=cases.CONV_CENTRAL, gradientScheme=cases.GRAD_GREEN_GAUSS,
                      useNonOrthCorrector=1, addConvectionTerm=0, maxIter=5000)
    L, R = 0.2, 0.01
    o = cases.polygon_outline([(0, 0), (L, 0), (L, R), (0, R)], [3, 1, 2, 0])
    out.append(("pipe_fd_hill_noconv", dict(groups=c.groups, settings=c.settings, blocks=c.blocks, outline=o)))
    pts, tris, classify = trimesh.bullet_in_pipe(nz=24, nr=6, seed=1)

    def leave_outlet(fz, fr):
        g = classify(fz, fr)
        g[g == 1] = -1            # an outlet the outline did not tag
        return g
    mesh = trimesh.pack_triangles(pts, tris, leave_outlet)
    c = cases.with_scalars(cases.bullet(scale=0.1), concentration=False, t_wall=320.0)
    for g, n in zip(c.groups, ["Inlet", "Outlet", "Wall/body", "Wall body"]):
        g.name = n
    c.groups[3].btype = cases.WALL   # the axis group tagged a wall: both names sanitize to Wall_body
    c.settings.update(convectionScheme=cases.CONV_QUICK)
    out.append(("bullet_triangles_unassigned", dict(groups=c.groups, settings=c.settings, points=pts, tris=tris,
                                                   mesh=mesh)))
    return out


def write_spec(spec, path):
    st = foam.case_setup(spec["settings"])
    with open(path, "w") as f:
        f.write("tol 1e-09\nwedge 5.0\n")
        for b in spec.get("blocks") or []:
            ax, rd = b["axial"], b["radial"]
            f.write("block %r %r %r %d %d %r %r %d %d %r %d %d %d %d\n" % (
                b["z0"], b["r0"], ax[0], ax[1], ax[2], ax[3], rd[0], rd[1], rd[2], rd[3], *b["edge_group"]))
        for g in spec["groups"]:
            items = []
            for var, bc in g.bcs.items():
                t, val = bc[0], bc[1]
                if t in (cases.MICHAELIS_MENTEN, cases.HILL):
                    val = 0.0
                amp, freq = (bc[2], bc[3]) if t == cases.PULSATILE else (0.0, 0.0)
                items.append(f"{VAR_NAMES[var]} {t} {float(val)!r} {amp!r} {freq!r}")
            name = g.name.encode("utf-8").hex() or "-"
            f.write(f"group {g.id} {g.btype} {float(np.float32(g.total_length))!r} {name} {len(items)} "
                    f"{' '.join(items)}\n")
            for var, bc in g.bcs.items():
                if bc[0] in (cases.MICHAELIS_MENTEN, cases.HILL):
                    k = bc[1]
                    inh = k.get("inhibition")
                    m, k2, v2 = inh if inh else (1.0, 0.0, 0.0)
                    f.write(f"kin {g.id} {VAR_NAMES[var]} {bc[0]} {k['Vmax']!r} {k['Km']!r} {k['n']!r} "
                            f"{1 if inh else 0} {m!r} {k2!r} {v2!r}\n")
        if spec.get("outline") is not None:
            verts, edges, groups = spec["outline"]
            for z, r in verts:
                f.write(f"vertex {float(z)!r} {float(r)!r}\n")
            for (a, b), g in zip(edges, groups):
                f.write(f"edge {int(a)} {int(b)} {int(g)}\n")
        if spec.get("tris") is not None:
            m = spec["mesh"]
            for z, r in spec["points"]:
                f.write(f"point {float(z)!r} {float(r)!r}\n")
            for t in spec["tris"]:
                f.write("tri %d %d %d\n" % tuple(int(v) for v in t))
            v01 = foam._fv_faces(spec["points"], spec["tris"], m)
            for k, (a, b) in enumerate(v01):
                f.write("face %d %d %d %d %r %r %d\n" % (a, b, m["faceOwner"][k], m["faceNeighbor"][k],
                                                        float(m["faceNormalZ"][k]), float(m["faceNormalR"][k]),
                                                        m["faceBoundaryGroupID"][k]))
        for k in SETUP_KEYS:
            f.write(f"set {k} {float(st[k])!r}\n")


def run_reference(spec):
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "spec.txt")
        write_spec(spec, path)
        case = os.path.join(d, "case")
        r = subprocess.run([FOAM_BIN, path, case], capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError(f"reference export failed: {r.stdout} {r.stderr}")
        files = {}
        for root, _, names in os.walk(case):
            for n in names:
                p = os.path.join(root, n)
                files[os.path.relpath(p, case)] = open(p, "rb").read().decode("utf-8")
        return files


def main(outdir=HERE):
    for name, spec in foam_cases():
        files = run_reference(spec)
        with open(os.path.join(outdir, "foam_" + name + ".json"), "w") as f:
            json.dump({"files": files}, f, indent=0, sort_keys=True)
        print(name, len(files), "files")


if __name__ == "__main__":
    main(*sys.argv[1:])
