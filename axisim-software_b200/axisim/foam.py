"""OpenFOAM case export, in the reference's layout and spelling.

Writes what the reference's `saveFoamCase` writes (manager/source/
file_manager.cpp:1153-1258, with the writers of manager/source/
file_converter.cpp): a wedge case, one cell thick and 5 degrees wide, that
simpleFoam / pimpleFoam run as the axisymmetric counterpart of a solve here.

- structured (multiblock) meshes go out as system/blockMeshDict: block
  corners welded into global labels, patches from the outline group nearest
  each external block edge, wedge planes "back" / "front";
- triangle meshes go out as constant/polyMesh: every point revolved onto the
  two wedge planes (one point on the axis), faces ordered as polyMesh wants;
- system/controlDict, fvSchemes, fvSolution, constant/transportProperties,
  turbulenceProperties, and 0/U, p (T, Conc) from the boundary groups.

Numbers are spelled as the reference spells them (17 significant digits in
mesh files, the shortest round-trip spelling in dictionaries), so an export
from here and one from the reference are byte-identical for the same case.
"""
import math
import os

from . import cases as _c

WEDGE_DEG = 5.0
CONC = "Conc"  # not "C": OpenFOAM writes cell centres under that name
_PI = 3.14159265358979323846

# BoundaryFOAMType
PATCH, WALL, WEDGE, SYMMETRY_PLANE = 1, 2, 3, 4
_TYPE_NAME = {WALL: "wall", WEDGE: "wedge", SYMMETRY_PLANE: "symmetryPlane", PATCH: "patch"}
# FoamConvection
UPWIND, LINEAR, LINEAR_UPWIND, QUICK = range(4)

_RULE = "// ************************************************************************* //\n"


def foam_number(x):
    """The shortest of %.15g, %.16g that reads back as x, else %.17g (foamNumber)."""
    for digits in (15, 16):
        s = "%.*g" % (digits, x)
        if float(s) == x:
            return s
    return "%.17g" % x


def _g17(x):
    """A double through an ostream at precision 17."""
    return "%.17g" % x


def _header(class_name, obj, location=None):
    """writeFoamHeader (file_converter.cpp:159-185)."""
    s = ("/*--------------------------------*- C++ -*----------------------------------*\\\n"
         "  Written by AxiSim. Axisymmetric wedge mesh, one cell thick in the\n"
         "  circumferential direction -- both wedge planes are patches of type wedge.\n"
         "\\*---------------------------------------------------------------------------*/\n"
         "FoamFile\n"
         "{\n"
         "    version     2.0;\n"
         "    format      ascii;\n"
         "    class       " + class_name + ";\n")
    if location:
        s += "    location    \"" + location + "\";\n"
    s += ("    object      " + obj + ";\n"
          "}\n"
          "// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //\n\n")
    return s


def patch_name(group):
    """foamPatchName: the group name squeezed into an OpenFOAM word."""
    name = ""
    for ch in group.name.encode("utf-8"):
        c = chr(ch)
        if (c.isascii() and c.isalnum()) or c == "_":
            name += c
        elif name and name[-1] != "_":
            name += "_"
    name = name.rstrip("_")
    if not name or name[0].isdigit():
        name = "group%d" % group.id + ("" if not name else "_" + name)
    return name


def _foam_type(btype):
    return WALL if btype == _c.WALL else SYMMETRY_PLANE if btype == _c.SYMMETRY else PATCH


def case_setup(settings):
    """foamCaseSetupFromSolver (file_manager.cpp:1264-1316) from a settings dict."""
    conv = {_c.CONV_CENTRAL: LINEAR, _c.CONV_SOU: LINEAR_UPWIND, _c.CONV_QUICK: LINEAR_UPWIND}
    return dict(rho=settings["rho"], mu=settings["mu"], D=settings.get("D", 3.0277e-9),
                cp=settings.get("cp", 4180.0), k=settings.get("k", 0.6),
                solveEnergy=bool(settings.get("solveEnergy")), solveConcentration=bool(settings.get("solveConcentration")),
                transient=bool(settings["transient"]), secondOrderTime=settings["timeScheme"] == _c.TIME_SECOND_ORDER,
                dt=settings["dt"], tEnd=settings["tEnd"], steadyIterations=max(int(settings["maxIter"]), 2000),
                convection=conv.get(settings["convectionScheme"], UPWIND),
                leastSquaresGradient=settings["gradientScheme"] == _c.GRAD_LSQ,
                addConvection=bool(settings["addConvectionTerm"]), nonOrthCorrector=bool(settings["useNonOrthCorrector"]),
                momentumRelaxation=settings["alphaU"], pressureRelaxation=settings["alphaP"],
                concentrationRelaxation=1.0)


# ---------------------------------------------------------------- outline
def _group_at_point(z, r, outline, tol):
    """groupAtPoint (math_func.cpp:175-196)."""
    verts, edges, groups = outline
    best, best_dist = -1, tol
    nv = len(verts)
    for (v0, v1), g in zip(edges, groups):
        if g < 0 or v0 < 0 or v1 < 0 or v0 >= nv or v1 >= nv:
            continue
        az, ar = float(verts[v0][0]), float(verts[v0][1])
        abz, abr = float(verts[v1][0]) - az, float(verts[v1][1]) - ar
        apz, apr = z - az, r - ar
        ab2 = abz * abz + abr * abr
        qz, qr = az, ar
        if not ab2 <= 1e-30:
            t = (apz * abz + apr * abr) / ab2
            t = min(max(t, 0.0), 1.0)
            qz, qr = az + t * abz, ar + t * abr
        dz, dr = qz - z, qr - r
        d = math.sqrt(dz * dz + dr * dr)
        if d < best_dist:
            best_dist, best = d, int(g)
    return best


# ---------------------------------------------------------------- blocks
def _zone_faces(length, n, grading, coef, start):
    """generateFaces (structs/multiblock.h:59-80)."""
    d = [length / n] * n
    if grading == _c.PROGRESSION and n > 1 and coef > 0.0 and coef != 1.0:
        d0 = length * (coef - 1.0) / (math.pow(coef, n) - 1.0)
        d = [d0 * math.pow(coef, k) for k in range(n)]
    x, out = start, [start]
    for k in range(n):
        x += d[k]
        out.append(x)
    return out


class _Block:
    def __init__(self, spec):
        ax, rd = spec["axial"], spec["radial"]
        self.zf = _zone_faces(ax[0], ax[1], ax[2], ax[3], spec["z0"])
        self.rf = _zone_faces(rd[0], rd[1], rd[2], rd[3], spec["r0"])
        self.nz, self.nr = ax[1], rd[1]
        self.axial, self.radial = ax, rd

    def node(self, i, j):
        return (self.zf[j], self.rf[i])


def _expansion_ratio(zone):
    """zoneExpansion: last cell over first."""
    length, cells, grading, coef = zone
    if grading != _c.PROGRESSION or cells < 2 or coef <= 0.0 or coef == 1.0:
        return 1.0
    return math.pow(coef, cells - 1)


def _llround(x):
    q = math.floor(x)
    frac = x - q
    if frac > 0.5 or (frac == 0.5 and x > 0):
        q += 1
    return int(q)


def _block_edge_ends(b, e):
    """West, East, South, North (multiblock.h:85) as (first, second)."""
    if e == 1:
        return b.node(0, b.nz), b.node(b.nr, b.nz)
    if e == 2:
        return b.node(0, 0), b.node(0, b.nz)
    if e == 3:
        return b.node(b.nr, 0), b.node(b.nr, b.nz)
    return b.node(0, 0), b.node(b.nr, 0)


def _interfaces(blocks, tol):
    """autoDetectInterfaces (multiblock.h:220-251): fully coincident edges of
    equal cell count; any coincident pair of unequal count drops them all."""
    tol2 = tol * tol

    def same(p, q):
        dz, dr = p[0] - q[0], p[1] - q[1]
        return dz * dz + dr * dr <= tol2
    claimed = set()
    for a in range(len(blocks)):
        for b in range(a + 1, len(blocks)):
            for ea in range(4):
                for eb in range(4):
                    as_, ae = _block_edge_ends(blocks[a], ea)
                    bs, be = _block_edge_ends(blocks[b], eb)
                    if not ((same(as_, bs) and same(ae, be)) or (same(as_, be) and same(ae, bs))):
                        continue
                    la = blocks[a].nr if ea <= 1 else blocks[a].nz
                    lb = blocks[b].nr if eb <= 1 else blocks[b].nz
                    if la != lb:
                        return set()
                    claimed.add((a, ea))
                    claimed.add((b, eb))
    return claimed


_BACK, _FRONT = (0, 3, 2, 1), (4, 5, 6, 7)
_EDGE_FACE = {1: (1, 2, 6, 5), 2: (0, 1, 5, 4), 3: (3, 7, 6, 2), 0: (0, 4, 7, 3)}


def _global_face(local, labels):
    out = [labels[k] for k in local]
    return out, len(set(out)) >= 3


def block_mesh_dict(blocks, groups, outline, tol=1e-9, wedge=WEDGE_DEG):
    """blockMeshDictFromMultiblock (file_converter.cpp:342-531): vertices,
    hexes and patches {name: (type, groupID, faces)}."""
    bl = [_Block(s) for s in blocks]
    extent = 0.0
    for b in bl:
        for z in b.zf:
            extent = max(extent, abs(z))
        for r in b.rf:
            extent = max(extent, abs(r))
    wtol = 1e-9 * (extent if extent > 0.0 else 1.0)
    half = 0.5 * wedge * (_PI / 180.0)
    ch, sh = math.cos(half), math.sin(half)
    points, grid, labels = [], {}, []
    for b in bl:
        corners = [b.node(0, 0), b.node(0, b.nz), b.node(b.nr, b.nz), b.node(b.nr, 0)]
        verts = [(c[0], c[1] * ch, sign * c[1] * sh) for sign in (-1.0, 1.0) for c in corners]
        lab = []
        for v in verts:
            home = (_llround(v[0] / wtol), _llround(v[1] / wtol), _llround(v[2] / wtol))
            match = -1
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        if match >= 0:
                            break
                        for cand in grid.get((home[0] + dx, home[1] + dy, home[2] + dz), ()):
                            q = points[cand]
                            if abs(q[0] - v[0]) <= wtol and abs(q[1] - v[1]) <= wtol and abs(q[2] - v[2]) <= wtol:
                                match = cand
                                break
                    if match >= 0:
                        break
                if match >= 0:
                    break
            if match < 0:
                match = len(points)
                points.append(v)
                grid.setdefault(home, []).append(match)
            lab.append(match)
        labels.append(lab)
    hexes = [(labels[i], (b.nz, b.nr, 1), (_expansion_ratio(b.axial), _expansion_ratio(b.radial), 1.0))
             for i, b in enumerate(bl)]
    patches = {"back": [WEDGE, -1, []], "front": [WEDGE, -1, []]}
    by_id = {g.id: g for g in groups}
    name_of = {}

    def patch_for(gid):
        if gid in name_of:
            return patches[name_of[gid]]
        grp = by_id.get(gid)
        stem = patch_name(grp) if grp else "unassigned"
        name, n = stem, 2
        while name in patches:
            name = "%s_%d" % (stem, n)
            n += 1
        name_of[gid] = name
        patches[name] = [_foam_type(grp.btype) if grp else PATCH, grp.id if grp else -1, []]
        return patches[name]
    claimed = _interfaces(bl, tol)
    match_tol = 1e-4 * max(extent, 1.0)
    for bi, b in enumerate(bl):
        lab = labels[bi]
        f, ok = _global_face(_BACK, lab)
        if ok:
            patches["back"][2].append(f)
        f, ok = _global_face(_FRONT, lab)
        if ok:
            patches["front"][2].append(f)
        for e in (0, 1, 2, 3):
            if (bi, e) in claimed:
                continue
            f, ok = _global_face(_EDGE_FACE[e], lab)
            if not ok:
                continue
            first, second = _block_edge_ends(b, e)
            t = 0.5
            gid = _group_at_point(first[0] + t * (second[0] - first[0]), first[1] + t * (second[1] - first[1]),
                                  outline, match_tol)
            patch_for(gid)[2].append(f)
    return points, hexes, patches


def _write_block_mesh_dict(path, points, hexes, patches):
    """writeBlockMeshDict (file_converter.cpp:858-989)."""
    s = _header("dictionary", "blockMeshDict")
    s += "scale   1;\n\n"
    s += "vertices\n(\n" + "".join("    (%s %s %s)\n" % tuple(_g17(c) for c in v) for v in points) + ");\n\n"
    s += "blocks\n(\n"
    for lab, size, grad in hexes:
        s += "    hex (" + " ".join(str(k) for k in lab) + ") (%d %d %d)" % size
        s += " simpleGrading (%s %s %s)\n" % tuple(_g17(g) for g in grad)
    s += ");\n\n"
    s += "edges\n(\n);\n\n"
    s += "boundary\n(\n"
    for name in sorted(patches):
        ptype, _, faces = patches[name]
        s += "    " + name + "\n    {\n        type    " + _TYPE_NAME[ptype] + ";\n        faces\n        (\n"
        s += "".join("            (%d %d %d %d)\n" % tuple(f) for f in faces)
        s += "        );\n    }\n"
    s += ");\n\n"
    s += "mergeType points;\n\n"
    s += _RULE
    _write(path, s)


# ---------------------------------------------------------------- triangles
def _fv_faces(points, tris, mesh):
    """The FVMesh faces createUnstructuredMesh builds (mesh.cpp:1848-2002):
    the first triangle edge of each face gives v0, v1."""
    seen, v01 = {}, []
    for t in tris:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            key = (min(a, b), max(a, b))
            if key not in seen:
                seen[key] = len(v01)
                v01.append((int(a), int(b)))
    if len(v01) != int(mesh["nFaces"]):
        raise ValueError("the packed mesh was not built from these triangles")
    return v01


def poly_mesh(points, tris, mesh, groups, wedge=WEDGE_DEG):
    """polyMeshFromUnstructured (file_converter.cpp:579-856)."""
    pts = [(float(z), float(r)) for z, r in points]
    tris = [tuple(int(v) for v in t) for t in tris]
    v01 = _fv_faces(pts, tris, mesh)
    extent = 0.0
    for z, r in pts:
        extent = max(extent, max(abs(z), abs(r)))
    axis_tol = 1e-9 * (extent if extent > 0.0 else 1.0)
    half = 0.5 * wedge * (_PI / 180.0)
    ch, sh = math.cos(half), math.sin(half)
    out_pts, back, front = [], [], []
    for z, r in pts:
        if r <= axis_tol:
            back.append(len(out_pts))
            front.append(len(out_pts))
            out_pts.append((z, 0.0, 0.0))
            continue
        back.append(len(out_pts))
        out_pts.append((z, r * ch, -r * sh))
        front.append(len(out_pts))
        out_pts.append((z, r * ch, r * sh))
    patches = {"back": [WEDGE, -1, []], "front": [WEDGE, -1, []]}
    by_id = {g.id: g for g in groups}
    name_of = {}

    def patch_for(gid):
        if gid in name_of:
            return patches[name_of[gid]]
        grp = by_id.get(gid)
        stem = patch_name(grp) if grp else "unassigned"
        name, n = stem, 2
        while name in patches:
            name = "%s_%d" % (stem, n)
            n += 1
        name_of[gid] = name
        patches[name] = [_foam_type(grp.btype) if grp else PATCH, grp.id if grp else -1, []]
        return patches[name]

    def collapse(*labels):
        out = []
        for x in labels:
            if not out or out[-1] != x:
                out.append(x)
        if len(out) > 1 and out[0] == out[-1]:
            out.pop()
        return out
    interior = []
    own, nbr = mesh["faceOwner"], mesh["faceNeighbor"]
    fnz, fnr, grp = mesh["faceNormalZ"], mesh["faceNormalR"], mesh["faceBoundaryGroupID"]
    for f, (a, b) in enumerate(v01):
        dz = pts[b][0] - pts[a][0]
        dr = pts[b][1] - pts[a][1]
        if dr * float(fnz[f]) - dz * float(fnr[f]) < 0.0:
            a, b = b, a
        lab = collapse(back[a], back[b], front[b], front[a])
        if len(lab) < 3:
            continue
        o, n = int(own[f]), int(nbr[f])
        if n >= 0:
            if o > n:
                o, n = n, o
                lab.reverse()
            interior.append((o, n, lab))
            continue
        patch_for(int(grp[f]))[2].append((o, lab))
    for c, (v0, v1, v2) in enumerate(tris):
        az, ar = pts[v0]
        bz, br = pts[v1]
        dz_, dr_ = pts[v2]
        twice = (bz - az) * (dr_ - ar) - (br - ar) * (dz_ - az)
        if twice < 0.0:
            v1, v2 = v2, v1
        patches["front"][2].append((c, [front[v0], front[v1], front[v2]]))
        patches["back"][2].append((c, [back[v0], back[v2], back[v1]]))
    interior.sort(key=lambda x: (x[0], x[1]))
    faces = [x[2] for x in interior]
    owner = [x[0] for x in interior]
    neighbour = [x[1] for x in interior]
    out_patches = []
    for name in sorted(patches):
        ptype, gid, pf = patches[name]
        if not pf:
            continue
        pf = sorted(pf, key=lambda x: x[0])   # stable: by owner only
        out_patches.append((name, ptype, gid, len(faces), len(pf)))
        for o, lab in pf:
            faces.append(lab)
            owner.append(o)
    return dict(points=out_pts, faces=faces, owner=owner, neighbour=neighbour, patches=out_patches,
                nCells=len(tris))


def _write_poly_mesh(d, pm):
    """writePolyMesh (file_converter.cpp:991-1207)."""
    os.makedirs(d, exist_ok=True)

    def put(obj, cls, body):
        _write(os.path.join(d, obj), _header(cls, obj, "constant/polyMesh") + body + "\n" + _RULE)
    put("points", "vectorField", "%d\n(\n" % len(pm["points"]) +
        "".join("(%s %s %s)\n" % tuple(_g17(c) for c in p) for p in pm["points"]) + ")\n")
    put("faces", "faceList", "%d\n(\n" % len(pm["faces"]) +
        "".join("%d(%s)\n" % (len(f), " ".join(str(k) for k in f)) for f in pm["faces"]) + ")\n")
    put("owner", "labelList", "%d\n(\n" % len(pm["owner"]) + "".join("%d\n" % o for o in pm["owner"]) + ")\n")
    put("neighbour", "labelList", "%d\n(\n" % len(pm["neighbour"]) +
        "".join("%d\n" % n for n in pm["neighbour"]) + ")\n")
    body = "%d\n(\n" % len(pm["patches"])
    for name, ptype, gid, start, n in pm["patches"]:
        body += "    " + name + "\n    {\n        type            " + _TYPE_NAME[ptype] + ";\n"
        if ptype == WALL:
            body += "        inGroups        1(wall);\n"
        body += "        nFaces          %d;\n        startFace       %d;\n    }\n" % (n, start)
    put("boundary", "polyBoundaryMesh", body + ")\n")


# ---------------------------------------------------------------- system / constant
def _scalar_transport(field, diffusivity):
    return ("    " + field + "\n    {\n        type            scalarTransport;\n"
            "        libs            (solverFunctionObjects);\n\n"
            "        field           " + field + ";\n"
            "        D               " + foam_number(diffusivity) + ";\n\n"
            "        // Defaults to true, which would clamp the field to [0,1].\n"
            "        bounded01       false;\n\n"
            "        resetOnStartUp  false;\n"
            "        writeControl    writeTime;\n"
            "    }\n")


def _alpha(st):
    return st["k"] / (st["rho"] * st["cp"]) if (st["rho"] != 0.0 and st["cp"] != 0.0) else 0.0


def _control_dict(st):
    """writeControlDict (file_converter.cpp:1237-1321)."""
    s = _header("dictionary", "controlDict", "system")
    s += ("// Written from the project's solver settings. pimpleFoam/simpleFoam follows\n"
          "// the Transient checkbox, and the relaxation factors come from the Solver\n"
          "// tab. On a transient run so do endTime and deltaT. On a steady run endTime\n"
          "// is an ITERATION CAP and is not the Solver tab's value: it is the larger of\n"
          "// that and 2000, because residualControl is what should stop this run and a\n"
          "// reference cut short is worse than one that iterates longer than AxiSim did.\n\n")
    s += "application     " + ("pimpleFoam" if st["transient"] else "simpleFoam") + ";\n\n"
    s += "startFrom       startTime;\nstartTime       0;\n\nstopAt          endTime;\n"
    if st["transient"]:
        s += "endTime         " + foam_number(st["tEnd"]) + ";\n\n"
        s += "deltaT          " + foam_number(st["dt"]) + ";\n\n"
        interval = st["tEnd"] / 10.0 if st["tEnd"] > 0.0 else st["dt"]
        s += "writeControl    runTime;\nwriteInterval   " + foam_number(interval) + ";\n"
    else:
        s += "endTime         %d;\n\ndeltaT          1;\n\nwriteControl    timeStep;\n" % st["steadyIterations"]
        s += "writeInterval   %d;\n" % st["steadyIterations"]
    s += ("purgeWrite      0;\n\nwriteFormat     ascii;\nwritePrecision  12;\nwriteCompression off;\n\n"
          "timeFormat      general;\ntimePrecision   6;\n\nrunTimeModifiable true;\n\n")
    if st["solveEnergy"] or st["solveConcentration"]:
        s += "functions\n{\n"
        if st["solveEnergy"]:
            s += _scalar_transport("T", _alpha(st))
        if st["solveEnergy"] and st["solveConcentration"]:
            s += "\n"
        if st["solveConcentration"]:
            s += _scalar_transport(CONC, st["D"])
        s += "}\n\n"
    return s + _RULE


def _fv_schemes(st):
    """writeFvSchemes (file_converter.cpp:1323-1435)."""
    s = _header("dictionary", "fvSchemes", "system")
    s += "ddtSchemes\n{\n"
    if not st["transient"]:
        s += "    default         steadyState;\n"
    else:
        s += "    default         " + ("backward" if st["secondOrderTime"] else "Euler") + ";\n"
    s += "}\n\n"
    s += "gradSchemes\n{\n    default         " + ("leastSquares" if st["leastSquaresGradient"] else "Gauss linear")
    s += ";\n}\n\n"
    bounded = "" if st["transient"] else "bounded "
    interp = {LINEAR: "linear", LINEAR_UPWIND: "linearUpwind", QUICK: "QUICK"}.get(st["convection"], "upwind")
    needs_grad = st["convection"] == LINEAR_UPWIND

    def div(field):
        key = "div(phi," + field + ")"
        e = "    " + key + " " * (16 - len(key) if len(key) < 16 else 1) + bounded + "Gauss " + interp
        if needs_grad:
            e += " grad(" + field + ")"
        return e + ";\n"
    s += "divSchemes\n{\n    default         none;\n"
    if not st["addConvection"]:
        s += ("\n    // AxiSim ran this case with convection DISABLED (Solver tab ->\n"
              "    // Add Convection Term). A stock OpenFOAM flow solver always\n"
              "    // assembles div(phi,U), so the entry below IS solved and the two\n"
              "    // codes are not solving the same equations. Convection is\n"
              "    // negligible at low Re, which is the only case where comparing\n"
              "    // them still means something.\n")
    s += div("U")
    if st["solveEnergy"]:
        s += div("T")
    if st["solveConcentration"]:
        s += div(CONC)
    s += "    div((nuEff*dev2(T(grad(U))))) Gauss linear;\n}\n\n"
    s += ("laplacianSchemes\n{\n    default         Gauss linear corrected;\n}\n\n"
          "interpolationSchemes\n{\n    default         linear;\n}\n\n"
          "snGradSchemes\n{\n    default         corrected;\n}\n\n")
    return s + _RULE


def _fv_solution(st):
    """writeFvSolution (file_converter.cpp:1437-1531)."""
    s = _header("dictionary", "fvSolution", "system")
    s += ("solvers\n{\n    \"p.*\"\n    {\n        solver          GAMG;\n        smoother        GaussSeidel;\n"
          "        tolerance       1e-08;\n        relTol          0.01;\n    }\n\n"
          "    \"(U|T|Conc).*\"\n    {\n        solver          smoothSolver;\n"
          "        smoother        symGaussSeidel;\n        tolerance       1e-08;\n        relTol          0.1;\n"
          "    }\n}\n\n")
    nno = 1 if st["nonOrthCorrector"] else 0
    if st["transient"]:
        s += ("PIMPLE\n{\n    nOuterCorrectors 1;\n    nCorrectors     2;\n"
              "    nNonOrthogonalCorrectors %d;\n}\n\n" % nno)
    else:
        s += ("SIMPLE\n{\n    nNonOrthogonalCorrectors %d;\n    consistent      no;\n\n"
              "    residualControl\n    {\n        p               1e-06;\n        U               1e-06;\n"
              "        \"(T|Conc)\"      1e-06;\n    }\n}\n\n" % nno)
        s += ("relaxationFactors\n{\n    fields\n    {\n        p               " + foam_number(st["pressureRelaxation"])
              + ";\n    }\n    equations\n    {\n        U               " + foam_number(st["momentumRelaxation"])
              + ";\n        T               " + foam_number(st["momentumRelaxation"]) + ";\n        "
              + CONC + "            " + foam_number(st["concentrationRelaxation"])
              + ";   // AxiSim solves concentration unrelaxed\n    }\n}\n\n")
    return s + _RULE


def _transport_properties(st):
    """writeTransportProperties (file_converter.cpp:1533-1567)."""
    s = _header("dictionary", "transportProperties", "constant")
    s += "transportModel  Newtonian;\n\n"
    nu = st["mu"] / st["rho"] if st["rho"] != 0.0 else 0.0
    s += "// nu = mu / rho = " + foam_number(st["mu"]) + " / " + foam_number(st["rho"]) + "\n"
    s += "nu              " + foam_number(nu) + ";\n"
    if st["solveConcentration"]:
        s += ("\n// mass diffusivity. The scalarTransport function object in controlDict\n"
              "// reads its own copy of this; the entry here is for utilities that expect it.\n"
              "DT              " + foam_number(st["D"]) + ";\n")
    return s + "\n" + _RULE


def _turbulence_properties():
    return _header("dictionary", "turbulenceProperties", "constant") + "simulationType  laminar;\n\n" + _RULE


# ---------------------------------------------------------------- 0/ fields
def _bc_value(bc):
    """BoundaryCondition::value(): 0 for the kinetics laws."""
    return 0.0 if bc[0] in (_c.MICHAELIS_MENTEN, _c.HILL) else float(bc[1])


def _scalar_patch(bc):
    """scalarPatch (file_converter.cpp:1602-1689): (type, entry, note)."""
    t = bc[0]
    if t == _c.DIRICHLET:
        return "fixedValue", "value           uniform " + foam_number(_bc_value(bc)) + ";", ""
    if t == _c.NEUMANN:
        if _bc_value(bc) != 0.0:
            return "fixedGradient", "gradient        uniform " + foam_number(_bc_value(bc)) + ";", ""
        return "zeroGradient", "", ""
    if t == _c.PULSATILE:
        note = "steady mean of a pulsatile condition"
        note += (": value*(1 + " + foam_number(bc[2]) + "*sin(2*pi*" + foam_number(bc[3]) + "*t))"
                 " -- reproduce with uniformFixedValue + a sine Function1")
        return "fixedValue", "value           uniform " + foam_number(_bc_value(bc)) + ";", note
    if t in (_c.MICHAELIS_MENTEN, _c.HILL):
        k = bc[1]
        note = "PLACEHOLDER, NOT THE SAME PROBLEM: AxiSim applies a saturating wall flux"
        if t == _c.MICHAELIS_MENTEN:
            note += " (Michaelis-Menten, Vmax=" + foam_number(k["Vmax"]) + " Km=" + foam_number(k["Km"]) + ")"
        else:
            note += (" (Hill, Vmax=" + foam_number(k["Vmax"]) + " Km=" + foam_number(k["Km"])
                     + " n=" + foam_number(k["n"]) + ")")
        return "zeroGradient", "", note + "; swap in a codedMixed to match it"
    if t == _c.FULLY_DEVELOPED:
        return "zeroGradient", "", ("AxiSim had a fully-developed (parabolic) profile on this scalar,"
                                    " which zeroGradient is NOT -- see the U file for the codedFixedValue form")
    return "zeroGradient", "", ""


def _velocity_component(bc, uniform, group, coord):
    def uniform_field(v):
        return "scalarField(Cf.size(), scalar(" + foam_number(v) + "))"
    if bc[0] != _c.FULLY_DEVELOPED:
        return uniform_field(uniform)
    length = float(__import__("numpy").float32(group.total_length))
    if not length > 0.0:
        return uniform_field(_bc_value(bc))
    return ("scalar(" + foam_number(_bc_value(bc)) + ")*(1.0 - sqr(" + coord + "/scalar("
            + foam_number(length) + ")))")


def _velocity_patch(group):
    """velocityPatch (file_converter.cpp:1716-1837)."""
    axial = _c.effective_bc(group, _c.U)
    radial = _c.effective_bc(group, _c.V)

    def fixed(bc):
        return bc[0] in (_c.DIRICHLET, _c.PULSATILE)
    if axial[0] == _c.FULLY_DEVELOPED or radial[0] == _c.FULLY_DEVELOPED:
        u = _velocity_component(axial, _bc_value(axial) if fixed(axial) else 0.0, group, "r")
        v = _velocity_component(radial, _bc_value(radial) if fixed(radial) else 0.0, group, "z")
        needs_z = radial[0] == _c.FULLY_DEVELOPED
        entry = ("value           uniform (0 0 0);\n"
                 "        name            axiInlet" + str(group.id) + ";\n"
                 "        code\n"
                 "        #{\n"
                 "            const vectorField& Cf = patch().Cf();\n"
                 "            const scalarField r(sqrt(sqr(Cf.component(1)) + sqr(Cf.component(2))));\n"
                 + ("            const scalarField z(Cf.component(0));\n" if needs_z else "") +
                 "\n"
                 "            const scalarField u(" + u + ");\n"
                 "            const scalarField v(" + v + ");\n"
                 "\n"
                 "            // r is a DIRECTION on the wedge, not an axis, so the radial\n"
                 "            // component is projected onto the local radial unit vector.\n"
                 "            // The max() only guards a face on the axis, where the\n"
                 "            // components it scales are zero anyway.\n"
                 "            const scalarField rHat(max(r, scalar(SMALL)));\n"
                 "\n"
                 "            vectorField out(Cf.size(), Zero);\n"
                 "            out.replace(0, u);\n"
                 "            out.replace(1, v*Cf.component(1)/rHat);\n"
                 "            out.replace(2, v*Cf.component(2)/rHat);\n"
                 "\n"
                 "            operator==(out);\n"
                 "        #};")
        note = ("fully-developed profile, matching AxiSim's"
                " value*(1-(x/L)^2). Needs allowSystemOperations 1 in etc/controlDict")
        other = radial if axial[0] == _c.FULLY_DEVELOPED else axial
        if not fixed(other):
            note += "; the other velocity component was free in AxiSim and is pinned to 0 here"
        return "codedFixedValue", entry, note
    if not fixed(axial) and not fixed(radial):
        return "zeroGradient", "", ""
    u = _bc_value(axial) if fixed(axial) else 0.0
    v = _bc_value(radial) if fixed(radial) else 0.0
    if fixed(axial) and fixed(radial) and u == 0.0 and v == 0.0:
        return "noSlip", "", ""
    entry = "value           uniform (" + foam_number(u) + " " + foam_number(v) + " 0);"
    note = ""
    if fixed(axial) != fixed(radial):
        note = "one velocity component was free in AxiSim; pinned to 0 here, because fixedValue takes the whole vector"
    elif axial[0] == _c.PULSATILE or radial[0] == _c.PULSATILE:
        note = "steady mean of a pulsatile inlet -- reproduce with uniformFixedValue + a sine Function1"
    return "fixedValue", entry, note


def initial_fields(patches, groups, st):
    """initialFields (file_converter.cpp:1861-1967): patches {name: (type, groupID)}."""
    def inlet_value(var):
        for g in groups:
            if g.btype != _c.VELOCITY_INLET:
                continue
            bc = g.bcs.get(var)
            if bc is not None and bc[0] == _c.DIRICHLET:
                return float(bc[1])
        return 0.0
    fields = [dict(name="U", var=None, cls="volVectorField", dims="[0 1 -1 0 0 0 0]", internal="uniform (0 0 0)",
                   note=""),
              dict(name="p", var=_c.P, cls="volScalarField", dims="[0 2 -2 0 0 0 0]", internal="uniform 0",
                   note="p is KINEMATIC (p/rho), which is what the incompressible solvers want."
                        " AxiSim stores pressure in Pa, so divide any non-zero value below by rho.")]
    if st["solveEnergy"]:
        fields.append(dict(name="T", var=_c.TEMP, cls="volScalarField", dims="[0 0 0 1 0 0 0]",
                           internal="uniform " + foam_number(inlet_value(_c.TEMP)), note=""))
    if st["solveConcentration"]:
        fields.append(dict(name=CONC, var=_c.CONC, cls="volScalarField", dims="[0 -3 0 0 1 0 0]",
                           internal="uniform " + foam_number(inlet_value(_c.CONC)),
                           note="dimensioned as mol/m^3, matching the base SI values AxiSim stores."))
    by_id = {g.id: g for g in groups}
    for f in fields:
        f["patches"] = {}
    for name in sorted(patches):
        ptype, gid = patches[name]
        constraint = _TYPE_NAME[ptype] if ptype in (WEDGE, SYMMETRY_PLANE) else None
        grp = by_id.get(gid)
        for f in fields:
            if constraint:
                fp = (constraint, "", "")
            elif grp is None:
                fp = ("zeroGradient", "", "no boundary group behind this patch. zeroGradient is a guess")
            elif f["name"] == "U":
                fp = _velocity_patch(grp)
            else:
                fp = _scalar_patch(_c.effective_bc(grp, f["var"]))
            f["patches"][name] = fp
    return fields


def _write_fields(d, fields):
    """writeInitialFields (file_converter.cpp:1997-2046)."""
    for f in fields:
        s = _header(f["cls"], f["name"], "0")
        if f["note"]:
            s += "// " + f["note"] + "\n\n"
        s += "dimensions      " + f["dims"] + ";\n\ninternalField   " + f["internal"] + ";\n\nboundaryField\n{\n"
        for name in sorted(f["patches"]):
            t, entry, note = f["patches"][name]
            s += "    " + name + "\n    {\n        type            " + t + ";\n"
            if entry:
                s += "        " + entry + "\n"
            if note:
                s += "        // " + note + "\n"
            s += "    }\n"
        s += "}\n\n" + _RULE
        _write(os.path.join(d, f["name"]), s)


def _write(path, text):
    with open(path, "wb") as fh:
        fh.write(text.encode("utf-8"))


def save_foam_case(directory, groups, settings, blocks=None, outline=None, tol=1e-9, points=None, tris=None,
                   mesh=None, wedge=WEDGE_DEG):
    """saveFoamCase: a multiblock mesh (`blocks` with the domain `outline`,
    interface tolerance `tol`) goes out as system/blockMeshDict; a triangle
    mesh (`points`, `tris` and the packed `mesh` built from them, which
    carries the boundary groups) as constant/polyMesh. Returns the case
    directory's file list."""
    st = case_setup(settings)
    sysd, cons, zero = (os.path.join(directory, x) for x in ("system", "constant", "0"))
    for d in (sysd, cons, zero):
        os.makedirs(d, exist_ok=True)
    if blocks is not None:
        pts, hexes, patches = block_mesh_dict(blocks, groups, outline, tol, wedge)
        _write_block_mesh_dict(os.path.join(sysd, "blockMeshDict"), pts, hexes, patches)
        refs = {name: (p[0], p[1]) for name, p in patches.items()}
    else:
        pm = poly_mesh(points, tris, mesh, groups, wedge)
        _write_poly_mesh(os.path.join(cons, "polyMesh"), pm)
        refs = {name: (ptype, gid) for name, ptype, gid, _, _ in pm["patches"]}
    _write(os.path.join(sysd, "controlDict"), _control_dict(st))
    _write(os.path.join(sysd, "fvSchemes"), _fv_schemes(st))
    _write(os.path.join(sysd, "fvSolution"), _fv_solution(st))
    _write(os.path.join(cons, "transportProperties"), _transport_properties(st))
    _write(os.path.join(cons, "turbulenceProperties"), _turbulence_properties())
    _write_fields(zero, initial_fields(refs, groups, st))
    out = []
    for root, _, files in os.walk(directory):
        out += [os.path.relpath(os.path.join(root, f), directory) for f in files]
    return sorted(out)
