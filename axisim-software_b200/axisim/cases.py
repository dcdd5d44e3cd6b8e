"""Synthetic cases for the SIMPLE path: mesh blocks, boundary groups, settings.

Each case is a plain description (multiblock block specs, boundary groups with
their per-variable conditions, solver settings) that both the CUDA path and the
CPU oracle consume. The boundary resolution follows the reference's
BoundaryDefaults (manager/source/boundary_func.cpp:104-201, 333-378) and the
pulsatile-to-Dirichlet mapping of createBoundaryFieldHost
(manager/source/memory_manger.cpp:51-152).
"""
from dataclasses import dataclass, field
import math

import numpy as np

# BCType (structs/boundary_struct.h:90-99)
DIRICHLET, NEUMANN, FULLY_DEVELOPED, MICHAELIS_MENTEN, HILL, NONE, PULSATILE = range(7)
# BoundaryType (structs/boundary_struct.h:342-348)
WALL, VELOCITY_INLET, PRESSURE_OUTLET, SYMMETRY, FAR_FIELD = range(5)
# BoundaryVariable: velocity components, pressure, static temperature, concentration
U, V, P, TEMP, CONC = "u", "v", "p", "T", "C"
SCALARS = (TEMP, CONC)
# ConvectionScheme / GradientScheme / LinearSolverType / TimeScheme
CONV_UPWIND, CONV_CENTRAL, CONV_SOU, CONV_QUICK = range(4)
GRAD_GREEN_GAUSS, GRAD_LSQ = range(2)
LINEAR_JACOBI, LINEAR_GS_RB = range(2)
TIME_FIRST_ORDER, TIME_SECOND_ORDER = range(2)
# Grading (structs/multiblock.h:46)
UNIFORM, PROGRESSION = range(2)
WEST, EAST, SOUTH, NORTH = range(4)


def default_bc_type(btype, var):
    """getDefaultBCType (boundary_func.cpp:117-201): the scalars are Dirichlet
    at a velocity inlet and zero-gradient everywhere else."""
    table = {
        VELOCITY_INLET: {U: DIRICHLET, V: DIRICHLET, P: NEUMANN, TEMP: DIRICHLET, CONC: DIRICHLET},
        PRESSURE_OUTLET: {U: NEUMANN, V: NEUMANN, P: DIRICHLET, TEMP: NEUMANN, CONC: NEUMANN},
        WALL: {U: DIRICHLET, V: DIRICHLET, P: NEUMANN, TEMP: NEUMANN, CONC: NEUMANN},
        SYMMETRY: {U: NEUMANN, V: DIRICHLET, P: NEUMANN, TEMP: NEUMANN, CONC: NEUMANN},
        FAR_FIELD: {U: DIRICHLET, V: DIRICHLET, P: NEUMANN, TEMP: NEUMANN, CONC: NEUMANN},
    }
    return table.get(btype, {}).get(var, NONE)


def variable_editable(var, btype):
    """isVariableInBoundaryType (boundary_func.cpp:333-378)."""
    if btype == WALL:
        return var in (U, V, TEMP, CONC)
    if btype == SYMMETRY:
        return False
    if btype == FAR_FIELD:
        return var in (U, V)
    if btype == VELOCITY_INLET:
        return var in (U, V, TEMP, CONC)
    if btype == PRESSURE_OUTLET:
        return var in (P, TEMP, CONC)
    return False


def michaelis_menten(vmax, km, inhibition=None):
    """MichaelisMentenParams (boundary_struct.h:111): J = Vmax c / (Km + c),
    times 1 - V2 c^m / (K2^m + c^m) when inhibition = (m, K2, V2) is given."""
    return (MICHAELIS_MENTEN, dict(Vmax=vmax, Km=km, n=1.0, inhibition=inhibition))


def hill(vmax, km, n, inhibition=None):
    """HillParams (boundary_struct.h:112): J = Vmax c^n / (Km^n + c^n)."""
    return (HILL, dict(Vmax=vmax, Km=km, n=n, inhibition=inhibition))


@dataclass
class Group:
    """BoundarySegmentGroup (boundary_struct.h:501-533): id, type, user BCs, totalLength.

    bcs maps variable -> (bcType, value), (PULSATILE, mean, amplitude, frequency)
    or a kinetics condition from michaelis_menten() / hill(). layers maps a
    scalar variable to its wall stack [(k, d), ...], a series resistance
    sum d / k (Layer::resistance, boundary_struct.h:24-39).
    total_length is stored as float32, as the reference's float totalLength is.
    """
    id: int
    btype: int
    bcs: dict = field(default_factory=dict)
    total_length: float = 0.0
    layers: dict = field(default_factory=dict)
    name: str = ""   # BoundarySegmentGroup::name (the OpenFOAM export derives patch names from it)


def effective_bc(group, var):
    """getEffectiveBC (boundary_func.cpp:104-115)."""
    if var in group.bcs and variable_editable(var, group.btype):
        return group.bcs[var]
    return (default_bc_type(group.btype, var), 0.0)


def resolve_bc_field(groups, var):
    """createBoundaryFieldHost (memory_manger.cpp:51-152) for one variable:
    per-group type/boundaryType/value/length arrays; PULSATILE maps to DIRICHLET
    with its mean value, and is flagged so the solver updates it per time step."""
    G = max(g.id for g in groups) + 1 if groups else 0
    out = dict(type=np.full(G, NONE, np.uint8), btype=np.full(G, WALL, np.uint8),
               value=np.zeros(G), length=np.zeros(G), puls=np.zeros(G, np.uint8),
               amp=np.zeros(G), freq=np.zeros(G))
    if var in SCALARS:  # kinetics defaults (memory_manger.cpp:72-83)
        out.update(vmax=np.zeros(G), km=np.zeros(G), n=np.ones(G), m=np.ones(G), k2=np.zeros(G),
                   v2=np.zeros(G), Rtot=np.zeros(G))
    for g in groups:
        if g.id < 0:
            continue
        bc = effective_bc(g, var)
        t = bc[0]
        out["type"][g.id] = DIRICHLET if t == PULSATILE else t
        out["btype"][g.id] = g.btype
        out["length"][g.id] = float(np.float32(g.total_length))
        if t in (MICHAELIS_MENTEN, HILL):
            # memory_manger.cpp:110-131: a kinetics condition has no single value
            k = bc[1]
            out["vmax"][g.id] = k["Vmax"]
            out["km"][g.id] = k["Km"]
            if t == HILL:
                out["n"][g.id] = k["n"]
            if k.get("inhibition"):
                out["m"][g.id], out["k2"][g.id], out["v2"][g.id] = k["inhibition"]
        else:
            out["value"][g.id] = bc[1]
        if var in SCALARS and var in g.layers:  # memory_manger.cpp:133-145
            R = 0.0
            for (k_layer, d_layer) in g.layers[var]:
                R += (d_layer / k_layer) if k_layer != 0.0 else 0.0
            out["Rtot"][g.id] = R
        if t == PULSATILE:
            out["puls"][g.id] = 1
            out["amp"][g.id] = bc[2]
            out["freq"][g.id] = bc[3]
    return out


def block(z0, r0, axial, radial, edge_group=(-1, -1, -1, -1)):
    """Block spec for makeRectBlock (multiblock.h:118-136). axial/radial are
    (length, cells, grading, coef) MeshZones."""
    def zone(z):
        z = tuple(z)
        if len(z) == 2:
            z = z + (UNIFORM, 1.0)
        return (float(z[0]), int(z[1]), int(z[2]), float(z[3]))
    return dict(z0=float(z0), r0=float(r0), axial=zone(axial), radial=zone(radial),
                edge_group=list(edge_group))


def default_settings():
    """ConfigSolver/ConfigSimple/ConfigMultigrid/ConfigResidual defaults
    (solver_struct.h:158-231, 240-258) plus SIMPLE relaxation (0.7 / 0.3)."""
    return dict(convectionScheme=CONV_UPWIND, gradientScheme=GRAD_LSQ, linearType=LINEAR_JACOBI,
                timeScheme=TIME_FIRST_ORDER, linearMaxIter=20, useMultigrid=1, addConvectionTerm=1,
                transient=0, useNonOrthCorrector=0, dt=0.1, tEnd=2.0, maxIter=50, checkConv=1,
                mgMaxIter=3, mgWeight=0.6, mgLinearSweep=30, mgPreSweep=1, mgPostSweep=1,
                rho=998.0, mu=0.0010518, alphaU=0.7, alphaP=0.3,
                resNorm=[0, 0, 0], resScale=[3, 3, 3], resEnabled=[1, 1, 1], resTol=[1e-3, 1e-3, 1e-3],
                solveEnergy=0, solveConcentration=0, cp=4180.0, k=0.6, D=3.0277e-9,
                scalarResNorm=[0, 0], scalarResScale=[3, 3], scalarResEnabled=[0, 0],
                scalarResTol=[1e-3, 1e-3])


@dataclass
class Case:
    name: str
    blocks: list
    groups: list
    settings: dict
    note: str = ""
    mesh: dict = None   # packed mesh for unstructured cases (blocks empty)

    def bc_fields(self):
        """Per-variable boundary fields: u, v, p, and T / C when the settings solve them."""
        out = {v: resolve_bc_field(self.groups, v) for v in (U, V, P)}
        if self.settings.get("solveEnergy"):
            out[TEMP] = resolve_bc_field(self.groups, TEMP)
        if self.settings.get("solveConcentration"):
            out[CONC] = resolve_bc_field(self.groups, CONC)
        return out

    def packed(self, builder):
        """The packed mesh: the stored one, or `builder(blocks)` (the C++ or the oracle packer)."""
        return self.mesh if self.mesh is not None else builder(self.blocks)


def pipe(nr=40, nz=200, R=0.01, L=0.2, U0=0.05, rho=1000.0, mu=1e-3, fully_developed=False,
         max_iter=50000, tol=1e-6):
    """Laminar pipe flow, Re_D = 1000 at the defaults (uniform r-z mesh, 40 x 200).
    Upwind convection, Green-Gauss gradients, alpha 0.7/0.3, multicolour GS for
    u and v, agglomeration multigrid for p'. fully_developed=True prescribes the
    parabolic inlet with peak 2*U0 (used for the analytic Poiseuille check)."""
    inlet_bc = (FULLY_DEVELOPED, 2.0 * U0) if fully_developed else (DIRICHLET, U0)
    groups = [Group(0, VELOCITY_INLET, {U: inlet_bc}, total_length=R),
              Group(1, PRESSURE_OUTLET, {P: (DIRICHLET, 0.0)}, total_length=R),
              Group(2, WALL, {}, total_length=L),
              Group(3, SYMMETRY, {}, total_length=L)]
    blocks = [block(0.0, 0.0, (L, nz), (R, nr), edge_group=(0, 1, 3, 2))]
    s = default_settings()
    s.update(convectionScheme=CONV_UPWIND, gradientScheme=GRAD_GREEN_GAUSS, linearType=LINEAR_GS_RB,
             rho=rho, mu=mu, alphaU=0.7, alphaP=0.3, maxIter=max_iter, resTol=[tol, tol, tol])
    return Case(f"pipe_{nr}x{nz}", blocks, groups, s)


def _prog(n, ratio, toward_end):
    """Progression coefficient giving max/min spacing `ratio` over n cells,
    smaller cells at the end of the band (toward_end) or at its start."""
    if n <= 1 or ratio == 1.0:
        return (UNIFORM, 1.0)
    c = ratio ** (1.0 / (n - 1))
    return (PROGRESSION, 1.0 / c if toward_end else c)


def expansion(nr_in=86, nr_out=170, nz_in=1024, nz_out=3072, r_in=0.002, r_out=0.006, l_in=0.04,
              l_out=0.12, rho=1056.0, mu=3.5e-3, re=500.0, bias=1.1, scheme=CONV_SOU,
              max_iter=50000, tol=1e-6, scale=1.0):
    """Sudden expansion on a three-block trellis mesh: inlet pipe (radius r_in,
    length l_in) then an abrupt step to r_out over l_out. Band totals default to
    256 radial x 4096 axial (874,496 cells; the block outside the domain is
    dropped, as Mesh::buildStructuredMultiBlock does, mesh.cpp:2717-2741).
    Grading: each band is a geometric progression whose end-to-end spacing ratio
    is `bias`, with the small cells at the step and at the walls. Fully developed
    inlet with peak 2*Ubar, Ubar from the throat Reynolds number. Second-order
    upwind by default. `scale` multiplies every cell count (for test sizes)."""
    nr_in, nr_out = max(1, round(nr_in * scale)), max(1, round(nr_out * scale))
    nz_in, nz_out = max(1, round(nz_in * scale)), max(1, round(nz_out * scale))
    ubar = re * mu / (rho * 2.0 * r_in)
    z_in = _prog(nz_in, bias, toward_end=True)       # small cells at the step
    z_out = _prog(nz_out, bias, toward_end=False)    # small cells at the step
    r_lo = _prog(nr_in, bias, toward_end=True)       # small cells at the inlet-pipe wall
    r_hi = _prog(nr_out, bias, toward_end=True)      # small cells at the outer wall
    g_in, g_out, g_wall, g_axis = 0, 1, 2, 3
    blocks = [
        block(0.0, 0.0, (l_in, nz_in) + z_in, (r_in, nr_in) + r_lo, edge_group=(g_in, -1, g_axis, g_wall)),
        block(l_in, 0.0, (l_out, nz_out) + z_out, (r_in, nr_in) + r_lo, edge_group=(-1, g_out, g_axis, -1)),
        block(l_in, r_in, (l_out, nz_out) + z_out, (r_out - r_in, nr_out) + r_hi,
              edge_group=(g_wall, g_out, -1, g_wall)),
    ]
    groups = [Group(g_in, VELOCITY_INLET, {U: (FULLY_DEVELOPED, 2.0 * ubar)}, total_length=r_in),
              Group(g_out, PRESSURE_OUTLET, {P: (DIRICHLET, 0.0)}, total_length=r_out),
              Group(g_wall, WALL, {}, total_length=l_in + (r_out - r_in) + l_out),
              Group(g_axis, SYMMETRY, {}, total_length=l_in + l_out)]
    s = default_settings()
    s.update(convectionScheme=scheme, gradientScheme=GRAD_LSQ, linearType=LINEAR_JACOBI, rho=rho, mu=mu,
             maxIter=max_iter, resTol=[tol, tol, tol])
    n = nr_in * nz_in + nr_in * nz_out + nr_out * nz_out
    return Case(f"expansion_{n}", blocks, groups, s,
                note=f"Ubar={ubar:.6g} m/s; bias={bias} end-to-end spacing ratio per band")


def pulsatile_expansion(scale=1.0, dt=1e-4, steps=2000, period=0.1, amplitude=0.5, **kw):
    """Transient pulsatile sudden expansion: the expansion geometry, BDF2 in
    time, inlet u(t) = U0 (1 + A sin(2 pi t / T)) as a uniform Dirichlet value
    (the reference maps PULSATILE to Dirichlet, memory_manger.cpp:96-100)."""
    c = expansion(scale=scale, **kw)
    rho, mu = c.settings["rho"], c.settings["mu"]
    u0 = 500.0 * mu / (rho * 0.004)
    c.groups[0].bcs[U] = (PULSATILE, u0, amplitude, 1.0 / period)
    c.settings.update(transient=1, timeScheme=TIME_SECOND_ORDER, dt=dt, tEnd=dt * steps)
    c.name = "pulsatile_" + c.name
    return c


def bullet(scale=1.0, rho=1000.0, mu=1e-3, re=200.0, seed=0, max_iter=50000, tol=1e-6):
    """Revolved bullet body (cylinder radius 5 mm, length 30 mm, hemispherical
    nose) on the axis of a pipe of radius 20 mm and length 300 mm, triangulated
    to ~485k cells at scale 1 (1250 x 200 quads split in two, body removed,
    interior vertices jittered +-10 % of the spacing from a fixed seed).
    Uniform inlet at Re 200 on the body diameter; the fluid is unstated in the
    case description, so water (rho 1000, mu 1e-3, U = 0.02 m/s). Least-squares
    gradients with the non-orthogonal corrector, agglomeration multigrid."""
    from . import trimesh
    nz, nr = max(8, round(1250 * scale)), max(4, round(200 * scale))
    pts, tris, classify = trimesh.bullet_in_pipe(nz=nz, nr=nr, seed=seed)
    mesh = trimesh.pack_triangles(pts, tris, classify)
    u_in = re * mu / (rho * 0.01)
    groups = [Group(0, VELOCITY_INLET, {U: (DIRICHLET, u_in)}, total_length=0.02),
              Group(1, PRESSURE_OUTLET, {P: (DIRICHLET, 0.0)}, total_length=0.02),
              Group(2, WALL, {}, total_length=0.3),
              Group(3, SYMMETRY, {}, total_length=0.3)]
    s = default_settings()
    s.update(convectionScheme=CONV_UPWIND, gradientScheme=GRAD_LSQ, linearType=LINEAR_JACOBI, useNonOrthCorrector=1,
             rho=rho, mu=mu, maxIter=max_iter, resTol=[tol, tol, tol])
    return Case(f"bullet_{mesh['nCells']}", [], groups, s, note=f"U_in={u_in:.4g} m/s", mesh=mesh)


def with_scalars(case, energy=True, concentration=True, t_in=310.0, t_wall=300.0, c_in=1.0, wall_c=None,
                 wall_layers=None, k=None, D=None):
    """Adds energy and/or concentration transport to a case: Dirichlet T and C
    at every velocity inlet; at every wall, T fixed at t_wall (None keeps the
    zero-gradient default) and C by wall_c (a michaelis_menten() / hill()
    condition, a (type, value) pair, or None for zero gradient) behind the
    layer stack wall_layers [(k, d), ...]. k / D override the conductivity and
    the mass diffusivity."""
    for g in case.groups:
        if g.btype == VELOCITY_INLET:
            if energy:
                g.bcs[TEMP] = (DIRICHLET, t_in)
            if concentration:
                g.bcs[CONC] = (DIRICHLET, c_in)
        elif g.btype == WALL:
            if energy and t_wall is not None:
                g.bcs[TEMP] = (DIRICHLET, t_wall)
            if concentration and wall_c is not None:
                g.bcs[CONC] = wall_c
            if concentration and wall_layers:
                g.layers[CONC] = list(wall_layers)
    case.settings.update(solveEnergy=int(bool(energy)), solveConcentration=int(bool(concentration)))
    if k is not None:
        case.settings["k"] = k
    if D is not None:
        case.settings["D"] = D
    case.name += "_scalars"
    return case


def polygon_outline(points, groups):
    """A closed outline loop: points [(z, r), ...] in order, groups[i] the
    boundary group of the edge from point i to point i + 1 (the last edge
    closes the loop). Returns (vertices, edges, groups) as the mesh builders
    take them."""
    n = len(points)
    edges = [(i, (i + 1) % n) for i in range(n)]
    return np.asarray(points, np.float64), np.asarray(edges, np.int32), np.asarray(groups, np.int32)


def expansion_outline(r_in=0.002, r_out=0.006, l_in=0.04, l_out=0.12, g_in=0, g_out=1, g_wall=2, g_axis=3):
    """The sudden expansion's outline with the groups expansion() uses."""
    L = l_in + l_out
    pts = [(0.0, 0.0), (L, 0.0), (L, r_out), (l_in, r_out), (l_in, r_in), (0.0, r_in)]
    return polygon_outline(pts, [g_axis, g_out, g_wall, g_wall, g_wall, g_in])


def cell_count(case):
    return sum(int(b["axial"][1]) * int(b["radial"][1]) for b in case.blocks)


def expansion_metrics(mesh, u, p, r_in=0.002, r_out=0.006, l_in=0.04, l_total=0.16):
    """Flow quantities of the sudden expansion used to compare precisions:
    centreline axial velocity u(z) (cells next to the axis), pressure drop
    (area-weighted p next to the inlet minus next to the outlet) and the corner
    recirculation length (from the step to where u next to the outer wall
    turns positive)."""
    zc, rc, vol = mesh["cellCenterZ"], mesh["cellCenterR"], mesh["cellVolume"]
    r_axis = rc.min()
    axis = np.isclose(rc, r_axis, rtol=0, atol=1e-12)
    order = np.argsort(zc[axis])
    centre_z, centre_u = zc[axis][order], u[axis][order]
    dz_in = np.sort(np.unique(zc))[:1]
    first_col = np.isclose(zc, zc.min(), rtol=0, atol=1e-12)
    last_col = np.isclose(zc, zc.max(), rtol=0, atol=1e-12)
    p_in = np.sum(p[first_col] * vol[first_col]) / np.sum(vol[first_col])
    p_out = np.sum(p[last_col] * vol[last_col]) / np.sum(vol[last_col])
    wall = np.isclose(rc, rc[zc > l_in].max(), rtol=0, atol=1e-12) & (zc > l_in)
    wz, wu = zc[wall], u[wall]
    o = np.argsort(wz)
    wz, wu = wz[o], wu[o]
    # primary recirculation: the longest run of reversed flow along the outer
    # wall (a small corner eddy can sit right at the step)
    recirc, to_outlet = 0.0, False
    neg = wu < 0
    if neg.any():
        edges = np.diff(np.concatenate([[0], neg.astype(np.int8), [0]]))
        starts, ends = np.nonzero(edges == 1)[0], np.nonzero(edges == -1)[0]
        k = int(np.argmax(ends - starts))
        to_outlet = ends[k] == len(wu)
        recirc = (l_total if to_outlet else wz[ends[k]]) - l_in
    del dz_in
    return {"centre_z": centre_z, "centre_u": centre_u, "dp": p_in - p_out, "recirculation_length": float(recirc),
            "recirculation_reaches_outlet": to_outlet}
