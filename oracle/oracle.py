"""ctypes binding of the CPU oracle (oracle/liborc.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, to compare against. The product path never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


class OrcMesh(C.Structure):
    _fields_ = [("nCells", C.c_int32), ("nFaces", C.c_int32),
                ("faceOwner", _i32p), ("faceNeighbor", _i32p),
                ("faceNormalZ", _f64p), ("faceNormalR", _f64p),
                ("faceCenterZ", _f64p), ("faceCenterR", _f64p), ("faceArea", _f64p),
                ("faceBoundaryGroupID", _i32p),
                ("cellCenterZ", _f64p), ("cellCenterR", _f64p),
                ("cellArea2D", _f64p), ("cellVolume", _f64p),
                ("cellFaceStart", _i32p), ("cellFaceIDs", _i32p)]


class OrcBC(C.Structure):
    _fields_ = [("nGroups", C.c_int32), ("typeByGroup", _u8p), ("boundaryTypeByGroup", _u8p),
                ("valueByGroup", _f64p), ("lengthByGroup", _f64p),
                ("pulsatileByGroup", _u8p), ("amplitudeByGroup", _f64p),
                ("frequencyByGroup", _f64p), ("vmaxByGroup", _f64p), ("kmByGroup", _f64p),
                ("nByGroup", _f64p), ("mByGroup", _f64p), ("k2ByGroup", _f64p), ("v2ByGroup", _f64p),
                ("RtotByGroup", _f64p)]


class OrcConfig(C.Structure):
    _fields_ = [("convectionScheme", C.c_int), ("gradientScheme", C.c_int), ("linearType", C.c_int),
                ("timeScheme", C.c_int), ("linearMaxIter", C.c_int), ("useMultigrid", C.c_int),
                ("addConvectionTerm", C.c_int), ("transient", C.c_int), ("useNonOrthCorrector", C.c_int),
                ("dt", C.c_double), ("tEnd", C.c_double), ("maxIter", C.c_int), ("checkConv", C.c_int),
                ("mgMaxIter", C.c_int), ("mgWeight", C.c_double), ("mgLinearSweep", C.c_int),
                ("mgPreSweep", C.c_int), ("mgPostSweep", C.c_int), ("rho", C.c_double), ("mu", C.c_double),
                ("alphaU", C.c_double), ("alphaP", C.c_double), ("resNorm", C.c_int * 3),
                ("resScale", C.c_int * 3), ("resEnabled", C.c_int * 3), ("resTol", C.c_double * 3),
                ("solveEnergy", C.c_int), ("solveConcentration", C.c_int), ("cp", C.c_double),
                ("k", C.c_double), ("D", C.c_double), ("scalarResNorm", C.c_int * 2),
                ("scalarResScale", C.c_int * 2), ("scalarResEnabled", C.c_int * 2),
                ("scalarResTol", C.c_double * 2), ("structuredMesh", C.c_int)]


class OrcBlock(C.Structure):
    _fields_ = [("z0", C.c_double), ("r0", C.c_double),
                ("axialLength", C.c_double), ("axialCells", C.c_int), ("axialGrading", C.c_int),
                ("axialCoef", C.c_double),
                ("radialLength", C.c_double), ("radialCells", C.c_int), ("radialGrading", C.c_int),
                ("radialCoef", C.c_double), ("edgeGroup", C.c_int * 4)]


def build(force=False):
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.orc_mb_build.restype = C.c_void_p
        L.orc_mb_build.argtypes = [C.c_int, C.POINTER(OrcBlock), C.c_double, C.c_int, C.POINTER(C.c_int)]
        L.orc_mb_sizes.argtypes = [C.c_void_p, _i32p, _i32p, _i32p]
        L.orc_mb_copy.argtypes = [C.c_void_p] + [C.c_void_p] * 14
        L.orc_mb_free.argtypes = [C.c_void_p]
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcBC), C.POINTER(OrcBC),
                                 C.POINTER(OrcBC), C.POINTER(OrcConfig)]
        L.orc_create_ex.restype = C.c_void_p
        L.orc_create_ex.argtypes = [C.POINTER(OrcMesh)] + [C.POINTER(OrcBC)] * 5 + [C.POINTER(OrcConfig)]
        L.orc_scalar_residuals.argtypes = [C.c_void_p, _f64p]
        L.orc_run.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.orc_get.argtypes = [C.c_void_p, C.c_char_p, _f64p, C.c_size_t]
        L.orc_set.argtypes = [C.c_void_p, C.c_char_p, _f64p, C.c_size_t]
        L.orc_last_residuals.argtypes = [C.c_void_p, _f64p]
        L.orc_iterations.argtypes = [C.c_void_p]
        L.orc_mg_levels.argtypes = [C.c_void_p, _i32p, C.c_int]
        L.orc_mg_level_maps.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_coloring.argtypes = [C.c_void_p, _i32p]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def multiblock(blocks, tol=1e-9, default_group=-1):
    """Pack a multiblock mesh with the oracle's restatement of multiblock.h.
    blocks: list of dicts with z0, r0, axial=(length, cells, grading, coef),
    radial=(...), edge_group=[W, E, S, N]. Returns dict of numpy arrays."""
    L = lib()
    arr = (OrcBlock * len(blocks))()
    for i, b in enumerate(blocks):
        ax, rd = b["axial"], b["radial"]
        arr[i] = OrcBlock(b["z0"], b["r0"], ax[0], ax[1], ax[2], ax[3], rd[0], rd[1], rd[2], rd[3],
                          (C.c_int * 4)(*b["edge_group"]))
    st = C.c_int(0)
    h = L.orc_mb_build(len(blocks), arr, tol, default_group, C.byref(st))
    n, f, r = C.c_int32(), C.c_int32(), C.c_int32()
    L.orc_mb_sizes(h, C.byref(n), C.byref(f), C.byref(r))
    n, f, r = n.value, f.value, r.value
    m = dict(nCells=n, nFaces=f,
             faceOwner=np.zeros(f, np.int32), faceNeighbor=np.zeros(f, np.int32),
             faceNormalZ=np.zeros(f), faceNormalR=np.zeros(f), faceCenterZ=np.zeros(f),
             faceCenterR=np.zeros(f), faceArea=np.zeros(f), faceBoundaryGroupID=np.zeros(f, np.int32),
             cellCenterZ=np.zeros(n), cellCenterR=np.zeros(n), cellArea2D=np.zeros(n),
             cellVolume=np.zeros(n), cellFaceStart=np.zeros(n + 1, np.int32),
             cellFaceIDs=np.zeros(r, np.int32))
    keys = ["faceOwner", "faceNeighbor", "faceNormalZ", "faceNormalR", "faceCenterZ", "faceCenterR",
            "faceArea", "faceBoundaryGroupID", "cellCenterZ", "cellCenterR", "cellArea2D", "cellVolume",
            "cellFaceStart", "cellFaceIDs"]
    L.orc_mb_copy(h, *[m[k].ctypes.data_as(C.c_void_p) for k in keys])
    L.orc_mb_free(h)
    m["status"] = st.value
    m["meshType"] = 0  # MeshType::Structured
    return m


def mesh_struct(m):
    keep = []

    def P(k, t):
        a = np.ascontiguousarray(m[k])
        keep.append(a)
        return a.ctypes.data_as(t)
    s = OrcMesh(m["nCells"], m["nFaces"], P("faceOwner", _i32p), P("faceNeighbor", _i32p),
                P("faceNormalZ", _f64p), P("faceNormalR", _f64p), P("faceCenterZ", _f64p),
                P("faceCenterR", _f64p), P("faceArea", _f64p), P("faceBoundaryGroupID", _i32p),
                P("cellCenterZ", _f64p), P("cellCenterR", _f64p), P("cellArea2D", _f64p),
                P("cellVolume", _f64p), P("cellFaceStart", _i32p), P("cellFaceIDs", _i32p))
    return s, keep


KINETICS_KEYS = ("vmax", "km", "n", "m", "k2", "v2", "Rtot")


def bc_struct(bc):
    """bc: dict type(u8[G]) btype(u8[G]) value(f64[G]) length(f64[G]) [puls amp freq]
    [vmax km n m k2 v2 Rtot] (the wall-kinetics arrays of a scalar field)"""
    keep = []

    def P(k, t, dt):
        if k not in bc or bc[k] is None:
            return None
        a = np.ascontiguousarray(bc[k], dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(t)
    G = len(bc["type"])
    s = OrcBC(G, P("type", _u8p, np.uint8), P("btype", _u8p, np.uint8), P("value", _f64p, np.float64),
              P("length", _f64p, np.float64), P("puls", _u8p, np.uint8), P("amp", _f64p, np.float64),
              P("freq", _f64p, np.float64), *[P(k, _f64p, np.float64) for k in KINETICS_KEYS])
    return s, keep


def config_struct(cfg):
    c = OrcConfig()
    for k, v in cfg.items():
        if k in ("resNorm", "resScale", "resEnabled"):
            setattr(c, k, (C.c_int * 3)(*v))
        elif k == "resTol":
            setattr(c, k, (C.c_double * 3)(*v))
        elif k in ("scalarResNorm", "scalarResScale", "scalarResEnabled"):
            setattr(c, k, (C.c_int * 2)(*v))
        elif k == "scalarResTol":
            setattr(c, k, (C.c_double * 2)(*v))
        else:
            setattr(c, k, v)
    return c


class Oracle:
    """One oracle solver instance on one case (mesh + bcs + config dicts)."""

    def __init__(self, mesh, bcs, cfg, threads=0):
        L = lib()
        if threads:
            L.orc_set_threads(threads)
        self._ms, self._mk = mesh_struct(mesh)
        self._b = [bc_struct(bcs[k]) if k in bcs else None for k in ("u", "v", "p", "T", "C")]
        # Mesh::currentMeshType: multiblock meshes are structured
        self._cfg = config_struct(dict(cfg, structuredMesh=int(mesh.get("meshType", 1) == 0)))
        self.mesh = mesh
        ref = [C.byref(b[0]) if b is not None else None for b in self._b]
        self.h = L.orc_create_ex(C.byref(self._ms), *ref, C.byref(self._cfg))
        if not self.h:
            raise RuntimeError("orc_create failed")

    def run(self, cont=False):
        conv = C.c_int(0)
        it = lib().orc_run(self.h, 1 if cont else 0, C.byref(conv))
        return it, bool(conv.value)

    def get(self, name):
        n = self.mesh["nCells"]
        size = max(n, self.mesh["nFaces"], len(self.mesh["cellFaceIDs"]))
        out = np.zeros(size)
        k = lib().orc_get(self.h, name.encode(), out.ctypes.data_as(_f64p), size)
        if k < 0:
            raise KeyError(name)
        return out[:k].copy()

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        k = lib().orc_set(self.h, name.encode(), a.ctypes.data_as(_f64p), a.size)
        if k < 0:
            raise KeyError(name)

    def residuals(self):
        out = np.zeros(3)
        lib().orc_last_residuals(self.h, out.ctypes.data_as(_f64p))
        return out

    def scalar_residuals(self):
        out = np.zeros(2)
        lib().orc_scalar_residuals(self.h, out.ctypes.data_as(_f64p))
        return out

    def iterations(self):
        return lib().orc_iterations(self.h)

    def mg_levels(self):
        cells = np.zeros(64, np.int32)
        n = lib().orc_mg_levels(self.h, cells.ctypes.data_as(_i32p), 64)
        return cells[:n].copy()

    def mg_level_maps(self, level):
        cells = self.mg_levels()
        nf = cells[level]
        S = len(self.mesh["cellFaceIDs"]) if level == 0 else None
        if S is None:
            # fine slot count of this level is the previous level's coarse slot count
            S = lib().orc_mg_level_maps(self.h, level - 1, None, None, None, None)
        c2c = np.zeros(nf, np.int32)
        f2c = np.zeros(S, np.int32)
        cfs = np.zeros(cells[level + 1] + 1, np.int32)
        Sc = lib().orc_mg_level_maps(self.h, level, None, None, None, None)
        cfn = np.zeros(max(Sc, 1), np.int32)
        lib().orc_mg_level_maps(self.h, level, c2c.ctypes.data_as(C.c_void_p), f2c.ctypes.data_as(C.c_void_p),
                                cfs.ctypes.data_as(C.c_void_p), cfn.ctypes.data_as(C.c_void_p))
        return c2c, f2c, cfs, cfn[:Sc]

    def coloring(self):
        out = np.zeros(self.mesh["nCells"], np.int32)
        nc = lib().orc_coloring(self.h, out.ctypes.data_as(_i32p))
        return out, nc

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
