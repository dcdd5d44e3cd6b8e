"""ctypes binding of libaxisim_b200.so (the C ABI declared in include/axisim_b200.h).

This is the Python mirror of the reference's Solver verbs (set mesh / bcs /
config, solve, continue, stop, read solutions). The compute path is the CUDA
library; there is no fallback: loading fails loudly when the library or a GPU
is missing.
"""
import ctypes as C
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libaxisim_b200.so")

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)

OK, E_ARG, E_CONFIG, E_MESH, E_CUDA, E_DIVERGED, E_STOPPED, E_STATE, E_TIMEOUT = range(9)
STATUS_NAMES = {0: "OK", 1: "E_ARG", 2: "E_CONFIG", 3: "E_MESH", 4: "E_CUDA", 5: "E_DIVERGED",
                6: "E_STOPPED", 7: "E_STATE", 8: "E_TIMEOUT"}
PREC_FP64, PREC_MIXED = 0, 1
VCYCLE_PER_PHASE, VCYCLE_RESIDENT = 0, 1
PSOLVE_VCYCLES, PSOLVE_FCG = 0, 1
LEARNED_OFF, LEARNED_FIRST_STEP, LEARNED_ALWAYS = 0, 1, 2
NET_FP32, NET_BF16, NET_BF16_WEIGHTS = 0, 1, 2

# Every entry point include/axisim_b200.h declares.
EXPORTS = [
    "axisim_abi_version", "axisim_create", "axisim_destroy", "axisim_last_error", "axisim_set_log",
    "axisim_set_mesh", "axisim_set_bc", "axisim_set_config", "axisim_set_fluid", "axisim_set_precision",
    "axisim_solve", "axisim_can_continue", "axisim_request_stop", "axisim_get_field", "axisim_set_field",
    "axisim_mg_levels", "axisim_mg_level_maps", "axisim_coloring", "axisim_multiblock_build",
    "axisim_mesh_sizes", "axisim_mesh_view", "axisim_mesh_free", "axisim_resolve_bc",
    "axisim_profile_iteration", "axisim_create_on", "axisim_set_batch", "axisim_batch_status",
    "axisim_set_pressure_solver", "axisim_residual_static", "axisim_pressure_stats",
    "axisim_learned_harvest", "axisim_learned_sample_count", "axisim_learned_add_sample",
    "axisim_learned_get_sample", "axisim_learned_init", "axisim_learned_params", "axisim_learned_grad",
    "axisim_learned_train", "axisim_learned_enable", "axisim_learned_stats", "axisim_learned_predict",
    "axisim_set_kinetics", "axisim_set_scalars", "axisim_scalar_residuals", "axisim_set_mesh_type",
    "axisim_trellis_build", "axisim_triangle_mesh_build", "axisim_classify_boundary_faces",
    "axisim_mg_levels_host", "axisim_mg_level_maps_host", "axisim_coloring_host",
    "axisim_set_autotune", "axisim_autotune_report", "axisim_setup_profile", "axisim_profile_levels",
    "axisim_mg_batch_levels_host", "axisim_set_vcycle_kernel", "axisim_test_barrier_timeout",
    "axisim_set_momentum_sweeps", "axisim_sweep_tiles", "axisim_sweep_tiles_host", "axisim_mesh_segments",
]
VAR_U, VAR_V, VAR_P, VAR_T, VAR_C = range(5)
VAR_INDEX = {"u": VAR_U, "v": VAR_V, "p": VAR_P, "T": VAR_T, "C": VAR_C}
MESH_STRUCTURED, MESH_UNSTRUCTURED = 0, 1


class MeshPacked(C.Structure):
    _fields_ = [("nCells", C.c_int32), ("nFaces", C.c_int32),
                ("faceOwner", _i32p), ("faceNeighbor", _i32p),
                ("faceNormalZ", _f64p), ("faceNormalR", _f64p),
                ("faceCenterZ", _f64p), ("faceCenterR", _f64p), ("faceArea", _f64p),
                ("faceBoundaryGroupID", _i32p),
                ("cellCenterZ", _f64p), ("cellCenterR", _f64p),
                ("cellArea2D", _f64p), ("cellVolume", _f64p),
                ("cellFaceStart", _i32p), ("cellFaceIDs", _i32p)]


class BCField(C.Structure):
    _fields_ = [("nGroups", C.c_int32), ("typeByGroup", _u8p), ("boundaryTypeByGroup", _u8p),
                ("valueByGroup", _f64p), ("lengthByGroup", _f64p), ("pulsatileByGroup", _u8p),
                ("amplitudeByGroup", _f64p), ("frequencyByGroup", _f64p)]


class Kinetics(C.Structure):
    _fields_ = [("nGroups", C.c_int32), ("vmaxByGroup", _f64p), ("kmByGroup", _f64p), ("nByGroup", _f64p),
                ("mByGroup", _f64p), ("k2ByGroup", _f64p), ("v2ByGroup", _f64p), ("RtotByGroup", _f64p)]


class OutlineC(C.Structure):
    _fields_ = [("nVertices", C.c_int32), ("vertexZ", _f64p), ("vertexR", _f64p), ("nEdges", C.c_int32),
                ("edgeV0", _i32p), ("edgeV1", _i32p), ("edgeGroup", _i32p)]


class ConfigSolver(C.Structure):
    _fields_ = [("velocitySolver", C.c_uint8), ("convectionScheme", C.c_uint8), ("gradientScheme", C.c_uint8),
                ("type", C.c_uint8), ("timeScheme", C.c_uint8), ("pad_", C.c_uint8 * 3),
                ("linearMaxIter", C.c_int32), ("useMultigrid", C.c_uint8), ("addConvectionTerm", C.c_uint8),
                ("transient", C.c_uint8), ("useNonOrthCorrector", C.c_uint8), ("dt", C.c_double),
                ("tEnd", C.c_double), ("saveKeyFrameIter", C.c_int32), ("pad2_", C.c_int32)]


class ConfigSimple(C.Structure):
    _fields_ = [("maxIter", C.c_int32), ("checkConv", C.c_int32), ("momTol", C.c_double), ("ppTol", C.c_double)]


class ConfigMultigrid(C.Structure):
    _fields_ = [("maxIter", C.c_int32), ("weight", C.c_double), ("linearSweep", C.c_int32),
                ("linearPreSweep", C.c_int32), ("linearPostSweep", C.c_int32)]


class ConfigResidual(C.Structure):
    _fields_ = [("type", C.c_uint8), ("normType", C.c_uint8), ("scaleType", C.c_uint8), ("enabled", C.c_uint8),
                ("tol", C.c_double)]


class Fluid(C.Structure):
    _fields_ = [("rho", C.c_double), ("mu", C.c_double), ("cp", C.c_double), ("k", C.c_double), ("D", C.c_double)]


class Result(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("totalIterations", C.c_int32), ("converged", C.c_int32),
                ("timeSteps", C.c_int32), ("residual", C.c_double * 3), ("solveMs", C.c_double)]


class BlockSpec(C.Structure):
    _fields_ = [("z0", C.c_double), ("r0", C.c_double),
                ("axialLength", C.c_double), ("axialCells", C.c_int32), ("axialGrading", C.c_int32),
                ("axialCoef", C.c_double),
                ("radialLength", C.c_double), ("radialCells", C.c_int32), ("radialGrading", C.c_int32),
                ("radialCoef", C.c_double), ("edgeGroup", C.c_int32 * 4)]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int32), ("ms", C.c_double), ("bytes", C.c_double)]


RESIDUAL_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int32, _f64p)
LOG_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_char_p)


def build(force=False):
    """Compile the library in-tree (nvcc for sm_100a); returns its path."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", PKG_DIR], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = {
            "axisim_abi_version": (C.c_int, []),
            "axisim_create": (C.c_int, [C.POINTER(Fluid), C.POINTER(vp)]),
            "axisim_create_on": (C.c_int, [C.c_int32, C.POINTER(Fluid), C.POINTER(vp)]),
            "axisim_destroy": (C.c_int, [vp]),
            "axisim_last_error": (C.c_char_p, [vp]),
            "axisim_set_log": (C.c_int, [vp, LOG_FN, RESIDUAL_FN, vp]),
            "axisim_set_mesh": (C.c_int, [vp, C.POINTER(MeshPacked)]),
            "axisim_set_bc": (C.c_int, [vp, C.c_int32, C.POINTER(BCField)]),
            "axisim_set_config": (C.c_int, [vp, C.POINTER(ConfigSolver), C.POINTER(ConfigSimple),
                                            C.POINTER(ConfigMultigrid), C.POINTER(ConfigResidual),
                                            C.c_double, C.c_double]),
            "axisim_set_fluid": (C.c_int, [vp, C.POINTER(Fluid)]),
            "axisim_set_kinetics": (C.c_int, [vp, C.c_int32, C.POINTER(Kinetics)]),
            "axisim_set_scalars": (C.c_int, [vp, C.c_int32, C.c_int32, C.POINTER(ConfigResidual)]),
            "axisim_scalar_residuals": (C.c_int, [vp, _f64p]),
            "axisim_set_mesh_type": (C.c_int, [vp, C.c_int32]),
            "axisim_set_precision": (C.c_int, [vp, C.c_int32]),
            "axisim_set_pressure_solver": (C.c_int, [vp, C.c_int32, C.c_double, C.c_double]),
            "axisim_set_autotune": (C.c_int, [vp, C.c_int32]),
            "axisim_set_vcycle_kernel": (C.c_int, [vp, C.c_int32]),
            "axisim_set_momentum_sweeps": (C.c_int, [vp, C.c_int32, C.c_int32]),
            "axisim_sweep_tiles": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "axisim_sweep_tiles_host": (C.c_int64, [C.POINTER(MeshPacked), C.c_int32, C.c_int32, C.c_int32,
                                                    C.POINTER(C.c_int32), _i32p, _i32p, _i32p,
                                                    C.POINTER(C.c_uint64), C.c_int64]),
            "axisim_test_barrier_timeout": (C.c_int, [vp, C.c_int32]),
            "axisim_autotune_report": (C.c_int, [vp, _i32p, _f64p, C.c_int32]),
            "axisim_pressure_stats": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
            "axisim_learned_harvest": (C.c_int, [vp, C.c_int32, C.c_int32]),
            "axisim_learned_sample_count": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "axisim_learned_add_sample": (C.c_int, [vp, vp, vp, vp, vp, vp]),
            "axisim_learned_get_sample": (C.c_int, [vp, C.c_int32, vp, vp, vp, vp, vp, vp]),
            "axisim_learned_init": (C.c_int, [vp, C.c_int32, C.c_uint64, C.POINTER(C.c_int64)]),
            "axisim_learned_params": (C.c_int, [vp, vp, C.c_int64, C.c_int32]),
            "axisim_learned_grad": (C.c_int, [vp, C.c_int32, vp, vp, C.c_int64]),
            "axisim_learned_train": (C.c_int, [vp, C.c_int32, C.c_float, C.c_uint64, C.c_int32, C.c_int32, vp]),
            "axisim_learned_enable": (C.c_int, [vp, C.c_int32]),
            "axisim_learned_predict": (C.c_int, [vp, vp, vp, vp, vp]),
            "axisim_learned_stats": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                               C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            # device pointers as integers (e.g. torch data_ptr()), stream as cudaStream_t
            "axisim_residual_static": (C.c_int, [C.c_int32] * 3 + [vp] * 12 + [C.c_int32] * 2 + [vp] * 5 +
                                       [C.c_char_p, C.c_size_t]),
            "axisim_solve": (C.c_int, [vp, C.c_int32, C.POINTER(Result)]),
            "axisim_can_continue": (C.c_int, [vp, C.c_char_p, C.c_size_t]),
            "axisim_request_stop": (C.c_int, [vp]),
            "axisim_get_field": (C.c_int64, [vp, C.c_char_p, _f64p, C.c_size_t]),
            "axisim_set_field": (C.c_int64, [vp, C.c_char_p, _f64p, C.c_size_t]),
            "axisim_mg_levels": (C.c_int, [vp, _i32p, C.c_int32]),
            "axisim_mg_level_maps": (C.c_int64, [vp, C.c_int32, vp, vp, vp, vp]),
            "axisim_coloring": (C.c_int, [vp, _i32p, C.c_size_t]),
            "axisim_multiblock_build": (C.c_int, [C.c_int32, C.POINTER(BlockSpec), C.c_double, C.c_int32,
                                                  C.POINTER(vp), _i32p]),
            "axisim_mesh_sizes": (C.c_int, [vp, _i32p, _i32p, _i32p]),
            "axisim_mesh_view": (C.c_int, [vp, C.POINTER(MeshPacked)]),
            "axisim_mesh_free": (C.c_int, [vp]),
            "axisim_resolve_bc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, _u8p,
                                            _f64p, _u8p]),
            "axisim_trellis_build": (C.c_int, [C.c_int32, _f64p, C.c_int32, _f64p, _i32p, _i32p,
                                               C.POINTER(OutlineC), C.c_double, C.c_double, C.c_int32, C.c_int32,
                                               C.POINTER(vp), _i32p]),
            "axisim_triangle_mesh_build": (C.c_int, [C.c_int32, _f64p, _f64p, C.c_int32, _i32p,
                                                     C.POINTER(OutlineC), C.c_double, C.c_double, C.POINTER(vp)]),
            "axisim_classify_boundary_faces": (C.c_int, [C.c_int32, _i32p, _f64p, _f64p, C.POINTER(OutlineC),
                                                         C.c_double, C.c_double, _i32p]),
            "axisim_mg_levels_host": (C.c_int, [C.POINTER(MeshPacked), _i32p, C.c_int32]),
            "axisim_mg_batch_levels_host": (C.c_int, [C.POINTER(MeshPacked), C.c_int32, _i32p, _i32p, _i32p,
                                                      C.c_int32]),
            "axisim_mg_level_maps_host": (C.c_int64, [C.POINTER(MeshPacked), C.c_int32, vp, vp, vp, vp]),
            "axisim_coloring_host": (C.c_int, [C.POINTER(MeshPacked), _i32p, C.c_size_t]),
            "axisim_profile_iteration": (C.c_int, [vp, C.c_int32, C.POINTER(KernelStat), C.c_int32, _i32p]),
            "axisim_setup_profile": (C.c_int, [vp, C.POINTER(KernelStat), C.c_int32, _i32p, C.c_int32]),
            "axisim_mesh_segments": (C.c_int, [vp, _i32p, _i32p, _i32p, _i32p]),
            "axisim_profile_levels": (C.c_int, [vp, C.c_int32, C.POINTER(KernelStat), C.c_int32, _i32p]),
            "axisim_set_batch": (C.c_int, [vp, C.c_int32, _i32p]),
            "axisim_batch_status": (C.c_int, [vp, _i32p, _f64p, C.c_int32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class AxisimError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


# ---------------------------------------------------------------- host prep
MESH_KEYS = ["faceOwner", "faceNeighbor", "faceNormalZ", "faceNormalR", "faceCenterZ", "faceCenterR",
             "faceArea", "faceBoundaryGroupID", "cellCenterZ", "cellCenterR", "cellArea2D", "cellVolume",
             "cellFaceStart", "cellFaceIDs"]


def multiblock(blocks, tol=1e-9, default_group=-1):
    """Pack a multiblock mesh with the library's C++ packer (structs/multiblock.h
    semantics). Returns a dict of numpy arrays (FVMeshHostPacked layout)."""
    L = lib()
    arr = (BlockSpec * len(blocks))()
    for i, b in enumerate(blocks):
        ax, rd = b["axial"], b["radial"]
        arr[i] = BlockSpec(b["z0"], b["r0"], ax[0], ax[1], ax[2], ax[3], rd[0], rd[1], rd[2], rd[3],
                           (C.c_int32 * 4)(*b["edge_group"]))
    h = C.c_void_p()
    seam = C.c_int32(0)
    st = L.axisim_multiblock_build(len(blocks), arr, tol, default_group, C.byref(h), C.byref(seam))
    if st != OK:
        raise AxisimError(st, "multiblock build failed")
    return _take_mesh(h, seam.value, MESH_STRUCTURED)


def _take_mesh(h, status, mesh_type):
    """Copies a library-built mesh into numpy arrays and frees it."""
    L = lib()
    v = MeshPacked()
    L.axisim_mesh_view(h, C.byref(v))
    n, f = v.nCells, v.nFaces
    r = v.cellFaceStart[n]
    m = {"nCells": n, "nFaces": f, "status": status, "meshType": mesh_type}
    sizes = dict(faceOwner=f, faceNeighbor=f, faceNormalZ=f, faceNormalR=f, faceCenterZ=f, faceCenterR=f,
                 faceArea=f, faceBoundaryGroupID=f, cellCenterZ=n, cellCenterR=n, cellArea2D=n, cellVolume=n,
                 cellFaceStart=n + 1, cellFaceIDs=r)
    for k in MESH_KEYS:
        ptr = getattr(v, k)
        m[k] = np.ctypeslib.as_array(ptr, shape=(sizes[k],)).copy()
    L.axisim_mesh_free(h)
    return m


def outline_struct(vertices, edges, groups):
    """vertices (V, 2) as (z, r); edges (E, 2) vertex ids; groups (E,) boundary
    group per edge (-1 = none). Returns (struct, arrays kept alive)."""
    v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 2)
    e = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 2)
    keep = [np.ascontiguousarray(v[:, 0]), np.ascontiguousarray(v[:, 1]), np.ascontiguousarray(e[:, 0]),
            np.ascontiguousarray(e[:, 1]), np.ascontiguousarray(groups, dtype=np.int32)]
    s = OutlineC(len(v), keep[0].ctypes.data_as(_f64p), keep[1].ctypes.data_as(_f64p), len(e),
                 keep[2].ctypes.data_as(_i32p), keep[3].ctypes.data_as(_i32p), keep[4].ctypes.data_as(_i32p))
    return s, keep


def trellis(z_lines, r_lines, z_cells, r_cells, outline, L, R, nz=1, nr=1):
    """Mesh::buildStructuredMultiBlock through the library: a uniform block per
    trellis cell inside `outline` ((vertices, edges, groups)), external faces
    classified by the nearest outline edge. Returns the packed-mesh dict."""
    z = np.ascontiguousarray(z_lines, dtype=np.float64)
    r = np.ascontiguousarray(r_lines, dtype=np.float64)
    zc = np.ascontiguousarray(z_cells, dtype=np.int32)
    rc = np.ascontiguousarray(r_cells, dtype=np.int32)
    o, keep = outline_struct(*outline)
    h = C.c_void_p()
    seam = C.c_int32(0)
    st = lib().axisim_trellis_build(len(z), z.ctypes.data_as(_f64p), len(r), r.ctypes.data_as(_f64p),
                                    zc.ctypes.data_as(_i32p), rc.ctypes.data_as(_i32p), C.byref(o), L, R, nz, nr,
                                    C.byref(h), C.byref(seam))
    if st != OK:
        raise AxisimError(st, "trellis build failed")
    return _take_mesh(h, seam.value, MESH_STRUCTURED)


def triangle_mesh(points, tris, outline, L, R):
    """Mesh::createUnstructuredMesh through the library, external faces
    classified by the nearest edge of `outline`."""
    p = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    pz, pr = np.ascontiguousarray(p[:, 0]), np.ascontiguousarray(p[:, 1])
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
    o, keep = outline_struct(*outline)
    h = C.c_void_p()
    st = lib().axisim_triangle_mesh_build(len(p), pz.ctypes.data_as(_f64p), pr.ctypes.data_as(_f64p), len(t),
                                          t.ctypes.data_as(_i32p), C.byref(o), L, R, C.byref(h))
    if st != OK:
        raise AxisimError(st, "triangle mesh build failed")
    return _take_mesh(h, 0, MESH_UNSTRUCTURED)


def classify_boundary_faces(mesh, outline, L, R):
    """Mesh::classifyBoundaryFaces on a packed-mesh dict (in place)."""
    o, keep = outline_struct(*outline)
    nb = np.ascontiguousarray(mesh["faceNeighbor"], dtype=np.int32)
    fz = np.ascontiguousarray(mesh["faceCenterZ"], dtype=np.float64)
    fr = np.ascontiguousarray(mesh["faceCenterR"], dtype=np.float64)
    g = np.ascontiguousarray(mesh["faceBoundaryGroupID"], dtype=np.int32).copy()
    st = lib().axisim_classify_boundary_faces(len(nb), nb.ctypes.data_as(_i32p), fz.ctypes.data_as(_f64p),
                                              fr.ctypes.data_as(_f64p), C.byref(o), L, R, g.ctypes.data_as(_i32p))
    if st != OK:
        raise AxisimError(st, "classification failed")
    mesh["faceBoundaryGroupID"] = g
    return mesh


def resolve_bc(boundary_type, variable, user=None):
    """BoundaryDefaults::getEffectiveBC through the library: returns (type, value, pulsatile)."""
    t = C.c_uint8()
    v = C.c_double()
    p = C.c_uint8()
    has = 0 if user is None else 1
    ut, uv = (0, 0.0) if user is None else (user[0], user[1])
    st = lib().axisim_resolve_bc(boundary_type, variable, has, ut, uv, C.byref(t), C.byref(v), C.byref(p))
    if st != OK:
        raise AxisimError(st, "resolve_bc failed")
    return t.value, v.value, p.value


def mg_levels_host(mesh):
    """Cells per multigrid level of `mesh`, built on the host without a device
    (the hierarchy a handle holding this mesh reports)."""
    s, keep = mesh_struct(mesh)
    cells = np.zeros(64, np.int32)
    n = lib().axisim_mg_levels_host(C.byref(s), cells.ctypes.data_as(_i32p), 64)
    if n < 0:
        raise AxisimError(-n, "mg_levels_host failed")
    return cells[:n].copy()


def mg_batch_levels_host(mesh, case_cell_start):
    """(cells per level, terminal cells per level) of the per-case hierarchy a batch solve builds."""
    s, keep = mesh_struct(mesh)
    cs = np.ascontiguousarray(case_cell_start, dtype=np.int32)
    cells = np.zeros(64, np.int32)
    term = np.zeros(64, np.int32)
    n = lib().axisim_mg_batch_levels_host(C.byref(s), len(cs) - 1, cs.ctypes.data_as(_i32p),
                                          cells.ctypes.data_as(_i32p), term.ctypes.data_as(_i32p), 64)
    if n < 0:
        raise AxisimError(-n, "mg_batch_levels_host failed")
    return cells[:n].copy(), term[:n].copy()


def sweep_tiles_host(mesh, S, cap, tile_cells):
    """The momentum sweep tiles (axisim_sweep_tiles_host): dict of tileStart,
    layerEnd (n_tiles x (S + 1)), gid and lnb (n_local x 4 local neighbours,
    -1 for none); n_tiles = 0 when no tiling fits."""
    s, keep = mesh_struct(mesh)
    f = lib().axisim_sweep_tiles_host
    nt = C.c_int32()
    total = int(f(C.byref(s), S, cap, tile_cells, C.byref(nt), None, None, None, None, 0))
    if total < 0:
        raise AxisimError(-total, "sweep_tiles_host failed")
    n = nt.value
    ts = np.zeros(n + 1, np.int32)
    le = np.zeros(max(n, 1) * (S + 1), np.int32)
    gid = np.zeros(max(total, 1), np.int32)
    lnb = np.zeros(max(total, 1), np.uint64)
    got = int(f(C.byref(s), S, cap, tile_cells, C.byref(nt), ts.ctypes.data_as(_i32p), le.ctypes.data_as(_i32p),
                gid.ctypes.data_as(_i32p), lnb.ctypes.data_as(C.POINTER(C.c_uint64)), total))
    if got != total:
        raise AxisimError(E_MESH, "sweep_tiles_host changed between calls")
    words = lnb[:total].view(np.uint16).reshape(total, 4).astype(np.int32)
    words[words == 0xFFFF] = -1
    return {"n_tiles": n, "tileStart": ts, "layerEnd": le[:n * (S + 1)].reshape(n, S + 1), "gid": gid[:total],
            "lnb": words}


def mg_level_maps_host(mesh, level):
    """(cellToCoarse, fineSlotToCoarseSlot, coarseFaceStart, coarseFaceNeighbor)
    of `level`, built on the host without a device."""
    s, keep = mesh_struct(mesh)
    cells = mg_levels_host(mesh)
    if not 0 <= level < len(cells) - 1:
        raise AxisimError(E_ARG, "level out of range")
    f = lib().axisim_mg_level_maps_host
    S = len(mesh["cellFaceIDs"]) if level == 0 else int(f(C.byref(s), level - 1, None, None, None, None))
    Sc = int(f(C.byref(s), level, None, None, None, None))
    if S < 0 or Sc < 0:
        raise AxisimError(-min(S, Sc), "mg_level_maps_host failed")
    out = (np.zeros(cells[level], np.int32), np.zeros(S, np.int32), np.zeros(cells[level + 1] + 1, np.int32),
           np.zeros(max(Sc, 1), np.int32))
    r = f(C.byref(s), level, *(a.ctypes.data_as(C.c_void_p) for a in out))
    if r < 0:
        raise AxisimError(-r, "mg_level_maps_host failed")
    return out[0], out[1], out[2], out[3][:Sc]


def coloring_host(mesh):
    """(colour per cell, number of colours) of `mesh`, on the host."""
    s, keep = mesh_struct(mesh)
    out = np.zeros(mesh["nCells"], np.int32)
    nc = lib().axisim_coloring_host(C.byref(s), out.ctypes.data_as(_i32p), out.size)
    if nc < 0:
        raise AxisimError(-nc, "coloring_host failed")
    return out, nc


def mesh_struct(m):
    keep = []

    def P(k, t, dt):
        a = np.ascontiguousarray(m[k], dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(t)
    s = MeshPacked(m["nCells"], m["nFaces"], P("faceOwner", _i32p, np.int32), P("faceNeighbor", _i32p, np.int32),
                   P("faceNormalZ", _f64p, np.float64), P("faceNormalR", _f64p, np.float64),
                   P("faceCenterZ", _f64p, np.float64), P("faceCenterR", _f64p, np.float64),
                   P("faceArea", _f64p, np.float64), P("faceBoundaryGroupID", _i32p, np.int32),
                   P("cellCenterZ", _f64p, np.float64), P("cellCenterR", _f64p, np.float64),
                   P("cellArea2D", _f64p, np.float64), P("cellVolume", _f64p, np.float64),
                   P("cellFaceStart", _i32p, np.int32), P("cellFaceIDs", _i32p, np.int32))
    return s, keep


def bc_struct(bc):
    keep = []

    def P(k, t, dt):
        if k not in bc or bc[k] is None:
            return None
        a = np.ascontiguousarray(bc[k], dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(t)
    s = BCField(len(bc["type"]), P("type", _u8p, np.uint8), P("btype", _u8p, np.uint8),
                P("value", _f64p, np.float64), P("length", _f64p, np.float64), P("puls", _u8p, np.uint8),
                P("amp", _f64p, np.float64), P("freq", _f64p, np.float64))
    return s, keep


KINETICS_KEYS = ("vmax", "km", "n", "m", "k2", "v2", "Rtot")


def kinetics_struct(bc):
    """The wall-kinetics arrays of a scalar's boundary field (None when it has none)."""
    if not any(k in bc for k in KINETICS_KEYS):
        return None, []
    keep = []

    def P(k):
        if k not in bc or bc[k] is None:
            return None
        a = np.ascontiguousarray(bc[k], dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(_f64p)
    return Kinetics(len(bc["type"]), *[P(k) for k in KINETICS_KEYS]), keep


def settings_structs(s):
    cs = ConfigSolver()
    cs.velocitySolver = 0
    cs.convectionScheme = s["convectionScheme"]
    cs.gradientScheme = s["gradientScheme"]
    cs.type = s["linearType"]
    cs.timeScheme = s["timeScheme"]
    cs.linearMaxIter = s["linearMaxIter"]
    cs.useMultigrid = s["useMultigrid"]
    cs.addConvectionTerm = s["addConvectionTerm"]
    cs.transient = s["transient"]
    cs.useNonOrthCorrector = s["useNonOrthCorrector"]
    cs.dt = s["dt"]
    cs.tEnd = s["tEnd"]
    cs.saveKeyFrameIter = 2
    sim = ConfigSimple(s["maxIter"], s["checkConv"], 1e-8, 1e-5)
    mg = ConfigMultigrid(s["mgMaxIter"], s["mgWeight"], s["mgLinearSweep"], s["mgPreSweep"], s["mgPostSweep"])
    res = (ConfigResidual * 3)()
    for i in range(3):
        res[i] = ConfigResidual(0, s["resNorm"][i], s["resScale"][i], s["resEnabled"][i], s["resTol"][i])
    fluid = Fluid(s["rho"], s["mu"], s.get("cp", 4180.0), s.get("k", 0.6), s.get("D", 3.0277e-9))
    return cs, sim, mg, res, fluid


def scalar_residual_structs(s):
    """The Temperature / Concentration ConfigResidual entries of a settings dict."""
    res = (ConfigResidual * 2)()
    norm = s.get("scalarResNorm", [0, 0])
    scale = s.get("scalarResScale", [3, 3])
    en = s.get("scalarResEnabled", [0, 0])
    tol = s.get("scalarResTol", [1e-3, 1e-3])
    for i in range(2):
        res[i] = ConfigResidual(0, norm[i], scale[i], en[i], tol[i])
    return res


class Solver:
    """One solver handle (Solver in the reference): case in, fields out."""

    def __init__(self, mesh, bcs, settings, precision=PREC_FP64, device=0, pressure_solver=PSOLVE_VCYCLES,
                 pressure_tol=0.0, prolong_scale=1.0, autotune=False):
        L = lib()
        cs, sim, mg, res, fluid = settings_structs(settings)
        self.h = C.c_void_p()
        st = L.axisim_create_on(device, C.byref(fluid), C.byref(self.h))
        if st != OK:
            raise AxisimError(st, "axisim_create failed (no CUDA device?)")
        self.mesh = mesh
        self.settings = dict(settings)
        self._residual_log = []
        ms, keep = mesh_struct(mesh)
        self._check(L.axisim_set_mesh(self.h, C.byref(ms)))
        # Mesh::currentMeshType (a packed mesh without the key counts as unstructured)
        self._check(L.axisim_set_mesh_type(self.h, int(mesh.get("meshType", MESH_UNSTRUCTURED))))
        for key in ("u", "v", "p", "T", "C"):
            if key not in bcs:
                continue
            b, keep2 = bc_struct(bcs[key])
            self._check(L.axisim_set_bc(self.h, VAR_INDEX[key], C.byref(b)))
            kin, keep3 = kinetics_struct(bcs[key])
            if kin is not None:
                self._check(L.axisim_set_kinetics(self.h, VAR_INDEX[key], C.byref(kin)))
        self._check(L.axisim_set_config(self.h, C.byref(cs), C.byref(sim), C.byref(mg), res,
                                        settings["alphaU"], settings["alphaP"]))
        if settings.get("solveEnergy") or settings.get("solveConcentration"):
            self._check(L.axisim_set_scalars(self.h, int(bool(settings.get("solveEnergy"))),
                                             int(bool(settings.get("solveConcentration"))),
                                             scalar_residual_structs(settings)))
        if precision != PREC_FP64:
            self._check(L.axisim_set_precision(self.h, precision))
        if pressure_solver != PSOLVE_VCYCLES:
            self._check(L.axisim_set_pressure_solver(self.h, pressure_solver, pressure_tol, prolong_scale))
        if autotune:
            self._check(L.axisim_set_autotune(self.h, 1))

    def _check(self, st):
        if st != OK:
            raise AxisimError(st, lib().axisim_last_error(self.h).decode())
        return st

    def solve(self, cont=False, allow=(OK,)):
        r = Result()
        st = lib().axisim_solve(self.h, 1 if cont else 0, C.byref(r))
        if st not in allow:
            self._check(st)
        return dict(status=st, iterations=r.iterations, total=r.totalIterations, converged=bool(r.converged),
                    steps=r.timeSteps, residual=list(r.residual), ms=r.solveMs)

    def scalar_residuals(self):
        """Temperature and Concentration residuals of the last check."""
        out = np.zeros(2)
        self._check(lib().axisim_scalar_residuals(self.h, out.ctypes.data_as(_f64p)))
        return out

    FACE_FIELDS = frozenset(("mDot", "invDPN", "wP", "dPB", "length2D", "lsqWZ", "lsqWR", "cw", "ocrWall"))

    def get(self, name, out=None):
        """Field `name` copied into `out` (a float64 array of the field's size,
        e.g. in pinned memory) or into a new array."""
        if name.startswith("AF_"):
            n = len(self.mesh["cellFaceIDs"])
        elif name in self.FACE_FIELDS:
            n = self.mesh["nFaces"]
        else:
            n = self.mesh["nCells"]
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size < n or not out.flags.c_contiguous:
            raise AxisimError(E_ARG, "out must be a contiguous float64 array of the field's size")
        k = lib().axisim_get_field(self.h, name.encode(), out.ctypes.data_as(_f64p), n)
        if k < 0:
            self._check(int(-k))
        return out if k == n else out[:k].copy()

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        k = lib().axisim_set_field(self.h, name.encode(), a.ctypes.data_as(_f64p), a.size)
        if k < 0:
            self._check(int(-k))

    def set_max_iter(self, max_iter, tol=None):
        """Change ConfigSimple.maxIter (and optionally every residual tolerance)
        without touching the settings baked into the captured iteration."""
        self.settings["maxIter"] = int(max_iter)
        if tol is not None:
            self.settings["resTol"] = [tol, tol, tol]
        cs, sim, mg, res, fluid = settings_structs(self.settings)
        self._check(lib().axisim_set_config(self.h, C.byref(cs), C.byref(sim), C.byref(mg), res,
                                            self.settings["alphaU"], self.settings["alphaP"]))

    def profile(self, iterations=1, by_level=False):
        """Per-kernel launches / CUDA-event ms / algorithmic bytes over `iterations`
        eagerly replayed SIMPLE iterations (advances the solution). by_level:
        multigrid launches are named "<kernel>@<level>"."""
        out = (KernelStat * 256)()
        n = C.c_int32(0)
        fn = lib().axisim_profile_levels if by_level else lib().axisim_profile_iteration
        self._check(fn(self.h, iterations, out, 256, C.byref(n)))
        return [dict(name=out[i].name.decode(), launches=out[i].launches, ms=out[i].ms, bytes=out[i].bytes)
                for i in range(min(n.value, 256))]

    def setup_profile(self, reset=False):
        """Host-clock ms and call count of each set-up stage since creation (or the last reset)."""
        out = (KernelStat * 64)()
        n = C.c_int32(0)
        self._check(lib().axisim_setup_profile(self.h, out, 64, C.byref(n), 1 if reset else 0))
        return {out[i].name.decode(): dict(calls=out[i].launches, ms=out[i].ms) for i in range(min(n.value, 64))}

    def set_batch(self, case_cell_start):
        cs = np.ascontiguousarray(case_cell_start, dtype=np.int32)
        self._check(lib().axisim_set_batch(self.h, len(cs) - 1, cs.ctypes.data_as(_i32p)))
        self.n_cases = len(cs) - 1

    def batch_status(self):
        n = self.n_cases
        conv = np.zeros(n, np.int32)
        res = np.zeros((n, 3))
        k = lib().axisim_batch_status(self.h, conv.ctypes.data_as(_i32p), res.ctypes.data_as(_f64p), n)
        if k < 0:
            self._check(-k)
        return conv, res

    def save_solution_npy(self, directory, quads=True, triangles=None, **kw):
        """The reference's NumPy export (solution.npy, points.npy, cells.npy,
        meta.json; see axisim.export) of this handle's current fields. quads:
        derive the corner polygons of an axis-aligned structured mesh;
        triangles: (points, tris) of an unstructured one."""
        from . import export
        s = self.settings
        fluid = {"rho": s["rho"], "mu": s["mu"], "cp": s.get("cp", 4180.0), "k": s.get("k", 0.6),
                 "D": s.get("D", 3.0277e-9)}
        sols = export.solutions_from(self.get, self.mesh, fluid, energy=bool(s.get("solveEnergy")),
                                     concentration=bool(s.get("solveConcentration")))
        kw.setdefault("transient", bool(s.get("transient", 0)))
        kw.setdefault("dt", s.get("dt", 0.0))
        q = export.quad_corners(self.mesh) if quads and triangles is None else None
        return export.save_solution_npy(directory, self.mesh, sols, fluid, quads=q, triangles=triangles, **kw)

    # ---- learned p' preconditioner ----
    def learned_harvest(self, every, capacity=0):
        self._check(lib().axisim_learned_harvest(self.h, every, capacity))

    def learned_sample_count(self):
        c = C.c_int32()
        self._check(lib().axisim_learned_sample_count(self.h, C.byref(c)))
        return c.value

    def learned_add_sample(self, b, target, ac, deficit, af):
        """af: off-diagonals in the mesh's slot order (len(cellFaceIDs))."""
        arrs = [np.ascontiguousarray(a, np.float32) for a in (b, target, ac, deficit, af)]
        self._check(lib().axisim_learned_add_sample(self.h, *[a.ctypes.data for a in arrs]))

    def learned_get_sample(self, i):
        """(b, target, A_C, deficit, A_F in slot order, relative residual of the
        solve that made it)."""
        n = self.mesh["nCells"]
        out = [np.zeros(n, np.float32) for _ in range(4)] + [np.zeros(len(self.mesh["cellFaceIDs"]), np.float32)]
        rr = np.zeros(1, np.float32)
        self._check(lib().axisim_learned_get_sample(self.h, i, *[a.ctypes.data for a in out], rr.ctypes.data))
        return out + [float(rr[0])]

    def learned_init(self, precision=NET_BF16_WEIGHTS, seed=0):
        n = C.c_int64()
        self._check(lib().axisim_learned_init(self.h, precision, seed, C.byref(n)))
        self._n_params = n.value
        return n.value

    def learned_params(self):
        p = np.zeros(self._n_params, np.float32)
        self._check(lib().axisim_learned_params(self.h, p.ctypes.data, p.size, 0))
        return p

    def learned_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(lib().axisim_learned_params(self.h, p.ctypes.data, p.size, 1))

    def learned_grad(self, i):
        loss = np.zeros(1, np.float32)
        g = np.zeros(self._n_params, np.float32)
        self._check(lib().axisim_learned_grad(self.h, i, loss.ctypes.data, g.ctypes.data, g.size))
        return float(loss[0]), g

    def learned_train(self, steps, lr=1e-3, seed=0, first=0, count=0):
        out = np.zeros(steps, np.float32)
        self._check(lib().axisim_learned_train(self.h, steps, lr, seed, first, count, out.ctypes.data))
        return out

    def learned_predict(self, r, ac, deficit):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (r, ac, deficit)]
        out = np.zeros(self.mesh["nCells"], np.float32)
        self._check(lib().axisim_learned_predict(self.h, *[a.ctypes.data for a in arrs], out.ctypes.data))
        return out

    def learned_enable(self, mode=LEARNED_FIRST_STEP):
        self._check(lib().axisim_learned_enable(self.h, mode))

    def learned_stats(self):
        """Solves with the network, fallbacks to the V-cycle, and the running
        scores (mean log residual reduction per Krylov iteration) of both."""
        a, f, sn, sv = C.c_int64(), C.c_int64(), C.c_double(), C.c_double()
        self._check(lib().axisim_learned_stats(self.h, C.byref(a), C.byref(f), C.byref(sn), C.byref(sv)))
        return dict(applied=a.value, fallbacks=f.value, score_net=sn.value, score_vcycle=sv.value)

    def set_momentum_sweeps(self, sweeps_per_launch, threads=0):
        """Momentum Jacobi sweeps per launch (default 1 = one launch per sweep; above 1 run
        on shared-memory tiles) and the CTA size of the tiled launches (0 = 1024)."""
        self._check(lib().axisim_set_momentum_sweeps(self.h, sweeps_per_launch, threads))

    def sweep_tiles(self):
        """Tiles the momentum sweeps of the last captured solve ran on (0: one launch per sweep)."""
        n = C.c_int32()
        self._check(lib().axisim_sweep_tiles(self.h, C.byref(n)))
        return n.value

    def set_vcycle_kernel(self, mode):
        """VCYCLE_PER_PHASE (default): one launch per phase; VCYCLE_RESIDENT: the coarser
        levels' V-cycle in one cooperative kernel."""
        self._check(lib().axisim_set_vcycle_kernel(self.h, mode))

    def set_autotune(self, on=True):
        """Tune the multigrid levels' launch shapes before the next solve captures its graph."""
        self._check(lib().axisim_set_autotune(self.h, 1 if on else 0))

    def autotune_report(self):
        """(block size per level, sweep microseconds per level and candidate 64/128/256)."""
        blocks = np.zeros(64, np.int32)
        us = np.zeros(64 * 3)
        n = lib().axisim_autotune_report(self.h, blocks.ctypes.data_as(_i32p), us.ctypes.data_as(_f64p), 64)
        if n < 0:
            self._check(-n)
        return blocks[:n].copy(), us[:3 * n].reshape(n, 3).copy()

    def pressure_stats(self):
        """(Krylov p' solves started, Krylov iterations completed)."""
        a, b = C.c_int64(), C.c_int64()
        self._check(lib().axisim_pressure_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def can_continue(self):
        buf = C.create_string_buffer(256)
        r = lib().axisim_can_continue(self.h, buf, 256)
        return r == 1, buf.value.decode()

    def request_stop(self):
        return lib().axisim_request_stop(self.h)

    def mesh_segments(self):
        """The mesh's 32-cell segments as set_mesh classified them: dict of
        segments, offset_segments (slot neighbours at fixed offsets),
        face_segments (also affine faces) and in_use (the tables are used)."""
        v = [C.c_int32(0) for _ in range(4)]
        self._check(lib().axisim_mesh_segments(self.h, *(C.byref(x) for x in v)))
        return dict(segments=v[0].value, offset_segments=v[1].value, face_segments=v[2].value,
                    in_use=bool(v[3].value))

    def mg_levels(self):
        cells = np.zeros(64, np.int32)
        n = lib().axisim_mg_levels(self.h, cells.ctypes.data_as(_i32p), 64)
        if n < 0:
            self._check(-n)
        return cells[:n].copy()

    def mg_level_maps(self, level):
        cells = self.mg_levels()
        S = int(lib().axisim_mg_level_maps(self.h, level - 1, None, None, None, None)) if level > 0 \
            else len(self.mesh["cellFaceIDs"])
        Sc = int(lib().axisim_mg_level_maps(self.h, level, None, None, None, None))
        c2c = np.zeros(cells[level], np.int32)
        f2c = np.zeros(S, np.int32)
        cfs = np.zeros(cells[level + 1] + 1, np.int32)
        cfn = np.zeros(max(Sc, 1), np.int32)
        lib().axisim_mg_level_maps(self.h, level, c2c.ctypes.data_as(C.c_void_p), f2c.ctypes.data_as(C.c_void_p),
                                   cfs.ctypes.data_as(C.c_void_p), cfn.ctypes.data_as(C.c_void_p))
        return c2c, f2c, cfs, cfn[:Sc]

    def coloring(self):
        out = np.zeros(self.mesh["nCells"], np.int32)
        nc = lib().axisim_coloring(self.h, out.ctypes.data_as(_i32p), out.size)
        if nc < 0:
            self._check(-nc)
        return out, nc

    def close(self):
        if self.h:
            lib().axisim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
