"""Shared test helpers: build one case for both the CUDA path and the oracle."""
import numpy as np

from axisim import cases
import axisim.abi as abi
import oracle

# intermediate state compared bit for bit between the FP64 CUDA path and the oracle
FIELDS = ["u", "v", "p", "pp", "mDot", "DU", "DV", "gradPZ", "gradPR", "gradUZ", "gradUR", "gradVZ", "gradVR",
          "AC_u", "b_u", "AF_u", "invAC_u", "AC_v", "b_v", "AF_v", "invAC_v", "AC_pp", "b_pp", "AF_pp",
          "invAC_pp", "res_U", "res_V", "res_Continuity"]
# the geometry precompute (memory_manger.cpp:512-617)
GEOM = ["invDPN", "wP", "dPB", "length2D", "lsqWZ", "lsqWR", "invA2D", "lsqInvZZ", "lsqInvZR", "lsqInvRR"]


def oracle_case(case, mesh=None):
    m = mesh if mesh is not None else oracle.multiblock(case.blocks)
    return m, oracle.Oracle(m, case.bc_fields(), case.settings)


def gpu_case(case, mesh=None, precision=abi.PREC_FP64):
    m = mesh if mesh is not None else abi.multiblock(case.blocks)
    return m, abi.Solver(m, case.bc_fields(), case.settings, precision=precision)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


# The 32-cell segment classification set_mesh makes for the kernels on a
# mesh's slots (k_build_seg, csrc/kernels_fp64.cu), restated in numpy.
def slot_arrays(mesh):
    """Slot faces and slot neighbours [W][N] in the cells' CSR face order (-1: none)."""
    N = int(mesh["nCells"])
    cfs = np.asarray(mesh["cellFaceStart"], np.int64)
    cfi = np.asarray(mesh["cellFaceIDs"], np.int64)
    own = np.asarray(mesh["faceOwner"], np.int64)
    nb = np.asarray(mesh["faceNeighbor"], np.int64)
    deg = np.diff(cfs)
    W = int(deg.max())
    sface = -np.ones((W, N), np.int64)
    snb = -np.ones((W, N), np.int64)
    for j in range(W):
        idx = np.nonzero(deg > j)[0]
        f = cfi[cfs[idx] + j]
        sface[j, idx] = f
        snb[j, idx] = np.where(own[f] == idx, nb[f], np.where(nb[f] == idx, own[f], -1))
    return W, sface, snb, own, nb


def segment_counts(mesh):
    """(segments, segments with slot offsets, of those with affine faces)."""
    N = int(mesh["nCells"])
    nseg = (N + 31) // 32
    W, sface, snb, own, nb = slot_arrays(mesh)
    if W not in (3, 4):
        return nseg, 0, 0
    full = N // 32
    c = np.arange(full * 32).reshape(full, 32)
    off_ok = np.ones(full, bool)
    face_ok = np.ones(full, bool)
    for j in range(W):
        k = snb[j, :full * 32].reshape(full, 32)
        d = k - c
        ok = (k >= 0).all(axis=1) & (d == d[:, :1]).all(axis=1)
        off_ok &= ok
        f = sface[j, :full * 32].reshape(full, 32)
        f0 = f[:, :1]
        t = f[:, 1:2] - f0
        aff = (f0[:, 0] >= 0) & ((t[:, 0] == 1) | (t[:, 0] == 2)) & (f == f0 + t * (c - c[:, :1])).all(axis=1)
        fs = np.where(f >= 0, f, 0)
        o = own[fs[:, :1]] == c[:, :1]
        side = np.where(o, (own[fs] == c) & (nb[fs] == c + d[:, :1]), (own[fs] == c + d[:, :1]) & (nb[fs] == c))
        face_ok &= aff & side.all(axis=1)
    return nseg, int(off_ok.sum()), int((off_ok & face_ok).sum())
