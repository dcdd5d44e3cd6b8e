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
