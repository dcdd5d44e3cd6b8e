"""Shared test helpers: build one case for both the CUDA path and the oracle."""
import numpy as np

from axisim import cases
import axisim.abi as abi
import oracle


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
