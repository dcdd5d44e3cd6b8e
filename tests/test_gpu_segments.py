"""The 32-cell segment tables set_mesh builds for the kernels on a mesh's slots
(segNeighbours / slotFaces in csrc/device.cuh): the device's classification
against a numpy restatement of it, and bit-exact FP64 parity with the oracle
on meshes that use the tables and on one that does not."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "axisim-software_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from axisim import abi, cases  # noqa: E402
from helpers import FIELDS, segment_counts  # noqa: E402

pytestmark = pytest.mark.gpu


def gpu_solver(mesh, case, **kw):
    return abi.Solver(mesh, case.bc_fields(), case.settings, **kw)


@pytest.mark.parametrize("name", ["expansion", "pipe", "pipe_ragged", "bullet"])
def test_segment_tables_match_restatement(name):
    if name == "expansion":
        case = cases.expansion(scale=1 / 8, max_iter=1, tol=1e-30)
    elif name == "pipe":
        case = cases.pipe(max_iter=1, tol=1e-30)
    elif name == "pipe_ragged":
        case = cases.pipe(nr=13, nz=37, max_iter=1, tol=1e-30)  # 481 cells: a partial last segment
    else:
        case = cases.bullet(scale=0.1, max_iter=1, tol=1e-30)
    mesh = case.packed(abi.multiblock)
    gpu = gpu_solver(mesh, case)
    got = gpu.mesh_segments()
    nseg, noff, nface = segment_counts(mesh)
    assert (got["segments"], got["offset_segments"], got["face_segments"]) == (nseg, noff, nface)
    assert got["in_use"] == (2 * (nseg - noff) <= nseg)
    if name == "expansion":
        assert got["in_use"] and noff >= 0.7 * nseg  # 0.97 at full size
    if name == "bullet":
        assert not got["in_use"]
    gpu.close()


@pytest.mark.parametrize("scale", [1 / 16, 1 / 5])
def test_fp64_bitexact_with_segment_tables(scale):
    import oracle

    case = cases.expansion(scale=scale, max_iter=6, tol=1e-30)
    mesh = case.packed(abi.multiblock)
    gpu = gpu_solver(mesh, case)
    seg = gpu.mesh_segments()
    assert seg["in_use"] and seg["face_segments"] > 0
    r = gpu.solve()
    orc = oracle.Oracle(mesh, case.bc_fields(), case.settings)
    it, _ = orc.run()
    assert r["iterations"] == it == 6
    for f in FIELDS:
        np.testing.assert_array_equal(gpu.get(f), orc.get(f), err_msg=f)
    gpu.close()
