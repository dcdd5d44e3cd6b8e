"""The 32-cell segment classification (restated in helpers.segment_counts) on
the workloads' own meshes, without a GPU: the structured expansion qualifies
almost everywhere, the jittered bullet's triangles nowhere, and a segment
with a boundary slot never qualifies."""
import numpy as np

from axisim import cases
import axisim.abi as abi
from helpers import segment_counts


def test_expansion_full_size_segments():
    mesh = cases.expansion().packed(abi.multiblock)
    assert mesh["nCells"] == 874496
    assert segment_counts(mesh) == (27328, 26396, 26396)


def test_bullet_has_no_regular_segments():
    mesh = cases.bullet(scale=0.25).mesh
    nseg, noff, nface = segment_counts(mesh)
    assert nseg > 500 and noff == 0 and nface == 0


def test_boundary_and_partial_segments_do_not_qualify():
    mesh = cases.pipe(nr=13, nz=37).packed(abi.multiblock)  # 481 cells: a partial last segment
    nseg, noff, nface = segment_counts(mesh)
    assert nseg == 16 and noff <= 15 and nface == noff
    big = cases.pipe(nr=64, nz=96).packed(abi.multiblock)
    nseg, noff, nface = segment_counts(big)
    assert 0 < noff < nseg and nface == noff
    # a segment whose cells have a boundary slot never qualifies
    cfs = np.asarray(big["cellFaceStart"])
    nb = np.asarray(big["faceNeighbor"])
    cfi = np.asarray(big["cellFaceIDs"])
    boundary_cell = np.zeros(big["nCells"], bool)
    for c in range(big["nCells"]):
        boundary_cell[c] = (nb[cfi[cfs[c]:cfs[c + 1]]] < 0).any()
    seg_has_boundary = boundary_cell[: (big["nCells"] // 32) * 32].reshape(-1, 32).any(axis=1)
    assert noff <= int((~seg_has_boundary).sum())
