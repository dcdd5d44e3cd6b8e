"""Agglomeration hierarchy and cell colouring built by the library on the host
(axisim_mg_levels_host, axisim_mg_level_maps_host, axisim_coloring_host) against
the oracle's restatement of buildAgglomerationMap / coarsenGrid / buildLevels
(multigrid.cu:79-325) and buildMeshColoring (memory_manger.cpp:334-409):
identical level sizes, fine-to-coarse maps, coarse CSR and colours on a
structured pipe, a graded multiblock expansion, a jittered triangle mesh and a
packed batch of uneven cases. No device is needed.
"""
import numpy as np
import pytest

import axisim.abi as abi
from axisim import batch, cases
import oracle


def _pipe():
    c = cases.pipe(max_iter=1)
    return oracle.multiblock(c.blocks), c.bc_fields(), c.settings


def _expansion():
    c = cases.expansion(scale=1 / 16, max_iter=1)
    return oracle.multiblock(c.blocks), c.bc_fields(), c.settings


def _bullet():
    c = cases.bullet(scale=0.05, max_iter=1)
    return c.mesh, c.bc_fields(), c.settings


def _batch():
    cs = batch.random_cases(5, seed=3, lo=2_000, hi=12_000)
    union, _, bcs = batch.pack_union([oracle.multiblock(c.blocks) for c in cs], [c.groups for c in cs])
    return union, bcs, cs[0].settings


@pytest.mark.parametrize("make", [_pipe, _expansion, _bullet, _batch], ids=["pipe", "expansion", "bullet", "batch"])
def test_host_hierarchy_and_coloring_match_oracle(make):
    mesh, bcs, settings = make()
    # the oracle colours the cells only for the red-black Gauss-Seidel smoother
    orc = oracle.Oracle(mesh, bcs, dict(settings, linearType=cases.LINEAR_GS_RB))
    levels = abi.mg_levels_host(mesh)
    np.testing.assert_array_equal(levels, orc.mg_levels())
    assert len(levels) >= 3
    for lvl in range(len(levels) - 1):
        for a, b in zip(abi.mg_level_maps_host(mesh, lvl), orc.mg_level_maps(lvl)):
            np.testing.assert_array_equal(a, b)
    colors, nc = abi.coloring_host(mesh)
    oc, onc = orc.coloring()
    assert nc == onc
    np.testing.assert_array_equal(colors, oc)


@pytest.mark.parametrize("nr,nz", [(2, 4), (8, 8), (3, 50), (1, 200)])
def test_host_hierarchy_small_and_thin_meshes_match_oracle(nr, nz):
    # 8 and 64 cells stay one level (coarsening stops at 64 cells); a one-cell
    # thick strip aggregates along its length only
    c = cases.pipe(nr=nr, nz=nz, max_iter=1)
    mesh = oracle.multiblock(c.blocks)
    orc = oracle.Oracle(mesh, c.bc_fields(), dict(c.settings, linearType=cases.LINEAR_GS_RB))
    levels = abi.mg_levels_host(mesh)
    np.testing.assert_array_equal(levels, orc.mg_levels())
    if nr * nz <= 64:
        assert len(levels) == 1
    for lvl in range(len(levels) - 1):
        for a, b in zip(abi.mg_level_maps_host(mesh, lvl), orc.mg_level_maps(lvl)):
            np.testing.assert_array_equal(a, b)
    colors, nc = abi.coloring_host(mesh)
    oc, onc = orc.coloring()
    assert nc == onc
    np.testing.assert_array_equal(colors, oc)


def test_host_hierarchy_rejects_bad_connectivity_and_levels():
    mesh, _, _ = _pipe()
    with pytest.raises(abi.AxisimError) as e:
        abi.mg_level_maps_host(mesh, len(abi.mg_levels_host(mesh)) - 1)
    assert e.value.status == abi.E_ARG
    bad = dict(mesh)
    ids = np.array(mesh["cellFaceIDs"], dtype=np.int32)
    ids[5] = mesh["nFaces"]  # a face id past the last face
    bad["cellFaceIDs"] = ids
    with pytest.raises(abi.AxisimError) as e:
        abi.mg_levels_host(bad)
    assert e.value.status == abi.E_MESH
    with pytest.raises(abi.AxisimError) as e:
        abi.coloring_host(bad)
    assert e.value.status == abi.E_MESH


def test_batch_hierarchy_is_each_case_coarsened_alone():
    """A batch solve coarsens every case on its own (multigrid.cu:298-325 per
    case) and merges the levels: each level holds the cells of every case that
    reaches it, and a case's coarsest level is terminal there."""
    cs = batch.random_cases(6, seed=5, lo=2_000, hi=40_000)
    meshes = [oracle.multiblock(c.blocks) for c in cs]
    union, start, _ = batch.pack_union(meshes, [c.groups for c in cs])
    cells, term = abi.mg_batch_levels_host(union, start)
    alone = [abi.mg_levels_host(m) for m in meshes]
    depth = max(len(a) for a in alone)
    assert len(cells) == depth
    assert len({len(a) for a in alone}) > 1, "the draw should hold cases of different depths"
    for lvl in range(depth):
        assert cells[lvl] == sum(int(a[lvl]) for a in alone if len(a) > lvl)
        want = sum(int(a[lvl]) for a in alone if len(a) == lvl + 1) if lvl < depth - 1 else 0
        assert term[lvl] == want, lvl
    # a one-case batch is the case's own hierarchy
    c1, t1 = abi.mg_batch_levels_host(meshes[0], [0, meshes[0]["nCells"]])
    np.testing.assert_array_equal(c1, alone[0])
    assert not t1.any()
