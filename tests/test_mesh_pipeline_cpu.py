"""The host mesh pipeline upstream of the solver, through the C ABI (no GPU).

Restates Mesh::buildStructuredMultiBlock (solver/source/mesh.cpp:2717-2762)
with Mesh::pointInsideDomain (mesh.cpp:1177-1205), Mesh::classifyBoundaryFaces
with groupAtPoint (mesh.cpp:1835-1846, manager/source/math_func.cpp:175-196)
and Mesh::createUnstructuredMesh (mesh.cpp:1848-2002). The reference runs
these inside its GUI's Mesh, which is not compiled here, so they are pinned by
identities: a trellis over the sudden expansion must reproduce, array for
array, the hand-built multiblock case whose edge groups are known; the
triangle builder must reproduce the Python packer the unstructured cases use.
"""
import numpy as np
import pytest

from axisim import cases, trimesh
import axisim.abi as abi


@pytest.fixture(scope="module")
def lib():
    return abi.lib()


def _same_mesh(a, b, groups=True):
    for k in abi.MESH_KEYS:
        if k == "faceBoundaryGroupID" and not groups:
            continue
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


@pytest.mark.parametrize("scale", [1 / 32, 1 / 8])
def test_trellis_reproduces_the_multiblock_expansion(lib, scale):
    case = cases.expansion(scale=scale, bias=1.0)
    ref = abi.multiblock(case.blocks)
    ax = [b["axial"][1] for b in case.blocks]
    rd = [b["radial"][1] for b in case.blocks]
    m = abi.trellis([0.0, 0.04, 0.16], [0.0, 0.002, 0.006], [ax[0], ax[1]], [rd[0], rd[2]],
                    cases.expansion_outline(), L=0.16, R=0.006)
    assert m["nCells"] == ref["nCells"] == ax[0] * rd[0] + ax[1] * rd[1] + ax[1] * rd[2]
    _same_mesh(m, ref)


def test_outline_holes_and_unassigned_edges(lib):
    # a pipe with a rectangular obstacle in the middle band: the trellis cell
    # inside the obstacle loop drops out and its faces take the obstacle's group
    L, R = 0.2, 0.01
    v = [(0, 0), (L, 0), (L, R), (0, R), (0.08, 0.004), (0.12, 0.004), (0.12, 0.007), (0.08, 0.007)]
    e = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4)]
    g = [3, 1, 2, 0, 5, 5, 5, 5]
    zl, rl = [0, 0.08, 0.12, L], [0, 0.004, 0.007, R]
    m = abi.trellis(zl, rl, [8, 4, 8], [4, 3, 3], (v, e, g), L=L, R=R)
    assert m["nCells"] == 20 * 10 - 4 * 3
    bnd = m["faceNeighbor"] < 0
    grp = m["faceBoundaryGroupID"][bnd]
    fz, fr = m["faceCenterZ"][bnd], m["faceCenterR"][bnd]
    hole = (fz > 0.079) & (fz < 0.121) & (fr > 0.0039) & (fr < 0.0071)
    assert hole.sum() == 2 * (4 + 3) and np.all(grp[hole] == 5)
    assert np.all(grp[~hole & (fz < 1e-12)] == 0) and np.all(grp[~hole & (fz > L - 1e-12)] == 1)
    assert np.all(grp[~hole & (fr < 1e-12)] == 3) and np.all(grp[~hole & (fr > R - 1e-12)] == 2)
    # an edge without a group never claims a face: those faces stay -1
    g2 = [3, 1, -1, 0, 5, 5, 5, 5]
    m2 = abi.trellis(zl, rl, [8, 4, 8], [4, 3, 3], (v, e, g2), L=L, R=R)
    top = (m2["faceNeighbor"] < 0) & (m2["faceCenterR"] > R - 1e-12)
    assert top.sum() == 20 and np.all(m2["faceBoundaryGroupID"][top] == -1)


def test_empty_trellis_falls_back_to_one_block(lib):
    L, R = 0.1, 0.01
    o = cases.polygon_outline([(0, 0), (L, 0), (L, R), (0, R)], [3, 1, 2, 0])
    m = abi.trellis([], [], [], [], o, L=L, R=R, nz=7, nr=3)
    assert m["nCells"] == 21
    g = m["faceBoundaryGroupID"][m["faceNeighbor"] < 0]
    assert sorted(np.unique(g)) == [0, 1, 2, 3]


def test_triangle_builder_matches_the_python_packer(lib):
    pts, tris, classify = trimesh.bullet_in_pipe(nz=40, nr=8, seed=3)
    ref = trimesh.pack_triangles(pts, tris, classify)
    # outline = the triangulation's own boundary edges, grouped by the same classifier
    E = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    key = np.sort(E, axis=1)
    uniq, cnt = np.unique(key, axis=0, return_counts=True)
    bedges = uniq[cnt == 1]
    mid = 0.5 * (pts[bedges[:, 0]] + pts[bedges[:, 1]])
    groups = classify(mid[:, 0], mid[:, 1])
    m = abi.triangle_mesh(pts, tris, (pts, bedges, groups), L=0.3, R=0.02)
    _same_mesh(m, ref)
    assert m["meshType"] == abi.MESH_UNSTRUCTURED


def test_classification_rewrites_only_external_faces(lib):
    case = cases.expansion(scale=1 / 32, bias=1.0)
    ref = abi.multiblock(case.blocks)
    blank = [dict(b, edge_group=[-1, -1, -1, -1]) for b in case.blocks]
    m = abi.multiblock(blank)
    assert np.all(m["faceBoundaryGroupID"] == -1)
    abi.classify_boundary_faces(m, cases.expansion_outline(), L=0.16, R=0.006)
    _same_mesh(m, ref)


def test_bad_inputs_are_statuses(lib):
    o = cases.expansion_outline()
    with pytest.raises(abi.AxisimError) as e:
        abi.trellis([0.0, 0.04, 0.02], [0.0, 0.006], [4, 4], [4], o, L=0.16, R=0.006)
    assert e.value.status == abi.E_ARG
    pts = np.array([[0, 0], [1, 0], [0, 1], [1, 1]], float)
    with pytest.raises(abi.AxisimError) as e:   # edge (0, 1) in three triangles
        abi.triangle_mesh(pts, [[0, 1, 2], [1, 0, 3], [0, 1, 3]], o, L=1, R=1)
    assert e.value.status == abi.E_MESH
    with pytest.raises(abi.AxisimError) as e:
        abi.triangle_mesh(pts, [[0, 1, 9]], o, L=1, R=1)
    assert e.value.status == abi.E_MESH
