"""Tiles of the momentum Jacobi sweeps, built on the host (no GPU).

Several sweeps per launch run on tiles of cells with halo layers
(axisim_sweep_tiles_host). These tests hold the tile lists to what the tile
kernel relies on:

* layer 0 of the tiles partitions the cells;
* every cell the kernel updates (layers 0..S-1) finds each slot neighbour of
  the [W][N] slot block (linear_solver.cu:9-33 gathers through it) inside its
  tile, at the local index the tile lists;
* S sweeps run tile by tile on those lists (a NumPy restatement of the tile
  kernel, same operation order) give layer 0 exactly the values of S
  whole-mesh sweeps, bit for bit, for every S up to the tiles' layer count;
* a cap too small for one cell and its halo gives no tiles.
"""
import numpy as np
import pytest

from axisim import batch, cases
import axisim.abi as abi


def _slot_neighbours(m):
    N = m["nCells"]
    cfs, cfi, own, nbr = m["cellFaceStart"], m["cellFaceIDs"], m["faceOwner"], m["faceNeighbor"]
    deg = np.diff(cfs)
    W = int(deg.max())
    nb = -np.ones((W, N), np.int64)
    for j in range(W):
        n = np.nonzero(deg > j)[0]
        f = cfi[cfs[n] + j]
        o, q = own[f], nbr[f]
        nb[j, n] = np.where(o == n, q, np.where(q == n, o, -1))
    return nb


def _meshes():
    e = cases.expansion(scale=1 / 8, max_iter=1, tol=0.0)
    b = cases.bullet(scale=0.1, max_iter=1, tol=0.0)
    cs = batch.random_cases(4, seed=3, scale=0.05, max_iter=1, tol=0.0)
    union, _, _ = batch.pack_union([abi.multiblock(c.blocks) for c in cs], [c.groups for c in cs])
    return [("expansion", abi.multiblock(e.blocks)), ("bullet", b.mesh), ("union4", union)]


MESHES = _meshes()


def _sweep(nb, a, b, inv, x):
    v = b.copy()
    for j in range(nb.shape[0]):
        k = nb[j]
        g = x[np.where(k >= 0, k, 0)]
        v = np.where(k >= 0, v - a[j] * g, v)
    return np.where(inv != 0.0, v * inv, x)


def _tiled(t, a, b, inv, x, sweeps):
    """The tile kernel over all tiles at once: flat local cells, neighbours by
    flat index, sweep s over the local cells below layerEnd[S' - s]."""
    gid, lnb = t["gid"], t["lnb"]
    ts, le = t["tileStart"], t["layerEnd"]
    n_tiles = t["n_tiles"]
    tile_of = np.repeat(np.arange(n_tiles), np.diff(ts))
    local = np.arange(len(gid)) - ts[tile_of]
    W = a.shape[0]
    flat_nb = np.where(lnb[:, :W] >= 0, ts[tile_of][:, None] + lnb[:, :W], -1).T
    X = x[gid]
    A = a[:, gid]
    B, I = b[gid], inv[gid]
    for s in range(1, sweeps + 1):
        upd = local < le[tile_of, sweeps - s]
        Y = _sweep(np.where(upd[None, :], flat_nb, -1), A, B, I, X)
        X = np.where(upd, Y, X)
    out = np.full(len(x), np.nan)
    own = local < le[tile_of, 0]
    out[gid[own]] = X[own]
    return out


@pytest.mark.parametrize("name,mesh", MESHES, ids=[n for n, _ in MESHES])
def test_tiles_partition_cells_and_hold_every_neighbour(name, mesh):
    S, cap = 4, 1024
    t = abi.sweep_tiles_host(mesh, S, cap, 600)
    N = mesh["nCells"]
    assert t["n_tiles"] > 1
    ts, le, gid, lnb = t["tileStart"], t["layerEnd"], t["gid"], t["lnb"]
    assert ts[0] == 0 and ts[-1] == len(gid)
    assert (np.diff(ts) <= cap).all() and (np.diff(ts) == le[:, S]).all()
    assert (np.diff(le, axis=1) >= 0).all()
    owned = np.concatenate([gid[ts[i]:ts[i] + le[i, 0]] for i in range(t["n_tiles"])])
    assert np.array_equal(np.sort(owned), np.arange(N))
    nb = _slot_neighbours(mesh)
    W = nb.shape[0]
    for i in range(t["n_tiles"]):
        g = gid[ts[i]:ts[i + 1]]
        assert len(np.unique(g)) == len(g)
        for k in range(S + 1):  # each layer in ascending cell order
            lay = g[(le[i, k - 1] if k else 0):le[i, k]]
            assert (np.diff(lay) > 0).all()
        inner = le[i, S - 1]
        loc = lnb[ts[i]:ts[i] + inner, :W]
        want = nb[:, g[:inner]].T
        assert np.array_equal(np.where(loc >= 0, g[np.maximum(loc, 0)], -1), want), (name, i)
        assert (lnb[ts[i]:ts[i + 1], W:] == -1).all()
        assert (lnb[ts[i] + inner:ts[i + 1]] == -1).all()


@pytest.mark.parametrize("name,mesh", MESHES, ids=[n for n, _ in MESHES])
def test_tiled_sweeps_equal_whole_mesh_sweeps_bitwise(name, mesh):
    S = 4
    t = abi.sweep_tiles_host(mesh, S, 2048, 1300)
    nb = _slot_neighbours(mesh)
    N = mesh["nCells"]
    rng = np.random.default_rng(7)
    a = np.where(nb >= 0, -rng.uniform(0.1, 1.0, nb.shape), 0.0)
    diag = -a.sum(0) + rng.uniform(0.0, 0.5, N)
    inv = np.where(rng.uniform(size=N) < 0.02, 0.0, 1.0 / diag)  # some rows keep their value
    b = rng.standard_normal(N)
    x0 = rng.standard_normal(N)
    for sweeps in range(1, S + 1):
        want = x0
        for _ in range(sweeps):
            want = _sweep(nb, a, b, inv, want)
        got = _tiled(t, a, b, inv, x0, sweeps)
        assert np.array_equal(got, want), (name, sweeps)


def test_cap_too_small_for_one_cell_gives_no_tiles():
    mesh = MESHES[0][1]
    t = abi.sweep_tiles_host(mesh, 4, 8, 4)
    assert t["n_tiles"] == 0 and len(t["tileStart"]) == 1


def test_bad_arguments_are_refused():
    mesh = MESHES[0][1]
    for S, cap, run in ((0, 1024, 100), (9, 1024, 100), (4, 0, 100), (4, 70000, 100), (4, 1024, 0)):
        with pytest.raises(abi.AxisimError):
            abi.sweep_tiles_host(mesh, S, cap, run)
