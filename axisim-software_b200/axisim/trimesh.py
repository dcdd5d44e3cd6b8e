"""Unstructured (triangle) r-z meshes in the reference's packed layout.

`pack_triangles` turns points + triangles into the face-based packed mesh the
solver takes, following Mesh::createUnstructuredMesh (solver/source/mesh.cpp:
1848-2002): cell centre = vertex average and volume = 2 pi r_c A (Pappus);
faces created per triangle in edge order (v0 v1), (v1 v2), (v2 v0), the first
triangle to reach an edge owning it; normal (dr, -dz)/|.| of the owner's edge
direction, flipped to point away from the owner centre; face area = 2 pi r_f L.
Boundary groups come from a caller-supplied classifier of the boundary face
centres (the reference matches them to the nearest sketch edge,
mesh.cpp:1835-1846).

`bullet_in_pipe` builds the unstructured bullet case: a revolved bullet body
(cylinder, hemispherical nose) on the axis of a pipe, triangulated from a quad
grid, the body removed cell by cell, interior vertices jittered from a fixed
seed.
"""
import numpy as np

PI = 3.14159265358979323846


def pack_triangles(points, tris, classify):
    """points: (P, 2) float64 (z, r); tris: (T, 3) int; classify(zf, rf) ->
    int group ids for boundary face centres. Returns the packed-mesh dict."""
    points = np.asarray(points, dtype=np.float64)
    tris = np.asarray(tris, dtype=np.int64)
    T = len(tris)
    a, b, c = points[tris[:, 0]], points[tris[:, 1]], points[tris[:, 2]]
    cz = (a[:, 0] + b[:, 0] + c[:, 0]) / 3.0
    cr = (a[:, 1] + b[:, 1] + c[:, 1]) / 3.0
    dz1, dr1 = b[:, 0] - a[:, 0], b[:, 1] - a[:, 1]
    dz2, dr2 = c[:, 0] - a[:, 0], c[:, 1] - a[:, 1]
    area2d = 0.5 * np.abs(dz1 * dr2 - dr1 * dz2)
    vol = 2.0 * PI * cr * area2d
    # edges in creation order: triangle t contributes 3t, 3t+1, 3t+2
    E = np.stack([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]], axis=1).reshape(-1, 2)
    P = len(points)
    key = np.minimum(E[:, 0], E[:, 1]) * P + np.maximum(E[:, 0], E[:, 1])
    uniq, first, inverse = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")          # face id -> unique edge
    face_of_uniq = np.empty(len(order), dtype=np.int64)
    face_of_uniq[order] = np.arange(len(order))
    face_of_edge = face_of_uniq[inverse.ravel()]
    F = len(order)
    first_edge = first[order]
    owner = (first_edge // 3).astype(np.int32)
    neighbor = np.full(F, -1, dtype=np.int32)
    second = np.arange(len(E)) != first[inverse.ravel()]
    neighbor[face_of_edge[second]] = (np.arange(len(E))[second] // 3).astype(np.int32)
    if np.bincount(face_of_edge, minlength=F).max() > 2:
        raise ValueError("an edge is shared by more than two triangles")
    p0, p1 = points[E[first_edge, 0]], points[E[first_edge, 1]]
    fz = 0.5 * (p0[:, 0] + p1[:, 0])
    fr = 0.5 * (p0[:, 1] + p1[:, 1])
    dz, dr = p1[:, 0] - p0[:, 0], p1[:, 1] - p0[:, 1]
    length = np.sqrt(dz * dz + dr * dr)
    farea = 2.0 * PI * fr * length
    nz, nr = dr.copy(), -dz
    mag = np.sqrt(nz * nz + nr * nr)
    ok = mag > 1e-30
    nz[ok] /= mag[ok]
    nr[ok] /= mag[ok]
    tz, tr = fz - cz[owner], fr - cr[owner]
    flip = nz * tz + nr * tr < 0.0
    nz[flip] *= -1.0
    nr[flip] *= -1.0
    group = np.full(F, -1, dtype=np.int32)
    bnd = neighbor < 0
    group[bnd] = classify(fz[bnd], fr[bnd]).astype(np.int32)
    return dict(nCells=T, nFaces=F, faceOwner=owner, faceNeighbor=neighbor, faceNormalZ=nz, faceNormalR=nr,
                faceCenterZ=fz, faceCenterR=fr, faceArea=farea, faceBoundaryGroupID=group, cellCenterZ=cz,
                cellCenterR=cr, cellArea2D=area2d, cellVolume=vol,
                cellFaceStart=(3 * np.arange(T + 1)).astype(np.int32),
                cellFaceIDs=face_of_edge.astype(np.int32), status=0, meshType=1)


def bullet_in_pipe(nz=1250, nr=200, L=0.3, R=0.02, body_r=0.005, body_len=0.03, nose_tip=0.1, jitter=0.1, seed=0):
    """Triangulated r-z domain [0,L] x [0,R] minus an axis-attached bullet:
    hemispherical nose of radius body_r with its tip at z = nose_tip, then a
    cylinder of radius body_r and length body_len. Returns (points, tris,
    classify); groups 0 inlet (z=0), 1 outlet (z=L), 2 wall (outer pipe and
    body), 3 axis (r=0)."""
    zc0 = nose_tip + body_r          # nose sphere centre / cylinder start
    zc1 = zc0 + body_len
    zs = np.linspace(0.0, L, nz + 1)
    rs = np.linspace(0.0, R, nr + 1)
    Z, Rg = np.meshgrid(zs, rs)      # (nr+1, nz+1)
    pts = np.stack([Z.ravel(), Rg.ravel()], axis=1)
    idx = np.arange((nr + 1) * (nz + 1)).reshape(nr + 1, nz + 1)
    a, b = idx[:-1, :-1], idx[:-1, 1:]
    c, d = idx[1:, 1:], idx[1:, :-1]
    alt = ((np.arange(nr)[:, None] + np.arange(nz)[None, :]) % 2) == 0
    t1 = np.where(alt[..., None], np.stack([a, b, c], -1), np.stack([a, b, d], -1))
    t2 = np.where(alt[..., None], np.stack([a, c, d], -1), np.stack([b, c, d], -1))
    tris = np.concatenate([t1.reshape(-1, 3), t2.reshape(-1, 3)], axis=0)
    cen = pts[tris].mean(axis=1)

    def inside(z, r):
        cyl = (z >= zc0) & (z <= zc1) & (r <= body_r)
        nose = (z < zc0) & ((z - zc0) ** 2 + r ** 2 <= body_r ** 2)
        return cyl | nose
    keep = ~inside(cen[:, 0], cen[:, 1])
    removed = tris[~keep]
    tris = tris[keep]
    # interior vertices jitter by +-jitter of the local spacing; boundary-line
    # vertices only along their line; vertices on the body stay put
    rng = np.random.default_rng(seed)
    dzs, drs = L / nz, R / nr
    jz = rng.uniform(-jitter, jitter, len(pts)) * dzs
    jr = rng.uniform(-jitter, jitter, len(pts)) * drs
    zi, ri = np.meshgrid(np.arange(nz + 1), np.arange(nr + 1))
    zi, ri = zi.ravel(), ri.ravel()
    on_z_edge = (zi == 0) | (zi == nz)
    on_r_edge = (ri == 0) | (ri == nr)
    fixed = np.zeros(len(pts), dtype=bool)
    fixed[np.unique(removed)] = True
    jz[on_z_edge | fixed] = 0.0
    jr[on_r_edge | fixed] = 0.0
    pts = pts + np.stack([jz, jr], axis=1)

    def classify(fz, fr):
        g = np.full(len(fz), 2)
        eps_z, eps_r = 1e-9 * L, 1e-9 * R
        g[fz < eps_z] = 0
        g[fz > L - eps_z] = 1
        g[fr < eps_r] = 3
        return g
    return pts, tris.astype(np.int64), classify
