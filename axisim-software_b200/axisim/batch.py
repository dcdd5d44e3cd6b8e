"""Batches of independent cases: generation, packing into one mesh, sharding.

A batch is solved as ONE packed mesh whose cases occupy contiguous cell ranges
and share no face (`pack_union`); the library advances every case in the same
kernels and graph nodes and monitors each case's residuals separately
(axisim_set_batch). Across GPUs, cases are independent units: `shard` assigns
them to ranks by a greedy longest-first bin pack on cell count, and the only
exchange is a gather of per-case results at the end (`gather_results`).
"""
import math

import numpy as np

from . import cases as C

GROUPS_PER_CASE = 4


def random_cases(n=256, seed=0, lo=8_000, hi=260_000, rho=1056.0, mu=3.5e-3, scale=1.0, max_iter=50000, tol=1e-6):
    """The batch workload: n cases with cell count log-uniform in [lo, hi]; each a
    pipe or a sudden expansion (expansion ratio uniform in [1.5, 4]), throat
    Reynolds number uniform in [50, 1500], inlet uniform or fully developed with
    50/50 odds; all drawn from `seed`. `scale` multiplies the cell counts."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        target = math.exp(rng.uniform(math.log(lo), math.log(hi))) * scale
        geom = "pipe" if rng.uniform() < 0.5 else "expansion"
        ratio = rng.uniform(1.5, 4.0)
        re = rng.uniform(50.0, 1500.0)
        fd = rng.uniform() < 0.5
        r_in = 0.002
        ubar = re * mu / (rho * 2.0 * r_in)
        if geom == "pipe":
            L = 20.0 * 2.0 * r_in
            nr = max(4, int(round(math.sqrt(target / 8.0))))
            nz = max(8, int(round(target / nr)))
            c = C.pipe(nr=nr, nz=nz, R=r_in, L=L, U0=ubar, rho=rho, mu=mu, fully_developed=fd,
                       max_iter=max_iter, tol=tol)
            c.settings.update(gradientScheme=C.GRAD_LSQ, linearType=C.LINEAR_JACOBI)
        else:
            r_out = ratio * r_in
            # cells split so that bands are near-square in spacing
            nr_in = max(2, int(round(math.sqrt(target / (8.0 * (1.0 + (ratio - 1.0) * 0.75 / 1.0 + 2.0))))))
            nr_out = max(2, int(round(nr_in * (ratio - 1.0))))
            nz_in = max(4, 2 * nr_in)
            nz_out = max(8, int(round((target - nr_in * nz_in) / max(1, nr_in + nr_out))))
            c = C.expansion(nr_in=nr_in, nr_out=nr_out, nz_in=nz_in, nz_out=nz_out, r_in=r_in, r_out=r_out,
                            l_in=10 * r_in, l_out=40 * r_in, rho=rho, mu=mu, re=re, bias=1.0,
                            scheme=C.CONV_UPWIND, max_iter=max_iter, tol=tol)
            if not fd:
                c.groups[0].bcs[C.U] = (C.DIRICHLET, ubar)
        c.name = f"case{i:03d}_{geom}"
        out.append(c)
    return out


def pack_union(meshes, groups_list):
    """Concatenate packed meshes (cell, face and group ids offset per case).
    groups_list[c] are case c's boundary groups (ids 0..3). Returns (mesh,
    caseCellStart, bc_fields) for the whole batch."""
    cell_off = np.cumsum([0] + [m["nCells"] for m in meshes])
    face_off = np.cumsum([0] + [m["nFaces"] for m in meshes])
    ref_off = np.cumsum([0] + [len(m["cellFaceIDs"]) for m in meshes])
    out = {"nCells": int(cell_off[-1]), "nFaces": int(face_off[-1]), "status": 0,
           "meshType": 0 if all(m.get("meshType", 1) == 0 for m in meshes) else 1}
    cat = lambda k: np.concatenate([m[k] for m in meshes])  # noqa: E731
    for k in ("faceNormalZ", "faceNormalR", "faceCenterZ", "faceCenterR", "faceArea", "cellCenterZ", "cellCenterR",
              "cellArea2D", "cellVolume"):
        out[k] = cat(k)
    out["faceOwner"] = np.concatenate([m["faceOwner"] + cell_off[i] for i, m in enumerate(meshes)]).astype(np.int32)
    out["faceNeighbor"] = np.concatenate([np.where(m["faceNeighbor"] >= 0, m["faceNeighbor"] + cell_off[i], -1)
                                          for i, m in enumerate(meshes)]).astype(np.int32)
    out["faceBoundaryGroupID"] = np.concatenate(
        [np.where(m["faceBoundaryGroupID"] >= 0, m["faceBoundaryGroupID"] + GROUPS_PER_CASE * i, -1)
         for i, m in enumerate(meshes)]).astype(np.int32)
    out["cellFaceIDs"] = np.concatenate([m["cellFaceIDs"] + face_off[i] for i, m in enumerate(meshes)]).astype(np.int32)
    out["cellFaceStart"] = np.concatenate([meshes[0]["cellFaceStart"][:1]] +
                                          [m["cellFaceStart"][1:] + ref_off[i] for i, m in enumerate(meshes)]).astype(np.int32)
    groups = []
    for i, gs in enumerate(groups_list):
        for g in gs:
            groups.append(C.Group(g.id + GROUPS_PER_CASE * i, g.btype, dict(g.bcs), g.total_length))
    bcs = {v: C.resolve_bc_field(groups, v) for v in (C.U, C.V, C.P)}
    return out, cell_off.astype(np.int32), bcs


def split_fields(arr, case_cell_start):
    return [arr[case_cell_start[i]:case_cell_start[i + 1]] for i in range(len(case_cell_start) - 1)]


def shard(sizes, world):
    """Greedy longest-first bin pack of case sizes onto `world` ranks.
    Returns a list of case-index lists, one per rank (each sorted)."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def gather_results(local, world, dist=None):
    """All ranks' per-case result dicts merged into one {case index: result};
    `dist` is torch.distributed (any backend) or None for one process."""
    if dist is None or world == 1:
        return dict(local)
    objs = [None] * world
    dist.all_gather_object(objs, dict(local))
    merged = {}
    for o in objs:
        merged.update(o)
    return merged
