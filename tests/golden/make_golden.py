"""Generate golden vectors from the REFERENCE's own SIMPLE solver.

Runs oracle/_ref/axisim_ref (the reference's solver translation units compiled
unchanged from their sources by oracle/ref_build/Makefile, driven headless by
oracle/ref_build/ref_driver.cu) on small cases and stores the solution fields
and residual history as .npz fixtures next to this script. Needs a GPU (the
reference is GPU-only); the committed fixtures are what the CPU tests read.

    python tests/golden/make_golden.py [outdir]
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "axisim-software_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from axisim import cases  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "axisim_ref")
VAR_NAMES = {cases.U: "u", cases.V: "v", cases.P: "p", cases.TEMP: "T", cases.CONC: "C"}


def fixture_cases():
    """(name, case, tolerance note) of every golden vector."""
    out = []
    out.append(("pipe10x50_fd_converged", cases.pipe(nr=10, nz=50, max_iter=5000, tol=1e-6, fully_developed=True)))
    out.append(("pipe10x50_5it", cases.pipe(nr=10, nz=50, max_iter=5, tol=1e-30)))
    c = cases.expansion(scale=1 / 32, max_iter=5, tol=1e-30)
    out.append(("expansion864_sou_5it", c))
    c = cases.expansion(scale=1 / 32, max_iter=20000, tol=1e-6)
    out.append(("expansion864_sou_converged", c))
    c = cases.expansion(scale=1 / 32, max_iter=4, tol=1e-30)
    c.settings.update(convectionScheme=cases.CONV_CENTRAL, gradientScheme=cases.GRAD_GREEN_GAUSS)
    out.append(("expansion864_gg_central_4it", c))
    c = cases.pipe(nr=8, nz=40, max_iter=4, tol=1e-30)
    c.settings.update(useMultigrid=0, linearType=cases.LINEAR_JACOBI, linearMaxIter=7)
    out.append(("pipe8x40_nomg_jacobi7_4it", c))
    c = cases.pulsatile_expansion(scale=1 / 32, dt=1e-3, steps=3, max_iter=3, tol=1e-30)
    out.append(("pulsatile864_bdf2_3x3", c))
    c = cases.pipe(max_iter=50000, tol=1e-6)
    out.append(("pipe40x200_config1_converged", c))
    # triangles (the bullet body, jittered): least-squares gradients with the
    # non-orthogonal corrector on an unstructured mesh, packed by this
    # project's createUnstructuredMesh restatement and handed to the reference
    # solver as packed arrays
    out.append(("bullet1205_lsq_nonortho_6it", cases.bullet(scale=0.05, max_iter=6, tol=1e-30)))
    out.append(("batch4_union6316_5it", batch_union()[0]))
    # the same four cases, each solved alone by the reference: a batched solve
    # coarsens every case on its own, so each case of it must give these
    for i, c in enumerate(batch_cases()):
        out.append((f"batch4_case{i}_{c.name.split('_')[-1]}_5it", c))
    out += scalar_fixture_cases()
    return out


def fullsize_fixture_cases():
    """Workloads at their own sizes. Their fields do not fit a small fixture, so
    compact() keeps a strided sample of cells, per-block sums and the norms."""
    return [("expansion874496_sou_5it", cases.expansion(scale=1.0, max_iter=5, tol=1e-30))]


SAMPLE_STRIDE = 211   # every 211th cell (4,145 of 874,496)
BLOCK = 4096          # consecutive cells per block sum
COMPACT_FIELDS = ("u", "v", "p", "gradPZ", "gradPR")


def compact(res):
    """The size-independent summary of a full-size run: for each field a
    strided sample, the sum and the sum of magnitudes over every block of
    BLOCK consecutive cells (so every cell contributes), and the L2 norm."""
    out = {k: res[k] for k in ("iterations", "converged", "residual_history")}
    for k in COMPACT_FIELDS:
        a = np.asarray(res[k], dtype=np.float64)
        starts = np.arange(0, a.size, BLOCK)
        out[k + "_sample"] = a[::SAMPLE_STRIDE].copy()
        out[k + "_blocksum"] = np.add.reduceat(a, starts)
        out[k + "_blockabs"] = np.add.reduceat(np.abs(a), starts)
        out[k + "_norm"] = np.array(np.linalg.norm(a))
    out["nCells"] = np.array(len(res["u"]))
    return out


def compact_mismatch(fields, g):
    """Largest relative disagreement between full fields and a compact fixture:
    samples and norms by relative L2 / relative difference, block sums against
    the block's sum of magnitudes (sums of signed values may cancel)."""
    worst = {}
    for k in COMPACT_FIELDS:
        a = np.asarray(fields[k], dtype=np.float64)
        starts = np.arange(0, a.size, BLOCK)
        smp = a[::SAMPLE_STRIDE]
        e_s = np.linalg.norm(smp - g[k + "_sample"]) / max(np.linalg.norm(g[k + "_sample"]), 1e-300)
        e_b = np.max(np.abs(np.add.reduceat(a, starts) - g[k + "_blocksum"]) / np.maximum(g[k + "_blockabs"], 1e-300))
        e_n = abs(np.linalg.norm(a) - float(g[k + "_norm"])) / max(float(g[k + "_norm"]), 1e-300)
        worst[k] = max(e_s, e_b, e_n)
    return worst


def batch_cases(n=4, seed=7, scale=0.02, iters=5):
    """The random cases of batch_union, each as a case of its own."""
    from axisim import batch
    return batch.random_cases(n, seed=seed, scale=scale, max_iter=iters, tol=1e-30)


def batch_union(n=4, seed=7, scale=0.02, iters=5):
    """Four random cases of the batch mix packed into one mesh (cell, face and
    group ids offset per case), as a Case the reference solves as one mesh;
    returns (case, caseCellStart). With the tolerance out of reach every case
    runs the same iterations, so a batched solve must give these fields."""
    from axisim import batch
    import oracle
    cs = batch.random_cases(n, seed=seed, scale=scale, max_iter=iters, tol=1e-30)
    union, start, _ = batch.pack_union([oracle.multiblock(c.blocks) for c in cs], [c.groups for c in cs])
    groups = [cases.Group(g.id + batch.GROUPS_PER_CASE * i, g.btype, dict(g.bcs), g.total_length)
              for i, c in enumerate(cs) for g in c.groups]
    return cases.Case(f"batch{n}_union{union['nCells']}", [], groups, dict(cs[0].settings), mesh=union), start


def scalar_fixture_cases():
    """Energy + concentration transport: Michaelis-Menten wall behind a layer
    (GS sweeps, upwind), Hill wall with substrate inhibition (Jacobi, SOU,
    non-integer exponents; the corrector flag is set and, on this structured
    mesh, cleared by runCheck), a BDF2 pulsatile run with both scalars, and a
    run to convergence."""
    out = []
    c = cases.with_scalars(cases.pipe(nr=10, nz=50, max_iter=10, tol=1e-30), wall_c=cases.michaelis_menten(1e-3, 0.2),
                           wall_layers=[(1e-6, 1e-4)], D=1e-6)
    c.settings.update(scalarResEnabled=[1, 1], scalarResTol=[1e-30, 1e-30])
    out.append(("pipe10x50_scalars_mm_10it", c))
    c = cases.with_scalars(cases.expansion(scale=1 / 32, max_iter=6, tol=1e-30),
                           wall_c=cases.hill(2e-3, 0.4, 2.5, inhibition=(2.0, 0.5, 0.3)), t_wall=None, D=2e-6,
                           k=0.6e2)
    c.settings.update(scalarResEnabled=[1, 0], scalarResNorm=[1, 0], useNonOrthCorrector=1)
    out.append(("expansion864_scalars_hill_sou_6it", c))
    c = cases.with_scalars(cases.pulsatile_expansion(scale=1 / 32, dt=1e-3, steps=3, max_iter=3, tol=1e-30),
                           wall_c=cases.michaelis_menten(1e-3, 0.2), D=1e-6)
    out.append(("pulsatile864_bdf2_scalars_3x3", c))
    c = cases.with_scalars(cases.pipe(nr=10, nz=50, max_iter=5000, tol=1e-6), wall_c=cases.michaelis_menten(1e-3, 0.2),
                           wall_layers=[(1e-6, 1e-4)], D=1e-6)
    c.settings.update(scalarResEnabled=[1, 1], scalarResTol=[1e-6, 1e-6])
    out.append(("pipe10x50_scalars_mm_converged", c))
    return out


PACKED_ORDER = [("faceOwner", np.int32), ("faceNeighbor", np.int32), ("faceNormalZ", np.float64),
                ("faceNormalR", np.float64), ("faceCenterZ", np.float64), ("faceCenterR", np.float64),
                ("faceArea", np.float64), ("faceBoundaryGroupID", np.int32), ("cellCenterZ", np.float64),
                ("cellCenterR", np.float64), ("cellArea2D", np.float64), ("cellVolume", np.float64),
                ("cellFaceStart", np.int32), ("cellFaceIDs", np.int32)]


def write_packed(mesh, path):
    """The driver's packed-mesh file: int32 nCells, nFaces, nRefs, then the
    FVMeshHostPacked arrays in declaration order."""
    with open(path, "wb") as f:
        np.array([mesh["nCells"], mesh["nFaces"], len(mesh["cellFaceIDs"])], np.int32).tofile(f)
        for k, dt in PACKED_ORDER:
            np.ascontiguousarray(mesh[k], dtype=dt).tofile(f)


def write_spec(case, path, tol=1e-9):
    with open(path, "w") as f:
        f.write(f"tol {tol!r}\n")
        if case.mesh is not None:
            mesh_path = os.path.join(os.path.dirname(path), "mesh.bin")
            write_packed(case.mesh, mesh_path)
            f.write(f"packed {mesh_path}\n")
        for b in case.blocks:
            ax, rd = b["axial"], b["radial"]
            f.write("block %r %r %r %d %d %r %r %d %d %r %d %d %d %d\n" % (
                b["z0"], b["r0"], ax[0], ax[1], ax[2], ax[3], rd[0], rd[1], rd[2], rd[3], *b["edge_group"]))
        for g in case.groups:
            items = []
            for var, bc in g.bcs.items():
                t, val = bc[0], bc[1]
                if t in (cases.MICHAELIS_MENTEN, cases.HILL):
                    val = 0.0  # parameters follow on a kin line
                amp, freq = (bc[2], bc[3]) if len(bc) > 2 else (0.0, 0.0)
                items.append(f"{VAR_NAMES[var]} {t} {val!r} {amp!r} {freq!r}")
            f.write(f"group {g.id} {g.btype} {float(np.float32(g.total_length))!r} {len(items)} {' '.join(items)}\n")
        for g in case.groups:
            for var, bc in g.bcs.items():
                if bc[0] in (cases.MICHAELIS_MENTEN, cases.HILL):
                    k = bc[1]
                    inh = k.get("inhibition")
                    m, k2, v2 = inh if inh else (1.0, 0.0, 0.0)
                    f.write(f"kin {g.id} {VAR_NAMES[var]} {bc[0]} {k['Vmax']!r} {k['Km']!r} {k['n']!r} "
                            f"{1 if inh else 0} {m!r} {k2!r} {v2!r}\n")
            for var, layers in g.layers.items():
                for (kl, dl) in layers:
                    f.write(f"layer {g.id} {VAR_NAMES[var]} {kl!r} {dl!r}\n")
        s = case.settings
        for k in ("convectionScheme", "gradientScheme", "linearType", "timeScheme", "linearMaxIter", "useMultigrid",
                  "addConvectionTerm", "transient", "useNonOrthCorrector", "dt", "tEnd", "maxIter", "checkConv",
                  "mgMaxIter", "mgWeight", "mgLinearSweep", "mgPreSweep", "mgPostSweep", "rho", "mu", "alphaU",
                  "alphaP", "cp", "k", "D", "solveEnergy", "solveConcentration"):
            f.write(f"set {k} {float(s[k])!r}\n")
        for i in range(3):
            f.write(f"set resNorm{i} {s['resNorm'][i]}\nset resScale{i} {s['resScale'][i]}\n"
                    f"set resEnabled{i} {s['resEnabled'][i]}\nset resTol{i} {s['resTol'][i]!r}\n")
        for j in range(2):
            i = 3 + j
            f.write(f"set resNorm{i} {s['scalarResNorm'][j]}\nset resScale{i} {s['scalarResScale'][j]}\n"
                    f"set resEnabled{i} {s['scalarResEnabled'][j]}\nset resTol{i} {s['scalarResTol'][j]!r}\n")


FIELDS = ["u", "v", "p", "continuity", "gradPZ", "gradPR", "gradUZ", "gradUR", "gradVZ", "gradVR"]


def read_out(path):
    raw = open(path, "rb").read()
    N, it, conv, rows = np.frombuffer(raw[:16], dtype=np.int32)
    off = 16
    out = {"iterations": int(it), "converged": int(conv)}
    for name in FIELDS:
        out[name] = np.frombuffer(raw[off:off + 8 * N], dtype=np.float64).copy()
        off += 8 * N
    # iteration, U, V, Continuity, Temperature, Concentration
    out["residual_history"] = np.frombuffer(raw[off:off + 48 * rows], dtype=np.float64).reshape(rows, 6).copy()
    off += 48 * rows
    flags = np.frombuffer(raw[off:off + 8], dtype=np.int32)
    off += 8
    for on, names in zip(flags, (("T", "gradTZ", "gradTR"), ("C", "gradCZ", "gradCR"))):
        if not on:
            continue
        for name in names:
            out[name] = np.frombuffer(raw[off:off + 8 * N], dtype=np.float64).copy()
            off += 8 * N
    return out


def run_reference(case):
    with tempfile.TemporaryDirectory() as d:
        spec, out = os.path.join(d, "spec.txt"), os.path.join(d, "out.bin")
        write_spec(case, spec)
        r = subprocess.run([REF_BIN, spec, out], capture_output=True, text=True, timeout=1200)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed: {r.stdout} {r.stderr}")
        res = read_out(out)
        res["log"] = r.stdout
        return res


def main(outdir=HERE, only=""):
    """Regenerates every fixture whose name contains `only` (the full-size
    ones only when `only` names them)."""
    for name, case in fullsize_fixture_cases():
        if not only or only not in name:
            continue
        res = run_reference(case)
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **compact(res))
        print(name, res["iterations"], res["converged"], res["log"].strip().splitlines()[0])
    for name, case in fixture_cases():
        if only not in name:
            continue
        res = run_reference(case)
        keep = {k: v for k, v in res.items() if k not in ("log",)}
        if name.startswith("pipe40x200") or name.startswith("batch4_union"):
            keep = {k: keep[k] for k in ("u", "v", "p", "iterations", "converged", "residual_history")}
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **keep)
        print(name, res["iterations"], res["converged"], res["log"].strip().splitlines()[0])


if __name__ == "__main__":
    main(*sys.argv[1:])
