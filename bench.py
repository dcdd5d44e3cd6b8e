#!/usr/bin/env python
"""SIMPLE iterations per second per Mcell on one B200 (or N replicas).

Workload: the sudden expansion on a three-block structured mesh (256 radial x
4096 axial band cells, 874,496 cells), rho 1056, mu 3.5e-3, fully developed
inlet at throat Re 500, second-order upwind, LSQ gradients, 20 Jacobi sweeps
per momentum solve, 3 agglomeration-multigrid V-cycles per pressure solve.
A step is one SIMPLE outer iteration over the whole mesh.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0). `value` is device time (CUDA events on the
solver's stream) of K steps after W warm-up steps; `e2e` is the same metric
through the public C API from host buffers (case upload + solve + field
download, host clock). `--impl reference` times the CPU restatement of the
reference algorithm (the reference has no CPU solver) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "axisim-software_b200"))

METRIC = "time-to-residual 1e-6 & SIMPLE iter/s per Mcell, learned+mixed vs plain, 1 B200"
UNIT = "Mcell-iter/s"


def _json_scalar(o):
    # numpy scalars (numpy's bool_ included) as plain Python values
    if hasattr(o, "item"):
        return o.item()
    raise TypeError(f"not JSON serializable: {type(o).__name__}")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="cell-count scale of the workload (1 = full size)")
    ap.add_argument("--no-extras", action="store_true", help="skip cpu baseline / e2e / time-to-residual legs")
    ap.add_argument("--network-only", action="store_true",
                    help="time the learned p' network alone (inference and training steps, 2M-cell mesh)")
    ap.add_argument("--scalars-only", action="store_true",
                    help="energy + concentration transport on the workload mesh: cost per SIMPLE iteration with "
                         "and without the scalars, and the scalar kernels' achieved bandwidth (--steps iterations)")
    ap.add_argument("--transient-only", action="store_true",
                    help="the 2M-cell pulsatile transient leg alone (time and error to the converged FP64 steps)")
    ap.add_argument("--bullet-only", action="store_true", help="the 485k-cell unstructured bullet leg alone")
    ap.add_argument("--accuracy-only", action="store_true",
                    help="time to 1e-6 relative L2 of the converged FP64 fields on the workload (all arms)")
    ap.add_argument("--momentum-sweeps", type=int, default=1,
                    help="momentum Jacobi sweeps per launch (above 1: shared-memory tiles; the default 1 is the "
                         "faster setting measured on a B200)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="mixed: FP32 inner solves inside FP64 refinement (the workload's setting); fp64: plain")
    return ap.parse_args()


def workload(scale):
    from axisim import cases
    c = cases.expansion(scale=scale, max_iter=10, tol=0.0)
    return c


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as D
        torch.cuda.set_device(local)
        D.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = D
    return world, rank, local, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    """CPU restatement of the reference's SIMPLE loop on all host threads."""
    world, rank, local, dist = dist_setup(args.gpus)
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    case = workload(args.scale)
    threads = os.cpu_count() or 1
    mesh = oracle.multiblock(case.blocks)
    s = dict(case.settings)
    s["maxIter"] = max(1, args.warmup)
    o = oracle.Oracle(mesh, case.bc_fields(), s, threads=threads)
    o.run()
    # timed sample: up to K iterations, bounded to about a minute of CPU time
    per = None
    done, t_total = 0, 0.0
    budget = 60.0
    while done < args.steps and t_total < budget:
        n = 1 if per is None else max(1, min(args.steps - done, int((budget - t_total) / max(per, 1e-6))))
        n = min(n, 25)
        o.close()
        s["maxIter"] = n
        o = oracle.Oracle(mesh, case.bc_fields(), s, threads=threads)
        t0 = time.perf_counter()
        o.run()
        dt = time.perf_counter() - t0
        done += n
        t_total += dt
        per = t_total / done
    value = mesh["nCells"] * done / t_total / 1e6
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": case.name, "cells": mesh["nCells"], "faces": mesh["nFaces"]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{done} SIMPLE iterations of {case.name} ({t_total:.1f} s)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU solver path; this arm runs the oracle's C restatement of it"}
    print(json.dumps(line, default=_json_scalar), flush=True)


def cpu_baseline_leg(case, mesh):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    s = dict(case.settings)
    s["maxIter"] = 2
    o = oracle.Oracle(mesh, case.bc_fields(), s, threads=threads)
    t0 = time.perf_counter()
    o.run()
    est = (time.perf_counter() - t0) / 2
    n = int(max(2, min(60, 12.0 / max(est, 1e-6))))
    s["maxIter"] = n
    o2 = oracle.Oracle(mesh, case.bc_fields(), s, threads=threads)
    t0 = time.perf_counter()
    o2.run()
    dt = time.perf_counter() - t0
    v = mesh["nCells"] * n / dt / 1e6
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} SIMPLE iterations of {case.name} from rest ({dt:.1f} s)"}


def reference_cuda_leg(case, iters, tol=0.0):
    """The reference's own CUDA solver (compiled unchanged from its sources,
    oracle/ref_build) on the same workload, timed by its CudaTimer span."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "axisim_ref")
    if not os.path.exists(ref_bin):
        return {"unavailable": "oracle/_ref/axisim_ref not built"}
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import tempfile
    import make_golden
    c = workload(1.0) if case is None else case
    c.settings["maxIter"] = iters
    c.settings["resTol"] = [tol, tol, tol]
    with tempfile.TemporaryDirectory() as d:
        spec, out = os.path.join(d, "spec.txt"), os.path.join(d, "out.bin")
        make_golden.write_spec(c, spec)
        r = subprocess.run([ref_bin, spec, out], capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return {"unavailable": "reference run failed: " + r.stderr.strip()[-200:]}
    # "reference solver: N cells, K iterations, converged C, T ms"
    import re
    m = re.search(r"reference solver: (\d+) cells, (\d+) iterations, converged (\d+), ([0-9.]+) ms", r.stdout)
    n, k, ms = int(m.group(1)), int(m.group(2)), float(m.group(4))
    return {"value": n * k / (ms / 1e3) / 1e6, "unit": UNIT, "iterations": k, "ms": ms,
            "note": "reference CUDA build (sm_100a, unchanged sources), CudaTimer over its SIMPLE loop"}


# DRAM bytes per launch per cell of the top kernels, from one ncu capture of this
# workload each (dram__bytes_read.sum + dram__bytes_write.sum per launch at
# 874,496 cells; FP64 sweep 88.4 MB).
NCU_TRAFFIC_PER_CELL = {"jacobi_uv": 88.36e6 / 874496,
                        # dram__bytes_read.sum 48.976 MB + dram__bytes_write.sum 0.179 MB per launch
                        "jacobi_uv32": (48.976384e6 + 0.178688e6) / 874496}


def pinned_like(a, fill=None):
    """A page-locked host array with a's shape and dtype, holding a copy of a
    (or `fill`): the host side of the e2e leg's copies."""
    import numpy as np
    import torch
    a = np.asarray(a)
    t = torch.empty(a.shape, dtype=torch.from_numpy(np.empty(0, a.dtype)).dtype, pin_memory=True)
    out = t.numpy()
    if fill is None:
        out[...] = a
    else:
        out.fill(fill)
    _PINNED.append(t)
    return out


_PINNED = []


def mesh_bytes(m):
    import numpy as np
    return int(sum(np.asarray(m[k]).nbytes for k in m if k not in ("nCells", "nFaces", "status")))


def measure(abi, mesh, bcs, settings, args, local, dist, prec, sampler=None):
    """W warm-up iterations, then K timed SIMPLE iterations (CUDA events inside
    the library) on one solver handle; returns the solver and the timing."""
    s = dict(settings)
    s["maxIter"] = max(3, args.warmup)
    s["resTol"] = [0.0, 0.0, 0.0]
    solver = abi.Solver(mesh, bcs, s, device=local, precision=prec)
    if args.momentum_sweeps != 1:
        solver.set_momentum_sweeps(args.momentum_sweeps)
    solver.solve()                       # warm-up (+ capture of the iteration graph)
    solver.set_max_iter(args.steps, tol=0.0)
    barrier(dist)
    if sampler:
        sampler.start()
        time.sleep(0.3)
    r = solver.solve(cont=True)          # K timed iterations
    barrier(dist)
    clocks = sampler.stop() if sampler else None
    assert r["iterations"] == args.steps, r
    return solver, max_over_ranks(dist, r["ms"]), clocks


def time_to_residual(abi, case, local, prec, tol=1e-6, fcg_iters=0):
    c = dict(case.settings)
    c["resTol"] = [tol, tol, tol]
    mesh = case.packed(abi.multiblock)
    if fcg_iters:
        c["mgMaxIter"] = fcg_iters
        s = abi.Solver(mesh, case.bc_fields(), c, device=local, precision=prec, pressure_solver=abi.PSOLVE_FCG)
    else:
        s = abi.Solver(mesh, case.bc_fields(), c, device=local, precision=prec)
    r = s.solve()
    out = {"iterations": r["iterations"], "converged": r["converged"], "seconds": r["ms"] / 1e3,
           "residuals": r["residual"]}
    fields = {f: s.get(f) for f in ("u", "v", "p")}
    s.close()
    return out, mesh, fields


def _rel(a, b):
    import numpy as np
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def converged_reference(abi, case, mesh, local, chunk=2000, change=1e-9, budget=60000):
    """The FP64 fixed point of the SIMPLE iteration on `case`: FP64 with the
    flexible-CG p' solve (a fixed point does not depend on the p' solver),
    iterated in chunks until u, v and p change by at most `change` relative L2
    over one chunk. Returns (fields, info)."""
    st = dict(case.settings)
    st.update(maxIter=chunk, resTol=[0.0] * 3, mgMaxIter=5)
    s = abi.Solver(mesh, case.bc_fields(), st, device=local, precision=abi.PREC_FP64,
                   pressure_solver=abi.PSOLVE_FCG)
    prev, iters, secs, d = None, 0, 0.0, None
    while iters < budget:
        r = s.solve(cont=iters > 0)
        iters += r["iterations"]
        secs += r["ms"] / 1e3
        cur = {f: s.get(f) for f in ("u", "v", "p")}
        if prev is not None:
            d = max(_rel(cur[f], prev[f]) for f in cur)
            if d <= change:
                break
        prev = cur
    s.close()
    return cur, {"iterations": iters, "seconds": secs, "last_chunk_change": d, "chunk": chunk,
                 "how": "FP64, flexible-CG p' solve (5 iterations), iterated until a chunk changes u, v, p by "
                        f"<= {change:g} relative L2"}


def run_to_accuracy(abi, case, mesh, ref, local, prec, psolve=None, fcg_iters=5, target=1e-6, chunk=500,
                    budget=40000):
    """Device time until u, v and p are all within `target` relative L2 of the
    converged FP64 fields `ref`: SIMPLE iterations in chunks of `chunk` (no
    residual stop), the fields compared after each chunk. Chunks continue one
    run, so the iterates are those of one uninterrupted solve."""
    st = dict(case.settings)
    st.update(maxIter=chunk, resTol=[0.0] * 3)
    kw = {}
    if psolve == abi.PSOLVE_FCG:
        st["mgMaxIter"] = fcg_iters
        kw = {"pressure_solver": abi.PSOLVE_FCG}
    s = abi.Solver(mesh, case.bc_fields(), st, device=local, precision=prec, **kw)
    iters, secs, err = 0, 0.0, None
    while iters < budget:
        r = s.solve(cont=iters > 0)
        iters += r["iterations"]
        secs += r["ms"] / 1e3
        err = {f: _rel(s.get(f), ref[f]) for f in ("u", "v", "p")}
        if max(err.values()) <= target:
            break
    s.close()
    return {"reached": max(err.values()) <= target, "seconds": secs, "iterations": iters, "error_vs_fp64": err,
            "chunk": chunk}


def accuracy_leg(abi, local, scale=1.0):
    """Time to fields within 1e-6 relative L2 (u, v, p) of the converged FP64
    solution of the steady expansion, for the reference method in FP64 and for
    the flexible-CG p' solve in FP64 and mixed precision."""
    from axisim import cases
    case = cases.expansion(scale=scale, max_iter=60000, tol=1e-6)
    mesh = abi.multiblock(case.blocks)
    ref, info = converged_reference(abi, case, mesh, local)
    out = {"workload": case.name, "cells": int(mesh["nCells"]), "target_rel_l2": 1e-6, "reference": info}
    out["plain_fp64"] = run_to_accuracy(abi, case, mesh, ref, local, abi.PREC_FP64, budget=45000)
    out["mixed_fcg"] = run_to_accuracy(abi, case, mesh, ref, local, abi.PREC_MIXED, abi.PSOLVE_FCG)
    out["fcg_fp64"] = run_to_accuracy(abi, case, mesh, ref, local, abi.PREC_FP64, abi.PSOLVE_FCG)
    for k in ("mixed_fcg", "fcg_fp64"):
        # the reference method's time over this arm's; where the reference
        # method misses the target the ratio is a lower bound on the speed-up
        out[k]["plain_seconds_over_arm_seconds"] = out["plain_fp64"]["seconds"] / out[k]["seconds"]
    return out


def precision_leg(abi, local, scale=1.0, iters=5000):
    """Mixed precision against the all-FP64 run of the same solver on the
    steady expansion: the same `iters` SIMPLE iterations from rest in both,
    then the relative L2 differences of u, v, p and of the flow quantities the
    case is judged by (centreline u(z), pressure drop, recirculation length)."""
    from axisim import cases
    case = cases.expansion(scale=scale, max_iter=iters, tol=0.0)
    mesh = abi.multiblock(case.blocks)
    f, t = {}, {}
    for name, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        s = abi.Solver(mesh, case.bc_fields(), dict(case.settings, resTol=[0.0] * 3), device=local, precision=prec)
        r = s.solve()
        t[name] = r["ms"] / 1e3
        f[name] = {k: s.get(k) for k in ("u", "v", "p")}
        s.close()
    e64 = cases.expansion_metrics(mesh, f["fp64"]["u"], f["fp64"]["p"])
    emx = cases.expansion_metrics(mesh, f["mixed"]["u"], f["mixed"]["p"])
    return {"iterations": iters, "seconds": t,
            "error_vs_fp64": {"u": _rel(f["mixed"]["u"], f["fp64"]["u"]), "v": _rel(f["mixed"]["v"], f["fp64"]["v"]),
                              "p": _rel(f["mixed"]["p"], f["fp64"]["p"]),
                              "centreline_u": _rel(emx["centre_u"], e64["centre_u"]),
                              "pressure_drop": abs(emx["dp"] - e64["dp"]) / abs(e64["dp"]),
                              "recirculation_length_m": abs(emx["recirculation_length"] - e64["recirculation_length"])},
            "fp64_pressure_drop_Pa": e64["dp"], "fp64_recirculation_length_m": e64["recirculation_length"]}


def bullet_leg(abi, local, scale=1.0, steps=20, warmup=3):
    """The unstructured bullet (485,868 triangles at scale 1): SIMPLE
    iterations per second in mixed precision and FP64 (device time of `steps`
    iterations after `warmup`), the mixed fields' error against the FP64 run
    of the same iterations, and the FP32 momentum sweep on W = 3 slots against
    the HBM peak (eager replay, CUDA events)."""
    from axisim import cases
    case = cases.bullet(scale=scale, max_iter=warmup, tol=0.0)
    mesh = case.mesh
    N = int(mesh["nCells"])
    peak, kind = peaks()
    out = {"workload": case.name, "cells": N, "steps": steps, "gradient": "least squares + non-orthogonal corrector"}
    fields = {}
    for name, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
        s = abi.Solver(mesh, case.bc_fields(), dict(case.settings, resTol=[0.0] * 3), device=local, precision=prec)
        s.solve()
        s.set_max_iter(steps, tol=0.0)
        r = s.solve(cont=True)
        out[name] = {"Mcell_iter_s": N * steps / (r["ms"] / 1e3) / 1e6, "ms_per_iter": r["ms"] / steps}
        fields[name] = {k: s.get(k) for k in ("u", "v", "p")}
        if name == "mixed":
            st = {k["name"]: k for k in s.profile(2)}
            for kname in ("jacobi_uv32_tiles", "jacobi_uv32"):
                j = st.get(kname)
                if j:
                    gbs = (j["bytes"] / j["launches"]) / (j["ms"] / j["launches"] / 1e3) / 1e9
                    out["sweep_roofline"] = {"kernel": kname + " (W=3)", "achieved": gbs, "peak": peak,
                                             "peak_kind": kind, "unit": "GB/s", "frac": gbs / peak,
                                             "launches_per_iter": j["launches"] / 2.0,
                                             "ms_per_iter": j["ms"] / 2.0}
                    break
        s.close()
    out["mixed_error_vs_fp64"] = {k: _rel(fields["mixed"][k], fields["fp64"][k]) for k in ("u", "v", "p")}
    out["note"] = f"both arms from rest, {warmup + steps} iterations; errors after the same iterations"
    return out


def batch_leg(abi, local, n_cases=256, steps=50, seq_sample=32):
    """Config 4 at its stated size: all `n_cases` cases of the random mix (seed
    0) packed into one mesh and advanced together for `steps` SIMPLE
    iterations (device time, per-case hierarchies), against one handle per case
    for a sample of `seq_sample` cases (every n_cases/seq_sample-th), whose
    device time per cell-iteration stands for the sequential solve of all."""
    from axisim import batch
    cs = batch.random_cases(n_cases, seed=0)
    meshes = [abi.multiblock(c.blocks) for c in cs]
    union, start, bcs = batch.pack_union(meshes, [c.groups for c in cs])
    settings = dict(cs[0].settings)
    settings.update(maxIter=3, resTol=[0.0] * 3)
    g = abi.Solver(union, bcs, settings, device=local)
    g.set_batch(start)
    g.solve()
    g.set_max_iter(steps, tol=0.0)
    rb = g.solve(cont=True)
    g.close()
    seq_ms, seq_cells = 0.0, 0
    pick = list(range(0, n_cases, max(1, n_cases // seq_sample)))[:seq_sample]
    for i in pick:
        c, m = cs[i], meshes[i]
        s = dict(c.settings)
        s.update(maxIter=3, resTol=[0.0] * 3)
        h = abi.Solver(m, c.bc_fields(), s, device=local)
        h.solve()
        h.set_max_iter(steps, tol=0.0)
        seq_ms += h.solve(cont=True)["ms"]
        seq_cells += int(m["nCells"])
        h.close()
    cells = int(union["nCells"])
    seq_rate = seq_cells * steps / (seq_ms / 1e3) / 1e6
    batched = cells * steps / (rb["ms"] / 1e3) / 1e6
    return {"cases": n_cases, "cells": cells, "steps": steps, "batched_Mcell_iter_s": batched,
            "sequential_Mcell_iter_s": seq_rate, "speedup": batched / seq_rate, "batched_ms": rb["ms"],
            "sequential_sample": {"cases": len(pick), "cells": seq_cells, "ms": seq_ms},
            "note": f"random pipe/expansion case mix (seed 0), all {n_cases} cases in one packed mesh; the "
                    f"sequential rate is one handle per case over every {max(1, n_cases // seq_sample)}th case"}


def batch_converge_leg(abi, local, n_cases=16, scale=0.05, max_iter=20000):
    """Time to all-converged for a small batch vs the sum of the sequential solves."""
    from axisim import batch
    cs = batch.random_cases(n_cases, seed=0, scale=scale, max_iter=max_iter, tol=1e-6)
    meshes = [abi.multiblock(c.blocks) for c in cs]
    union, start, bcs = batch.pack_union(meshes, [c.groups for c in cs])
    g = abi.Solver(union, bcs, cs[0].settings, device=local)
    g.set_batch(start)
    rb = g.solve()
    conv_at, _ = g.batch_status()
    g.close()
    seq_ms, seq_conv = 0.0, 0
    for c, m in zip(cs, meshes):
        h = abi.Solver(m, c.bc_fields(), c.settings, device=local)
        r = h.solve()
        seq_ms += r["ms"]
        seq_conv += int(r["converged"])
        h.close()
    return {"cases": n_cases, "cells": int(union["nCells"]), "batched_seconds": rb["ms"] / 1e3,
            "batched_iterations": rb["iterations"], "batched_converged_cases": int((conv_at >= 0).sum()),
            "sequential_seconds": seq_ms / 1e3, "sequential_converged_cases": seq_conv,
            "note": f"random pipe/expansion case mix at scale {scale}, tolerance 1e-6, at most {max_iter} iterations"}


def transient_leg(abi, local, scale=1.512, warm_steps=2, timed_steps=3, max_iter=300, train_steps=600):
    """The transient pulsatile sudden expansion (1,998,855 cells at scale
    1.512, BDF2, dt 1e-4): after `warm_steps` untimed steps, the device time of
    `timed_steps` steps per arm, and the error of each arm's u, v, p after the
    last step against the converged FP64 solution of the same steps (FP64,
    flexible-CG p' solve with a tight Krylov tolerance, every step to a 1e-9
    residual or 400 iterations). Arms: the reference method (FP64, 3 V-cycles; at most
    `max_iter` SIMPLE iterations per step, which takes about the wall time of
    the Krylov arms), FP64 and mixed precision with the flexible-CG p' solve,
    and mixed with the learned first Krylov step (network trained on the GPU on
    p' systems harvested during its warm-up steps). Each Krylov arm runs with
    the loosest per-step residual tolerance of 1e-6, 1e-7, 1e-8 that puts its
    fields within 1e-6 relative L2 of the converged ones."""
    import numpy as np
    from axisim import cases
    case = cases.pulsatile_expansion(scale=scale, dt=1e-4, steps=warm_steps, max_iter=max_iter, tol=1e-6)
    mesh = case.packed(abi.multiblock)
    dt = case.settings["dt"]

    def arm(prec, psolve, tol=1e-6, ptol=1e-2, learned=False, cap=max_iter, fcg_cap=100):
        st = dict(case.settings)
        st["maxIter"] = cap
        st["resTol"] = [tol] * 3
        if psolve == abi.PSOLVE_FCG:
            st["mgMaxIter"] = 300 if learned else fcg_cap  # the learned arm harvests converged p' while warming up
        s = abi.Solver(mesh, case.bc_fields(), st, device=local, precision=prec, pressure_solver=psolve,
                       pressure_tol=ptol if not learned else 1e-6, prolong_scale=2.0)
        info = {"step_tol": tol}
        if learned:
            s.learned_harvest(1, 64)
        s.solve()  # warm-up steps (harvesting for the learned arm)
        if learned:
            s.learned_harvest(0)
            n = s.learned_sample_count()
            s.learned_init(abi.NET_BF16_WEIGHTS, seed=1)
            t0 = time.perf_counter()
            losses = s.learned_train(train_steps, lr=1e-3, seed=0, first=0, count=max(1, n - 8))
            t_train = time.perf_counter() - t0
            held = [s.learned_grad(i)[0] for i in range(max(1, n - 8), n)]
            info["training"] = {"samples": n, "steps": train_steps, "seconds": t_train,
                                "loss_first_50": float(np.mean(losses[:50])),
                                "loss_last_50": float(np.mean(losses[-50:])),
                                "held_out_loss": float(np.mean(held)) if held else None,
                                "loss": "energy-norm error left after the best scaling of the output"}
            s.settings["mgMaxIter"] = fcg_cap
            abi.lib().axisim_set_pressure_solver(s.h, abi.PSOLVE_FCG, ptol, 2.0)
            s.learned_enable(abi.LEARNED_FIRST_STEP)
        s.settings["tEnd"] = dt
        steps, secs, iters = [], 0.0, 0
        pp0 = s.pressure_stats() if psolve == abi.PSOLVE_FCG else (0, 0)
        for _ in range(timed_steps):
            s.set_max_iter(cap, tol=tol)
            r = s.solve(cont=True)
            steps.append([r["iterations"], bool(r["converged"]), round(r["ms"] / 1e3, 4)])
            secs += r["ms"] / 1e3
            iters += r["iterations"]
        info.update(seconds=secs, iterations=iters, steps_converged=sum(1 for x in steps if x[1]),
                    steps=steps, final_residual=r["residual"])
        if psolve == abi.PSOLVE_FCG:
            pp1 = s.pressure_stats()
            info["krylov_iterations_per_solve"] = (pp1[1] - pp0[1]) / max(1, pp1[0] - pp0[0])
        if learned:
            info["learned"] = s.learned_stats()
            a, f = info["learned"]["applied"], info["learned"]["fallbacks"]
            info["fallback_rate"] = f / max(1, a + f)
        fields = {k: s.get(k) for k in ("u", "v", "p")}
        s.close()
        return info, fields

    out = {"workload": case.name, "cells": int(mesh["nCells"]), "dt": dt, "warm_steps": warm_steps,
           "timed_steps": timed_steps, "max_iter_per_step": max_iter, "target_rel_l2": 1e-6}
    ref_info, ref = arm(abi.PREC_FP64, abi.PSOLVE_FCG, tol=1e-9, ptol=1e-3, cap=400, fcg_cap=200)
    out["reference"] = {k: ref_info[k] for k in ("seconds", "iterations", "steps_converged", "step_tol",
                                                 "final_residual")}
    out["reference"]["how"] = ("FP64, flexible-CG p' solve (relative tolerance 1e-3), every step to a 1e-9 "
                               "residual or 400 iterations")

    def err(f):
        return {k: _rel(f[k], ref[k]) for k in ("u", "v", "p")}

    out["plain_fp64"], f = arm(abi.PREC_FP64, abi.PSOLVE_VCYCLES)
    out["plain_fp64"]["error_vs_fp64"] = err(f)
    # the reference method given ten times the iterations per step
    out["plain_fp64_long"], f = arm(abi.PREC_FP64, abi.PSOLVE_VCYCLES, cap=10 * max_iter)
    out["plain_fp64_long"]["error_vs_fp64"] = err(f)
    out["plain_fp64_long"]["within_target"] = max(out["plain_fp64_long"]["error_vs_fp64"].values()) <= 1e-6
    chosen = None
    for tol in (1e-6, 1e-7, 1e-8):
        info, f = arm(abi.PREC_MIXED, abi.PSOLVE_FCG, tol=tol, cap=3000)
        info["error_vs_fp64"] = err(f)
        out.setdefault("mixed_fcg_ladder", []).append(
            {"step_tol": tol, "seconds": info["seconds"], "max_error": max(info["error_vs_fp64"].values())})
        out["mixed_fcg"] = info
        chosen = tol
        if max(info["error_vs_fp64"].values()) <= 1e-6:
            break
    out["fcg_fp64"], f = arm(abi.PREC_FP64, abi.PSOLVE_FCG, tol=chosen, cap=3000)
    out["fcg_fp64"]["error_vs_fp64"] = err(f)
    out["learned_mixed_fcg"], f = arm(abi.PREC_MIXED, abi.PSOLVE_FCG, tol=chosen, cap=3000, learned=True)
    out["learned_mixed_fcg"]["error_vs_fp64"] = err(f)
    out["plain_fp64"]["within_target"] = max(out["plain_fp64"]["error_vs_fp64"].values()) <= 1e-6
    longer = out["plain_fp64_long"]
    for k in ("mixed_fcg", "fcg_fp64", "learned_mixed_fcg"):
        out[k]["within_target"] = max(out[k]["error_vs_fp64"].values()) <= 1e-6
        # the reference method's time (ten times the iteration cap) over this
        # arm's; where the reference method still misses the target the ratio
        # is a lower bound on the speed-up
        out[k]["plain_seconds_over_arm_seconds"] = longer["seconds"] / out[k]["seconds"]
        out[k]["plain_ratio_is_lower_bound"] = not longer["within_target"]
    return out


def network_leg(abi, local, scale=1.512, infer=5, train=5):
    """The learned p' network alone on the transient mesh (1,998,855 cells at
    scale 1.512): mean host-clock time of `infer` predictions and `train` Adam
    steps on a synthetic sample (after one warm-up of each)."""
    import numpy as np
    from axisim import cases
    case = cases.pulsatile_expansion(scale=scale, dt=1e-4, steps=1, max_iter=1, tol=1e-30)
    mesh = case.packed(abi.multiblock)
    N = int(mesh["nCells"])
    s = abi.Solver(mesh, case.bc_fields(), case.settings, device=local)
    rng = np.random.default_rng(0)
    af = np.where(mesh["faceNeighbor"][mesh["cellFaceIDs"]] >= 0, -1.0, 0.0)
    s.learned_harvest(0, 1)
    s.learned_add_sample(rng.standard_normal(N), rng.standard_normal(N), np.full(N, 4.1), np.zeros(N), af)
    n_params = s.learned_init(abi.NET_BF16_WEIGHTS, seed=0)
    r, ac, d = rng.standard_normal(N), np.full(N, 4.1), np.zeros(N)
    s.learned_predict(r, ac, d)
    s.learned_train(1)
    t0 = time.perf_counter()
    for _ in range(infer):
        s.learned_predict(r, ac, d)
    t_inf = (time.perf_counter() - t0) / infer
    t0 = time.perf_counter()
    s.learned_train(train)
    t_tr = (time.perf_counter() - t0) / train
    s.close()
    return {"cells": N, "parameters": n_params,
            "predict_ms": t_inf * 1e3, "train_step_ms": t_tr * 1e3,
            "note": "predict includes the host copies of r, A_C, deficit and the result"}


def scalars_leg(abi, local, scale=1.0, iters=20):
    """Energy + concentration (Michaelis-Menten wall behind a layer) on the
    workload mesh, FP64 SIMPLE iterations: device time per iteration with and
    without the scalars (CUDA events over `iters` iterations after a warm run
    of the same length), and the per-kernel profile of the scalar step
    (algorithmic bytes / CUDA-event time, eager replay)."""
    from axisim import cases
    hbm, src = peaks()
    flow = workload(scale)
    flow.settings.update(maxIter=iters)
    both = cases.with_scalars(workload(scale), wall_c=cases.michaelis_menten(1e-3, 0.2),
                              wall_layers=[(1e-6, 1e-4)], D=1e-6)
    both.settings.update(maxIter=iters)
    mesh = abi.multiblock(flow.blocks)
    out = {"cells": int(mesh["nCells"]), "iterations": iters, "peak_gbs": hbm, "peak_source": src}
    for name, case in (("flow", flow), ("flow_T_C", both)):
        s = abi.Solver(mesh, case.bc_fields(), case.settings, device=local)
        s.solve()
        r = s.solve(cont=True)
        out[name + "_ms_per_iter"] = r["ms"] / max(1, r["iterations"])
        if name == "flow_T_C":
            prof = {}
            for k in s.profile(3):
                if k["name"] in ("scalar", "scalar_wall", "jacobi_TC", "gs_TC", "jacobi_T", "jacobi_C", "gs_T", "gs_C",
                                 "scalar_residual", "momentum"):
                    gbs = k["bytes"] / (k["ms"] * 1e-3) / 1e9 if k["ms"] > 0 else 0.0
                    prof[k["name"]] = {"launches": k["launches"], "ms_per_launch": k["ms"] / k["launches"],
                                       "GBps": gbs, "frac_of_peak": gbs / hbm}
            out["kernels"] = prof
        s.close()
    out["scalar_overhead"] = out["flow_T_C_ms_per_iter"] / out["flow_ms_per_iter"] - 1.0
    return out


def _r(x, n=4):
    """x to n significant digits (JSON-compact)."""
    if isinstance(x, float):
        return float(f"{x:.{n}g}")
    return x


def summary(line):
    """The like-for-like numbers in one short object, printed last in the line
    (the end of a long line is what survives truncation)."""
    out = {"Mcell_iter_s": {"mixed": _r(line["value"])}}
    if "plain_fp64" in line:
        out["Mcell_iter_s"]["fp64"] = _r(line["plain_fp64"]["value"])
    rc = line.get("reference_cuda", {})
    if "value" in rc:
        out["Mcell_iter_s"]["reference_cuda_build"] = _r(rc["value"])
    if "cpu_baseline" in line:
        out["Mcell_iter_s"]["cpu_port"] = _r(line["cpu_baseline"]["value"])
    if "e2e" in line:
        out["e2e_Mcell_iter_s"] = _r(line["e2e"]["value"])
    pr = line.get("precision")
    if pr:
        e = pr["error_vs_fp64"]
        out["mixed_vs_fp64_same_iterations"] = {"it": pr["iterations"], "uvp": _r(max(e["u"], e["v"], e["p"]), 2),
                                                "dp": _r(e["pressure_drop"], 2)}
    acc = line.get("accuracy")
    if acc:
        out["to_1e-6_of_fp64_fields_874k"] = {
            k: {"s": _r(acc[k]["seconds"]), "it": acc[k]["iterations"], "reached": acc[k]["reached"],
                "err": _r(max(acc[k]["error_vs_fp64"].values()), 2)}
            for k in ("plain_fp64", "fcg_fp64", "mixed_fcg") if k in acc}
    tr = line.get("transient")
    if tr:
        t = {}
        for k in ("plain_fp64", "plain_fp64_long", "fcg_fp64", "mixed_fcg", "learned_mixed_fcg"):
            if k not in tr:
                continue
            a = tr[k]
            t[k] = {"s": _r(a["seconds"]), "steps_conv": a["steps_converged"],
                    "err": _r(max(a["error_vs_fp64"].values()), 2)}
            if "plain_seconds_over_arm_seconds" in a:
                t[k]["plain_long_s_over_s"] = _r(a["plain_seconds_over_arm_seconds"], 3)
                t[k]["lower_bound"] = a.get("plain_ratio_is_lower_bound", False)
            if "fallback_rate" in a:
                t[k]["fallback_rate"] = _r(a["fallback_rate"], 3)
        t["step_tol"] = tr.get("mixed_fcg", {}).get("step_tol")
        out["transient_2M_3steps"] = t
    b = line.get("batch")
    if b:
        out["batch"] = {"cases": b["cases"], "cells": b["cells"], "batched": _r(b["batched_Mcell_iter_s"]),
                        "sequential": _r(b["sequential_Mcell_iter_s"])}
    bc = line.get("batch_to_converged")
    if bc:
        out["batch_to_converged"] = {"cases": bc["cases"], "s": _r(bc["batched_seconds"]),
                                     "seq_s": _r(bc["sequential_seconds"]),
                                     "conv": [bc["batched_converged_cases"], bc["sequential_converged_cases"]]}
    bu = line.get("bullet")
    if bu:
        out["bullet_485k"] = {"mixed": _r(bu["mixed"]["Mcell_iter_s"]), "fp64": _r(bu["fp64"]["Mcell_iter_s"]),
                              "err": _r(max(bu["mixed_error_vs_fp64"].values()), 2),
                              "sweep_frac": _r(bu.get("sweep_roofline", {}).get("frac"), 3)}
    return out


def run_b200(args):
    world, rank, local, dist = dist_setup(args.gpus)
    import numpy as np
    import axisim.abi as abi
    from axisim import cases
    if not os.path.exists(abi.LIB_PATH):
        abi.build()
    if args.network_only:
        if rank == 0:
            print(json.dumps(network_leg(abi, local, scale=1.512 * args.scale), default=_json_scalar), flush=True)
        return
    if args.transient_only:
        if rank == 0:
            print(json.dumps(transient_leg(abi, local, scale=1.512 * args.scale), default=_json_scalar), flush=True)
        return
    if args.bullet_only:
        if rank == 0:
            print(json.dumps(bullet_leg(abi, local, scale=args.scale, steps=max(1, args.steps)),
                             default=_json_scalar), flush=True)
        return
    if args.accuracy_only:
        if rank == 0:
            print(json.dumps(accuracy_leg(abi, local, scale=args.scale), default=_json_scalar), flush=True)
        return
    if args.scalars_only:
        if rank == 0:
            print(json.dumps(scalars_leg(abi, local, scale=args.scale, iters=max(1, args.steps)),
                             default=_json_scalar), flush=True)
        return
    case = workload(args.scale)
    mesh = abi.multiblock(case.blocks)
    N = mesh["nCells"]
    bcs = case.bc_fields()
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    sampler = ClockSampler(local) if rank == 0 else None
    solver, ms, clocks = measure(abi, mesh, bcs, case.settings, args, local, dist, prec, sampler)
    value = world * N * args.steps / (ms / 1e3) / 1e6

    # per-kernel roofline: two eagerly replayed iterations with events after every launch
    stats = solver.profile(iterations=2)
    solver.close()
    launches_per_iter = sum(k["launches"] for k in stats) / 2.0
    top = max(stats, key=lambda k: k["ms"])
    peak, peak_kind = peaks()
    achieved = (top["bytes"] / top["launches"]) / (top["ms"] / top["launches"] / 1e3) / 1e9
    total_bytes = sum(k["bytes"] for k in stats) / 2.0
    total_ms = sum(k["ms"] for k in stats) / 2.0
    traffic = NCU_TRAFFIC_PER_CELL.get(top["name"])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32" if prec == abi.PREC_MIXED else "f64", "data": "synthetic",
        "config": {"workload": case.name, "cells": N, "faces": mesh["nFaces"], "precision": args.precision,
                   "convection": "second-order upwind", "gradient": "least squares",
                   "momentum_solver": "Jacobi x20 (u,v fused)" + (
                       ", %d sweeps per launch" % args.momentum_sweeps if args.momentum_sweeps != 1 else ""),
                   "pressure_solver": "agglomeration MG, 3 V-cycles",
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": "inputs larger than L2 (mesh + fields ~%.0f MB per iteration)" % (
                       (mesh_bytes(mesh) + N * 8 * 40) / 1e6)},
        "roofline": {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic * N if traffic else None,
                     "bytes_per_launch": top["bytes"] / top["launches"],
                     "ms_per_launch": top["ms"] / top["launches"],
                     "iteration_algorithmic_GBps": total_bytes / (total_ms / 1e3) / 1e9},
        "kernels": {k["name"]: {"launches_per_iter": k["launches"] / 2.0, "ms_per_iter": k["ms"] / 2.0,
                                "GBps": (k["bytes"] / (k["ms"] / 1e3) / 1e9) if k["ms"] > 0 else 0.0}
                    for k in stats},
        "gpu_launches": int(round(launches_per_iter * args.steps)),
        "clocks": clocks,
    }
    if prec == abi.PREC_MIXED:
        s64, ms64, _ = measure(abi, mesh, bcs, case.settings, args, local, dist, abi.PREC_FP64)
        s64.close()
        line["plain_fp64"] = {"value": world * N * args.steps / (ms64 / 1e3) / 1e6, "unit": UNIT,
                              "ms_per_step": ms64 / args.steps}
    if rank == 0 and not args.no_extras and world == 1:
        # e2e through the public API from pinned host buffers: case upload + K
        # iterations + field download
        pmesh = {k: (pinned_like(v) if isinstance(v, np.ndarray) else v) for k, v in mesh.items()}
        zeros = pinned_like(np.empty(N), fill=0.0)
        zf = pinned_like(np.empty(mesh["nFaces"]), fill=0.0)
        outs = [pinned_like(np.empty(N), fill=0.0) for _ in range(3)]
        s2 = dict(case.settings)
        s2["maxIter"] = args.steps
        s2["resTol"] = [0.0, 0.0, 0.0]
        t0 = time.perf_counter()
        sol2 = abi.Solver(pmesh, bcs, s2, device=local, precision=prec)
        for f in ("u", "v", "p"):
            sol2.set(f, zeros)
        sol2.set("mDot", zf)
        r2 = sol2.solve(cont=True)
        for f, o in zip(("u", "v", "p"), outs):
            sol2.get(f, out=o)
        t_e2e = time.perf_counter() - t0
        setup = sol2.setup_profile()
        sol2.close()
        h2d = mesh_bytes(mesh) + sum(b[k].nbytes for b in bcs.values() for k in b) + 3 * N * 8 + mesh["nFaces"] * 8
        d2h = sum(o.nbytes for o in outs)
        line["e2e"] = {"value": N * r2["iterations"] / t_e2e / 1e6, "unit": UNIT,
                       "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                       "seconds": t_e2e,
                       "note": "host clock around set_mesh/set_bc/set_field/solve/get_field, host arrays page-locked",
                       "setup_ms": {k: round(v["ms"], 2) for k, v in setup.items()}}
        line["cpu_baseline"] = cpu_baseline_leg(case, mesh)
        line["precision"] = precision_leg(abi, local, scale=args.scale)
        line["accuracy"] = accuracy_leg(abi, local, scale=args.scale)
        ttr = {}
        pc = cases.pipe(max_iter=50000, tol=1e-6)
        p64, _, _ = time_to_residual(abi, pc, local, abi.PREC_FP64)
        pmx, _, _ = time_to_residual(abi, pc, local, abi.PREC_MIXED)
        ref_pipe = reference_cuda_leg(cases.pipe(max_iter=50000, tol=1e-6), 50000, tol=1e-6)
        ttr[pc.name] = {"plain_fp64": p64, "mixed": pmx}
        if "ms" in ref_pipe:
            ttr[pc.name]["reference_cuda"] = {"seconds": ref_pipe["ms"] / 1e3, "iterations": ref_pipe["iterations"]}
        line["time_to_residual"] = ttr
        line["transient"] = transient_leg(abi, local, scale=1.512 * args.scale)
        line["batch"] = batch_leg(abi, local)
        line["batch_to_converged"] = batch_converge_leg(abi, local)
        line["bullet"] = bullet_leg(abi, local, scale=args.scale)
        line["reference_cuda"] = reference_cuda_leg(workload(args.scale), min(args.steps, 100))
    if "plain_fp64" in line:
        line["plain_fp64"] = line.pop("plain_fp64")  # like-for-like numbers go to the end of the line
    if rank == 0 and world == 1:
        line["summary"] = summary(line)
    if rank == 0:
        print(json.dumps(line, default=_json_scalar), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
