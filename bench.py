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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="cell-count scale of the workload (1 = full size)")
    ap.add_argument("--no-extras", action="store_true", help="skip cpu baseline / e2e / time-to-residual legs")
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
    print(json.dumps(line), flush=True)


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


def reference_cuda_leg(case, iters):
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
    c.settings["resTol"] = [0.0, 0.0, 0.0]
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


def mesh_bytes(m):
    import numpy as np
    return int(sum(np.asarray(m[k]).nbytes for k in m if k not in ("nCells", "nFaces", "status")))


def run_b200(args):
    world, rank, local, dist = dist_setup(args.gpus)
    import numpy as np
    import axisim.abi as abi
    if not os.path.exists(abi.LIB_PATH):
        abi.build()
    case = workload(args.scale)
    mesh = abi.multiblock(case.blocks)
    N = mesh["nCells"]
    bcs = case.bc_fields()
    s = dict(case.settings)
    s["maxIter"] = max(3, args.warmup)
    s["resTol"] = [0.0, 0.0, 0.0]
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    solver = abi.Solver(mesh, bcs, s, device=local, precision=prec)
    solver.solve()                       # warm-up: W SIMPLE iterations (+ capture of the iteration graph)
    solver.set_max_iter(args.steps, tol=0.0)
    sampler = ClockSampler(local) if rank == 0 else None
    barrier(dist)
    if sampler:
        sampler.start()
        time.sleep(0.3)
    r = solver.solve(cont=True)          # K timed SIMPLE iterations (CUDA events inside)
    barrier(dist)
    clocks = sampler.stop() if sampler else None
    assert r["iterations"] == args.steps, r
    ms = max_over_ranks(dist, r["ms"])
    value = world * N * args.steps / (ms / 1e3) / 1e6

    # per-kernel roofline: two eagerly replayed iterations with events after every launch
    stats = solver.profile(iterations=2)
    launches_per_iter = sum(k["launches"] for k in stats) / 2.0
    top = max(stats, key=lambda k: k["ms"])
    peak, peak_kind = peaks()
    achieved = (top["bytes"] / top["launches"]) / (top["ms"] / top["launches"] / 1e3) / 1e9
    total_bytes = sum(k["bytes"] for k in stats) / 2.0
    total_ms = sum(k["ms"] for k in stats) / 2.0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": case.name, "cells": N, "faces": mesh["nFaces"], "precision": args.precision,
                   "convection": "second-order upwind", "gradient": "least squares",
                   "momentum_solver": "Jacobi x20 (u,v fused)", "pressure_solver": "agglomeration MG, 3 V-cycles",
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": "inputs larger than L2 (mesh + fields ~%.0f MB per iteration)" % (
                       (mesh_bytes(mesh) + N * 8 * 40) / 1e6)},
        "roofline": {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "bytes_per_launch": top["bytes"] / top["launches"],
                     "ms_per_launch": top["ms"] / top["launches"],
                     "iteration_algorithmic_GBps": total_bytes / (total_ms / 1e3) / 1e9},
        "kernels": {k["name"]: {"launches_per_iter": k["launches"] / 2.0, "ms_per_iter": k["ms"] / 2.0,
                                "GBps": (k["bytes"] / (k["ms"] / 1e3) / 1e9) if k["ms"] > 0 else 0.0}
                    for k in stats},
        "gpu_launches": int(round(launches_per_iter * args.steps)),
        "clocks": clocks,
    }
    solver.close()
    if rank == 0 and not args.no_extras and world == 1:
        # e2e through the public API from host buffers: case upload + K iterations + field download
        t0 = time.perf_counter()
        s2 = dict(case.settings)
        s2["maxIter"] = args.steps
        s2["resTol"] = [0.0, 0.0, 0.0]
        sol2 = abi.Solver(mesh, bcs, s2, device=local)
        zeros = np.zeros(N)
        for f in ("u", "v", "p"):
            sol2.set(f, zeros)
        sol2.set("mDot", np.zeros(mesh["nFaces"]))
        r2 = sol2.solve(cont=True)
        outs = [sol2.get(f) for f in ("u", "v", "p")]
        t_e2e = time.perf_counter() - t0
        sol2.close()
        h2d = mesh_bytes(mesh) + sum(b[k].nbytes for b in bcs.values() for k in b) + 3 * N * 8 + mesh["nFaces"] * 8
        d2h = sum(o.nbytes for o in outs)
        line["e2e"] = {"value": N * r2["iterations"] / t_e2e / 1e6, "unit": UNIT,
                       "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                       "seconds": t_e2e, "note": "host clock around set_mesh/set_bc/set_field/solve/get_field"}
        line["cpu_baseline"] = cpu_baseline_leg(case, mesh)
        line["reference_cuda"] = reference_cuda_leg(workload(args.scale), min(args.steps, 100))
        # time to residual 1e-6 on the pipe, CUDA-event time inside solve
        from axisim import cases
        pc = cases.pipe(max_iter=50000, tol=1e-6)
        pm = abi.multiblock(pc.blocks)
        ps = abi.Solver(pm, pc.bc_fields(), pc.settings, device=local)
        rr = ps.solve()
        line["time_to_residual"] = {"case": pc.name, "cells": pm["nCells"], "iterations": rr["iterations"],
                                    "converged": rr["converged"], "seconds": rr["ms"] / 1e3,
                                    "residuals": rr["residual"]}
        ps.close()
        ref_pipe = reference_cuda_leg(cases.pipe(max_iter=50000, tol=1e-6), 50000)
        if "ms" in ref_pipe:
            line["time_to_residual"]["reference_cuda_seconds"] = ref_pipe["ms"] / 1e3
            line["time_to_residual"]["reference_cuda_iterations"] = ref_pipe["iterations"]
    if rank == 0:
        print(json.dumps(line), flush=True)
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
