#!/usr/bin/env python
"""SIMPLE cell-iterations/s on the 2M-cell jittered lid-driven cavity.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

A step is one SIMPLE outer iteration (momentum predictor with its non-
orthogonal passes, predictor flux, pressure equation with its passes, flux
correction, relaxed updates) over the whole 128^3 mesh, on fields that stay
resident in HBM between steps.  N > 1 runs independent replicas, one per GPU
(one case per GPU: the SIMPLE loop is not split across GPUs), launched
by torchrun; value is the whole job's cells*iterations / max-over-ranks time.

The workload: 128^3 = 2,097,152 hex cells in the unit box, interior mesh
points jittered by a seeded uniform +-10% of the cell size, lid (ymax)
U = (1 0 0), other walls no-slip, nu = 1/400 (Re 400), schemes upwind /
corrected / corrected, 1 non-orthogonal corrector, relaxU 0.7, relaxP 0.3,
pRelaxStart 0.02, pressure Jacobi-PCG to 1e-8 (infinity norm relative to the
right-hand side, the reference's test) with at most 2000 iterations, and a
pressure reference cell (cell 0) -- without it the reference's singular
Neumann pressure system, made inconsistent by its own boundary
non-orthogonal correction, drives p to ~1e12 in the first iteration.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CELLS = 128
JITTER, SEED = 0.1, 7
NU = 1.0 / 400.0
NAMES = ["left", "right", "bottom", "lid", "front", "back"]
SIDES = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
METRIC = "SIMPLE cell-iter/s at 2M cells; time to 1e-8 p-residual, learned vs plain PCG"


def workload_config(n):
    return {"workload": f"lid-driven cavity {n}^3 hex ({n ** 3} cells), interior points jittered +-10% "
                        f"(seed {SEED}), Re 400, upwind/corrected/corrected, nonOrth 1, relaxU 0.7 relaxP 0.3 "
                        f"pRelaxStart 0.02, pressure Jacobi-PCG tol 1e-8 maxIter 2000, pRefCell 0",
            "cells": n ** 3, "step": "one SIMPLE outer iteration",
            "l2": "inputs larger than L2 (about 1.3 GB of fields, matrices and mesh resident in HBM)",
            "precision": "FP64 throughout"}


def make_case(n, device, precond="Jacobi"):
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (n, n, n), {s: (nm, "wall") for s, nm in zip(SIDES, NAMES)})
    mesh.jitter_interior(JITTER, SEED)
    case = cf.SimpleCase(mesh, device)
    for nm in NAMES:
        case.set_patch_bc("U", nm, "fixedValue", (1.0, 0, 0) if nm == "lid" else (0, 0, 0))
        case.set_patch_bc("p", nm, "zeroGradient", 0.0)
    case.init_flux()
    ctl = cf.SimpleControls(max_iterations=1, relax_u=0.7, relax_p=0.3, p_relax_start=0.02, non_orth_correctors=1,
                            linear_tol=1e-8, linear_max_iter=2000, nu=NU, p_ref_cell=0, p_ref_value=0.0,
                            p_preconditioner=precond)
    return mesh, case, ctl


def case_dict(n):
    sides = "\n".join(f"    {s} {{ name {nm}; type wall; }}" for s, nm in zip(SIDES, NAMES))
    pats = "\n".join(f"    {nm} {{ U ({'1' if nm == 'lid' else '0'} 0 0); }}" for nm in NAMES)
    return (f"block\n{{\n    min (0 0 0);\n    max (1 1 1);\n    cells ({n} {n} {n});\n{sides}\n}}\n"
            f"nu {NU!r};\npatches\n{{\n{pats}\n}}\n"
            "schemes { ddt steady; div upwind; laplacian corrected; grad corrected; }\n"
            "simple { maxIterations 1; relaxU 0.7; relaxP 0.3; pRelaxStart 0.02; nonOrthCorrectors 1; "
            "linearTol 1e-08; linearMaxIter 2000; }\n")


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except OSError:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local, dist


def allreduce_max(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def run_reference_cpu(n, points, timeout=3600):
    """One SIMPLE outer iteration of the reference's own build on this host."""
    drv = os.path.join(ROOT, "oracle", "_ref", "cf_ref_driver")
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(case_dict(n))
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(points).tofile(pp)
        if os.path.exists(drv):
            r = subprocess.run([drv, "simple", cp, td, pp], capture_output=True, text=True, timeout=timeout)
            if r.returncode != 0:
                raise RuntimeError(r.stderr)
            res = open(os.path.join(td, "result.txt")).read().split()
            return float(res[4]), "reference", "oracle/_ref/cf_ref_driver (the reference's sources, g++ -O3)"
        # the C restatement of the same algorithm, when the reference was not built
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import _oracle as O
        m = O.block_mesh((0, 0, 0), (1, 1, 1), (n, n, n), NAMES, ["wall"] * 6).with_points(points)
        case = O.Case(m, u_type=["fixedValue"] * 6,
                      u_value=[(1.0, 0, 0) if nm == "lid" else (0, 0, 0) for nm in m.patch_names],
                      p_type=["zeroGradient"] * 6, p_value=[0] * 6, nu=NU, max_iterations=1, linear_tol=1e-8,
                      non_orth=1, relax_u=0.7, relax_p=0.3, p_relax_start=0.02)
        t0 = time.perf_counter()
        case.run()
        return time.perf_counter() - t0, "port", "oracle/cfo.c (C restatement)"


def cpu_info():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main_reference(args, world, rank, dist):
    """The reference's CPU SIMPLE on the same workload: one outer iteration of
    the 128^3 case from rest per step, single thread (the reference is serial)."""
    if rank != 0:
        return
    n = args.cells
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (n, n, n), {s: (nm, "wall") for s, nm in zip(SIDES, NAMES)})
    mesh.jitter_interior(JITTER, SEED)
    pts = mesh.addressing()["points"]
    del mesh
    steps = 1
    secs, kind, what = run_reference_cpu(n, pts)
    v = n ** 3 * steps / secs
    out = {"metric": METRIC, "impl": "reference", "value": v, "unit": "cell-iter/s", "n_gpus": args.gpus,
           "steps": steps, "warmup": 0, "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(n),
           "cpu_baseline": {"value": v, "unit": "cell-iter/s", "cores": 1, "kind": kind,
                            "sample": f"one SIMPLE outer iteration of the {n}^3 case from rest (a step of the "
                                      f"timed loop); the reference has no pressure reference cell, so its "
                                      f"pressure solve runs the unpinned system; {what}; {cpu_info()}"},
           "e2e": {"value": v, "unit": "cell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--cells", type=int, default=CELLS)
    ap.add_argument("--cpu-sample-cells", type=int, default=48)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--p-precond", default="Jacobi", choices=["Jacobi", "DIC"])
    ap.add_argument("--profile", action="store_true",
                    help="run --steps outer iterations from the initial state with no warm-up, timing or "
                         "baselines: the command line the ncu captures run")
    args = ap.parse_args()
    world, rank, local, dist = dist_setup()
    if args.impl == "reference":
        main_reference(args, world, rank, dist)
        if dist is not None:
            dist.destroy_process_group()
        return

    n = args.cells
    mesh, case, ctl = make_case(n, local, args.p_precond)
    ncell = mesh.n_cells
    if args.profile:
        for _ in range(args.steps):
            r = case.solve(ctl)
        print(json.dumps({"profile": workload_config(n)["workload"], "steps": args.steps,
                          "u_inner": r.u_inner_iterations, "p_inner": r.p_inner_iterations}))
        return
    for _ in range(max(3, args.warmup)):
        case.solve(ctl)
    # the state every leg starts from: the timed, end-to-end and kernel-timing
    # legs all run the same K outer iterations from it
    U0, p0, phi0 = case.download()
    # ---- timed region: K outer iterations on device-resident fields ----
    barrier(dist)
    dev_ms = 0.0
    launches = 0
    u_inner = p_inner = 0
    with Clocks(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r = case.solve(ctl)
            ms, nl = case.last_timing()
            dev_ms += ms[7]
            launches += nl
            u_inner += r.u_inner_iterations
            p_inner += r.p_inner_iterations
        wall = time.perf_counter() - t0
    barrier(dist)
    t_max = allreduce_max(dist, dev_ms / 1e3)
    value = world * ncell * args.steps / t_max

    # ---- end to end through the public API with host buffers: the same K
    # iterations, each uploading its input from pinned host memory and
    # downloading its result ----
    try:
        import torch
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    except Exception:
        pin = np.ascontiguousarray
    U, p, phi = pin(U0), pin(p0), pin(phi0)
    h2d = (U.nbytes + p.nbytes + phi.nbytes)
    e2e_steps = args.steps
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        case.upload(U, p, phi)
        case.solve(ctl)
        U2, p2, phi2 = case.download()
        U[...], p[...], phi[...] = U2, p2, phi2
    e2e_wall = allreduce_max(dist, time.perf_counter() - t0)
    e2e = world * ncell * e2e_steps / e2e_wall

    # ---- per-kernel event timing (outside the timed region: the events
    # keep the solver chunks out of CUDA graphs) over the first iteration ----
    case.upload(U0, p0, phi0)
    case.kernel_timing(True)
    case.solve(ctl)
    kstats = case.kernel_stats()
    case.kernel_timing(False)

    # ---- roofline of the dominant kernel: the pressure-PCG SpMV (+ p.Ap) ----
    nI = mesh.n_internal_faces
    s, i = 8, 4
    alg_spmv = 3 * s * ncell + s * nI + 2 * i * nI          # SpMV symmetric LDU, FP64
    alg_iter = alg_spmv + 11 * s * ncell                     # one Jacobi-PCG iteration
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    cnt, tot = kstats["cg_spmv"]
    spmv_ms = tot / max(cnt, 1)
    it_ms = sum(kstats[k][1] for k in kstats) / max(cnt, 1)
    achieved = alg_spmv / (spmv_ms * 1e-3) / 1e9 if cnt else 0.0
    traffic = None
    tp = os.environ.get("CFG_SPMV_TRAFFIC_BYTES")
    if tp:
        traffic = float(tp)
    roof = {"kernel": "k_cg_spmv (pressure Jacobi-PCG: SELL-32 SpMV + p.Ap)", "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_src, "traffic": traffic,
            "algorithmic_bytes_per_launch": alg_spmv, "launches_timed": cnt, "avg_launch_us": spmv_ms * 1e3,
            "pcg_iteration": {"algorithmic_bytes": alg_iter, "avg_us": it_ms * 1e3,
                              "achieved_gbs": alg_iter / (it_ms * 1e-3) / 1e9 if cnt else 0.0}}

    out = {"metric": METRIC, "value": value, "unit": "cell-iter/s", "n_gpus": world, "steps": args.steps,
           "warmup": max(3, args.warmup), "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": dict(workload_config(n), parallelism=f"replicas x{world}"),
           "e2e": {"value": e2e, "unit": "cell-iter/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                   "steps": e2e_steps},
           "gpu_launches": launches, "roofline": roof, "clocks": clk.summary(),
           "inner_iterations_per_step": {"momentum_bicgstab_sum_over_components": u_inner / args.steps,
                                         "pressure_pcg": p_inner / args.steps},
           "wall_s_timed": wall}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        m2 = args.cpu_sample_cells
        import chuanflow_b200 as cf
        sm = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (m2, m2, m2), {s_: (nm, "wall") for s_, nm in zip(SIDES, NAMES)})
        sm.jitter_interior(JITTER, SEED)
        secs, kind, what = run_reference_cpu(m2, sm.addressing()["points"])
        out["cpu_baseline"] = {"value": m2 ** 3 / secs, "unit": "cell-iter/s", "cores": 1, "kind": kind,
                               "sample": f"one SIMPLE outer iteration of the same case family on a {m2}^3 mesh "
                                         f"({secs:.1f} s; the full {n}^3 iteration takes minutes on one core); "
                                         f"unpinned pressure (the reference has no reference cell); {what}; "
                                         f"{cpu_info()}"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
