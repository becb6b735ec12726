#!/usr/bin/env python
"""SIMPLE cell-iterations/s on a 2M-cell jittered channel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

A step is one SIMPLE outer iteration (momentum predictor with its non-
orthogonal passes, predictor flux, pressure equation with its passes, flux
correction, relaxed updates) over the whole mesh, on fields that stay
resident in HBM between steps.  N > 1 runs independent replicas, one per GPU
(one case per GPU: the SIMPLE loop is not split across GPUs), launched
by torchrun; value is the whole job's cells*iterations / max-over-ranks time.

The workload: the 16,000-cell verification channel's family (2.0 x 0.1 x
0.1 m, inlet 0.1 m/s, fixed-p outlet, no-slip walls, nu 1e-4) at 512 x 64 x
64 = 2,097,152 hex cells -- the cell count of the 128^3 cavity -- with the
cavity's mesh treatment (interior points jittered by a seeded uniform +-10%
of the cell size, so every face is non-orthogonal), schemes upwind /
corrected / corrected, 1 non-orthogonal corrector, and the reference's own
channel relaxation (relaxU 0.9, relaxP 0.03) with the startup floor of its
adaptive pressure relaxation at pRelaxStart 0.002 (its 16,000-cell value,
0.02, lets the 2M-cell SIMPLE diverge within five iterations).  Both linear
solves stop on the reference's test (infinity norm relative to the right-
hand side, 1e-8, FP64) with at most 2000 iterations; both are preconditioned
by FP32 aggregation-AMG V-cycles inside FP64 Krylov loops: the momentum
components by BiCGStab with the momentum matrix's V-cycle (--u-precond; the
line's `momentum_jacobi` runs the same steps with the reference's Jacobi-
BiCGStab), the pressure by flexible CG (--p-precond; `variant` runs the
same steps with FP64 multicolour DIC-PCG, FP64 throughout, whose fields the
headline's are measured against).  The pressure hierarchy aggregates by
strength of connection (--amg-theta 0.25: couplings under a quarter of a
row's largest are left out, which here are those along the channel); the
momentum hierarchy aggregates plainly.  `--workload cavity` times the lid-driven cavity of the same cell
count (128^3, Re 400, relaxation 0.7 / 0.3 / pRelaxStart 5e-4, pressure
reference cell 0), which the reference cannot run as such: it has no
reference cell.

Every leg counts the outer iterations that diverged (simpleSolver.cpp:360-364:
non-finite continuity, pressure step or fields; and, before a blow-up
overflows, a continuity error 100x the first warm-up step's); the JSON line
carries them and the run exits 1 when any did.
"""
import argparse
import dataclasses
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CELLS = 64                      # the channel's cells across; 8x along: 512 x 64 x 64 = 2,097,152
LENGTH = (2.0, 0.1, 0.1)
U_IN, NU = 0.1, 1e-4            # Re 100 on the channel height
JITTER, SEED = 0.1, 7
SIDES = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
CH_NAMES = ["inlet", "outlet", "bottom", "top", "front", "back"]
CH_TYPES = ["inlet", "outlet", "wall", "wall", "wall", "wall"]
# the reference's channel relaxation; the startup floor of its adaptive
# pressure relaxation lowered from its 16,000-cell value 0.02, with which its
# SIMPLE diverges at 2M cells
RELAX = {"relax_u": 0.9, "relax_p": 0.03, "p_relax_start": 0.002}
# the detail blocks: k-epsilon blocks' Re_H; the startup floor of the
# adaptive pressure relaxation (with 0.02 the reference's own DetailBlock
# diverges on these ducts, laminar and k-epsilon); the outer iterations that
# develop every block before the one-iteration coupling passes
RE_KEPS = 2e4
BLOCK_P_RELAX_START = 0.002
BLOCK_START = 60
# the pressure AMG hierarchy aggregates by strength of connection: across
# the channel the cells are 2.5x thinner than along it, so the couplings
# along it are 0.16x the others and fall under this threshold
AMG_THETA = 0.25
METRIC = "SIMPLE cell-iter/s at 2M cells; time to 1e-8 p-residual, learned vs plain PCG"
REFERENCE_ARM = ("the reference's CPU SIMPLE (its own sources, its Jacobi-PCG pressure and Jacobi-BiCGStab "
                 "momentum) on the same mesh, boundary conditions and settings, one outer iteration from rest as "
                 "a bounded sample (a whole 2M-cell iteration takes minutes on one core); one core, pinned")
# the lid-driven cavity the tests still run (the reference's SIMPLE diverges on it at these sizes)
CAV_NAMES = ["left", "right", "bottom", "lid", "front", "back"]
CAV_NU = 1.0 / 400.0


def dims(n):
    return (8 * n, n, n)


def workload_config(n, precond="DIC", u_precond="Jacobi", amg_theta=0.0):
    solve = (("FP64 flexible CG with an FP32 aggregation-AMG V-cycle" +
              (f" (aggregates by strength of connection, theta {amg_theta})" if amg_theta else " (plain aggregation)"))
             if precond == "AMG" else f"{precond}-PCG")
    usolve = ("FP64 BiCGStab with the FP32 aggregation-AMG V-cycle of the momentum matrix (3 components per V-cycle)"
              if u_precond == "AMG" else "Jacobi-BiCGStab (the reference's)")
    nx, ny, nz = dims(n)
    fp32 = [w for w, on in (("momentum", u_precond == "AMG"), ("pressure", precond == "AMG")) if on]
    return {"workload": f"3D channel {LENGTH[0]} x {LENGTH[1]} x {LENGTH[2]} m, {nx} x {ny} x {nz} hex "
                        f"({nx * ny * nz} cells), interior points jittered +-10% (seed {SEED}), inlet {U_IN} m/s, "
                        f"fixed-p outlet, no-slip walls, nu {NU} (Re 100), upwind/corrected/corrected, nonOrth 1, "
                        f"relaxU 0.9 relaxP 0.03 pRelaxStart 0.002, momentum {usolve}, pressure {solve}, "
                        f"both to 1e-8 (|r|inf/|b|inf, FP64), maxIter 2000",
            "cells": nx * ny * nz, "step": "one SIMPLE outer iteration",
            "l2": "inputs larger than L2 (about 1.3 GB of fields, matrices and mesh resident in HBM)",
            "precision": (f"FP64 Krylov vectors, dot products and stopping tests; the {' and '.join(fp32)} "
                          f"preconditioner{'s' if len(fp32) > 1 else ''} FP32" if fp32 else "FP64 throughout"),
            "parallelism": "one case per GPU (replicas); the reference arm on one host core",
            "reference_arm": REFERENCE_ARM}


KERNEL_NAMES = {
    "cg_spmv": "k_cg_spmv (pressure PCG: SELL-32 SpMV + p.Ap)",
    "cg_update": "k_cg_update (pressure PCG: x, r update + norms + r.z)",
    "cg_p": "k_cg_p (pressure PCG: search direction)",
    "bi_p": "k_bi_p (momentum BiCGStab, 3 components: p, z update)",
    "bi_spmv1": "k_bi_spmv1 (momentum BiCGStab, 3 components: v = A z + r0.v)",
    "bi_spmv2": "k_bi_spmv2 (momentum BiCGStab, 3 components: t = A s^, s^ formed per column, + t.t, t.s)",
    "bi_x": "k_bi_x (momentum BiCGStab, 3 components: x += alpha z + omega s^, r update + |r| + r0.r)",
    "dic_apply": "k_dic_fwd/k_dic_bwd (multicolour DIC z = M^-1 r, all colour phases)",
    "bia_p": "k_bia_p (AMG momentum BiCGStab, 3 components: p update)",
    "amgv_pre0": "k_amgv_pre0 (momentum V-cycle, finest level, 3 components: x = w D^-1 b, r = b - A x, FP32)",
    "amgv_coarse": "the momentum V-cycle's restriction, coarse levels, tail and prolongations (several kernels)",
    "amgv_post0": "k_amgv_post0 (momentum V-cycle, finest level, 3 components: z = y + w D^-1 (b - A y), FP32 in, "
                  "FP64 out)",
    "bia_spmv1": "k_bi_spmv1 (AMG momentum BiCGStab, 3 components: v = A z + r0.v)",
    "bia_s": "k_bia_s (AMG momentum BiCGStab, 3 components: s = r - alpha v)",
    "bia_spmv2": "k_bia_spmv2 (AMG momentum BiCGStab, 3 components: t = A s^ + t.t, t.s)",
    "bia_x": "k_bia_x (AMG momentum BiCGStab, 3 components: x += alpha z + omega s^, r update + |r| + r0.r)",
}


# DRAM bytes (read + write) per launch from one full-set ncu capture of
# k_bi_spmv2 on the 2M-cell channel (launches 21-22 of its third outer
# iteration: 334.2 and 333.3 MB)
# DRAM bytes (read + write) per launch from one ncu capture of this
# workload (profiles/), with what that launch carried
MEASURED_TRAFFIC = {"bi_spmv2": (334.2e6, "all three components; profiles/k_bi_spmv2_channel2M_full.md"),
                    "amgv_pre0": (219.3e6, "a launch with two of three components iterating (algorithmic 192.7 MB); "
                                           "profiles/k_amgv_pre0_channel2M_full.md")}


def kernel_bytes(N, F, s=8, i=4):
    """Algorithmic bytes of one launch of each solver kernel as (shared,
    per component): every array counted once per read and once per write,
    gathers as one N-stream; the three momentum components share one matrix
    read and D^-1.  k_bi_p and k_bi_x skip a converged component's rows, the
    two SpMVs always carry all three."""
    spmv_sym = 3 * s * N + s * F + 2 * i * F       # x in, y out, diag + one coefficient per face, indices
    mat3 = s * N + 2 * s * F + 2 * i * F           # diag + both coefficients + indices, shared by 3 components
    # the three-component V-cycle's finest passes: an FP32 SELL read (value
    # and column per entry, N + 2F entries) and D^-1 each; per component the
    # pre-sweep reads the FP64 input (gathered) and writes the FP32 sweep and
    # residual, the post-sweep reads the FP64 input and the prolongated FP32
    # correction (gathered) and writes the FP64 output.  The level vectors
    # hold a float4 per row; only the three components' 12 bytes are
    # counted, not the fourth word.  Everything between (restriction of the
    # residual with the member list, the coarse levels, the prolongation:
    # the sweep, the aggregate map and the coarse output read, the
    # correction written) is counted at its finest-level streams plus about
    # 30% for the coarser levels.
    f4 = 4
    sell32 = (N + 2 * F) * 2 * f4 + f4 * N
    coarse3 = (1.3 * 3 * f4 * N, 1.3 * 3 * f4 * N)
    return {"cg_spmv": (spmv_sym, 0), "cg_update": (7 * s * N, 0), "cg_p": (4 * s * N, 0),
            # invD in; per component r, p, v in, p, z out
            "bi_p": (s * N, 5 * s * N),
            # matrix; per component z in (gathered), v out, r0 in
            "bi_spmv1": (mat3, 3 * s * N),
            # matrix, invD (gathered); per component r, v in (gathered), t out
            "bi_spmv2": (mat3 + s * N, 3 * s * N),
            # invD; per component x, z, r, v, t, r0 in, x, r out
            "bi_x": (s * N, 8 * s * N),
            "dic_apply": (3 * s * N + 2 * (s * F + 2 * i * F), 0),
            # the AMG-preconditioned momentum BiCGStab: per component r, p, v
            # in, p out
            "bia_p": (0, 4 * s * N),
            "amgv_pre0": (sell32, s * N + 2 * f4 * N),
            "amgv_coarse": coarse3,
            "amgv_post0": (sell32, s * N + f4 * N + s * N),
            "bia_spmv1": (mat3, 3 * s * N),
            # per component r, v in, s out
            "bia_s": (0, 3 * s * N),
            # matrix; per component s^ in (gathered), s in, t out
            "bia_spmv2": (mat3, 3 * s * N),
            # per component x, z, s, s^, t, r0 in, x, r out
            "bia_x": (0, 8 * s * N)}


COMPOSITE = ("amgv_coarse",)
SKIPS_DONE = ("bi_p", "bi_x", "bia_p", "amgv_pre0", "amgv_coarse", "amgv_post0", "bia_s", "bia_x")


def simple_step_bytes(N, F, Fb, n_orth, it_p, precond, solver_bytes, s=8, i=4):
    """Algorithmic bytes of one SIMPLE outer iteration: the fixed face and
    cell passes (gradients, correctors, assemblies, fluxes, updates) plus
    `solver_bytes`, the solver kernels' own per-launch bytes times their
    launches; with the AMG pressure (whose kernels are not event-timed) its
    flexible-CG iterations are added at the model's per-iteration bytes."""
    Ft = F + Fb
    grad_plain = Ft * (2 * i + 4 * s) + 5 * s * N
    grad_corr = grad_plain + 2 * (Ft * (2 * i + 7 * s) + 8 * s * N)
    corrector = Ft * (2 * i + 5 * s) + 5 * s * N
    fixed = (2 * grad_corr + (n_orth + 1) * 3 * (grad_corr + corrector) + (n_orth + 1) * (grad_corr + corrector)
             + Ft * (2 * i + 5 * s) + 8 * s * N          # momentum assembly
             + Ft * (2 * i + 4 * s) + 3 * s * N          # pressure assembly
             + Ft * (2 * i + 5 * s) + 3 * s * N          # predictor flux
             + Ft * (2 * i + 9 * s) + 4 * s * N          # correctFluxes
             + 21 * s * N                                # cell updates
             + Ft * (i + s) + s * N)                     # divPhi
    extra = 0
    if precond == "AMG":
        # flexible CG: FP64 SpMV + 9 vector streams, and the V-cycle: at the
        # finest level two FP32 SELL passes (value + column per entry, N + 2F
        # entries) and 12 four-byte vector streams; the coarser levels add
        # about 30% (their rows are 1/7 as many but longer)
        fine = 2 * (N + 2 * F) * 8 + 12 * 4 * N
        extra = it_p * (3 * s * N + s * F + 2 * i * F + 9 * s * N + 1.3 * fine)
    return fixed + solver_bytes + extra


def cavity_config(n, precond="DIC"):
    solve = ("FP64 flexible CG with an FP32 aggregation-AMG V-cycle" if precond == "AMG" else f"{precond}-PCG")
    return {"workload": f"lid-driven cavity {n}^3 hex ({n ** 3} cells), interior points jittered +-10% (seed {SEED}), "
                        f"Re 400, upwind/corrected/corrected, nonOrth 1, relaxU 0.7 relaxP 0.3 pRelaxStart 5e-4, "
                        f"pressure {solve} tol 1e-8 (|r|inf/|b|inf) maxIter 2000, pressure reference cell 0",
            "cells": n ** 3, "step": "one SIMPLE outer iteration",
            "l2": "inputs larger than L2 (about 1.3 GB of fields, matrices and mesh resident in HBM)",
            "precision": ("FP64, the pressure preconditioner FP32" if precond == "AMG" else "FP64 throughout"),
            "parallelism": "one case per GPU (replicas)",
            "reference_arm": "none for this workload: the reference has no pressure reference cell"}


def make_case(n, device, precond="Jacobi", amg_theta=0.0):
    """The headline channel on `device`, at rest with its boundary flux;
    amg_theta > 0 aggregates the pressure AMG hierarchy by strength of
    connection at that threshold."""
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), LENGTH, dims(n), {s: (nm, t) for s, nm, t in zip(SIDES, CH_NAMES, CH_TYPES)})
    mesh.jitter_interior(JITTER, SEED)
    case = cf.SimpleCase(mesh, device)
    if amg_theta:
        case.amg_strength(amg_theta)
    case.set_patch_bc("U", "inlet", "fixedValue", (U_IN, 0, 0))
    case.set_patch_bc("p", "inlet", "zeroGradient", 0.0)
    case.set_patch_bc("U", "outlet", "zeroGradient", (0, 0, 0))
    case.set_patch_bc("p", "outlet", "fixedValue", 0.0)
    for nm in CH_NAMES[2:]:
        case.set_patch_bc("U", nm, "fixedValue", (0, 0, 0))
        case.set_patch_bc("p", nm, "zeroGradient", 0.0)
    case.init_flux()
    ctl = cf.SimpleControls(max_iterations=1, non_orth_correctors=1, linear_tol=1e-8, linear_max_iter=2000, nu=NU,
                            p_preconditioner=precond, **RELAX)
    return mesh, case, ctl


def make_cavity_case(n, device, precond="Jacobi", p_relax_start=0.02):
    """The jittered n^3 lid-driven cavity (Re 400, relaxation 0.7 / 0.3,
    pressure reference cell 0); pRelaxStart 0.02 by default (the golden
    fixtures' value), 5e-4 for the 128^3 workload, where 0.02 diverges."""
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (n, n, n), {s: (nm, "wall") for s, nm in zip(SIDES, CAV_NAMES)})
    mesh.jitter_interior(JITTER, SEED)
    case = cf.SimpleCase(mesh, device)
    for nm in CAV_NAMES:
        case.set_patch_bc("U", nm, "fixedValue", (1.0, 0, 0) if nm == "lid" else (0, 0, 0))
        case.set_patch_bc("p", nm, "zeroGradient", 0.0)
    case.init_flux()
    ctl = cf.SimpleControls(max_iterations=1, relax_u=0.7, relax_p=0.3, p_relax_start=p_relax_start,
                            non_orth_correctors=1, linear_tol=1e-8, linear_max_iter=2000, nu=CAV_NU, p_ref_cell=0,
                            p_ref_value=0.0, p_preconditioner=precond)
    return mesh, case, ctl


def _splitmix64(x):
    """splitmix64 over a uint64 array (numpy wraps on overflow)."""
    x = x + np.uint64(0x9E3779B97F4A7C15)
    z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def block_points(cells, length, fraction=JITTER, seed=SEED):
    """The points of a jittered block mesh from the origin to `length`,
    computed in numpy with the same IEEE operations as BlockMesh::create's
    coordAt (blockMesh.cpp:52-57) and cfg_mesh_jitter_interior (every
    interior point moves by (2u - 1) fraction h per axis, u =
    splitmix64(seed * 0x100000001B3 ^ (3 point + axis)) >> 11 over 2^53), so
    the reference arm needs no product library to build the same mesh."""
    nx, ny, nz = cells
    cx, cy, cz = (0.0 + (length[a] - 0.0) * np.arange(cells[a] + 1, dtype=np.float64) / float(cells[a])
                  for a in range(3))
    z, y, x = np.meshgrid(cz, cy, cx, indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    k, j, i = np.meshgrid(np.arange(1, nz), np.arange(1, ny), np.arange(1, nx), indexing="ij")
    pid = (i + (nx + 1) * (j + (ny + 1) * k)).ravel().astype(np.uint64)
    s0 = np.uint64((seed * 0x100000001B3) & ((1 << 64) - 1))
    with np.errstate(over="ignore"):
        for a in range(3):
            h = (length[a] - 0.0) / float(cells[a])
            r = _splitmix64(s0 ^ (pid * np.uint64(3) + np.uint64(a)))
            u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            pts[pid.astype(np.int64), a] += (u * 2.0 - 1.0) * fraction * h
    return pts


def cavity_points(n, fraction=JITTER, seed=SEED):
    return block_points((n, n, n), (1.0, 1.0, 1.0), fraction, seed)


def case_dict(n):
    """The headline channel as a reference case dictionary (simpleFoamApp's
    keys); its points come separately (the jitter)."""
    nx, ny, nz = dims(n)
    sides = "\n".join(f"    {s} {{ name {nm}; type {t}; }}" for s, nm, t in zip(SIDES, CH_NAMES, CH_TYPES))
    return (f"block\n{{\n    min (0 0 0);\n    max ({LENGTH[0]!r} {LENGTH[1]!r} {LENGTH[2]!r});\n"
            f"    cells ({nx} {ny} {nz});\n{sides}\n}}\n"
            f"nu {NU!r};\npatches\n{{\n"
            f"    inlet  {{ U ({U_IN!r} 0 0); UType fixedValue; pType zeroGradient; }}\n"
            f"    outlet {{ UType zeroGradient; p 0; pType fixedValue; }}\n"
            + "".join(f"    {nm} {{ U (0 0 0); }}\n" for nm in CH_NAMES[2:]) +
            "}\n"
            "schemes { ddt steady; div upwind; laplacian corrected; grad corrected; }\n"
            "simple { maxIterations 1; relaxU 0.9; relaxP 0.03; pRelaxStart 0.002; nonOrthCorrectors 1; "
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


def dist_setup(backend=None):
    """Replicas: one process per GPU from torchrun's RANK / LOCAL_RANK /
    WORLD_SIZE, NCCL between them (gloo on a host without CUDA, which the
    host-side tests use).  No data-path collective: only the barriers and
    the max-over-ranks reduction of the timings."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local, dist


def allreduce_max(dist, v):
    """The largest of the ranks' values (every rank gets it)."""
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, seconds):
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units: all units over the slowest rank's time."""
    return world * units_per_rank / seconds


def barrier(dist):
    if dist is not None:
        dist.barrier()


def pinned_core():
    """The core the CPU baseline runs on: the first one this process may use
    (the reference is serial), when taskset is there to pin it."""
    try:
        return min(os.sched_getaffinity(0)) if shutil.which("taskset") else None
    except (AttributeError, OSError, ValueError):
        return None


def run_reference_cpu(n, points, timeout=3600, fields=False):
    """One SIMPLE outer iteration from rest of the headline channel by the
    reference's own build (oracle/_ref/cf_ref_driver, its sources compiled
    with g++ -O3) on this host, pinned to one core (the reference is serial),
    with its Jacobi-PCG pressure.  Returns (seconds, kind, what, (U, p, phi)
    or None)."""
    drv = os.path.join(ROOT, "oracle", "_ref", "cf_ref_driver")
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(case_dict(n))
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(points).tofile(pp)
        if os.path.exists(drv):
            core = pinned_core()
            pin = ["taskset", "-c", str(core)] if core is not None else []
            r = subprocess.run(pin + [drv, "simple", cp, td, pp], capture_output=True, text=True, timeout=timeout)
            if r.returncode != 0:
                raise RuntimeError(r.stderr)
            res = open(os.path.join(td, "result.txt")).read().split()
            out = None
            if fields:
                out = (np.fromfile(os.path.join(td, "U.f64")).reshape(-1, 3), np.fromfile(os.path.join(td, "p.f64")),
                       np.fromfile(os.path.join(td, "phi.f64")))
            return float(res[4]), "reference", "oracle/_ref/cf_ref_driver (the reference's sources, g++ -O3)", out
        # the C restatement of the same algorithm, when the reference was not built
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import _oracle as O
        m = O.block_mesh((0, 0, 0), LENGTH, dims(n), CH_NAMES, CH_TYPES).with_points(points)
        case = O.Case(m, u_type=["fixedValue", "zeroGradient"] + ["fixedValue"] * 4,
                      u_value=[(U_IN, 0, 0)] + [(0, 0, 0)] * 5, p_type=["zeroGradient", "fixedValue"] +
                      ["zeroGradient"] * 4, p_value=[0] * 6, nu=NU, max_iterations=1, linear_tol=1e-8,
                      non_orth=1, **RELAX)
        t0 = time.perf_counter()
        U, p, phi, _ = case.run()
        return time.perf_counter() - t0, "port", "oracle/cfo.c (C restatement)", ((U, p, phi) if fields else None)


def cpu_info():
    """The CPU model, the host's core count and the core the baseline ran on."""
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    core = pinned_core()
    where = f"pinned to core {core}" if core is not None else "unpinned"
    return f"{model}, {os.cpu_count()} host cores, {where}"


def main_reference(args, world, rank, dist):
    """The reference arm: the reference's CPU SIMPLE on the workload's mesh
    (built here in numpy, without the product library) -- one outer
    iteration from rest, single thread (the reference is serial)."""
    if rank != 0:
        return
    n = args.cells
    steps = 1
    secs, kind, what, _ = run_reference_cpu(n, block_points(dims(n), LENGTH))
    v = float(np.prod(dims(n))) * steps / secs
    out = {"metric": METRIC, "impl": "reference", "value": v, "unit": "cell-iter/s", "n_gpus": args.gpus,
           "steps": steps, "warmup": 0, "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(n, args.p_precond, args.u_precond, args.amg_theta),
           "cpu_baseline": {"value": v, "unit": "cell-iter/s", "cores": 1, "kind": kind,
                            "sample": f"one SIMPLE outer iteration of the headline channel from rest; {what}; "
                                      f"{cpu_info()}"},
           "e2e": {"value": v, "unit": "cell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main_transient(args, world, rank, local, dist):
    """The learned part in a transient run: a 2D-extruded channel (nx x
    nx/4 x 4 hex cells) with a square obstacle of a quarter of the height,
    Re 200 on the obstacle, implicit-Euler PISO at CFL 0.5.  The first 75%
    of the steps run with DIC-PCG pressure and keep (residual each pressure
    solve starts from, correction it converges to) pairs; the network trains
    on them in the energy norm; the last 25% then run four times from the
    same fields -- DIC-PCG, the FP32-AMG flexible CG, the network's initial
    guess followed by the AMG flexible CG, and the network's guess followed
    by flexible CG with the network -- to the same 1e-8 test."""
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    nx = args.transient_nx
    ny = nx // 4
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "obstacle.msh")
        ncell, h = meshgen.obstacle_channel_msh(path, nx, ny, 4)
        mesh = cf.PolyMesh.read_gmsh(path, {"inlet": "inlet", "outlet": "outlet"})
    case = cf.SimpleCase(mesh, local)
    for name, _, _, _ in mesh.patches:
        if name == "inlet":
            case.set_patch_bc("U", name, "fixedValue", (1.0, 0, 0))
            case.set_patch_bc("p", name, "zeroGradient", 0.0)
        elif name == "outlet":
            case.set_patch_bc("U", name, "zeroGradient", 0.0)
            case.set_patch_bc("p", name, "fixedValue", 0.0)
        elif name in ("walls", "obstacle"):
            case.set_patch_bc("U", name, "fixedValue", (0, 0, 0))
            case.set_patch_bc("p", name, "zeroGradient", 0.0)
        else:
            case.set_patch_bc("U", name, "zeroGradient", 0.0)
            case.set_patch_bc("p", name, "zeroGradient", 0.0)
    case.init_flux()
    nu = 1.0 * 0.25 / 200.0
    dt = 0.5 * h / 1.0
    ctl = cf.PisoControls(dt=dt, correctors=2, continuity_tol=1e-10, linear_tol=1e-8, non_orth_correctors=0, nu=nu,
                          p_preconditioner="DIC")
    steps = args.transient_steps
    n_train = (3 * steps) // 4
    every = max(1, n_train // args.train_pairs)
    case.mpnn_create(4, seed=3)
    t0 = time.perf_counter()
    for s in range(n_train):
        case.mpnn_collect(2 if s == 0 else (1 if s % every == 0 else 0), args.train_pairs)
        case.piso_step(ctl)
    n_pairs = case.mpnn_collect(0, args.train_pairs)
    sim_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    losses = case.mpnn_train_collected(args.train_epochs, 2e-3)
    train_s = time.perf_counter() - t0
    batch = cf.Batch([case])
    batch.save()
    legs = {}
    for name, pre in (("dic64", "DIC"), ("amg32", "AMG"), ("learned_guess_amg32", "AMG_MPNN"),
                      ("learned_guess_fcg", "MPNN")):
        batch.restore()
        c2 = dataclasses.replace(ctl, p_preconditioner=pre)
        ms, pit, fin, div = [], 0, None, 0
        for s in range(n_train, steps):
            r = case.piso_step(c2)
            ms.append(r["device_ms"])
            pit += r["p_inner_iterations"]
            div += int(r.get("diverged", 0))
            fin = r
        U, p, phi = case.download()
        legs[name] = {"ms_per_step": statistics.mean(ms), "pressure_iterations_per_step": pit / max(1, len(ms)),
                      "continuity_last": fin["continuity_error"], "diverged_steps": div, "U": U}
    for k in legs:
        if k != "dic64":
            legs[k]["rel_L2_U_vs_dic64"] = float(np.linalg.norm(legs[k]["U"] - legs["dic64"]["U"]) /
                                                 np.linalg.norm(legs["dic64"]["U"]))
    for v in legs.values():
        v.pop("U")
    # the network's own cost on this mesh: one application, and one
    # message-passing layer against its algorithmic bytes (state in, the
    # neighbours' states as one stream, state out, mask; the matrix row; the
    # diagonal)
    app_ms, layer_ms = case.mpnn_time(20)
    entries = mesh.n_cells + 2 * mesh.n_internal_faces
    layer_bytes = mesh.n_cells * (3 * 128 + 4 + 8) + 12 * entries
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    if rank == 0:
        base = legs["amg32"]["ms_per_step"]
        out = {"metric": "transient obstacle channel: device ms per PISO step, learned initial guess + FP32-AMG "
                         "flexible CG vs the FP32-AMG flexible CG alone",
               "value": legs["learned_guess_amg32"]["ms_per_step"], "unit": "ms", "n_gpus": world,
               "steps": steps - n_train, "warmup": n_train, "higher_is_better": False, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64 (network: bf16 weights and tensor-core operands, f32 accumulation)",
               "data": "synthetic",
               "config": {"workload": f"2D-extruded channel {nx}x{ny}x4 hex with a square obstacle (blockage 0.25), "
                                      f"{ncell} cells, Re 200 on the obstacle, implicit Euler PISO (2 correctors) "
                                      f"at CFL 0.5 (dt {dt:g}), {steps} steps: the first {n_train} with DIC-PCG "
                                      f"generate the training pairs, the rest are timed four times from the same "
                                      f"fields", "cells": ncell},
               "legs": legs, "simulation_s_training_steps": sim_s, "train_s": train_s,
               "train_pairs": n_pairs,
               "train_loss_first": float(losses[0]), "train_loss_last": float(losses[-1]),
               "network": {"ms_per_application": app_ms, "layer_ms": layer_ms, "layer_alg_bytes": layer_bytes,
                           "layer_achieved_gbs": layer_bytes / (layer_ms * 1e-3) / 1e9,
                           "layer_frac_of_hbm_peak": layer_bytes / (layer_ms * 1e-3) / 1e9 / peak, "peak": peak},
               "speedup_learned_guess_amg_vs_amg": base / legs["learned_guess_amg32"]["ms_per_step"],
               "speedup_amg32_vs_dic": legs["dic64"]["ms_per_step"] / base,
               "speedup_learned_guess_fcg_vs_dic": legs["dic64"]["ms_per_step"] /
                                                   legs["learned_guess_fcg"]["ms_per_step"]}
        print(json.dumps(out), flush=True)


def main_blocks(args, world, rank, local, dist):
    """Detail blocks of a coupled 1D-3D network: N straight ducts with cell
    counts log-uniform in [2e3, 2e5], aspect 5-20, inlet profiles flat /
    parabolic / 1/7-power, mean inlet speeds uniform in [0.05, 0.5] m/s
    (seeded); even blocks laminar, odd blocks k-epsilon at Re_H RE_KEPS.
    Every block is first developed by one lossAt of BLOCK_START outer
    iterations at its rate.  A step is then one coupling pass: every block's
    lossAt(q) with one SIMPLE outer iteration (DIC-PCG pressure to 1e-8)
    from its previous state.  Timed with the autotuned batch schedule, as
    one CUDA-graph launch, and one block after another (the reference's
    order), each from the same saved fields; any diverged block solve makes
    the run exit 1."""
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    spec = meshgen.detail_block_set(args.blocks, seed=2024 + rank)
    cases, qs, ctls = [], [], []
    for s_ in spec:
        m = meshgen.channel_block(s_["cells"], s_["aspect"])
        c = cf.SimpleCase(m, local)
        c.detail_setup(s_["shape"], rho=998.0)
        # laminar blocks nu 1e-4; k-epsilon blocks at Re_H = U H / nu = RE_KEPS
        nu = 1e-4 if s_["laminar"] else s_["speed"] * 0.1 / RE_KEPS
        if not s_["laminar"]:
            c.detail_turbulence("kEpsilon", intensity=0.05, length_scale=-1.0, relaxation=0.7, nu=nu)
        cases.append(c)
        qs.append(s_["speed"] * 0.1 * 0.1)
        ctls.append(cf.SimpleControls(max_iterations=1, relax_u=0.7, relax_p=0.3, p_relax_start=BLOCK_P_RELAX_START,
                                      non_orth_correctors=1, linear_tol=1e-8, linear_max_iter=2000, nu=nu,
                                      p_preconditioner="DIC"))
    cells = sum(c.mesh.n_cells for c in cases)
    batch = cf.Batch(cases)
    batch.set_schedule(8, 1)
    # the coupled passes start from developed blocks: one lossAt of
    # BLOCK_START outer iterations each (untimed); one-iteration passes from
    # rest give the reference's DetailBlock non-positive and non-finite drops
    r0, _ = batch.loss(qs, [dataclasses.replace(c, max_iterations=BLOCK_START) for c in ctls])
    start_div = sum(int(x["diverged"]) for x in r0)
    warm_div = 0
    for _ in range(max(3, args.warmup)):
        rw, _ = batch.loss(qs, ctls)
        warm_div += sum(int(x["diverged"]) for x in rw)
    sched, cand = batch.autotune(qs, ctls)
    # the single-graph pass, timed on its own whether or not the autotuner
    # picked it (its first pass captures the graph)
    graph_sched = (0, -1)
    batch.save()
    batch.set_schedule(*graph_sched)
    batch.loss(qs, ctls)
    batch.restore()
    barrier(dist)
    # each step: the same pass from the same fields, one block after another,
    # as one graph launch, and under the autotuned schedule, the last kept
    batched, serial, graphed = [], [], []
    timed_div = 0
    for _ in range(args.steps):
        batch.save()
        batch.set_schedule(1, 0)
        r2, ms = batch.loss(qs, ctls)
        serial.append(ms)
        batch.restore()
        batch.set_schedule(*graph_sched)
        r3, ms = batch.loss(qs, ctls)
        graphed.append(ms)
        batch.restore()
        batch.set_schedule(*sched)
        r, ms = batch.loss(qs, ctls)
        batched.append(ms)
        timed_div += sum(int(x["diverged"]) for x in r + r2 + r3)
    barrier(dist)
    t_b = allreduce_max(dist, statistics.median(batched))
    t_s = allreduce_max(dist, statistics.median(serial))
    t_g = allreduce_max(dist, statistics.median(graphed))
    # the pass's algorithmic bytes: per block its fixed face and cell passes,
    # its momentum BiCGStab component-iterations (each the component's share
    # of both matrix reads plus its vector streams) and its DIC-PCG
    # iterations; the k-epsilon blocks' two scalar solves are not counted
    byts = 0.0
    for c, x in zip(cases, r):
        if x["diverged"]:
            continue  # a non-finite solve stops early and reports maxIter
        N, F, Fb = c.mesh.n_cells, c.mesh.n_internal_faces, c.mesh.n_boundary_faces
        kb = kernel_bytes(N, F)
        per_u = (kb["bi_spmv1"][0] + kb["bi_spmv2"][0] + kb["bi_p"][0] + kb["bi_x"][0]) / 3 + \
            kb["bi_p"][1] + kb["bi_spmv1"][1] + kb["bi_spmv2"][1] + kb["bi_x"][1]
        per_p = kb["cg_spmv"][0] + kb["cg_update"][0] + kb["cg_p"][0] + kb["dic_apply"][0]
        byts += simple_step_bytes(N, F, Fb, 1, 0, "DIC", x["u_inner_iterations"] * per_u +
                                  x["p_inner_iterations"] * per_p)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    if rank == 0:
        out = {"metric": "coupling pass time, 64 detail blocks x one SIMPLE outer iteration", "value": t_b,
               "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
               "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic",
               "config": {"workload": f"{len(cases)} straight hex ducts, {cells} cells in all, log-uniform "
                                      f"2e3-2e5 cells, aspect 5-20, flat/parabolic/1-7 power inlets, 0.05-0.5 m/s "
                                      f"(seed 2024), even blocks laminar nu 1e-4, odd blocks k-epsilon at Re_H {RE_KEPS:g}; every block "
                                      f"developed by one {BLOCK_START}-iteration lossAt, then one SIMPLE outer iteration per "
                                      f"block per pass; relaxU 0.7 relaxP 0.3 pRelaxStart {BLOCK_P_RELAX_START:g}",
                          "cells": cells, "schedule": {"workers": sched[0], "row_blocks_per_sm": sched[1]},
                          "autotune_ms": {f"{w}x{r}": v for (w, r), v in cand.items()}},
               "one_after_another_ms": t_s, "speedup_vs_one_after_another": t_s / t_b,
               "single_graph_ms": t_g, "speedup_single_graph_vs_one_after_another": t_s / t_g,
               "roofline": {"bound": "hbm", "achieved": byts / (t_b * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                            "frac": byts / (t_b * 1e-3) / 1e9 / peak, "traffic": None,
                            "model": "sum over blocks of the outer iteration's fixed passes plus the measured inner "
                                     "iterations at this build's per-kernel bytes (k-epsilon solves not counted), "
                                     "over the pass's wall time"},
               "cell_iter_per_s": cells / (t_b * 1e-3),
               "inner_iterations_last_pass": {"u": sum(x["u_inner_iterations"] for x in r),
                                              "p": sum(x["p_inner_iterations"] for x in r)},
               "blocks_with_rejected_drop": sum(1 for x in r if x["status"] != 0),
               "diverged_block_solves": {"start": start_div, "warmup": warm_div, "timed": timed_div},
               "valid": start_div + warm_div + timed_div == 0}
        print(json.dumps(out), flush=True)
    return 1 if start_div + warm_div + timed_div else 0


def main_poisson(args, world, rank, local, dist):
    """The mixed-precision pressure solve: a Delaunay tetrahedralisation of a
    seeded jittered (n+1)^3 lattice in the unit box, the orthogonal
    laplacianFace(1) operator with zero-gradient walls and one reference
    cell, a seeded standard-normal right-hand side with its mean removed.
    Each method runs from x = 0 to a 1e-8 FP64 true relative residual
    |b - Ax|2 / |b|2; a step is one such solve per method."""
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    t0 = time.perf_counter()
    mesh, pts, tets = meshgen.tet_mesh(args.tet_n, 0.1, 3)
    mesh_s = time.perf_counter() - t0
    case = cf.SimpleCase(mesh, local)
    case.poisson_setup(ref_cell=0)
    rng = np.random.default_rng(5)
    b = rng.normal(size=mesh.n_cells)
    b -= b.mean()
    methods = ["dic64", "ir32", "jacobi64", "fcg_amg"]
    # the AMG hierarchy: host structure once per mesh, device values once per
    # matrix, both outside the timed solves as the DIC factors are
    amg_info = case.poisson_amg_setup()
    if args.profile:
        # one solve of each of the two FP64-tolerance leaders, inside the
        # profiler range (ncu --profile-from-start off)
        import torch
        torch.cuda.synchronize(local)
        torch.cuda.profiler.start()
        x, rep = case.poisson_solve(b, "dic64", tol=1e-8)
        x, rep2 = case.poisson_solve(b, "fcg_amg", tol=1e-8)
        torch.cuda.synchronize(local)
        torch.cuda.profiler.stop()
        print(json.dumps({"profile": f"poisson {mesh.n_cells} tets", "dic64": rep, "fcg_amg": rep2}))
        return
    x_ref, _ = case.poisson_solve(b, "dic64", tol=1e-12, max_iter=50000)
    res = {}
    for m in methods:
        for _ in range(max(3, args.warmup)):
            case.poisson_solve(b, m, tol=1e-8, inner_tol=1e-3)
        times, reps = [], []
        barrier(dist)
        for _ in range(args.steps):
            x, rep = case.poisson_solve(b, m, tol=1e-8, inner_tol=1e-3)
            times.append(rep["device_ms"])
            reps.append(rep)
        barrier(dist)
        t_ms = allreduce_max(dist, statistics.median(times))
        res[m] = {"ms": t_ms, "inner_iterations": reps[-1]["inner_iterations"],
                  "outer_iterations": reps[-1]["outer_iterations"], "true_rel_residual": reps[-1]["true_rel_residual"],
                  "rel_err_vs_fp64_1e-12": float(np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref))}
    # the learned preconditioner: trained on residuals of the plain solver's
    # iterates (Jacobi-PCG after 0, 5, 20, 60 iterations of 6 right-hand
    # sides), then flexible CG with it (DIC-PCG fallback) on the timed rhs
    learned = learned_amg = None
    if not args.no_learned:
        rng2 = np.random.default_rng(11)
        samples = []
        for k in range(6):
            b2 = rng2.normal(size=mesh.n_cells)
            b2 -= b2.mean()
            for it in (0, 5, 20, 60):
                x2 = case.poisson_solve(b2, "jacobi64", tol=1e-14, max_iter=it)[0] if it else np.zeros_like(b2)
                samples.append(case.poisson_residual(b2, x2))
        # the learned correction of the AMG cycle: a second network trained
        # on what one V-cycle leaves of the same residuals, r - A V(r)
        amg_samples = [case.poisson_residual(s, case.poisson_amg_apply(s)) for s in samples]
        case.mpnn_create(4, seed=3)
        _, rep_u = case.poisson_solve(b, "fcg_mpnn", tol=1e-8)
        t0 = time.perf_counter()
        losses = case.mpnn_train(np.array(samples), epochs=args.train_epochs, lr=2e-3)
        train_s = time.perf_counter() - t0
        times, reps = [], []
        for _ in range(args.steps):
            x, rep = case.poisson_solve(b, "fcg_mpnn", tol=1e-8)
            times.append(rep["device_ms"])
            reps.append(rep)
        learned = {"ms": statistics.median(times), "inner_iterations": reps[-1]["inner_iterations"],
                   "outer_iterations": reps[-1]["outer_iterations"],
                   "true_rel_residual": reps[-1]["true_rel_residual"],
                   "rel_err_vs_fp64_1e-12": float(np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)),
                   "untrained_inner_iterations": rep_u["inner_iterations"], "untrained_ms": rep_u["device_ms"],
                   "train_s": train_s, "train_samples": len(samples), "train_epochs": args.train_epochs,
                   "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
                   "network": "4 message-passing layers, width 32, BF16 weights, FP32 activations",
                   "note": "outer_iterations 2 means the DIC-PCG fallback finished the solve"}
        # learned plus mixed precision: FCG preconditioned by the FP32 V-cycle
        # and the network applied to the residual each cycle leaves
        case.mpnn_create(4, seed=3)
        _, rep_u = case.poisson_solve(b, "fcg_amg_mpnn", tol=1e-8)
        t0 = time.perf_counter()
        losses = case.mpnn_train(np.array(amg_samples), epochs=args.train_epochs, lr=2e-3)
        train_s = time.perf_counter() - t0
        times, reps = [], []
        for _ in range(args.steps):
            x, rep = case.poisson_solve(b, "fcg_amg_mpnn", tol=1e-8)
            times.append(rep["device_ms"])
            reps.append(rep)
        learned_amg = {"ms": statistics.median(times), "inner_iterations": reps[-1]["inner_iterations"],
                       "outer_iterations": reps[-1]["outer_iterations"],
                       "true_rel_residual": reps[-1]["true_rel_residual"],
                       "rel_err_vs_fp64_1e-12": float(np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)),
                       "untrained_inner_iterations": rep_u["inner_iterations"], "untrained_ms": rep_u["device_ms"],
                       "train_s": train_s, "train_samples": len(amg_samples), "train_epochs": args.train_epochs,
                       "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
                       "preconditioner": "FP32 aggregation-AMG V-cycle, then the network on the residual it "
                                         "leaves; FP64 flexible CG"}
    if rank == 0:
        best = min(res, key=lambda k: res[k]["ms"])
        out = {"metric": "pressure-Poisson time to 1e-8 FP64 true relative residual", "value": res[best]["ms"],
               "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
               "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
               "data": "synthetic",
               "config": {"workload": f"Delaunay tets of a jittered {args.tet_n + 1}^3 lattice, unit box "
                                      f"({mesh.n_cells} cells), laplacianFace(1), zero-gradient walls, "
                                      f"reference cell 0, N(0,1) rhs mean-removed (seed 5)",
                          "cells": mesh.n_cells, "mesh_build_s": mesh_s, "best": best,
                          "l2": "inputs larger than L2"},
               "methods": res, "amg": amg_info, "learned_fcg": learned, "learned_amg_fcg": learned_amg,
               "speedup_ir32_vs_dic64": res["dic64"]["ms"] / res["ir32"]["ms"],
               "speedup_amg32_vs_dic64": res["dic64"]["ms"] / res["fcg_amg"]["ms"],
               "speedup_learned_vs_dic64": (res["dic64"]["ms"] / learned["ms"]) if learned else None,
               "speedup_learned_mixed_vs_dic64": (res["dic64"]["ms"] / learned_amg["ms"]) if learned_amg else None,
               "network_gain_over_amg32": (res["fcg_amg"]["ms"] / learned_amg["ms"]) if learned_amg else None}
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--cells", type=int, default=CELLS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--p-precond", default="AMG", choices=["Jacobi", "DIC", "AMG"])
    ap.add_argument("--u-precond", default="AMG", choices=["Jacobi", "AMG"],
                    help="simple: the momentum BiCGStab's preconditioner (Jacobi: the reference's; AMG: the FP32 "
                         "V-cycle of the momentum matrix)")
    ap.add_argument("--amg-theta", type=float, default=AMG_THETA,
                    help="strength threshold of the pressure AMG aggregation (0: plain aggregation)")
    ap.add_argument("--no-variant", action="store_true",
                    help="simple: skip the second pressure solver's timing from the same start state")
    ap.add_argument("--profile", action="store_true",
                    help="run --steps outer iterations from the initial state with no warm-up, timing or "
                         "baselines: the command line the ncu captures run")
    ap.add_argument("--profile-warm", type=int, default=0,
                    help="with --profile: outer iterations run before the profiler range opens")
    ap.add_argument("--workload", default="simple", choices=["simple", "cavity", "poisson", "blocks", "transient"],
                    help="simple: the 2M-cell SIMPLE channel (the headline); poisson: the ~4M-tet "
                         "pressure-Poisson solve, FP64 DIC-PCG vs FP32-in-FP64 refinement; blocks: 64 detail "
                         "blocks of a coupled network, one coupling pass per step, batched vs one after another")
    ap.add_argument("--blocks", type=int, default=64, help="blocks: number of detail blocks")
    ap.add_argument("--transient-steps", type=int, default=2000, help="transient: PISO steps in all")
    ap.add_argument("--transient-nx", type=int, default=800, help="transient: cells along the channel")
    ap.add_argument("--tet-n", type=int, default=84, help="poisson: lattice intervals per axis (6 n^3 tets)")
    ap.add_argument("--no-learned", action="store_true", help="poisson: skip the learned preconditioner")
    ap.add_argument("--train-epochs", type=int, default=30, help="poisson: training epochs of the network")
    ap.add_argument("--train-pairs", type=int, default=64, help="transient: training pairs kept from the first 75%%")
    args = ap.parse_args()
    world, rank, local, dist = dist_setup()
    if args.workload == "transient":
        main_transient(args, world, rank, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.workload == "blocks":
        rc = main_blocks(args, world, rank, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        sys.exit(rc)
    if args.workload == "poisson":
        main_poisson(args, world, rank, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.impl == "reference" and args.workload == "cavity":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no pressure reference cell, "
                                                                  "which the cavity workload needs"}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        main_reference(args, world, rank, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    rc = main_simple(args, world, rank, local, dist)
    if dist is not None:
        dist.destroy_process_group()
    sys.exit(rc)


# a step whose continuity error is this many times the first warm-up
# step's also counts as diverged: a blow-up stays finite (1e17, 1e30) for
# several iterations before it overflows into the reference's test
GROWTH = 100.0


class Steps:
    """K outer iterations with their device time, launches, inner counts and
    the divergence test of simpleSolver.cpp:360-364 (non-finite continuity,
    pressure step or fields), which SimpleResult.diverged carries, plus a
    growth test against `ref`, the first warm-up step's continuity error."""

    ref = None

    def __init__(self):
        self.ms, self.launches, self.u, self.p, self.diverged, self.cont = 0.0, 0, 0, 0, 0, []

    def run(self, case, ctl, k):
        for _ in range(k):
            r = case.solve(ctl)
            ms, nl = case.last_timing()
            self.ms += ms[7]
            self.launches += nl
            self.u += r.u_inner_iterations
            self.p += r.p_inner_iterations
            c = r.final_continuity_error
            if Steps.ref is None and np.isfinite(c):
                Steps.ref = c
            self.diverged += int(r.diverged or not np.isfinite(c) or grown(c))
            self.cont.append(c)
        return self


def grown(c):
    return Steps.ref is not None and c > GROWTH * max(Steps.ref, 1e-300)


def rel_l2(a, b):
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))


def field_errors(U, p, phi, U0, p0, phi0, mean_free=False):
    """Relative L2 errors per field (p mean-removed when no cell pins it)."""
    if mean_free:
        p, p0 = p - p.mean(), p0 - p0.mean()
    return {"U": rel_l2(U, U0), "p": rel_l2(p, p0), "phi": rel_l2(phi, phi0)}


def main_simple(args, world, rank, local, dist):
    """The headline: K SIMPLE outer iterations of the 2M-cell channel on
    device-resident fields after W warm-up iterations.  Every leg counts
    its diverged iterations; a run with any is reported and exits 1."""
    cavity = args.workload == "cavity"
    n = args.cells if not cavity else 2 * args.cells
    if cavity:
        mesh, case, ctl = make_cavity_case(n, local, args.p_precond, p_relax_start=5e-4)
    else:
        mesh, case, ctl = make_case(n, local, args.p_precond, args.amg_theta)
    ctl = dataclasses.replace(ctl, u_preconditioner=args.u_precond)
    config = (cavity_config(n, args.p_precond) if cavity else
              workload_config(n, args.p_precond, args.u_precond, args.amg_theta))
    ncell = mesh.n_cells
    if args.profile:
        import torch
        # --profile-warm W outer iterations first, outside the profiler range
        # (ncu --profile-from-start off captures only the --steps after them)
        for _ in range(args.profile_warm):
            case.solve(ctl)
        torch.cuda.synchronize(local)
        torch.cuda.profiler.start()
        for _ in range(args.steps):
            r = case.solve(ctl)
        torch.cuda.synchronize(local)
        torch.cuda.profiler.stop()
        print(json.dumps({"profile": config["workload"], "steps": args.steps,
                          "warm": args.profile_warm, "u_inner": r.u_inner_iterations,
                          "p_inner": r.p_inner_iterations}))
        return 0
    W = max(3, args.warmup)
    warm = Steps().run(case, ctl, W)
    # the state every leg starts from: the timed, end-to-end, kernel-timing
    # and comparison legs all run the same K outer iterations from it
    U0, p0, phi0 = case.download()

    # ---- timed region: K outer iterations on device-resident fields ----
    barrier(dist)
    with Clocks(local) as clk:
        t0 = time.perf_counter()
        timed = Steps().run(case, ctl, args.steps)
        wall = time.perf_counter() - t0
    barrier(dist)
    U1, p1, phi1 = case.download()
    t_max = allreduce_max(dist, timed.ms / 1e3)
    value = job_rate(world, ncell * args.steps, t_max)

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
    e2e_div = 0
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        case.upload(U, p, phi)
        r = case.solve(ctl)
        case.download(U, p, phi)
        e2e_div += int(r.diverged or not np.isfinite(r.final_continuity_error) or grown(r.final_continuity_error))
    e2e_wall = allreduce_max(dist, time.perf_counter() - t0)
    e2e = job_rate(world, ncell * args.steps, e2e_wall)
    e2e_same = bool(np.array_equal(U, U1) and np.array_equal(p, p1) and np.array_equal(phi, phi1))

    # ---- per-kernel event timing (outside the timed region: the events
    # keep the solver chunks out of CUDA graphs) over the first iteration ----
    case.upload(U0, p0, phi0)
    case.kernel_timing(True)
    ktimed = Steps().run(case, ctl, 1)
    kstats = case.kernel_stats()
    kcomp = case.kernel_components()
    case.kernel_timing(False)

    # ---- rooflines: every solver kernel, the dominant one, and the whole step ----
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    alg = kernel_bytes(ncell, mesh.n_internal_faces)
    kernels = {}
    solver_bytes = 0.0
    for k, (cnt, tot) in kstats.items():
        if cnt:
            us = tot / cnt * 1e3
            shared, per = alg[k]
            comps = kcomp[k] / cnt if k in SKIPS_DONE else (3 if k.startswith(("bi", "amgv")) else 0)
            b = shared + per * comps
            kernels[k] = {"launches": cnt, "total_ms": tot, "avg_us": us, "alg_bytes": b,
                          "components_per_launch": comps if k.startswith(("bi", "amgv")) else None,
                          "achieved_gbs": b / (us * 1e-6) / 1e9}
            # scaled from the kernel-timing iteration to the timed region's
            # mean inner counts
            scale = ((timed.u / args.steps) / max(1, ktimed.u) if k.startswith(("bi", "amgv"))
                     else (timed.p / args.steps) / max(1, ktimed.p))
            solver_bytes += cnt * b * scale
    # the dominant single kernel (the V-cycle's coarse slot spans several)
    top = max((k for k in kernels if k not in COMPOSITE), key=lambda k: kernels[k]["total_ms"])
    kt = kernels[top]
    # DRAM bytes per launch of the top kernel from one ncu capture of this
    # workload (profiles/), null for a kernel without one
    traffic, traffic_note = MEASURED_TRAFFIC.get(top, (None, None)) if n == CELLS else (None, None)
    roof = {"kernel": KERNEL_NAMES[top], "bound": "hbm", "achieved": kt["achieved_gbs"], "peak": peak,
            "unit": "GB/s", "frac": kt["achieved_gbs"] / peak, "peak_source": peak_src, "traffic": traffic,
            "traffic_note": traffic_note,
            "algorithmic_bytes_per_launch": kt["alg_bytes"], "launches_timed": kt["launches"],
            "avg_launch_us": kt["avg_us"], "timing": "CUDA events around each launch over one outer iteration "
                                                     "from the timed region's start state",
            "kernels": kernels}
    step_bytes = simple_step_bytes(ncell, mesh.n_internal_faces, mesh.n_boundary_faces, 1, timed.p / args.steps,
                                   args.p_precond, solver_bytes)
    step_s = t_max / args.steps
    simple_roof = {"bytes_per_step": step_bytes, "achieved_gbs": step_bytes / step_s / 1e9,
                   "frac": step_bytes / step_s / 1e9 / peak, "peak": peak,
                   "model": "this build's per-kernel algorithmic bytes (roofline.kernels) per solver iteration times "
                            "the timed region's inner iteration counts, plus the fixed face and cell passes of an "
                            "outer iteration, over the device time per step"}

    out = {"metric": METRIC, "value": value, "unit": "cell-iter/s", "n_gpus": world, "steps": args.steps,
           "warmup": W, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": config,
           "e2e": {"value": e2e, "unit": "cell-iter/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                   "steps": args.steps, "same_fields_as_timed": e2e_same},
           "gpu_launches": timed.launches, "roofline": roof, "simple_roofline": simple_roof, "clocks": clk.summary(),
           "inner_iterations_per_step": {"momentum_bicgstab_sum_over_components": timed.u / args.steps,
                                         "pressure": timed.p / args.steps},
           "continuity": {"first": timed.cont[0], "last": timed.cont[-1], "max": max(timed.cont)},
           "diverged_steps": {"warmup": warm.diverged, "timed": timed.diverged, "e2e": e2e_div},
           "wall_s_timed": wall}
    diverged = warm.diverged + timed.diverged + e2e_div

    # ---- the same K outer iterations from the same start state with the
    # other FP64-tolerance pressure solver, after one untimed iteration that
    # sets it up; with FP64 DIC-PCG (FP64 throughout) as the other solver,
    # its fields are the FP64 solve the headline's fields are measured
    # against ----
    if not args.no_variant:
        other = "DIC" if args.p_precond == "AMG" else "AMG"
        # with DIC pressure the variant runs FP64 throughout: the reference's
        # Jacobi-BiCGStab momentum as well
        c2 = dataclasses.replace(ctl, p_preconditioner=other,
                                 u_preconditioner="Jacobi" if other == "DIC" else ctl.u_preconditioner)
        case.upload(U0, p0, phi0)
        case.solve(c2)
        case.upload(U0, p0, phi0)
        barrier(dist)
        var = Steps().run(case, c2, args.steps)
        barrier(dist)
        U2, p2, phi2 = case.download()
        v_t = allreduce_max(dist, var.ms / 1e3)
        out["variant"] = {"pressure": other + (" (FP64 flexible CG, FP32 AMG V-cycle)" if other == "AMG" else
                                               " (FP64 multicolour DIC-PCG)"),
                          "momentum": c2.u_preconditioner + "-BiCGStab" + (" (FP64 throughout)" if other == "DIC"
                                                                           else ""),
                          "value": world * ncell * args.steps / v_t, "ms_per_step": v_t * 1e3 / args.steps,
                          "inner_iterations_per_step": {"momentum_bicgstab_sum_over_components": var.u / args.steps,
                                                        "pressure": var.p / args.steps},
                          "continuity": {"first": var.cont[0], "last": var.cont[-1]},
                          "diverged_steps": var.diverged,
                          "note": "same start state and steps as the headline, timed the same way"}
        diverged += var.diverged
        fp64 = (U2, p2, phi2) if other == "DIC" else (U1, p1, phi1)
        test = (U1, p1, phi1) if other == "DIC" else (U2, p2, phi2)
        out["field_error"] = dict(field_errors(*test, *fp64),
                                  against="FP64 throughout (Jacobi-BiCGStab momentum, DIC-PCG pressure), the same K "
                                          "iterations from the same start state; relative L2")

    # ---- the other momentum preconditioner: the same K iterations from the
    # same start state with the reference's Jacobi-BiCGStab momentum solve
    # or the AMG-preconditioned one, against the FP64 DIC fields ----
    if not args.no_variant:
        other_u = "AMG" if args.u_precond == "Jacobi" else "Jacobi"
        c4 = dataclasses.replace(ctl, u_preconditioner=other_u)
        case.upload(U0, p0, phi0)
        case.solve(c4)
        case.upload(U0, p0, phi0)
        barrier(dist)
        mom = Steps().run(case, c4, args.steps)
        barrier(dist)
        U4, p4, phi4 = case.download()
        u_t = allreduce_max(dist, mom.ms / 1e3)
        out["momentum_" + other_u.lower()] = {
            "momentum": ("BiCGStab with the FP32 AMG V-cycle of the momentum matrix as right preconditioner (one "
                         "V-cycle for the three components), FP64 vectors and |r|inf/|b|inf test at 1e-8"
                         if other_u == "AMG" else "the reference's Jacobi-BiCGStab"),
            "value": world * ncell * args.steps / u_t, "ms_per_step": u_t * 1e3 / args.steps,
            "inner_iterations_per_step": {"momentum_bicgstab_sum_over_components": mom.u / args.steps,
                                          "pressure": mom.p / args.steps},
            "continuity": {"first": mom.cont[0], "last": mom.cont[-1]},
            "diverged_steps": mom.diverged,
            "field_error_vs_fp64_dic": field_errors(U4, p4, phi4, *fp64)}
        diverged += mom.diverged

    # ---- mixed precision: the same K iterations with the pressure matrix
    # rounded to FP32 and FP32 DIC-PCG corrections inside FP64 refinement
    # (FP64 residual and infinity-norm test), against the FP64 DIC fields ----
    if not args.no_variant:
        c3 = dataclasses.replace(ctl, p_preconditioner="IR32")
        case.upload(U0, p0, phi0)
        case.solve(c3)
        case.upload(U0, p0, phi0)
        barrier(dist)
        mix = Steps().run(case, c3, args.steps)
        barrier(dist)
        U3, p3, phi3 = case.download()
        m_t = allreduce_max(dist, mix.ms / 1e3)
        out["mixed_precision"] = {
            "pressure": "matrix rounded to FP32, FP32 multicolour DIC-PCG corrections to 1e-4 inside FP64 iterative "
                        "refinement, FP64 residual and |r|inf/|b|inf test at 1e-8",
            "value": world * ncell * args.steps / m_t, "ms_per_step": m_t * 1e3 / args.steps,
            "inner_iterations_per_step": {"momentum_bicgstab_sum_over_components": mix.u / args.steps,
                                          "pressure_fp32": mix.p / args.steps},
            "diverged_steps": mix.diverged,
            "field_error_vs_fp64_dic": field_errors(U3, p3, phi3, *fp64)}
        diverged += mix.diverged

    # ---- the reference's own work on the GPU: its first outer iteration
    # from rest exactly as it runs it (no pressure reference cell, Jacobi-
    # PCG), timed and compared with the reference's CPU run of that
    # iteration (the cpu_baseline leg) ----
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not cavity:
        case.upload(np.zeros((ncell, 3)), np.zeros(ncell), np.zeros(mesh.n_faces))
        case.init_flux()
        rc = dataclasses.replace(ctl, p_preconditioner="Jacobi", u_preconditioner="Jacobi")
        same = Steps().run(case, rc, 1)
        Ug, pg, phig = case.download()
        secs, kind, what, ref_fields = run_reference_cpu(n, mesh.addressing()["points"], fields=True)
        out["cpu_baseline"] = {"value": ncell / secs, "unit": "cell-iter/s", "cores": 1, "kind": kind,
                               "sample": f"one SIMPLE outer iteration of the same mesh and settings from rest "
                                         f"({secs:.1f} s), with the reference's Jacobi-PCG pressure; {what}; "
                                         f"{cpu_info()}"}
        out["reference_step_same_work"] = {
            "what": "the reference's first outer iteration from rest with its own solvers (Jacobi-BiCGStab momentum, "
                    "Jacobi-PCG pressure), on this GPU and by the reference on one core",
            "gpu_ms": same.ms, "cpu_ms": secs * 1e3, "speedup": secs * 1e3 / same.ms,
            "inner_iterations_gpu": {"momentum": same.u, "pressure": same.p},
            "field_error_vs_reference": (field_errors(Ug, pg, phig, *ref_fields) if ref_fields else None),
            "diverged": same.diverged}
    if rank == 0:
        out["valid"] = diverged == 0
        print(json.dumps(out), flush=True)
    return 1 if diverged else 0


if __name__ == "__main__":
    main()
