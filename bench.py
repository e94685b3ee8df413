"""Benchmark: solve time to FP64 relative residual 1e-10 on the large 3-D
elasticity cantilever (box [0,4]x[0,1]x[0,1], box_mesh [280,70,70] -> 1,416,521
nodes, 8,232,000 tets, 4,234,440 free dofs; per-tet E = 1e-3 + (1-1e-3) rho^3
from a seeded smoothed density; nu = 0.3; x = 0 clamped; traction (0,0,-1e-3)
on x = 4).  Inputs are synthetic (seeded), no dataset exists for this path.

A step is one complete solve from x = 0 of the device-resident reduced system
with the two-level learned preconditioner -- learned FSAI factor (network
forward on this system, FP16 factor) plus the rigid-body aggregation coarse
space (A_c = P^T A P assembled and inverted on this system) -- and FP64 PCG,
set-up included, stopping on the TRUE FP64 residual.  --no-coarse times the
single-level learned FSAI instead.  `value`
is the median device time of a step (CUDA events on the library's stream);
`e2e` runs the same solve through the C ABI from host arrays (mesh upload,
assembly, traction, Dirichlet reduction, learned factor, solve, solution
download).  The plain method (FP64 Jacobi-PCG, CSR operator) is timed on the
same GPU in the same run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank solves its own replica: the path is one
SPD solve per GPU (replicas only), value = max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tpt-fem_b200"))

METRIC = "solve time to FP64 rel. residual 1e-10: learned mixed-prec PCG vs FP64 Jacobi-PCG"
WORKLOAD = "cantilever_280x70x70"
TOL = 1e-10


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    """One process per GPU (torchrun env); NCCL on GPUs, gloo where there are none."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier_max(value, world):
    """Max over ranks (every rank reports its own device-timed value)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cuda_sync():
    try:
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except Exception:
        pass


# ---- CPU baseline (oracle port) --------------------------------------------------

CPU_SOLVE_BUDGET_S = 150.0  # reference arm: complete CPU solves are timed until this much has been spent


def host_system(S):
    """The device-resident reduced system as host int32 CSR + right-hand side
    (the same bits the GPU solves; input generation, never timed)."""
    rp, ci, va, fred, _ = S.download()
    return rp.astype(np.int32), ci.astype(np.int32), va, fred


def cpu_full_solve(sysh, tol, threads):
    """One complete oracle FP64 Jacobi-PCG solve (all `threads` host cores,
    int32 CSR) from x = 0 to the TRUE relative residual `tol`: (seconds,
    iterations, true relative residual)."""
    from oracle import oracle as O
    rp, ci, va, b = sysh
    t0 = time.perf_counter()
    _, it, rel = O.pcg_jacobi_i32(len(b), rp, ci, va, b, tol=tol, max_it=200000, nthreads=threads)
    return time.perf_counter() - t0, it, rel


def cpu_ms_per_iteration(sysh, threads, iters=10):
    """Measured milliseconds per oracle Jacobi-PCG iteration on this system
    with `threads` cores (a fixed iteration count, no convergence)."""
    from oracle import oracle as O
    rp, ci, va, b = sysh
    t0 = time.perf_counter()
    _, it, _ = O.pcg_jacobi_i32(len(b), rp, ci, va, b, tol=1e-300, max_it=iters, nthreads=threads)
    return (time.perf_counter() - t0) / abs(it) * 1e3


def cpu_threads():
    from oracle import oracle as O
    return O.max_threads()


# ---- our arm -----------------------------------------------------------------------

def build_system(F, W, ctx, mesh_cells=None):
    mn, mx, n = W.CANTILEVERS[WORKLOAD]
    if mesh_cells:
        n = list(mesh_cells)
    E = W.cantilever_young(n)
    mesh = F.Mesh.box_mesh(mn, mx, n, ctx=ctx)
    K = F.assemble_elasticity(mesh, "3d", E, 0.3, 2)
    coords = W.box_coords(mn, mx, n)
    rhs = F.apply_traction(mesh, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(coords)
    S = F.reduce_system(K, rhs, list(zip(dof, val)))
    return mesh, K, S, E, rhs, dof, val


WEIGHTS = os.path.join(ROOT, "tpt-fem_b200", "weights", "lfsai_elasticity.bin")
# DRAM bytes (read + write) of one nb_spmv_sym<3> launch measured by ncu on the
# 200x50x50 cantilever (520,200 node groups; profiles/ has the capture); the
# bench case is scaled by its node-group count.
NBS_TRAFFIC_200 = (359.652352 + 12.161024) * 1e6
NBS_GROUPS_200 = 520200


def e2e_once(F, LF, W, ctx, solver, host, model, coarse, phases=None):
    """Host arrays -> C ABI -> host solution; returns (seconds, h2d bytes, d2h bytes, stats).
    Mesh upload, assembly, traction, Dirichlet reduction, the learned factor and
    the solve all run inside the timed region.  With `phases` (a dict), each
    step is synchronised and its wall time recorded there (an untimed run)."""
    coords, conn, E, dof, val = host
    cuda_sync()
    t0 = time.perf_counter()
    last = [t0]

    def mark(name):
        if phases is not None:
            ctx.synchronize()
            t = time.perf_counter()
            phases[name] = round((t - last[0]) * 1e3, 2)
            last[0] = t

    mesh = F.Mesh.from_arrays(F.CELL_TET4, coords, conn, ctx=ctx)
    mark("mesh_upload")
    K = F.assemble_elasticity(mesh, "3d", E, 0.3, 2)
    mark("assembly")
    rhs = F.apply_traction(mesh, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    mark("traction")
    S = F.reduce_system(K, rhs, list(zip(dof, val)))
    mark("reduction")
    if solver == F.SOLVER_LEARNED_FSAI_PCG:
        model.attach(S)
    st = S.solve(solver=solver, tol=TOL, fresh_setup=True, coarse=coarse)
    mark("first_solve")
    u = S.solution()
    ctx.synchronize()
    mark("solution_download")
    dt = time.perf_counter() - t0
    h2d = coords.nbytes + conn.nbytes + E.nbytes + 2 * rhs.nbytes + dof.nbytes + val.nbytes
    d2h = u.nbytes + rhs.nbytes
    return dt, h2d, d2h, st


def seconds(st):
    return (st["setup_ms"] + st["solve_ms"]) / 1e3


def run_ours(args, world, rank, local):
    import tpt_fem as F
    from tpt_fem import lfsai as LF
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    mesh, K, S, E, rhs, dof, val = build_system(F, W, ctx, args.mesh if args.profile else None)
    model = LF.LearnedFsai.load(ctx, WEIGHTS)
    model.attach(S)
    solver = {"learned": F.SOLVER_LEARNED_FSAI_PCG, "fsai": F.SOLVER_FSAI_MP_PCG, "jacobi": F.SOLVER_JACOBI_PCG,
              "mp": F.SOLVER_MP_PCG}[args.solver]
    coarse = not args.no_coarse and solver in (F.SOLVER_LEARNED_FSAI_PCG, F.SOLVER_FSAI_MP_PCG)
    if args.profile:  # kernels of the timed steps only (for an ncu launch list)
        for _ in range(args.steps):
            S.solve(solver=solver, tol=TOL, fresh_setup=True, coarse=coarse)
        ctx.synchronize()
        return None
    # The plain method the metric compares against: FP64 Jacobi-PCG with the
    # CSR operator (warp-per-row SpMV); also the same method on the node-block
    # operator, and classic FSAI, for the record.
    S.solve(solver=F.SOLVER_JACOBI_PCG, tol=TOL, fresh_setup=True, csr_only=True)
    jac = S.solve(solver=F.SOLVER_JACOBI_PCG, tol=TOL, fresh_setup=True, csr_only=True)
    jac_nb = S.solve(solver=F.SOLVER_JACOBI_PCG, tol=TOL, fresh_setup=True)
    S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=TOL, fresh_setup=True)
    fsai = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=TOL, fresh_setup=True)
    S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=TOL, fresh_setup=True, coarse=True)  # builds the coarse geometry
    fsai2 = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=TOL, fresh_setup=True, coarse=True)
    lrn1 = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=TOL, fresh_setup=True)
    lrn1 = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=TOL, fresh_setup=True)
    for _ in range(args.warmup):
        S.solve(solver=solver, tol=TOL, fresh_setup=True, coarse=coarse)
    barrier(world)
    cuda_sync()
    steps = []
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            steps.append(S.solve(solver=solver, tol=TOL, fresh_setup=True, coarse=coarse))
        cuda_sync()
        t_wall = time.perf_counter() - t_wall
    barrier(world)
    step_s = barrier_max(statistics.median([seconds(st) for st in steps]), world)
    # roofline of the dominant kernel: the Krylov operator y = K x
    prof = S.profile_spmv(20)
    n, nnz = S.n_free, S.nnz
    csr_bytes = nnz * (8 + 4) + 4 * (n + 1) + 8 * n + 8 * n  # CSR formula: values, int32 cols, row ptrs, x, y
    peak, peak_kind = measured_peaks()
    traffic = None
    if prof["nbs_ms"] > 0:
        op_ms, op_bytes = prof["nbs_ms"], prof["nbs_bytes"]
        op_name = "nb_spmv_sym<3> (node-block sliced ELL, symmetric half storage, FP64)"
        traffic = NBS_TRAFFIC_200 * (n / 3) / NBS_GROUPS_200
    elif prof["nb_ms"] > 0:
        op_ms, op_bytes = prof["nb_ms"], prof["nb_bytes"]
        op_name = "nb_spmv<3> (node-block sliced ELL, FP64)"
    else:
        op_ms, op_bytes = prof["csr_f64_ms"], csr_bytes
        op_name = "spmv_kernel<double> (CSR, FP64)"
    achieved = op_bytes / (op_ms * 1e-3) / 1e9
    # end to end through the C ABI from host arrays, on every rank's replica
    # (max over ranks): one untimed run pays the first-use costs (the pinned
    # staging buffer, library module loads); then the median of three timed runs
    coords = mesh.coords_array.copy()
    conn = mesh.conn_array.copy()
    e2e_once(F, LF, W, ctx, solver, (coords, conn, E, dof, val), model, coarse)
    barrier(world)
    e2e = [e2e_once(F, LF, W, ctx, solver, (coords, conn, E, dof, val), model, coarse) for _ in range(3)]
    e2e_s, h2d, d2h, e2e_st = sorted(e2e, key=lambda t: t[0])[1]
    e2e_s = barrier_max(e2e_s, world)
    out = None
    if rank == 0:
        phases = {}
        e2e_once(F, LF, W, ctx, solver, (coords, conn, E, dof, val), model, coarse, phases)
        # the plain method on the host cores (at N = 1 only: the other ranks
        # would wait on rank 0 at the next collective): one complete solve of
        # this exact system, measured (no scaling), and the one-core iteration cost
        cpu = None
        if world == 1:
            sysh = host_system(S)
            nthr = cpu_threads()
            cpu_ms_per_iteration(sysh, nthr, 3)  # page in, start the thread team
            cpu_s, cpu_it, cpu_rel = cpu_full_solve(sysh, TOL, nthr)
            cpu_1core_ms = cpu_ms_per_iteration(sysh, 1, 5)
            del sysh
            cpu = {"value": cpu_s, "unit": "s", "cores": nthr, "kind": "port", "iterations": cpu_it,
                   "rel_residual": cpu_rel, "one_core_ms_per_iteration": cpu_1core_ms,
                   "sample": f"one complete oracle FP64 Jacobi-PCG solve (int32 CSR, OpenMP, {nthr} host "
                             f"threads) of this exact reduced system from x = 0 to true rel. residual "
                             f"{TOL:g}: {abs(cpu_it)} iterations, measured, not scaled; one core measured "
                             f"at {cpu_1core_ms:.1f} ms per iteration over 5 iterations"}
        its = [st["iterations"] for st in steps]
        fsai_like = solver in (F.SOLVER_FSAI_MP_PCG, F.SOLVER_LEARNED_FSAI_PCG)
        kernels_per_it = (5 if fsai_like else 3) + (3 if coarse else 0)
        setup_kernels = (40 if solver == F.SOLVER_LEARNED_FSAI_PCG else 12) + (4 * 27 + 8 if coarse else 0)
        launches = sum(st["iterations"] * kernels_per_it + st["outer_steps"] * 6 + setup_kernels for st in steps)
        out = {
            "metric": METRIC, "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (factor f16/f32, network f32)",
            "data": "synthetic (seeded density field)",
            "config": {"workload": WORKLOAD, "mesh": [280, 70, 70], "nodes": int(mesh.n_nodes),
                       "tets": int(mesh.n_elems), "free_dofs": int(n), "nnz_reduced": int(nnz),
                       "solver": args.solver + ("+coarse" if coarse else ""),
                       "preconditioner": ("learned FSAI (FP16 factor) + " if solver == F.SOLVER_LEARNED_FSAI_PCG
                                          else "FSAI + ") + ("rigid-body aggregation coarse space (FP32 inverse)"
                                                             if coarse else "single level"),
                       "weights": os.path.relpath(WEIGHTS, ROOT), "tol": TOL,
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (matrix 1.85 GB)"},
            "solver_stats": {"iterations_median": statistics.median(its), "rel_residual": steps[-1]["rel_residual"],
                             "setup_ms": steps[-1]["setup_ms"], "solve_ms": steps[-1]["solve_ms"],
                             "reliable_updates": steps[-1]["outer_steps"], "fell_back": steps[-1]["fell_back"],
                             "coarse_size": steps[-1]["coarse_size"],
                             "step_s": [round(seconds(st), 4) for st in steps],
                             "setup_ms_steps": [round(st["setup_ms"], 2) for st in steps]},
            "fp64_jacobi_pcg": {"seconds": seconds(jac), "iterations": jac["iterations"],
                                "rel_residual": jac["rel_residual"], "operator": "CSR"},
            "fp64_jacobi_pcg_node_block": {"seconds": seconds(jac_nb), "iterations": jac_nb["iterations"],
                                           "rel_residual": jac_nb["rel_residual"]},
            "classic_fsai_pcg": {"seconds": seconds(fsai), "iterations": fsai["iterations"],
                                 "rel_residual": fsai["rel_residual"]},
            "classic_fsai_coarse_pcg": {"seconds": seconds(fsai2), "iterations": fsai2["iterations"],
                                        "rel_residual": fsai2["rel_residual"], "coarse_size": fsai2["coarse_size"]},
            "learned_fsai_single_level": {"seconds": seconds(lrn1), "iterations": lrn1["iterations"],
                                          "rel_residual": lrn1["rel_residual"]},
            "speedup_vs_fp64_jacobi": seconds(jac) / step_s,
            "speedup_vs_fp64_jacobi_node_block": seconds(jac_nb) / step_s,
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "iterations": e2e_st["iterations"], "runs_s": [round(t[0], 4) for t in e2e],
                    "phases_ms_untimed_run": phases},
            "roofline": {"bound": "hbm", "kernel": op_name, "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_source": "ncu dram__bytes_read+write of nb_spmv_sym at "
                         "200x50x50 (371.8 MB) scaled by node groups", "algorithmic_bytes": op_bytes, "ms": op_ms,
                         "csr_formula_bytes": csr_bytes,
                         "csr_formula_gbs": csr_bytes / (op_ms * 1e-3) / 1e9,
                         "nb_full_ms": prof["nb_ms"], "csr_f64_ms": prof["csr_f64_ms"],
                         "csr_f64_gbs": csr_bytes / (prof["csr_f64_ms"] * 1e-3) / 1e9},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "wall_s_timed_region": t_wall,
        }
        if cpu is not None:
            out["cpu_baseline"] = cpu
    return out


def run_partitioned(args, world, rank, local):
    """The row-partitioned two-level PCG (tptfem_dist_*: block learned FSAI of
    each rank's x-slab plus the coarse space from the ranks' summed partial
    coarse matrices) on the headline system, 1, 2, 4 and 8 ranks run in lock
    step on this process's GPU (tpt_fem.distributed with LocalComm: the
    exchanges are device copies, the sums host additions).  What it measures
    is how the partition changes the iteration count; its wall time includes
    the Python driver's per-step host round trips, so it is no multi-GPU
    timing."""
    import tpt_fem as F
    from tpt_fem import distributed as D
    from tpt_fem import lfsai as LF
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    mesh, K, S, E, rhs, dof, val = build_system(F, W, ctx, args.mesh)
    model = LF.LearnedFsai.load(ctx, WEIGHTS)
    model.attach(S)
    one = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=TOL, fresh_setup=True, coarse=True)
    rec = {"one_gpu_engine": {"iterations": one["iterations"], "rel_residual": one["rel_residual"],
                              "coarse_size": one["coarse_size"]}}
    import scipy.sparse as sp
    rp, ci, va, fred, _ = S.download()
    A = sp.csr_matrix((va, ci, rp), shape=(S.n_free, S.n_free))
    del rp, ci, va
    for nranks in (1, 2, 4, 8):
        starts = D.partition_rows(S.n_free, 3, nranks)
        ranks = [D.LibRank(S, k, nranks, starts) for k in range(nranks)]
        t0 = time.perf_counter()
        nc = {r.set_precond("learned", 0) for r in ranks}
        t1 = time.perf_counter()
        it, rel = D.solve(ranks, D.LocalComm(), tol=TOL, max_iter=2000)
        t2 = time.perf_counter()
        x = np.concatenate([r.solution() for r in ranks])
        rec[f"ranks_{nranks}"] = {"iterations": it, "rel_residual": rel, "coarse_size": max(nc),
                                 "host_rel_residual": float(np.linalg.norm(fred - A @ x) / np.linalg.norm(fred)),
                                 "setup_s": t1 - t0, "solve_wall_s": t2 - t1}
        del ranks
    if rank != 0:
        return None
    return {"metric": "iterations to FP64 rel. residual 1e-10 of the row-partitioned two-level PCG "
                      "(lock-step ranks on one GPU)", "value": rec["ranks_8"]["iterations"], "unit": "iterations",
            "higher_is_better": False,
            "config": {"workload": "partitioned_" + WORKLOAD, "free_dofs": int(S.n_free),
                       "preconditioner": "block learned FSAI per x-slab + rigid-body coarse space (summed partial "
                                         "coarse matrices)", "tol": TOL},
            "runs": rec}


def run_cantilever_sizes(args, world, rank, local):
    """The cantilever family at its other sizes: [200,50,50] (1.56M free dofs)
    and [400,100,100] (12.27M free dofs), same density recipe, clamp and
    traction.  Per size: the headline solver (learned FSAI + coarse space,
    fresh set-up) and FP64 Jacobi-PCG (node-block operator), each to the FP64
    relative residual 1e-10, one untimed warm-up solve then one timed solve."""
    import tpt_fem as F
    from tpt_fem import lfsai as LF
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    model = LF.LearnedFsai.load(ctx, WEIGHTS)
    out = {}
    for name in ("cantilever_200x50x50", "cantilever_400x100x100"):
        mesh, K, S, E, rhs, dof, val = build_system(F, W, ctx, W.CANTILEVERS[name][2])
        model.attach(S)
        rec = {"mesh": W.CANTILEVERS[name][2], "free_dofs": int(S.n_free), "nnz_reduced": int(S.nnz)}
        for meth, kw in (("learned_coarse", dict(solver=F.SOLVER_LEARNED_FSAI_PCG, coarse=True)),
                         ("fp64_jacobi_node_block", dict(solver=F.SOLVER_JACOBI_PCG))):
            S.solve(tol=TOL, fresh_setup=True, **kw)
            barrier(world)
            st = S.solve(tol=TOL, fresh_setup=True, **kw)
            rec[meth] = {"seconds": barrier_max(seconds(st), world), "iterations": st["iterations"],
                         "rel_residual": st["rel_residual"], "setup_ms": st["setup_ms"],
                         "fell_back": st["fell_back"]}
        rec["speedup"] = rec["fp64_jacobi_node_block"]["seconds"] / rec["learned_coarse"]["seconds"]
        out[name] = rec
        del mesh, K, S
    return out if rank == 0 else None


CUBE_TOL_REF = 1e-12  # the FP64 reference solution the cube's solutions are measured against


def run_box8(args, world, rank, local):
    """The reference's CPU-runnable case: Poisson on the unit cube, box_mesh
    [8,8,8] P1 tets (729 nodes), k = 1, f = 1, order 2, u = 0 on all six
    faces.  Through the library: device mesh, assembly, load, reduction and
    FP64 Jacobi-PCG to 1e-14 (solve_with_dirichlet); on the host: the oracle's
    solve_with_dirichlet, which is the reference's own path here (COO assembly,
    to_csr, dense LU; one core).  Both timed end to end over the same repeated
    calls; the solution agrees with the LU to 1e-12 relative."""
    import tpt_fem as F
    from oracle import oracle as O
    ctx = F.Context(local)
    n = [8, 8, 8]
    c, e = O.box_mesh([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], n)
    bcs = []
    for axis in range(3):
        for coord in (0.0, 1.0):
            bcs += [(int(i), 0.0) for i in O.nodes_on_plane(c, axis, coord, 1e-9)]

    def gpu_once():
        mesh = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], n, ctx=ctx)
        K = F.assemble_poisson(mesh, 1.0, 2)
        rhs = F.load_poisson_source(mesh, 1.0, 2)
        return F.solve_with_dirichlet(K, rhs, bcs, tol=1e-14)

    def cpu_once():
        om = O.Mesh(O.CELL_TET, c, e)
        coo = O.assemble_poisson(om, 1.0, 2)
        return O.solve_with_dirichlet(coo, O.load_poisson_source(om, 1.0, 2), bcs)

    reps = 20
    for _ in range(3):
        u, st = gpu_once()
    t0 = time.perf_counter()
    for _ in range(reps):
        u, st = gpu_once()
    gpu_s = barrier_max((time.perf_counter() - t0) / reps, world)
    if rank != 0:
        return None
    u_ref = cpu_once()
    rec = {"metric": "solve_poisson end to end (mesh, assembly, load, reduction, solve)", "value": gpu_s,
           "unit": "s", "higher_is_better": False,
           "config": {"workload": "poisson_box8", "mesh": n, "nodes": len(c), "free_dofs": 343, "tol": 1e-14},
           "max_rel_error_vs_dense_lu": float(np.max(np.abs(u - u_ref)) / np.max(np.abs(u_ref))),
           "iterations": st["iterations"]}
    if world == 1:
        t0 = time.perf_counter()
        for _ in range(3):
            cpu_once()
        rec["cpu_baseline"] = {"value": (time.perf_counter() - t0) / 3, "unit": "s", "cores": 1, "kind": "port",
                               "sample": "oracle solve_with_dirichlet on the same case (COO assembly, to_csr, "
                                         "dense LU -- the reference's own path), 3 calls, measured"}
    return rec


def run_cube(args, world, rank, local):
    """Unit-cube elasticity: box_mesh [64,64,64] P1 tets (274,625 nodes,
    823,875 dofs, 811,200 free), E = 1, nu = 0.3, x = 0 clamped, traction
    (0, 0, -1e-3) on x = 1, FP64 assembly.  The plain FP64 Jacobi-PCG (CSR
    operator) against the FP32-inner / FP64-refinement PCG (MP_PCG: FP32
    operator values, vectors and SpMV inside; FP64 true residual, solution
    accumulation and refinement outside) to FP64 relative residual 1e-10, each
    with its max error against an FP64 reference solution (FP64 Jacobi-PCG to
    1e-12); assembly Melem/s and SpMV GB/s of both precisions."""
    import tpt_fem as F
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    mn, mx, n = W.CANTILEVERS["cube_elasticity_64"]
    mesh = F.Mesh.box_mesh(mn, mx, n, ctx=ctx)
    K = F.assemble_elasticity(mesh, "3d", 1.0, 0.3, 2)
    K.profile_assembly(2)
    asm_ms = barrier_max(K.profile_assembly(10), world)
    rhs = F.apply_traction(mesh, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(mesh.coords_array)
    S = F.reduce_system(K, rhs, list(zip(dof, val)))
    free = np.setdiff1d(np.arange(K.nrows), dof)
    S.solve(solver=F.SOLVER_JACOBI_PCG, tol=CUBE_TOL_REF, csr_only=True, fresh_setup=True)
    u_ref = S.solution()[free]
    steps = max(1, min(args.steps, 5))
    rec = {}
    for name, kw in (("fp64_jacobi_pcg", dict(solver=F.SOLVER_JACOBI_PCG, csr_only=True)),
                     ("fp32_inner_fp64_refinement_pcg", dict(solver=F.SOLVER_MP_PCG))):
        try:  # every rank solves the same replica, so a failure is the same on all of them
            S.solve(tol=TOL, fresh_setup=True, **kw)
            barrier(world)
            runs = [S.solve(tol=TOL, fresh_setup=True, **kw) for _ in range(steps)]
        except F.TptFemError as e:
            rec[name] = {"error": str(e)}
            continue
        u = S.solution()[free]
        sec = barrier_max(statistics.median(seconds(st) for st in runs), world)
        rec[name] = {"seconds": sec, "iterations": runs[-1]["iterations"], "rel_residual": runs[-1]["rel_residual"],
                     "refinement_steps": runs[-1]["outer_steps"],
                     "max_rel_error_vs_fp64_reference": float(np.max(np.abs(u - u_ref)) / np.max(np.abs(u_ref)))}
    prof = S.profile_spmv(20)
    nf, nnz = S.n_free, S.nnz
    b64 = nnz * 12 + 4 * (nf + 1) + 16 * nf
    b32 = nnz * 8 + 4 * (nf + 1) + 8 * nf
    peak, kind = measured_peaks()
    if rank != 0:
        return None
    mp, fp = rec["fp32_inner_fp64_refinement_pcg"], rec["fp64_jacobi_pcg"]
    return {"metric": "solve time to FP64 rel. residual 1e-10: FP64 Jacobi-PCG vs FP32-inner/FP64-refinement PCG",
            "value": mp.get("seconds"), "unit": "s", "higher_is_better": False,
            "config": {"workload": "cube_elasticity_64", "mesh": list(n), "tets": int(mesh.n_elems),
                       "free_dofs": int(nf), "nnz_reduced": int(nnz), "tol": TOL,
                       "reference_solution": f"FP64 Jacobi-PCG to {CUBE_TOL_REF:g}"},
            "solvers": rec,
            "speedup_mp_vs_fp64": fp["seconds"] / mp["seconds"] if "seconds" in mp and "seconds" in fp else None,
            "assembly": {"ms": asm_ms, "melem_per_s": mesh.n_elems / (asm_ms * 1e-3) / 1e6,
                         "algorithmic_bytes": 24.0 * mesh.n_nodes + 16.0 * mesh.n_elems + 8.0 * K.nnz},
            "spmv": {"csr_f64_ms": prof["csr_f64_ms"], "csr_f64_gbs": b64 / (prof["csr_f64_ms"] * 1e-3) / 1e9,
                     "csr_f32_ms": prof["csr_f32_ms"], "csr_f32_gbs": b32 / (prof["csr_f32_ms"] * 1e-3) / 1e9,
                     "peak_gbs": peak, "peak_kind": kind,
                     "bytes_formula": "nnz (Vw + 4) + 4 (n + 1) + 2 Vw n, Vw = 8 (FP64) / 4 (FP32)"}}


POISSON_WEIGHTS = os.path.join(ROOT, "tpt-fem_b200", "weights", "lfsai_poisson.bin")
POISSON_TOL = 1e-8


def poisson_cpu_baseline(S, seed):
    """The plain method on the host cores: one complete oracle FP64 Jacobi-PCG
    solve (all host threads) of the reduced system of field `seed` (the last
    field timed on the GPU), from x = 0 to the true relative residual 1e-8,
    measured."""
    sysh = host_system(S)
    nthr = cpu_threads()
    cpu_ms_per_iteration(sysh, nthr, 3)
    sec, it, rel = cpu_full_solve(sysh, POISSON_TOL, nthr)
    return {"value": sec, "unit": "s", "cores": nthr, "kind": "port", "iterations": it, "rel_residual": rel,
            "sample": f"one complete oracle FP64 Jacobi-PCG solve of field {seed} ({len(sysh[3])} dofs) to true rel. "
                      f"residual {POISSON_TOL:g}, {abs(it)} iterations, measured, not scaled"}


def run_poisson_grf(args, world, rank, local):
    """Heterogeneous Poisson on 128^3 (2,000,376 free dofs) over unseen seeded
    Gaussian-random-field conductivities: mean solve time to FP64 relative
    residual 1e-8 with the learned preconditioner (Poisson weights, trained on
    32^3 / 64^3 fields) vs FP64 Jacobi-PCG, per field, set-up included."""
    import tpt_fem as F
    from tpt_fem import lfsai as LF
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    model = LF.LearnedFsai.load(ctx, POISSON_WEIGHTS)
    n = args.poisson_n
    seeds = list(range(5000 + 100 * rank, 5000 + 100 * rank + args.fields))
    methods = {"jacobi_csr": dict(solver=F.SOLVER_JACOBI_PCG, csr_only=True),
               "learned": dict(solver=F.SOLVER_LEARNED_FSAI_PCG),
               "learned_coarse": dict(solver=F.SOLVER_LEARNED_FSAI_PCG, coarse=True),
               "classic_fsai": dict(solver=F.SOLVER_FSAI_MP_PCG)}
    # one mesh and one reduced system; each field replaces the system's values
    # (tptfem_system_refresh), keeping its structures, as a loop over fields does
    prob = W.GrfPoisson(ctx, n)
    S = prob.system(4999)
    model.attach(S)
    if args.profile:  # the headline method's solves only, on one field (for an ncu launch list)
        S.refresh(prob.matrix(seeds[0]), prob.rhs)
        for _ in range(args.steps):
            S.solve(tol=POISSON_TOL, fresh_setup=True, **methods["learned_coarse"])
        ctx.synchronize()
        return None
    for _ in range(args.warmup):
        for kw in methods.values():
            S.solve(tol=POISSON_TOL, fresh_setup=True, **kw)
    rec = {m: {"s": [], "it": [], "res": [], "fell_back": 0} for m in methods}
    barrier(world)
    with ClockSampler(local) as clk:
        for sd in seeds:
            S.refresh(prob.matrix(sd), prob.rhs)
            for m, kw in methods.items():
                st = S.solve(tol=POISSON_TOL, fresh_setup=True, **kw)
                rec[m]["s"].append(seconds(st))
                rec[m]["it"].append(st["iterations"])
                rec[m]["res"].append(st["rel_residual"])
                rec[m]["fell_back"] += st["fell_back"]
    barrier(world)
    mean = {m: barrier_max(float(np.mean(r["s"])), world) for m, r in rec.items()}
    out = None
    if rank == 0:
        out = {"metric": "mean solve time to FP64 rel. residual 1e-8 over unseen GRF fields: learned vs FP64 Jacobi-PCG",
               "value": mean["learned_coarse"], "unit": "s", "n_gpus": world, "steps": len(seeds),
               "warmup": args.warmup, "ms_per_step": mean["learned_coarse"] * 1e3, "higher_is_better": False,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64 (factor f16/f32, network f32)",
               "data": "synthetic (seeded Gaussian random fields, random Fourier features M=1024, l=0.1)",
               "config": {"workload": f"poisson_grf_{n}^3", "mesh": [n, n, n], "fields": len(seeds),
                          "field_seeds": [seeds[0], seeds[-1]], "weights": os.path.relpath(POISSON_WEIGHTS, ROOT),
                          "tol": POISSON_TOL, "parallelism": f"replicas{world}"},
               "methods": {m: {"mean_s": mean[m], "mean_iterations": float(np.mean(r["it"])),
                               "max_rel_residual": float(np.max(r["res"])), "fell_back": r["fell_back"]}
                           for m, r in rec.items()},
               "cpu_baseline": poisson_cpu_baseline(S, seeds[-1]) if world == 1 else None,
               "speedup_learned_vs_jacobi": mean["jacobi_csr"] / mean["learned"],
               "speedup_learned_coarse_vs_jacobi": mean["jacobi_csr"] / mean["learned_coarse"],
               "clocks": clk.summary()}
    return out


def topopt_cpu_baseline(probs, gpu_rate, its=10):
    """The reference algorithm on one host core (oracle restatement of
    topopt_simp in the batch's density-filter mode, banded Cholesky in place of
    its infeasible dense LU): the first instance of each grid size in the batch,
    `its` OC iterations each.  The sizes are drawn uniformly, so one of each
    is a representative sample; the rate is measured, not scaled."""
    from oracle import oracle as O
    from tpt_fem import workloads as W
    sample = [next(p for p in probs if (p[0].grid.nelx, p[0].grid.nely) == sz) for sz in W.TOPOPT_SIZES
              if any((p[0].grid.nelx, p[0].grid.nely) == sz for p in probs)]
    t0 = time.perf_counter()
    for P, f, bcs in sample:
        O.topopt(P.grid.nelx, P.grid.nely, P.vol_frac, P.filter_radius, its, f, bcs, emin=P.emin,
                 density_filter=True, banded=True)
    dt = time.perf_counter() - t0
    rate = len(sample) * its / dt
    return {"value": rate, "unit": "instance-iterations/s", "cores": 1, "kind": "port",
            "sample": f"oracle topopt_simp (density-filter mode, banded Cholesky), {its} OC iterations of one "
                      f"instance of each size ({len(sample)} instances, {dt:.1f} s), measured",
            "gpu_speedup": gpu_rate / rate}


def run_topopt(args, world, rank, local):
    """The batched 2-D SIMP workload (512 uneven cantilever instances, 100 OC
    iterations, density filter, Emin 1e-9) as one tptfem_topopt_batch call:
    device time of the whole batch (CUDA events inside the library)."""
    import tpt_fem as F
    from tpt_fem import topopt as T
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    probs = W.topopt_batch_problems(args.instances, seed=7 + rank, max_iter=args.oc_iters)
    warm = W.topopt_batch_problems(min(args.instances, 32), seed=99, max_iter=2)
    for _ in range(max(1, args.warmup)):
        T.topopt_batch(ctx, warm, rel_tol=1e-10)
    barrier(world)
    with ClockSampler(local) as clk:
        res, st = T.topopt_batch(ctx, probs, rel_tol=1e-10)
    barrier(world)
    sec = barrier_max(st["total_ms"] / 1e3, world)
    out = None
    if rank == 0:
        dofs = sum(2 * P.grid.n_nodes() for P, _, _ in probs)
        ratio = [r.compliance[-1] / r.compliance[0] for r in res]
        out = {"metric": "batched SIMP topology optimisation: instance-iterations per second",
               "value": world * args.instances * args.oc_iters / sec, "unit": "instance-iterations/s",
               "n_gpus": world, "steps": 1, "warmup": args.warmup, "ms_per_step": sec * 1e3,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (seeded sizes and volume fractions)",
               "config": {"workload": "topopt_batch", "instances": args.instances, "oc_iterations": args.oc_iters,
                          "sizes": "nelx x nely from {60x20, 90x30, 120x40, 180x60, 240x80}",
                          "emin": 1e-9, "filter": "density, R 1.5", "dofs_per_iteration": dofs,
                          "solver": "banded Cholesky per instance (FP64, factor on the FP64 tensor cores, residual "
                                    "checked and refined to rel. tol 1e-10); two-level PCG for grids too wide for the band",
                          "direct_instances": st["direct_instances"], "refinement_steps": st["refinement_steps"],
                          "parallelism": f"replicas{world}"},
               "batch_seconds": sec, "tune_ms": st["tune_ms"], "threads_per_instance": st["block_threads"],
               "cpu_baseline": (topopt_cpu_baseline(probs, world * args.instances * args.oc_iters / sec)
                                if world == 1 else None),
               "pcg_iterations": st["pcg_iterations"],
               "compliance_final_over_initial": {"min": min(ratio), "median": float(np.median(ratio)),
                                                 "max": max(ratio)},
               "clocks": clk.summary()}
    return out


# ncu DRAM read + write of one numeric tet_node_rows launch on the
# 140x35x35 cantilever (1,029,000 tets); scaled by tets to the measured mesh
ASM_TRAFFIC_140 = (84.786688 + 110.981888) * 1e6
ASM_TETS_140 = 1029000


def assembly_cpu_baseline(n_sample=(40, 10, 10)):
    """The reference's assembly on the host: the oracle restatement of
    try_assemble (zero-skip COO over elements in id order) + Coo::to_csr (stable
    sort, duplicate sum), one core, on a bounded cantilever sample; returns
    (Melem/s, sample description)."""
    from oracle import oracle as O
    from tpt_fem import workloads as W
    c, e = O.box_mesh([0.0, 0.0, 0.0], [4.0, 1.0, 1.0], list(n_sample))
    m = O.Mesh(O.CELL_TET, c, e)
    E = W.cantilever_young(list(n_sample))
    O.assemble_elasticity(m, O.MODEL_3D, E, 0.3, 2).to_csr()  # warm
    reps, t0 = 0, time.perf_counter()
    while reps < 2 or time.perf_counter() - t0 < 10.0:
        O.assemble_elasticity(m, O.MODEL_3D, E, 0.3, 2).to_csr()
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    return len(e) / dt / 1e6, (f"oracle assemble_elasticity + to_csr on the {list(n_sample)} cantilever "
                               f"({len(e)} tets), {reps} repetitions, one core")


def run_assembly(args, world, rank, local):
    """Tet4 elasticity assembly of the 280x70x70 cantilever (8,232,000 tets,
    per-element E): element throughput of the numeric re-assembly kernel
    (pattern fixed, inputs resident; CUDA events in the library), and end to end
    through the C ABI from host arrays (mesh upload, pattern and values)."""
    import tpt_fem as F
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    mn, mx, n = W.CANTILEVERS[WORKLOAD]
    if args.mesh:  # a smaller cantilever of the same family (ncu captures)
        n = list(args.mesh)
    E = W.cantilever_young(n)
    m0 = F.Mesh.box_mesh(mn, mx, n, ctx=ctx)
    coords, conn = m0.coords_array.copy(), m0.conn_array.copy()
    del m0
    mesh = F.Mesh.from_arrays(F.CELL_TET4, coords, conn, ctx=ctx)
    K = F.assemble_elasticity(mesh, "3d", E, 0.3, 2)
    n_el, n_nodes, nnz = len(conn), len(coords), K.nnz
    K.profile_assembly(max(1, args.warmup))
    barrier(world)
    with ClockSampler(local) as clk:
        ms = K.profile_assembly(args.steps)
    barrier(world)
    ms = barrier_max(ms, world)
    # end to end: host arrays -> mesh -> assembled matrix (its size read back)
    walls = []
    for _ in range(3):
        cuda_sync()
        t0 = time.perf_counter()
        mh = F.Mesh.from_arrays(F.CELL_TET4, coords, conn, ctx=ctx)
        Kh = F.assemble_elasticity(mh, "3d", E, 0.3, 2)
        _ = Kh.nnz
        ctx.synchronize()
        walls.append(time.perf_counter() - t0)
        del Kh, mh
    e2e_s = min(walls)
    peak, kind = measured_peaks()
    alg = 24.0 * n_nodes + 16.0 * n_el + 8.0 * n_el + 8.0 * nnz
    out = None
    if rank == 0:
        cpu, sample = assembly_cpu_baseline() if world == 1 else (None, None)
        out = {"metric": "Tet4 elasticity assembly throughput (numeric, pattern fixed)",
               "value": world * n_el / (ms * 1e-3) / 1e6, "unit": "Melem/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded density field)",
               "config": {"workload": "assembly_cantilever_%dx%dx%d" % tuple(n), "mesh": list(n), "tets": n_el,
                          "nodes": n_nodes,
                          "nnz": nnz, "per_element_E": True, "parallelism": f"replicas{world}",
                          "l2": "inputs and output larger than L2 (values %.2f GB)" % (8e-9 * nnz)},
               "roofline": {"bound": "hbm", "kernel": "tet_node_rows<1,3,24,16> (NUMERIC: bit-exact FP64, no FMA)",
                            "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "peak_kind": kind, "unit": "GB/s",
                            "frac": alg / (ms * 1e-3) / 1e9 / peak, "traffic": ASM_TRAFFIC_140 * n_el / ASM_TETS_140,
                            "traffic_source": "ncu dram__bytes_read+write of the kernel at 140x35x35 scaled by tets",
                            "algorithmic_bytes": alg,
                            "algorithmic_formula": "24 N + 16 E + 8 E + 8 nnz (coords, connectivity, E, values)"},
               "e2e": {"value": n_el / e2e_s / 1e6, "unit": "Melem/s", "seconds": e2e_s,
                       "h2d_bytes_per_step": int(coords.nbytes + conn.nbytes + E.nbytes), "d2h_bytes_per_step": 8},
               "cpu_baseline": ({"value": cpu, "unit": "Melem/s", "cores": 1, "kind": "port", "sample": sample}
                                if world == 1 else None),
               "gpu_launches": args.steps,
               "clocks": clk.summary()}
    return out


def run_reference(args, world, rank, local):
    """The plain method on the host cores, on the headline system.

    The reference's own solver is a dense LU (crates/tpt-fem-sparse/src/lib.rs:225-278),
    which cannot run at 4.2M dofs (143 TB), and the Rust workspace cannot be
    built here; the reference arm therefore times the oracle port of the plain
    method, FP64 Jacobi-PCG, on ALL host cores, solving the exact 280x70x70
    reduced system from x = 0 to the true relative residual 1e-10.  Every timed
    step is one complete solve, measured; complete solves are timed until
    CPU_SOLVE_BUDGET_S is spent (at least one, at most --steps), and `steps`
    reports how many ran.  Warm-up steps are short fixed-iteration runs on the
    same system.  The system is built by the library on the GPU (input
    generation, outside the timed region; the configuration-size parity tests
    pin its rows bit for bit against the oracle)."""
    if rank != 0:
        return None
    import tpt_fem as F
    from tpt_fem import workloads as W
    ctx = F.Context(local)
    mesh, K, S, E, rhs, dof, val = build_system(F, W, ctx)
    sysh = host_system(S)
    n, nnz = S.n_free, S.nnz
    del mesh, K, S
    nthr = cpu_threads()
    for _ in range(max(1, args.warmup)):
        cpu_ms_per_iteration(sysh, nthr, 3)
    solves, spent = [], 0.0
    while len(solves) < max(1, args.steps) and (not solves or spent + solves[-1][0] <= CPU_SOLVE_BUDGET_S):
        solves.append(cpu_full_solve(sysh, TOL, nthr))
        spent += solves[-1][0]
    one_core = cpu_ms_per_iteration(sysh, 1, 5)
    v = statistics.median(t for t, _, _ in solves)
    its = [it for _, it, _ in solves]
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": len(solves),
            "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded density field)",
            "config": {"workload": WORKLOAD, "mesh": [280, 70, 70], "free_dofs": int(n), "nnz_reduced": int(nnz),
                       "solver": "FP64 Jacobi-PCG (oracle port of the plain method, int32 CSR, OpenMP)",
                       "tol": TOL},
            "step_s": [round(t, 3) for t, _, _ in solves], "iterations": its,
            "rel_residual": [r for _, _, r in solves],
            "cpu_baseline": {"value": v, "unit": "s", "cores": nthr, "kind": "port",
                             "one_core_ms_per_iteration": one_core,
                             "sample": f"{len(solves)} complete solves of the 280x70x70 reduced system to true rel. "
                                       f"residual {TOL:g} ({its[0]} iterations each), measured, not scaled; the "
                                       f"reference's dense LU is infeasible at this size; one core measured at "
                                       f"{one_core:.1f} ms per iteration"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solver", default="learned", choices=["learned", "fsai", "jacobi", "mp"])
    ap.add_argument("--profile", action="store_true",
                    help="cantilever / poisson_grf: run only the headline method's solves (ncu launch list)")
    ap.add_argument("--no-coarse", action="store_true", help="single-level preconditioner (no coarse space)")
    ap.add_argument("--workload", default="cantilever",
                    choices=["cantilever", "poisson_grf", "topopt", "assembly", "cube", "partitioned"],
                    help="poisson_grf: the heterogeneous-Poisson learned-preconditioner configuration; cube: the "
                         "64^3 elasticity cube, FP64 vs FP32-inner PCG")
    ap.add_argument("--headline-only", action="store_true",
                    help="cantilever: skip the other configurations' records in the JSON line")
    ap.add_argument("--fields", type=int, default=32, help="poisson_grf: unseen fields timed")
    ap.add_argument("--instances", type=int, default=512, help="topopt: instances in the batch")
    ap.add_argument("--oc-iters", type=int, default=100, help="topopt: OC iterations")
    ap.add_argument("--poisson-n", type=int, default=128, help="poisson_grf: box_mesh cells per axis")
    ap.add_argument("--mesh", type=int, nargs=3, default=None,
                    help="with --profile (or --workload partitioned): cantilever cells, a smaller case")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        out = run_reference(args, world, rank, local)
    elif args.workload == "poisson_grf":
        out = run_poisson_grf(args, world, rank, local)
    elif args.workload == "topopt":
        out = run_topopt(args, world, rank, local)
    elif args.workload == "assembly":
        out = run_assembly(args, world, rank, local)
    elif args.workload == "cube":
        out = run_cube(args, world, rank, local)
    elif args.workload == "partitioned":
        out = run_partitioned(args, world, rank, local)
    else:
        out = run_ours(args, world, rank, local)
        if not (args.headline_only or args.profile):
            # every other configuration, measured in the same run (records beside the headline)
            sub = {"poisson_box8": run_box8, "cube_elasticity_64": run_cube,
                   "assembly_cantilever_280x70x70": run_assembly,
                   "poisson_grf_128": run_poisson_grf, "topopt_batch": run_topopt,
                   "cantilever_other_sizes": run_cantilever_sizes}
            recs = {name: fn(args, world, rank, local) for name, fn in sub.items()}
            if rank == 0:
                out["configs"] = recs
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
