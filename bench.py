#!/usr/bin/env python
"""Stokes solves/s on the 128x1024 anisotropic annulus (B200).

A step is one complete Stokes solve of the workload: material upload from
device-resident inputs, element assembly, multigrid setup, the Schur PCG to
1e-8 relative residual (StokesPcCG semantics) and the rigid-rotation removal,
i.e. one call of the reference's solveStokes (src/Stokes/StokesSolver.jl:7-54).

Workload (the reference's headline configuration that fits one GPU): 128 x
1024 cells, 262,144 P2 elements, 1,052,672 velocity DOF, 786,432
discontinuous-P1 pressure DOF; transversely isotropic viscosity with eta(T)
contrast 1e5, weak-plane factor delta ~ U[1,10] per element, director from a
seeded 8-mode Fourier field; free slip with the rigid rotation pinned.  Inputs
are seeded synthetic arrays (dimspers_b200.inputs).

value     fast path (FP32 bulk / FP64 residual refinement) solves/s over all
          ranks, inputs resident in HBM, device time (CUDA events, max over ranks)
e2e       the same solve through the public API with pinned host buffers:
          the step's inputs are copied host->device and U, P device->host
fp64      the plain FP64 GPU path on the same inputs (comparison field)
roofline  the fine-level FP32 element-by-element A-apply, the dominant kernel
cpu_baseline  the FP64 CPU oracle (NumPy/SciPy port of the reference path) on
          a bounded sample of the same workload

--impl reference times the CPU oracle (the reference itself is Julia and
cannot run here) on the same workload and prints the same JSON line.
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
sys.path.insert(0, ROOT)

METRIC = "Stokes solves/s at 1e-8 rel. residual: learned+FP32 vs plain FP64, 1 B200"
UNIT = "solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nr", type=int, default=128)
    ap.add_argument("--nt", type=int, default=1024)
    ap.add_argument("--pressure", default="discontinuous")
    ap.add_argument("--kind", default="aniso")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--itmax", type=int, default=20000)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--fp64-warmup", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end arm (for the large single-shot measurements; not a bench line)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=3)
    ap.add_argument("--cpu-sample-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the solver loops from the host (same kernels, one launch each; for ncu launch lists,"
                         " which cannot see inside graphs with conditional nodes)")
    ap.add_argument("--no-clocks", action="store_true", help="do not sample nvidia-smi (for profiler runs)")
    ap.add_argument("--no-guess", action="store_true", help="fast arm without the learned initial guess")
    ap.add_argument("--profile-apply", action="store_true",
                    help="assemble the workload and launch the fine-level FP32 A-apply 3 times (for ncu)")
    ap.add_argument("--postprocess", action="store_true",
                    help="the kernels around the solve (stress, viscosity, DEM tensor, thermal step) on the GPU "
                         "beside the oracle's CPU restatements, one JSON line each")
    return ap.parse_args()


# solver options of the two arms
FAST = dict(precision=1, cheb_degree=3, cheb_lo=0.05, inner_rtol=1e-10, inner_relax=1e-2, relax_base=1e-8, schur_pc=1)
PLAIN = dict(precision=0, cheb_degree=3, cheb_lo=0.05, inner_rtol=1e-10, inner_relax=0.0, schur_pc=0)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(ms, device, world):
    """The job's time: the largest per-rank time (one all-reduce, MAX)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(units_per_rank, world, ms):
    """Whole-job throughput: units of all ranks over the max-over-ranks time."""
    return world * units_per_rank / (ms / 1e3)


# ---------------------------------------------------------------- clocks ----
REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
           0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
           0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}


class ClockSampler:
    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 3:
                try:
                    self.samples.append((float(parts[0]), float(parts[1]), int(parts[2], 16)))
                except ValueError:
                    pass

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        busy = [s for s in self.samples if not (s[2] & 0x1)] or self.samples
        mask = 0
        for s in busy:
            mask |= s[2]
        return {"sm_mhz": statistics.median(s[0] for s in busy), "sm_max_mhz": max(s[1] for s in busy),
                "reasons": [n for b, n in REASONS.items() if mask & b and b != 0x1], "samples": len(busy)}


# ------------------------------------------------------------ workload ----
def make_inputs(args, seed):
    from dimspers_b200 import build_mesh, inputs
    mesh = build_mesh(args.nr, args.nt, args.pressure, pin_rotation=True, colors=False)
    mat = inputs.make_material(mesh, args.kind, seed=seed)
    return mesh, mat


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profiles(nr, nt):
    """DRAM bytes per launch of the roofline kernel from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d.get(f"{nr}x{nt}")
        return None if e is None else float(e["dram_bytes_per_launch"])
    except Exception:
        return None


def start_cpu_sample(args):
    """The CPU oracle sample runs in its own process, concurrently with the GPU
    timing, on one host thread (the GPU path needs one more)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-sample-only", "--nr", str(args.nr), "--nt", str(args.nt),
           "--pressure", args.pressure, "--kind", args.kind, "--cpu-iters", str(args.cpu_iters)]
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", MKL_NUM_THREADS="1")
    return subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=env)


def finish_cpu_sample(proc, args, n_outer):
    try:
        out, _ = proc.communicate(timeout=900)
        d = json.loads(out.strip().splitlines()[-1])
    except Exception as e:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "port", "sample": f"failed: {e}"}
    per_solve = d["t_setup"] + n_outer * d["t_iter"]
    return {"value": 1.0 / per_solve, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"FP64 oracle on one thread: C element blocks, SciPy assembly + SuperLU factorisation "
                      f"({d['t_setup']:.1f} s) + "
                      f"{args.cpu_iters} outer iterations ({d['t_iter']:.2f} s each) of the {args.nr}x{args.nt} "
                      f"workload, extrapolated to {n_outer} outer iterations (lumped-mass StokesPcCG)"}


def run_ours(args, rank, world, local):
    import numpy as np
    import torch

    cpu_proc = start_cpu_sample(args) if (rank == 0 and world == 1 and not args.no_cpu) else None

    from dimspers_b200 import StokesContext
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    mesh, mat = make_inputs(args, seed=1 + rank)
    nel, nnod, npres = mesh.nel, mesh.nnod, mesh.npres
    ctx = StokesContext(args.nr, args.nt, args.pressure, device=local, pin_rotation=True)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    # device-resident inputs
    eta_d = torch.from_numpy(np.asfortranarray(mat.eta_ip).T.copy()).to(dev)     # (7, nel) == nel x 7 col-major
    dl_d = torch.from_numpy(mat.delta).to(dev)
    dx_d = torch.from_numpy(mat.dir_x).to(dev)
    dy_d = torch.from_numpy(mat.dir_y).to(dev)
    rho_d = torch.from_numpy(mat.rho).to(dev)
    U_d = torch.zeros(2 * nnod, dtype=torch.float64, device=dev)
    P_d = torch.zeros(npres, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    opts = dict(rtol=args.rtol, itmax=args.itmax, itmin=10, host_loop=1 if args.host_loop else 0)
    if args.pressure != "discontinuous":
        FAST["schur_pc"] = 0

    # learned initial guess (trained weights for this mesh, if present)
    from dimspers_b200 import learned
    guess = None
    wpath = learned.weights_path(args.nr, args.nt)
    if not args.no_guess:
        if os.path.exists(wpath):
            guess = learned.LearnedGuess(learned.GuessNet.load(wpath, max_batch=1, device=local), ctx)
        elif os.path.exists(learned.weights_path(128, 1024)):
            # no network trained on this mesh: the 128x1024 one, run on this grid
            # (its layers are convolutions); the solver still keeps the guess only
            # if it starts below the zero guess
            wpath = learned.weights_path(128, 1024)
            net = learned.GuessNet.load(wpath, max_batch=1, device=local)
            guess = learned.LearnedGuess(net.for_grid(*learned.grid_shape(args.nr, args.nt), device=local), ctx)

    def step(precision):
        arm = FAST if precision else PLAIN
        ctx.set_material_ti_device(eta_d.data_ptr(), nel, rho_d.data_ptr(), mat.g, dl_d.data_ptr(),
                                   dx_d.data_ptr(), dy_d.data_ptr())
        ctx.assemble(arm["precision"])
        if precision and guess is not None:
            guess.predict(mat.g, P_d.data_ptr())
            return ctx.solve_device(U_d.data_ptr(), P_d.data_ptr(), None, use_guess=2, **opts, **arm)
        return ctx.solve_device(U_d.data_ptr(), P_d.data_ptr(), None, **opts, **arm)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(precision, warm, steps, sampler=None):
        for _ in range(warm):
            step(precision)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = []
        with (sampler if sampler is not None else _Null()):
            e0.record(stream)
            for _ in range(steps):
                reps.append(step(precision))
            e1.record(stream)
            barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dev, world)
        return ms, reps

    sampler = ClockSampler(local) if not args.no_clocks else None
    ms32, reps32 = timed(1, args.warmup, args.steps, sampler)
    value = aggregate_value(args.steps, world, ms32)
    ms_per_step = ms32 / args.steps
    U32, P32 = U_d.clone(), P_d.clone()   # the fast path's solution, for its error against FP64

    fp64 = None
    if not args.no_fp64:
        ms64, reps64 = timed(0, args.fp64_warmup, args.fp64_steps)
        fp64 = {"value": aggregate_value(args.fp64_steps, world, ms64), "ms_per_step": ms64 / args.fp64_steps,
                "outer_iterations": reps64[-1]["iterations"], "inner_iterations": reps64[-1]["inner_iterations"],
                "status": reps64[-1]["status"], "relres": reps64[-1]["relres"],
                "mom_residual": reps64[-1]["mom_residual"]}
        U64 = U_d.clone()
        P64 = P_d.clone()

    # ---- e2e through the public API with pinned host buffers ---------------------
    eta_h = torch.from_numpy(np.asfortranarray(mat.eta_ip).T.copy()).pin_memory()
    dl_h, dx_h, dy_h, rho_h = (torch.from_numpy(a).pin_memory() for a in (mat.delta, mat.dir_x, mat.dir_y, mat.rho))
    U_h = torch.zeros(2 * nnod, dtype=torch.float64).pin_memory()
    P_h = torch.zeros(npres, dtype=torch.float64).pin_memory()
    from dimspers_b200._lib import DP_MEM_HOST, SolveReport, lib
    import ctypes as C

    def e2e_step():
        ctx._chk(lib().dp_set_material_ti(ctx.h, C.c_void_p(eta_h.data_ptr()), nel, C.c_void_p(dl_h.data_ptr()),
                                          C.c_void_p(dx_h.data_ptr()), C.c_void_p(dy_h.data_ptr()),
                                          C.c_void_p(rho_h.data_ptr()), float(mat.g), DP_MEM_HOST))
        ctx.assemble(1)
        o = __import__("dimspers_b200").default_opts(**opts, **FAST)
        if guess is not None:
            guess.predict(mat.g, P_h.data_ptr(), mem=0)
            o.use_guess = 2
        rep = SolveReport()
        st = lib().dp_solve(ctx.h, C.c_void_p(U_h.data_ptr()), C.c_void_p(P_h.data_ptr()), None, C.byref(o),
                            C.byref(rep), DP_MEM_HOST)
        if st >= 3:
            ctx._chk(st)
        return rep

    ms_e2e = None
    if not args.no_e2e:
        e2e_step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        barrier()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1), dev, world)
    h2d = (eta_h.numel() + dl_h.numel() + dx_h.numel() + dy_h.numel() + rho_h.numel()) * 8
    d2h = (U_h.numel() + P_h.numel()) * 8

    # accuracy of the fast path against the plain FP64 path (same inputs)
    err = None
    if fp64 is not None:
        err = {"u_rel_l2": float(torch.linalg.norm(U32 - U64) / torch.linalg.norm(U64)),
               "p_rel_l2": float(torch.linalg.norm(P32 - P64) / torch.linalg.norm(P64))}

    # ---- roofline of the dominant kernel: fine-level FP32 EBE A-apply ---------------
    # The solve is one CUDA graph (events cannot sit inside its loop bodies), so
    # the kernel is timed right after the timed region on the same stream:
    # cold (L2 overwritten before each launch -> the DRAM-bound figure used for
    # the HBM roofline) and warm (back-to-back, element blocks L2-resident).
    ms_cold = ctx.profile_kernel(0, reps=50, flush_l2=True)
    ms_warm = ctx.profile_kernel(0, reps=200)
    alg_bytes = nel * 78 * 4 + nnod * 2 * 4 * 2
    pk, pk_kind = peaks()
    achieved = alg_bytes / (ms_cold * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_apply_K<float,float> (fine level)", "achieved": achieved,
                "peak": pk, "peak_kind": pk_kind, "unit": "GB/s", "frac": achieved / pk,
                "traffic": traffic_from_profiles(args.nr, args.nt), "algorithmic_bytes": alg_bytes,
                "ms_per_launch": ms_cold, "ms_per_launch_warm_l2": ms_warm,
                "achieved_warm_l2": alg_bytes / (ms_warm * 1e-3) / 1e9}

    clocks = sampler.summary() if sampler is not None else {"sm_mhz": None, "reasons": ["not sampled"]}
    last = reps32[-1]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": {"workload": f"annulus {args.nr}x{args.nt} cells, {nel} P2 elements, {2 * nnod} velocity DOF, "
                               f"{npres} {args.pressure} P1 pressure DOF, {args.kind} viscosity",
                   "nr_cells": args.nr, "ntheta_cells": args.nt, "pressure": args.pressure, "material": args.kind,
                   "rtol": args.rtol,
                   "guess": ("learned (" + os.path.basename(wpath) + ")") if guess is not None else "zero",
                   "fast_arm": FAST, "plain_arm": PLAIN,
                   "parallelism": f"replicas x{world}",
                   "l2": "each step re-assembles > 400 MB of element blocks (L2 is 126 MB); no extra flush"},
        "outer_iterations": last["iterations"], "inner_iterations": last["inner_iterations"],
        "refinements": last["refinements"], "status": last["status"], "relres": last["relres"],
        "guess_fallback": last["fallback_used"], "r0_guess_over_r0": (last["r0_guess"] / last["r0"]) if guess else None,
        "mom_residual": last["mom_residual"], "mg_levels": last["mg_levels"],
        "fp64": fp64, "fast_vs_fp64": (value / fp64["value"]) if fp64 else None, "fast_vs_fp64_error": err,
        "e2e": ({"value": aggregate_value(args.steps, world, ms_e2e), "unit": UNIT, "h2d_bytes_per_step": h2d,
                 "d2h_bytes_per_step": d2h} if ms_e2e is not None else None),
        "gpu_launches": int(sum(r["kernel_launches"] for r in reps32)),
        "roofline": roofline, "clocks": clocks,
    }
    try:   # the whole solve against the HBM roofline, from a per-kernel byte model
        sb = solve_bytes_model(args.nr, args.nt, last["iterations"], last["inner_iterations"], args.pressure,
                               FAST["cheb_degree"])
        sgbs = sb / (ms_per_step * 1e-3) / 1e9
        line["solve_model"] = {"bytes_per_solve": sb, "achieved": sgbs, "unit": "GB/s", "frac": sgbs / pk,
                               "note": "algorithmic bytes of every kernel of one fast solve (bench.solve_bytes_model)"}
    except Exception as e:  # a model must never cost the measured line
        line["solve_model"] = {"error": str(e)}
    if cpu_proc is not None:
        line["cpu_baseline"] = finish_cpu_sample(cpu_proc, args, fp64["outer_iterations"] if fp64 else
                                                 last["iterations"])
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def solve_bytes_model(nr, nt, outer, inner, pressure="discontinuous", cheb_degree=3, coarse_max=1536):
    """Algorithmic HBM bytes of one fast-path solve (FP64 Krylov, FP32 multigrid
    V-cycle per inner iteration): every kernel's reads and writes once, from
    the measured iteration counts.  Per-kernel figures (the kernel table):
    FP32 apply 312 B/element + 16 B/node; FP64 apply 624 B/element + 48 B/node;
    Chebyshev vector step 76 B/node; restriction 16 B/fine node + 40 B/coarse
    node; prolongation 24 B/fine node; dense coarsest n^2 x 8 B; inner PCG
    vector passes 128 B/DOF; outer: G and G^T 288 B/element + vectors, the
    fused Schur update (5 N_P + 2 N_U) x 8 B and its dots; assembly and
    set-up excluded."""
    levels = []
    r_, t_ = nr, nt
    while True:
        nel, nnod = 2 * r_ * t_, (2 * r_ + 1) * 2 * t_
        levels.append((nel, nnod))
        if 2 * nnod <= coarse_max or r_ % 2 or t_ % 2:
            break
        r_, t_ = r_ // 2, t_ // 2
    vcycle = 0.0
    for i, (nel, nnod) in enumerate(levels):
        if i == len(levels) - 1:
            vcycle += (2 * nnod) ** 2 * 8.0
            break
        cn = levels[i + 1][1]
        vcycle += 2 * cheb_degree * (312.0 * nel + 16.0 * nnod)          # smoothing and residual applies
        vcycle += 2 * cheb_degree * 76.0 * nnod                          # Chebyshev vector steps
        vcycle += 16.0 * nnod + 40.0 * cn + 24.0 * nnod                  # restriction, prolongation
    nel, nnod = levels[0]
    n_u = 2 * nnod
    n_p = 3 * nel if pressure == "discontinuous" else (nr + 1) * nt
    per_inner = vcycle + 624.0 * nel + 48.0 * nnod + 128.0 * n_u
    per_outer = 2 * (288.0 * nel + 16.0 * nnod + 8.0 * n_p) + (5 * n_p + 2 * n_u) * 8.0 + 4 * 16.0 * n_p
    return inner * per_inner + outer * per_outer


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


# ------------------------------------------------------------ CPU oracle ----
def cpu_sample(args, n_outer, iters):
    """Oracle port on a bounded sample: assembly + sparse LU + `iters` outer
    iterations of this workload; solve time = setup + n_outer * (time per
    outer iteration)."""
    import numpy as np
    import scipy.sparse.linalg as spla
    import oracle.c_elements as OC
    import oracle.solver as OS
    from dimspers_b200 import inputs

    prob = OS.make_problem(args.nr, args.nt, args.pressure, pin_rotation=True)

    class MV:
        theta, r, e2n, th_el, r_el = prob.gr.theta, prob.gr.r, prob.gr.e2n, prob.th, prob.r

    mat = inputs.make_material(MV, args.kind, seed=1)
    t0 = time.perf_counter()
    A = OS.assemble(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, elements=OC.element_matrices)
    Kf = A["KK"][prob.ifree][:, prob.ifree].tocsc()
    lu = spla.splu(Kf, permc_spec="MMD_AT_PLUS_A")
    t1 = time.perf_counter()
    y = np.random.default_rng(0).standard_normal(Kf.shape[0])
    GT = A["GG"].T.tocsr()
    for _ in range(iters):
        z = lu.solve(y)
        zz = np.zeros(A["GG"].shape[0])
        zz[prob.ifree] = z
        GT @ zz
        A["GG"] @ np.ones(A["GG"].shape[1])
    t2 = time.perf_counter()
    t_setup, t_iter = t1 - t0, (t2 - t1) / iters
    return t_setup, t_iter


def profile_apply(args):
    """Assemble the workload and launch the fine-level FP32 A-apply 3 times."""
    from dimspers_b200 import StokesContext
    mesh, mat = make_inputs(args, seed=1)
    with StokesContext(args.nr, args.nt, args.pressure, pin_rotation=True) as ctx:
        ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
        ctx.assemble(1)
        ms = ctx.profile_kernel(0, reps=3)
    print(json.dumps({"profile_apply_ms": ms}))


def run_reference(args, rank, world):
    if rank != 0:
        return
    n_outer = reference_outer_iterations(args)
    t_setup, t_iter = cpu_sample(args, n_outer, args.cpu_iters)
    per_solve = t_setup + n_outer * t_iter
    value = 1.0 / per_solve
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_solve * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": f"annulus {args.nr}x{args.nt} cells, {args.pressure} P1 pressure, {args.kind}",
                   "nr_cells": args.nr, "ntheta_cells": args.nt},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": f"element blocks on {os.cpu_count()} threads (C/OpenMP restatement), sparse "
                                   f"assembly + rotation + SuperLU factorisation (single-threaded) ({t_setup:.1f} s) + "
                                   f"{args.cpu_iters} outer iterations ({t_iter:.2f} s each), extrapolated to "
                                   f"{n_outer} outer iterations"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------ kernels around the solve ----
def cpu_postprocess(args):
    """The oracle's CPU restatements on the inputs the GPU timing uses: ms per
    call (best of 2), on one thread (BLAS pools limited to 1; the DEM lookup
    is the plain-C restatement run on one OpenMP thread)."""
    from threadpoolctl import threadpool_limits
    with threadpool_limits(1):
        return _cpu_postprocess(args)


def _cpu_postprocess(args):
    import numpy as np
    import oracle.c_elements as OC
    import oracle.fabric as OF
    import oracle.rheology as RH
    import oracle.solver as OS
    import oracle.stress as ST
    import oracle.thermal as OT
    from dimspers_b200 import inputs, kernel_times as KT

    def best(fn, reps=2):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return 1e3 * min(ts)

    nr, nt = args.nr, args.nt
    out = {}
    prob = OS.make_problem(nr, nt, "discontinuous")
    gr = prob.gr

    class MV:
        theta, r, e2n, th_el, r_el = gr.theta, gr.r, gr.e2n, prob.th, prob.r
        nel, nnod = gr.e2n.shape[1], gr.nnod

    m = inputs.make_material(MV, "aniso", seed=1)
    rng = np.random.default_rng(0)
    U = rng.standard_normal(2 * gr.nnod)
    out["k_stress"] = (best(lambda: ST.stress(U, m.eta_ip, prob.th, prob.r, gr.e2n, m.C6)), "whole mesh")
    T, P, r, eps, tau, coh = KT.inputs_viscosity(MV, nr, nt, rng)
    eta0 = np.full((MV.nel, 7), 3.3e21)
    out["k_viscosity_arrhenius"] = (best(lambda: RH.arrhenius_viscosity(
        eta0, T, P, r, gr.e2n, eps, tau, coh, 5e20, 8.314, 100e3, 1e-6, 1600.0, 30.0)), "whole mesh")
    d = np.load(KT.DEM_FIXTURE)
    tab = OF.dem_tables(d["C"], d["ax"])
    x1, y1, r1, r2 = KT.inputs_dem(MV.nel, rng)
    out["k_dem_tensor"] = (best(lambda: OC.anisotropic_tensor(x1, y1, r1, r2, tab, 0.02, nthreads=1)),
                           "whole mesh (plain C, one thread)")
    pc = OS.make_problem(nr, nt, "continuous")
    T, rho, dt = KT.inputs_thermal(pc.gr, nr, np.random.default_rng(0))
    fixed, tfix = OT.boundary(pc.gr, 300.0, 4000.0)
    out["k_th_apply"] = (best(lambda: OT.thermal_step(pc.gr, pc.th, pc.r, T, rho, 3.3, 1.2e3, dt, fixed, tfix,
                                                      solver="gmres"), reps=1),
                         "whole step: assembly + the reference's full GMRES")
    return out


def postprocess(args):
    import torch
    size = f"{args.nr}x{args.nt}"
    gpu = {}
    if torch.cuda.is_available():
        from dimspers_b200 import kernel_times
        gpu = {rec["kernel"]: rec for rec in kernel_times.measure([size])}
    cpu = cpu_postprocess(args)
    for k, (ms, sample) in cpu.items():
        line = {"postprocess": k, "size": size, "gpu": gpu.get(k),
                "cpu_baseline": {"value": ms, "unit": "ms per call", "cores": 1, "kind": "port", "sample": sample}}
        print(json.dumps(line), flush=True)


def reference_outer_iterations(args):
    path = os.path.join(ROOT, "tests", "golden", "outer_iterations.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return int(d[f"{args.nr}x{args.nt}_{args.pressure}_{args.kind}"])
    except Exception:
        return 200


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.cpu_sample_only:
        t_setup, t_iter = cpu_sample(args, 0, args.cpu_iters)
        print(json.dumps({"t_setup": t_setup, "t_iter": t_iter}), flush=True)
        return
    if args.profile_apply:
        profile_apply(args)
        return
    if args.postprocess:
        if rank == 0:
            postprocess(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
