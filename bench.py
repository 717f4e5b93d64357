#!/usr/bin/env python
"""Stokes solves/s on the 512x4096 anisotropic (fabric) annulus (B200).

A step is one complete Stokes solve of the workload: material upload from
device-resident inputs, element assembly, multigrid setup, the Schur PCG to
1e-8 relative residual (StokesPcCG semantics) and the rigid-rotation removal,
i.e. one call of the reference's solveStokes (src/Stokes/StokesSolver.jl:7-54).

Headline workload (the configuration the metric's target is stated on):
512 x 4096 cells, 4,194,304 P2 elements, 16,793,600 velocity DOF, 12,582,912
discontinuous-P1 pressure DOF; director = major eigenvector of F F^T per
element with F = I + 0.5 G, G a seeded smooth 8-mode 2x2 field; viscosity
contrast 1e6, weak-plane factor delta ~ U[1,10]; free slip with the rigid
rotation pinned.  Inputs are seeded synthetic arrays (dimspers_b200.inputs).

value       fast path (FP32 element data and multigrid, FP64 Krylov/residual,
            compensated Schur dots, learned guess) solves/s over all ranks,
            inputs resident in HBM, device time (CUDA events, max over ranks)
e2e         the same solve through the public C ABI with pinned host buffers:
            the step's inputs are copied host->device and U, P device->host
fp64        the plain FP64 GPU path (the reference's algorithm: lumped-mass
            Schur preconditioner, inner solves to 1e-10) on the same inputs
fp64_same_algorithm
            FP64 with exactly the fast arm's algorithm (element-mass Schur
            preconditioner, relaxed inner solves, true-residual restarts,
            learned guess); value / this = the gain of the precision pattern
secondary   the 128x1024 anisotropic workload: both arms, and their errors
            against the tightly converged FP64 oracle solution committed in
            tests/golden (the yardstick), plus the fast arm at rtol 1e-9..1e-12
roofline    the fine-level FP32 element-by-element A-apply, the dominant kernel
cpu_baseline  the reference's CPU algorithm (the FP64 oracle) by a cost model
            fitted on oracle solves of two smaller meshes (oracle.refmodel)

--impl reference prints the same line for the CPU reference (modelled, the
reference itself is Julia and a 16.8M-DOF sparse LU cannot complete here).
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
    ap.add_argument("--nr", type=int, default=512)
    ap.add_argument("--nt", type=int, default=4096)
    ap.add_argument("--pressure", default="discontinuous")
    ap.add_argument("--kind", default="fabric")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--itmax", type=int, default=20000)
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="timed end-to-end solves (default min(steps, 5): one e2e solve of the headline "
                         "workload takes as long as a device-resident one)")
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--fp64-warmup", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end arm (for single-shot measurements; not a bench line)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-same-algorithm", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
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


# solver options of the arms
FAST = dict(precision=1, cheb_degree=3, cheb_lo=0.05, inner_rtol=1e-10, inner_relax=1e-2, relax_base=1e-8, schur_pc=1)
PLAIN = dict(precision=0, cheb_degree=3, cheb_lo=0.05, inner_rtol=1e-10, inner_relax=0.0, schur_pc=0)
SAME_ALGO = dict(FAST, precision=0)          # the fast arm's algorithm, all FP64
SECONDARY = (128, 1024, "aniso")             # the 1.05M-DOF workload with a committed oracle yardstick
TIGHT_FIXTURE = os.path.join(ROOT, "tests", "golden", "tight_128x1024_aniso.npz")
REF_SAMPLES = ((32, 256), (64, 512))        # meshes the CPU reference model measures


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
def make_inputs(nr, nt, pressure, kind, seed):
    from dimspers_b200 import build_mesh, inputs
    mesh = build_mesh(nr, nt, pressure, pin_rotation=True, colors=False)
    mat = inputs.make_material(mesh, kind, seed=seed)
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


def spread(vals):
    vals = [int(v) for v in vals]
    return {"min": min(vals), "median": statistics.median(vals), "max": max(vals), "n": len(vals)} if vals else None


# ------------------------------------------------------------ CPU reference ----
def reference_outer_iterations(nr, nt, pressure, kind):
    """Outer count of the reference algorithm (lumped-mass StokesPcCG, exact
    inner solves, rtol 1e-8) on this workload, as committed."""
    path = os.path.join(ROOT, "tests", "golden", "outer_iterations.json")
    with open(path) as f:
        d = json.load(f)
    return int(d[f"{nr}x{nt}_{pressure}_{kind}"]), d.get("source", "")


def reference_validation():
    """The model checked against an oracle solve that ran to completion
    (fitted on the 32x256 and 64x512 completed solves, predicting 128x1024)."""
    try:
        from oracle import refmodel
        with open(os.path.join(ROOT, "tests", "golden", "tight.json")) as f:
            rec = json.load(f)["refsolve"]
        return refmodel.validate(rec, "32x256_aniso", "64x512_aniso", "128x1024_aniso")
    except Exception as e:
        return {"error": str(e)}


def cpu_model(args, kind, threads_note):
    """The reference's CPU solve time on the headline workload by the cost
    model: the oracle's phases measured on two smaller meshes of the same
    workload, power laws in the DOF count, times the outer count."""
    from oracle import refmodel
    el = refmodel.default_elements()
    t0 = time.perf_counter()
    a = refmodel.measure(*REF_SAMPLES[0], kind=kind, elements=el)
    b = refmodel.measure(*REF_SAMPLES[1], kind=kind, elements=el)
    fit = refmodel.fit(a, b)
    n_outer, src = reference_outer_iterations(args.nr, args.nt, args.pressure, kind)
    pred = refmodel.predict(fit, args.nr, args.nt, n_outer)
    return dict(seconds_per_solve=pred["total"], phases=pred, n_outer=n_outer,
                exponents={k: v for k, v in fit.items() if k.startswith("p_")},
                samples=[{k: a[k] for k in ("nr", "nt", "asm", "setup", "iter")},
                         {k: b[k] for k in ("nr", "nt", "asm", "setup", "iter")}],
                sample_seconds=time.perf_counter() - t0, threads=threads_note)


def start_cpu_sample(args):
    """The CPU model's sample runs in its own process, concurrently with the
    GPU timing, on one host thread (the GPU path needs one more)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-sample-only", "--nr", str(args.nr), "--nt", str(args.nt),
           "--pressure", args.pressure, "--kind", args.kind]
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", MKL_NUM_THREADS="1")
    return subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=env)


def finish_cpu_sample(proc):
    try:
        out, _ = proc.communicate(timeout=900)
        d = json.loads(out.strip().splitlines()[-1])
    except Exception as e:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "port", "sample": f"failed: {e}"}
    return {"value": 1.0 / d["seconds_per_solve"], "unit": UNIT, "cores": 1, "kind": "port", "modelled": True,
            "sample": _model_sample_text(d), "model": d}


def _model_sample_text(d):
    s = d["samples"]
    return (f"FP64 oracle (the reference's StokesPcCG with a SuperLU inner solve) run on the {s[0]['nr']}x{s[0]['nt']} "
            f"and {s[1]['nr']}x{s[1]['nt']} meshes of this workload ({d['sample_seconds']:.1f} s): assembly, "
            f"factorisation and 4 whole outer iterations each, fitted as power laws in the DOF count "
            f"(exponents {d['exponents']['p_asm']:.2f}, {d['exponents']['p_setup']:.2f}, "
            f"{d['exponents']['p_iter']:.2f}) and extrapolated to this mesh at {d['n_outer']} outer iterations; "
            f"{d['threads']}")


# ------------------------------------------------------------ GPU workload ----
class Workload:
    """One mesh on the device: context, device-resident inputs, learned guess."""

    def __init__(self, nr, nt, pressure, kind, seed, local, opts, use_guess=True):
        import numpy as np
        import torch
        from dimspers_b200 import StokesContext, learned
        self.np, self.torch = np, torch
        self.nr, self.nt, self.kind = nr, nt, kind
        self.dev = torch.device("cuda", local)
        self.mesh, self.mat = make_inputs(nr, nt, pressure, kind, seed)
        m = self.mesh
        self.nel, self.nnod, self.npres = m.nel, m.nnod, m.npres
        self.ctx = StokesContext(nr, nt, pressure, device=local, pin_rotation=True)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream, device=self.dev)
        mat = self.mat
        self.eta_d = torch.from_numpy(np.asfortranarray(mat.eta_ip).T.copy()).to(self.dev)  # (7, nel) == nel x 7
        self.dl_d, self.dx_d, self.dy_d, self.rho_d = (torch.from_numpy(a).to(self.dev)
                                                       for a in (mat.delta, mat.dir_x, mat.dir_y, mat.rho))
        self.U_d = torch.zeros(2 * self.nnod, dtype=torch.float64, device=self.dev)
        self.P_d = torch.zeros(self.npres, dtype=torch.float64, device=self.dev)
        self.opts = opts
        self.guess, self.wpath = None, None
        if use_guess:
            wpath = learned.weights_path(nr, nt)
            if os.path.exists(wpath):
                self.guess = learned.LearnedGuess(learned.GuessNet.load(wpath, max_batch=1, device=local), self.ctx)
                self.wpath = wpath
            elif os.path.exists(learned.weights_path(128, 1024)):
                # no network trained on this mesh: the 128x1024 one run on this grid (its
                # layers are convolutions); the solver keeps the guess only if it starts
                # below the zero guess
                wpath = learned.weights_path(128, 1024)
                net = learned.GuessNet.load(wpath, max_batch=1, device=local)
                self.guess = learned.LearnedGuess(net.for_grid(*learned.grid_shape(nr, nt), device=local), self.ctx)
                self.wpath = wpath
        torch.cuda.synchronize()

    def step(self, arm, guess=True, **extra):
        m = self.mat
        self.ctx.set_material_ti_device(self.eta_d.data_ptr(), self.nel, self.rho_d.data_ptr(), m.g,
                                        self.dl_d.data_ptr(), self.dx_d.data_ptr(), self.dy_d.data_ptr())
        self.ctx.assemble(arm["precision"])
        o = {**self.opts, **arm, **extra}
        if guess and self.guess is not None:
            self.guess.predict(m.g, self.P_d.data_ptr())
            return self.ctx.solve_device(self.U_d.data_ptr(), self.P_d.data_ptr(), None, use_guess=2, **o)
        return self.ctx.solve_device(self.U_d.data_ptr(), self.P_d.data_ptr(), None, **o)

    def timed(self, arm, warm, steps, barrier, sampler=None, guess=True, **extra):
        torch = self.torch
        for _ in range(warm):
            self.step(arm, guess, **extra)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = []
        with (sampler if sampler is not None else _Null()):
            e0.record(self.stream)
            for _ in range(steps):
                reps.append(self.step(arm, guess, **extra))
            e1.record(self.stream)
            barrier()
        return e0.elapsed_time(e1), reps

    def solution(self):
        return self.U_d.clone(), self.P_d.clone()

    def close(self):
        self.ctx.close()


def rel_l2(a, b):
    import torch
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def err_vs_fixture(U, P, fx):
    """Relative L2 error against the committed oracle yardstick, estimated on
    its strided subsample (every `stride`-th entry of U and of P)."""
    import numpy as np
    st = int(fx["stride"])
    u = U.cpu().numpy()[::st]
    p = P.cpu().numpy()[::st]
    return {"u_rel_l2": float(np.linalg.norm(u - fx["U_sub"]) / np.linalg.norm(fx["U_sub"])),
            "p_rel_l2": float(np.linalg.norm(p - fx["P_sub"]) / np.linalg.norm(fx["P_sub"]))}


def run_secondary(local, barrier, host_loop):
    """The 128x1024 anisotropic workload: fast arm, plain FP64 arm, their
    errors against the committed tightly converged oracle solution, and the
    fast arm at tighter tolerances (the rtol where it meets 1e-7)."""
    import numpy as np
    nr, nt, kind = SECONDARY
    opts = dict(rtol=1e-8, itmax=20000, itmin=10, host_loop=1 if host_loop else 0)
    w = Workload(nr, nt, "discontinuous", kind, 1, local, opts)
    out = {"workload": f"annulus {nr}x{nt} cells, {w.nel} P2 elements, {2 * w.nnod} velocity DOF, {w.npres} "
                       f"discontinuous P1 pressure DOF, {kind} viscosity (contrast 1e5)"}
    fx = np.load(TIGHT_FIXTURE) if os.path.exists(TIGHT_FIXTURE) else None
    if fx is not None:
        out["yardstick"] = "FP64 oracle (SuperLU inner solve, element-mass Schur preconditioner) at rtol 1e-12, " \
                           "tests/golden/tight_128x1024_aniso.npz (every 15th entry)"
    ms, reps = w.timed(FAST, 1, 3, barrier)
    out["fast"] = {"value": 3 / (ms / 1e3), "ms_per_step": ms / 3,
                   "outer": spread(r["iterations"] for r in reps), "inner": spread(r["inner_iterations"] for r in reps)}
    Uf, Pf = w.solution()
    ms64, reps64 = w.timed(PLAIN, 0, 1, barrier, guess=False)
    out["fp64"] = {"value": 1 / (ms64 / 1e3), "ms_per_step": ms64, "outer": reps64[0]["iterations"],
                   "inner": reps64[0]["inner_iterations"]}
    U64, P64 = w.solution()
    out["fast_vs_fp64"] = out["fast"]["value"] / out["fp64"]["value"]
    out["fast_vs_fp64_error"] = {"u_rel_l2": rel_l2(Uf, U64), "p_rel_l2": rel_l2(Pf, P64)}
    if fx is not None:
        out["fast_err_vs_tight"] = err_vs_fixture(Uf, Pf, fx)
        out["fp64_err_vs_tight"] = err_vs_fixture(U64, P64, fx)
        sweep = []
        for rt in (1e-9, 1e-10, 1e-11, 1e-12):
            ms_t, rep_t = w.timed(FAST, 0, 1, barrier, rtol=rt, inner_rtol=min(1e-10, rt * 1e-2), relax_base=rt)
            Ut, Pt = w.solution()
            e = err_vs_fixture(Ut, Pt, fx)
            sweep.append({"rtol": rt, "value": 1 / (ms_t / 1e3), "outer": rep_t[0]["iterations"],
                          "inner": rep_t[0]["inner_iterations"], **e})
        out["fast_rtol_sweep"] = sweep
        ok = [s for s in sweep if max(s["u_rel_l2"], s["p_rel_l2"]) <= 1e-7]
        out["fast_meets_1e-7_at"] = ({"rtol": ok[0]["rtol"], "value": ok[0]["value"]} if ok else None)
    w.close()
    return out


def run_ours(args, rank, world, local):
    import torch

    cpu_proc = start_cpu_sample(args) if (rank == 0 and world == 1 and not args.no_cpu) else None
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    opts = dict(rtol=args.rtol, itmax=args.itmax, itmin=10, host_loop=1 if args.host_loop else 0)
    fast = dict(FAST) if args.pressure == "discontinuous" else dict(FAST, schur_pc=0)
    w = Workload(args.nr, args.nt, args.pressure, args.kind, 1 + rank, local, opts, use_guess=not args.no_guess)
    nel, nnod, npres = w.nel, w.nnod, w.npres

    sampler = ClockSampler(local) if not args.no_clocks else None
    ms32, reps32 = w.timed(fast, args.warmup, args.steps, barrier, sampler)
    ms32 = max_over_ranks(ms32, dev, world)
    value = aggregate_value(args.steps, world, ms32)
    ms_per_step = ms32 / args.steps
    U32, P32 = w.solution()   # the fast path's solution, for its error against FP64

    # ---- e2e through the public API with pinned host buffers ---------------------
    import ctypes as C
    import numpy as np
    from dimspers_b200 import default_opts
    from dimspers_b200._lib import DP_MEM_HOST, SolveReport, lib
    mat, ctx = w.mat, w.ctx
    eta_h = torch.from_numpy(np.asfortranarray(mat.eta_ip).T.copy()).pin_memory()
    dl_h, dx_h, dy_h, rho_h = (torch.from_numpy(a).pin_memory() for a in (mat.delta, mat.dir_x, mat.dir_y, mat.rho))
    U_h = torch.zeros(2 * nnod, dtype=torch.float64).pin_memory()
    P_h = torch.zeros(npres, dtype=torch.float64).pin_memory()

    def e2e_step():
        ctx._chk(lib().dp_set_material_ti(ctx.h, C.c_void_p(eta_h.data_ptr()), nel, C.c_void_p(dl_h.data_ptr()),
                                          C.c_void_p(dx_h.data_ptr()), C.c_void_p(dy_h.data_ptr()),
                                          C.c_void_p(rho_h.data_ptr()), float(mat.g), DP_MEM_HOST))
        ctx.assemble(1)
        o = default_opts(**opts, **fast)
        if w.guess is not None:
            w.guess.predict(mat.g, P_h.data_ptr(), mem=0)
            o.use_guess = 2
        rep = SolveReport()
        st = lib().dp_solve(ctx.h, C.c_void_p(U_h.data_ptr()), C.c_void_p(P_h.data_ptr()), None, C.byref(o),
                            C.byref(rep), DP_MEM_HOST)
        if st >= 3:
            ctx._chk(st)
        return rep.as_dict()

    e2e_steps = args.e2e_steps if args.e2e_steps is not None else min(args.steps, 5)
    ms_e2e, reps_e2e = None, []
    if not args.no_e2e:
        e2e_step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(w.stream)
        for _ in range(e2e_steps):
            reps_e2e.append(e2e_step())
        e1.record(w.stream)
        barrier()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1), dev, world)
    h2d = (eta_h.numel() + dl_h.numel() + dx_h.numel() + dy_h.numel() + rho_h.numel()) * 8
    d2h = (U_h.numel() + P_h.numel()) * 8

    # ---- FP64 arms: the reference's algorithm, and the fast arm's algorithm ---------
    fp64, err, same = None, None, None
    if not args.no_fp64:
        ms64, reps64 = w.timed(PLAIN, args.fp64_warmup, args.fp64_steps, barrier, guess=False)
        ms64 = max_over_ranks(ms64, dev, world)
        r = reps64[-1]
        fp64 = {"value": aggregate_value(args.fp64_steps, world, ms64), "ms_per_step": ms64 / args.fp64_steps,
                "outer_iterations": r["iterations"], "inner_iterations": r["inner_iterations"],
                "status": r["status"], "relres": r["relres"], "mom_residual": r["mom_residual"]}
        U64, P64 = w.solution()
        err = {"u_rel_l2": rel_l2(U32, U64), "p_rel_l2": rel_l2(P32, P64)}
    if not args.no_same_algorithm:
        same_arm = dict(SAME_ALGO) if args.pressure == "discontinuous" else dict(SAME_ALGO, schur_pc=0)
        ms_s, reps_s = w.timed(same_arm, 0, 1, barrier)
        ms_s = max_over_ranks(ms_s, dev, world)
        r = reps_s[-1]
        Us, Ps = w.solution()
        same = {"value": aggregate_value(1, world, ms_s), "ms_per_step": ms_s, "outer_iterations": r["iterations"],
                "inner_iterations": r["inner_iterations"], "status": r["status"],
                "options": same_arm, "error_vs_fast": {"u_rel_l2": rel_l2(U32, Us), "p_rel_l2": rel_l2(P32, Ps)}}

    # ---- roofline of the dominant kernel: fine-level FP32 EBE A-apply ---------------
    # The solve is one CUDA graph (events cannot sit inside its loop bodies), so
    # the kernel is timed right after the timed region on the same stream:
    # cold (L2 overwritten before each launch -> the DRAM-bound figure used for
    # the HBM roofline) and warm (back-to-back).
    w.ctx.assemble(1)
    ms_cold = ctx.profile_kernel(0, reps=20, flush_l2=True)
    ms_warm = ctx.profile_kernel(0, reps=50)
    alg_bytes = nel * 78 * 4 + nnod * 2 * 4 * 2
    pk, pk_kind = peaks()
    achieved = alg_bytes / (ms_cold * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_apply_K<float,float> (fine level)", "achieved": achieved,
                "peak": pk, "peak_kind": pk_kind, "unit": "GB/s", "frac": achieved / pk,
                "traffic": traffic_from_profiles(args.nr, args.nt), "algorithmic_bytes": alg_bytes,
                "ms_per_launch": ms_cold, "ms_per_launch_warm_l2": ms_warm,
                "achieved_warm_l2": alg_bytes / (ms_warm * 1e-3) / 1e9}
    w.ctx.assemble(0)
    ms64_apply = ctx.profile_kernel(1, reps=20, flush_l2=True)
    alg64 = nel * 78 * 8 + nnod * 2 * 8 * 2
    roofline["fp64_apply"] = {"kernel": "k_apply_K<double,double> (fine level)", "ms_per_launch": ms64_apply,
                              "achieved": alg64 / (ms64_apply * 1e-3) / 1e9,
                              "frac": alg64 / (ms64_apply * 1e-3) / 1e9 / pk}

    clocks = sampler.summary() if sampler is not None else {"sm_mhz": None, "reasons": ["not sampled"]}
    last = reps32[-1]
    allreps = reps32 + reps_e2e
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": {"workload": f"annulus {args.nr}x{args.nt} cells, {nel} P2 elements, {2 * nnod} velocity DOF, "
                               f"{npres} {args.pressure} P1 pressure DOF, {args.kind} viscosity",
                   "nr_cells": args.nr, "ntheta_cells": args.nt, "pressure": args.pressure, "material": args.kind,
                   "rtol": args.rtol,
                   "guess": ("learned (" + os.path.basename(w.wpath) + ")") if w.guess is not None else "zero",
                   "fast_arm": fast, "plain_arm": PLAIN,
                   "parallelism": f"replicas x{world}", "e2e_steps": e2e_steps,
                   "l2": "inputs larger than L2: every step re-assembles and streams the element blocks "
                         f"({nel * 78 * 4 / 1e9:.2f} GB FP32 + {nel * 78 * 8 / 1e9:.2f} GB FP64; L2 is 126 MB)"},
        "outer_iterations": last["iterations"], "inner_iterations": last["inner_iterations"],
        "iterations": {"outer": spread(r["iterations"] for r in allreps),
                       "inner": spread(r["inner_iterations"] for r in allreps),
                       "note": "timed device-resident and e2e solves; the FP32 applies scatter with atomics, so "
                               "counts vary between runs"},
        "refinements": last["refinements"], "status": last["status"], "relres": last["relres"],
        "guess_fallback": last["fallback_used"],
        "r0_guess_over_r0": (last["r0_guess"] / last["r0"]) if w.guess is not None and last["r0"] else None,
        "mom_residual": last["mom_residual"], "mg_levels": last["mg_levels"],
        "fp64": fp64, "fast_vs_fp64": (value / fp64["value"]) if fp64 else None, "fast_vs_fp64_error": err,
        "fp64_same_algorithm": same, "precision_gain": (value / same["value"]) if same else None,
        "e2e": ({"value": aggregate_value(e2e_steps, world, ms_e2e), "unit": UNIT, "h2d_bytes_per_step": h2d,
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
    w.close()
    if not args.no_secondary and world == 1:
        try:
            line["secondary"] = run_secondary(local, barrier, args.host_loop)
        except Exception as e:
            line["secondary"] = {"error": str(e)}
    if cpu_proc is not None:
        line["cpu_baseline"] = finish_cpu_sample(cpu_proc)
        line["cpu_baseline"]["validation"] = reference_validation()
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
    Chebyshev vector steps 52 B/node, first steps 44 B/node (on the coarse
    levels the first is fused into the restriction); restriction 8 B/fine node
    + 44 B/coarse node; prolongation 32 B/fine node; dense coarsest n^2 x 8 B; inner PCG
    vector passes 108 B/DOF; outer: G and G^T 288 B/element + vectors, the
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
        vcycle += (44.0 if i == 0 else 0.0) * nnod + 44.0 * nnod         # first steps (pre on the top level, post)
        vcycle += 2 * (cheb_degree - 1) * 52.0 * nnod                    # Chebyshev vector steps
        vcycle += 8.0 * nnod + 44.0 * cn + 32.0 * nnod                   # restriction, prolongation
    nel, nnod = levels[0]
    n_u = 2 * nnod
    n_p = 3 * nel if pressure == "discontinuous" else (nr + 1) * nt
    per_inner = vcycle + 624.0 * nel + 48.0 * nnod + 108.0 * n_u
    per_outer = 2 * (288.0 * nel + 16.0 * nnod + 8.0 * n_p) + (5 * n_p + 2 * n_u) * 8.0 + 4 * 16.0 * n_p
    return inner * per_inner + outer * per_outer


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def profile_apply(args):
    """Assemble the workload and launch the fine-level FP32 A-apply 3 times."""
    from dimspers_b200 import StokesContext
    mesh, mat = make_inputs(args.nr, args.nt, args.pressure, args.kind, seed=1)
    with StokesContext(args.nr, args.nt, args.pressure, pin_rotation=True) as ctx:
        ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
        ctx.assemble(1)
        ms = ctx.profile_kernel(0, reps=3)
    print(json.dumps({"profile_apply_ms": ms}))


def run_reference(args, rank, world):
    """The reference's CPU algorithm on this workload, by the cost model: each
    step measures the oracle's phases on the two sample meshes (element blocks
    on every host thread, SuperLU single-threaded) and predicts the solve."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    note = (f"element blocks on {threads} threads (C/OpenMP restatement); sparse assembly, SuperLU and the "
            f"outer iterations single-threaded")
    per = []
    d = None
    for i in range(args.warmup + args.steps):
        d = cpu_model(args, args.kind, note)
        if i >= args.warmup:
            per.append(d["seconds_per_solve"])
    per_solve = statistics.mean(per)
    value = 1.0 / per_solve
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_solve * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
        "modelled": True,
        "config": {"workload": f"annulus {args.nr}x{args.nt} cells, {args.pressure} P1 pressure, {args.kind}",
                   "nr_cells": args.nr, "ntheta_cells": args.nt, "pressure": args.pressure, "material": args.kind,
                   "rtol": args.rtol},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "modelled": True,
                         "sample": _model_sample_text(d), "model": d, "validation": reference_validation()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "ms_per_step is the modelled time of one reference solve; each of the warmup + steps passes "
                "measured the two sample meshes anew",
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


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.cpu_sample_only:
        print(json.dumps(cpu_model(args, args.kind, "one host thread")), flush=True)
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
