"""Independent Stokes solves of uneven resolution in one graph launch.

The reference solves one Stokes problem per call (solveStokes,
src/Stokes/StokesSolver.jl:7-54); it has no batched form.  ``SolveBatch``
wraps ``dp_batch_create`` / ``dp_batch_run``: one CUDA graph with one branch
per problem, each branch that problem's whole Schur PCG solve with its own
device-side loop control, so the 1-thread control kernels, reductions and
coarse-level work of small problems overlap with the other problems' kernels
instead of each problem running alone.

``autotune`` chooses the per-resolution settings the batch replays: the tile
of the element-by-element applies (warps per CTA, warps stacked along theta),
the Chebyshev degree and the size of the dense coarsest system.  Each
candidate runs a short solve with a fixed number of outer iterations and is
scored by milliseconds per outer iteration: the outer iteration count is set
by the Schur preconditioner, not by these settings, so this ranks candidates
as a full solve would at a small fraction of its cost.  Results are recorded
to JSON (keyed "NRxNT/pressure") and replayed with ``load_tuning``.

``python -m dimspers_b200.batch`` runs the 24-problem comparison (6 problems
each at 32x256, 64x512, 128x1024 and 256x2048 cells; plume temperatures,
Ra log-uniform in [1e5, 1e7], delta in [1, 10], anisotropic viscosity;
FP32-refined multigrid inner solves with the learned initial guess, to 1e-8):
the batch in one launch against the same problems one launch each, reporting
solves/s, per-solve iterations and p50/p99 completion latency.
"""
import argparse
import ctypes as C
import itertools
import json
import os
import time

import numpy as np

from . import inputs
from ._lib import DP_MEM_DEVICE, DP_MEM_HOST, SolveOpts, SolveReport, check, lib
from .stokes import StokesContext, default_opts

SIZES = ((32, 256), (64, 512), (128, 1024), (256, 2048))
FAST = dict(precision=1, cheb_degree=3, cheb_lo=0.05, inner_rtol=1e-10, inner_relax=1e-2, relax_base=1e-8, schur_pc=1)
TUNE_SPACE = dict(apply=((4, 1), (8, 1), (4, 4), (8, 2)), cheb_degree=(2, 3, 4), coarse_max=(1024, 1536))


def tuning_key(ctx):
    d = ctx.desc
    return f"{d.nr_cells}x{d.ntheta_cells}/{'discontinuous' if d.pressure_space == 1 else 'continuous'}"


class SolveBatch:
    """dp_batch over StokesContexts (all assembled, one device).  ``opts``: one
    dict of dp_solve_opts fields per context (or one dict for all)."""

    def __init__(self, contexts, opts=None):
        self.contexts = list(contexts)
        n = len(self.contexts)
        if isinstance(opts, dict) or opts is None:
            opts = [opts or {}] * n
        self._opts = (SolveOpts * n)(*[default_opts(**o) for o in opts])
        ptrs = (C.c_void_p * n)(*[c.h.value for c in self.contexts])
        self.h = C.c_void_p()
        check(lib().dp_batch_create(C.cast(ptrs, C.POINTER(C.c_void_p)), n, C.cast(self._opts, C.c_void_p),
                                    C.byref(self.h)))

    def close(self):
        if self.h:
            lib().dp_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, guesses=None, U=None, P=None, mem=DP_MEM_HOST):
        """One launch of the whole batch.  guesses / U / P: lists of numpy
        arrays (mem = host) or device pointers as ints (mem = device), entries
        may be None.  Returns (reports, done_ms): per-problem report dicts and
        completion times in ms from the launch."""
        n = len(self.contexts)

        def ptrs(lst):
            if lst is None:
                return None
            arr = (C.c_void_p * n)()
            for i, a in enumerate(lst):
                if a is None:
                    arr[i] = None
                elif isinstance(a, np.ndarray):
                    arr[i] = a.ctypes.data
                else:
                    arr[i] = int(a)
            return C.cast(arr, C.POINTER(C.c_void_p))

        reps = (SolveReport * n)()
        done = (C.c_double * n)()
        keep = (guesses, U, P)  # the arrays stay alive for the call
        st = lib().dp_batch_run(self.h, ptrs(guesses), ptrs(U), ptrs(P), int(mem), C.cast(reps, C.c_void_p), done)
        del keep
        check(st)
        return [r.as_dict() for r in reps], np.array(done[:], dtype=np.float64)


# ---- autotuner ------------------------------------------------------------------------
def autotune(ctx, base=None, outer_its=30, reps=2, space=None, log=None):
    """Best settings for one assembled context: ms per outer iteration of a
    fixed-length solve, best of ``reps``, over ``space``."""
    base = dict(FAST if base is None else base)
    space = space or TUNE_SPACE
    trials = []
    for (w, wt), deg, cmax in itertools.product(space["apply"], space["cheb_degree"], space["coarse_max"]):
        o = dict(base, apply_warps=w, apply_warps_t=wt, cheb_degree=deg, coarse_max=cmax,
                 rtol=1e-30, itmin=outer_its, itmax=outer_its, use_guess=0)
        best = None
        for _ in range(reps + 1):  # first run captures the graph
            _, _, _, r = ctx.solve(want_cart=False, raise_on_status=False, **o)
            if r["status"] >= 2:
                break
            ms = r["t_solve_ms"] / max(r["iterations"], 1)
            best = ms if best is None else min(best, ms)
        if best is None:
            continue
        trials.append(dict(apply_warps=w, apply_warps_t=wt, cheb_degree=deg, coarse_max=cmax, ms_per_outer=best))
        if log:
            log(f"  {tuning_key(ctx)} warps={w} warps_t={wt} cheb={deg} coarse={cmax}: {best:.3f} ms/outer")
    trials.sort(key=lambda t: t["ms_per_outer"])
    return trials


def tune_all(contexts, path=None, **kw):
    """Tunes one context per distinct resolution and records {key: settings}."""
    table = {}
    for c in contexts:
        key = tuning_key(c)
        if key in table:
            continue
        trials = autotune(c, **kw)
        table[key] = dict(trials[0], trials=len(trials), default=next(
            (t for t in trials if (t["apply_warps"], t["apply_warps_t"], t["cheb_degree"], t["coarse_max"]) ==
             (4, 1, FAST["cheb_degree"], 1536)), None))
    if path:
        with open(path, "w") as f:
            json.dump(table, f, indent=1)
    return table


def load_tuning(path):
    with open(path) as f:
        return json.load(f)


def tuned_opts(ctx, table, base=None):
    """Replay: base options with the recorded settings of the context's resolution."""
    o = dict(FAST if base is None else base)
    t = table.get(tuning_key(ctx)) if table else None
    if t:
        o.update({k: t[k] for k in ("apply_warps", "apply_warps_t", "cheb_degree", "coarse_max")})
    return o


# ---- the 24-problem comparison --------------------------------------------------------
def make_problems(sizes=SIZES, per_size=6, seed0=5000, device=0):
    """StokesContexts with plume temperatures, assembled (FP64 elements, FP32 copy on demand)."""
    ctxs = []
    for s, (nr, nt) in enumerate(sizes):
        for k in range(per_size):
            seed = seed0 + 100 * s + k
            c = StokesContext(nr, nt, "discontinuous", device)
            m = inputs.make_material(c.mesh, "plumes", seed=seed)
            c.set_material_ti(m.eta_ip, m.rho, m.g, m.delta, m.dir_x, m.dir_y)
            c.assemble(0)
            c.seed, c.g = seed, m.g
            ctxs.append(c)
    return ctxs


def learned_guesses(ctxs, device=0):
    """Device guess vectors (torch tensors) from the trained network, run at each
    context's own grid; None where no weights exist."""
    import torch

    from .learned import GuessNet, LearnedGuess, grid_shape, weights_path
    path = weights_path(128, 1024)
    if not os.path.exists(path):
        return [None] * len(ctxs)
    base = GuessNet.load(path, max_batch=1, device=device)
    nets, out = {}, []
    for c in ctxs:
        shape = grid_shape(c.desc.nr_cells, c.desc.ntheta_cells)
        if shape not in nets:
            nets[shape] = base if shape == (base.nrg, base.ntg) else base.for_grid(*shape, device=device)
        P0 = torch.zeros(c.npres, dtype=torch.float64, device=torch.device("cuda", device))
        LearnedGuess(nets[shape], c).predict(c.g, P0.data_ptr())
        out.append(P0)
    torch.cuda.synchronize()
    return out


def compare(ctxs, table, guesses, rtol=1e-8, itmax=20000, log=print):
    """Sequential (one launch per problem) vs batched (one launch) on the same problems."""
    import torch
    n = len(ctxs)
    use_guess = 2 if any(g is not None for g in guesses) else 0
    opts = [dict(tuned_opts(c, table), rtol=rtol, itmax=itmax, use_guess=use_guess if guesses[i] is not None else 0)
            for i, c in enumerate(ctxs)]
    dev = torch.device("cuda", ctxs[0].desc.device)
    Us = [torch.empty(2 * c.nnod, dtype=torch.float64, device=dev) for c in ctxs]
    Ps = [torch.empty(c.npres, dtype=torch.float64, device=dev) for c in ctxs]

    def load_guesses():
        for i in range(n):
            if guesses[i] is not None:
                Ps[i].copy_(guesses[i])
        torch.cuda.synchronize()

    # sequential: one-iteration warm solves capture each context's graph, then timed
    seq = []
    for i, c in enumerate(ctxs):
        load_guesses()
        c.solve_device(Us[i].data_ptr(), Ps[i].data_ptr(), **dict(opts[i], itmax=1, itmin=1))
    load_guesses()
    t0 = time.perf_counter()
    done_seq = []
    for i, c in enumerate(ctxs):
        r = c.solve_device(Us[i].data_ptr(), Ps[i].data_ptr(), **opts[i])
        done_seq.append((time.perf_counter() - t0) * 1e3)
        seq.append(r)
    t_seq = time.perf_counter() - t0
    U_seq = [u.clone() for u in Us]
    P_seq = [p.clone() for p in Ps]

    with SolveBatch(ctxs, opts) as b:
        g_ptrs = [g.data_ptr() if g is not None else None for g in guesses]
        t0 = time.perf_counter()
        bat, done_bat = b.run(g_ptrs, [u.data_ptr() for u in Us], [p.data_ptr() for p in Ps], DP_MEM_DEVICE)
        t_bat = time.perf_counter() - t0
    dU = max(float((Us[i] - U_seq[i]).norm() / U_seq[i].norm()) for i in range(n))
    dP = max(float((Ps[i] - P_seq[i]).norm() / P_seq[i].norm()) for i in range(n))

    def pct(a, q):
        return float(np.percentile(np.asarray(a), q))

    res = dict(
        problems=[dict(size=f"{c.desc.nr_cells}x{c.desc.ntheta_cells}", seed=c.seed,
                       seq_outer=seq[i]["iterations"], batch_outer=bat[i]["iterations"],
                       seq_status=seq[i]["status"], batch_status=bat[i]["status"],
                       seq_ms=seq[i]["t_solve_ms"], seq_done_ms=done_seq[i], batch_done_ms=float(done_bat[i]),
                       fallback=bat[i]["fallback_used"], relres=bat[i]["relres"]) for i, c in enumerate(ctxs)],
        sequential=dict(seconds=t_seq, solves_per_s=n / t_seq, p50_done_ms=pct(done_seq, 50),
                        p99_done_ms=pct(done_seq, 99),
                        p50_solve_ms=pct([r["t_solve_ms"] for r in seq], 50),
                        p99_solve_ms=pct([r["t_solve_ms"] for r in seq], 99)),
        batched=dict(seconds=t_bat, solves_per_s=n / t_bat, p50_done_ms=pct(done_bat, 50),
                     p99_done_ms=pct(done_bat, 99)),
        speedup=t_seq / t_bat, max_rel_diff_U=dU, max_rel_diff_P=dP, tuning=table)
    if log:
        log(f"sequential {t_seq:.2f} s ({n / t_seq:.3f} solves/s), batched {t_bat:.2f} s ({n / t_bat:.3f} solves/s), "
            f"x{t_seq / t_bat:.2f}; max rel diff U {dU:.2e} P {dP:.2e}")
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--per-size", type=int, default=6)
    ap.add_argument("--sizes", default="32x256,64x512,128x1024,256x2048")
    ap.add_argument("--tune", default=None, help="tuning JSON to replay (written by --retune)")
    ap.add_argument("--retune", action="store_true", help="run the autotuner and write --tune (or the report)")
    ap.add_argument("--no-guess", action="store_true")
    ap.add_argument("--out", default=None)
    ap.add_argument("--rtol", type=float, default=1e-8)
    a = ap.parse_args(argv)
    sizes = tuple(tuple(int(v) for v in s.split("x")) for s in a.sizes.split(","))
    ctxs = make_problems(sizes, a.per_size)
    t0 = time.perf_counter()
    if a.retune or not (a.tune and os.path.exists(a.tune)):
        table = tune_all(ctxs, a.tune, log=print)
    else:
        table = load_tuning(a.tune)
    t_tune = time.perf_counter() - t0
    guesses = [None] * len(ctxs) if a.no_guess else learned_guesses(ctxs)
    res = compare(ctxs, table, guesses, rtol=a.rtol)
    res["tune_seconds"] = t_tune
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    for c in ctxs:
        c.close()
    return res


if __name__ == "__main__":
    main()
