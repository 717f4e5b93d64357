"""Cost model of the reference's CPU solve (test and benchmark infrastructure).

The reference path (solveStokes with StokesPcCG and a direct LU inner solve,
src/Stokes/StokesSolver.jl:7-54, src/IterativeSolvers.jl:94-168,
src/PardisoSolvers.jl:247-256, 274-278) is restated by oracle.solver.  A solve
at the large workloads (4.2M elements, 16.8M velocity DOF) cannot be completed
on the host: the sparse LU alone would need tens of GB and its ~2,400
back-substitutions hours.  This module therefore measures the oracle's three
phases on two smaller meshes of the same workload, each phase on solves that
really run (the C/OpenMP element blocks with SciPy's sparse assembly and
rotation; SuperLU's factorisation and first solve; whole StokesPcCG outer
iterations -- back-solve, G and G^T products, Schur vector updates, means and
dots), fits each phase a power law in the number of velocity DOF, and predicts

    T(N) = T_asm(N) + T_setup(N) + n_outer * T_iter(N)

with n_outer the outer count of the reference algorithm on the target mesh.
``validate`` checks the prediction against oracle solves that ran to
completion (tests/golden/tight.json, "refsolve").  Nothing here is on the
product path.
"""
import math
import os
import time

import numpy as np

from . import solver as OS


def _dof(nr, nt):
    return 2 * (2 * nr + 1) * 2 * nt


class _MeshView:
    def __init__(self, prob):
        self.theta, self.r, self.e2n = prob.gr.theta, prob.gr.r, prob.gr.e2n
        self.th_el, self.r_el = prob.th, prob.r


def measure(nr, nt, kind="fabric", iters=4, seed=1, elements=None):
    """Phase times (s) of the oracle solve on an nr x nt mesh: assembly,
    factorisation + first solve, and the mean of `iters` whole outer
    iterations (the loop runs exactly `iters` iterations)."""
    from dimspers_b200 import inputs
    prob = OS.make_problem(nr, nt, "discontinuous", pin_rotation=True)
    mat = inputs.make_material(_MeshView(prob), kind, seed=seed)
    tm = {}
    t0 = time.perf_counter()
    OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-300, itmax=iters, itmin=iters,
                    remove_rotation=False, elements=elements, timing=tm)
    return dict(nr=nr, nt=nt, dof=_dof(nr, nt), asm=tm["assembly"], setup=tm["setup"],
                iter=float(np.mean(tm["iters"])), wall=time.perf_counter() - t0, iters=len(tm["iters"]))


def fit(a, b):
    """Per-phase power laws T = T_b * (N / N_b)^p from two measurements."""
    out = {"anchor": b}
    lr = math.log(b["dof"] / a["dof"])
    for ph in ("asm", "setup", "iter"):
        out["p_" + ph] = math.log(max(b[ph], 1e-9) / max(a[ph], 1e-9)) / lr
    return out


def predict(f, nr, nt, n_outer):
    b = f["anchor"]
    x = _dof(nr, nt) / b["dof"]
    asm = b["asm"] * x ** f["p_asm"]
    setup = b["setup"] * x ** f["p_setup"]
    it = b["iter"] * x ** f["p_iter"]
    return dict(total=asm + setup + n_outer * it, asm=asm, setup=setup, iter=it, n_outer=n_outer)


def validate(records, small, mid, target):
    """Model fitted on two completed solves' phases, checked against a third
    completed solve: relative error of the predicted total time."""
    def as_meas(key):
        r = records[key]
        nr, nt = (int(v) for v in key.split("_")[0].split("x"))
        return dict(nr=nr, nt=nt, dof=_dof(nr, nt), asm=r["assembly_s"], setup=r["setup_s"], iter=r["iter_mean_s"])
    f = fit(as_meas(small), as_meas(mid))
    t = records[target]
    nr, nt = (int(v) for v in target.split("_")[0].split("x"))
    p = predict(f, nr, nt, t["outer"])
    return dict(predicted_s=p["total"], measured_s=t["total_s"], rel_error=p["total"] / t["total_s"] - 1.0,
                fit={k: v for k, v in f.items() if k.startswith("p_")}, small=small, mid=mid, target=target)


def default_elements():
    """The threaded C restatement of the element blocks (all host threads)."""
    from . import c_elements as OC
    OC.build()
    return OC.element_matrices


def host_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
