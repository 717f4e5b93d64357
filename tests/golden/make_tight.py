"""Tightly converged oracle solutions and completed CPU reference solves
(test infrastructure).

The reference ships no golden vectors, so the yardstick every solve is
measured against is the FP64 oracle (a direct LU inner solve, the reference's
StokesPcCG) run far below the 1e-8 stopping tolerance.  This script makes:

  config1   32x256 isotropic workload (contrast 1e3, Ra 1e5, discontinuous P1,
            free slip, rotation removed, T = conductive + 0.01 cos4θ sin(π(r-r_in))
            + U(±1e-3), seed 1): full U and P at rtol 1e-12, the reference
            algorithm's rtol-1e-8 solution and outer count, and the oracle's own
            noise floor (the same solve with a second column ordering of the LU)
            -> config1_32x256_iso_disc.npz + tight.json["config1"]
  tight128  128x1024 anisotropic workload (contrast 1e5, seed 1, discontinuous
            P1): U and P at rtol 1e-12 with the exact element-mass Schur
            preconditioner; every 15th entry is kept (odd stride: both velocity
            components) with the full norms -> tight_128x1024_aniso.npz
  refsolve  completed oracle solves of the reference algorithm (lumped Schur
            preconditioner, rtol 1e-8) with their phase times: assembly,
            factorisation, seconds per outer iteration, outer count, total
            -> tight.json["refsolve"][size]; these validate the reference arm's
            cost model (oracle/refmodel.py) on solves that ran to completion

Run from the repository root, e.g.:
  python tests/golden/make_tight.py config1
  python tests/golden/make_tight.py tight128
  python tests/golden/make_tight.py refsolve 32x256 64x512 128x1024
Each command merges its results into tests/golden/tight.json.
"""
import fcntl
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dimspers_b200 import inputs  # noqa: E402
from oracle import solver as OS  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
META = os.path.join(HERE, "tight.json")
STRIDE = 15


class MeshView:
    def __init__(self, prob):
        self.theta, self.r, self.e2n = prob.gr.theta, prob.gr.r, prob.gr.e2n
        self.th_el, self.r_el = prob.th, prob.r


def merge(key, value):
    with open(META + ".lock", "w") as lk:
        fcntl.flock(lk, fcntl.LOCK_EX)
        d = {}
        if os.path.exists(META):
            with open(META) as f:
                d = json.load(f)
        if isinstance(value, dict) and isinstance(d.get(key), dict):
            d[key].update(value)
        else:
            d[key] = value
        with open(META, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
    os.remove(META + ".lock")


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def elements():
    import oracle.c_elements as OC
    OC.build()
    return OC.element_matrices


def config1():
    prob = OS.make_problem(32, 256, "discontinuous", pin_rotation=True)
    mat = inputs.make_material(MeshView(prob), "iso", seed=1)
    el = elements()
    out = {}
    sols = {}
    for permc in ("MMD_AT_PLUS_A", "COLAMD"):
        for rtol in (1e-12, 1e-8):
            t0 = time.perf_counter()
            s = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, None, rtol=rtol, itmax=20000,
                                permc=permc, elements=el)
            sols[(permc, rtol)] = s
            out[f"{permc}_rtol{rtol:g}"] = dict(iterations=s["report"].iterations, relres=s["report"].relres,
                                                seconds=time.perf_counter() - t0)
            print(permc, rtol, s["report"].iterations, flush=True)
    T = sols[("MMD_AT_PLUS_A", 1e-12)]
    for (permc, rtol), s in sols.items():
        out[f"{permc}_rtol{rtol:g}"].update(u_vs_tight=rel(s["U"], T["U"]), p_vs_tight=rel(s["P"], T["P"]))
    out["noise_floor_rtol1e-12"] = dict(
        u=rel(sols[("COLAMD", 1e-12)]["U"], T["U"]), p=rel(sols[("COLAMD", 1e-12)]["P"], T["P"]),
        note="the same rtol-1e-12 oracle solve with two LU column orderings")
    out["noise_floor_rtol1e-8"] = dict(
        u=rel(sols[("COLAMD", 1e-8)]["U"], sols[("MMD_AT_PLUS_A", 1e-8)]["U"]),
        p=rel(sols[("COLAMD", 1e-8)]["P"], sols[("MMD_AT_PLUS_A", 1e-8)]["P"]),
        note="two rtol-1e-8 oracle solves that differ only in the LU column ordering")
    out.update(nr_cells=32, ntheta_cells=256, pressure="discontinuous", kind="iso", seed=1, schur_pc="lumped")
    R8 = sols[("MMD_AT_PLUS_A", 1e-8)]
    np.savez_compressed(os.path.join(HERE, "config1_32x256_iso_disc.npz"), U=T["U"], P=T["P"],
                        U8=R8["U"], P8=R8["P"])
    merge("config1", out)


def tight128():
    prob = OS.make_problem(128, 1024, "discontinuous", pin_rotation=True)
    mat = inputs.make_material(MeshView(prob), "aniso", seed=1)
    tm = {}
    t0 = time.perf_counter()
    s = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-12, itmax=20000, schur_pc="mass",
                        elements=elements(), timing=tm)
    U, P = s["U"], s["P"]
    np.savez_compressed(os.path.join(HERE, "tight_128x1024_aniso.npz"), U_sub=U[::STRIDE], P_sub=P[::STRIDE],
                        U_norm=np.linalg.norm(U), P_norm=np.linalg.norm(P), stride=STRIDE)
    merge("tight128", dict(nr_cells=128, ntheta_cells=1024, pressure="discontinuous", kind="aniso", seed=1,
                           schur_pc="mass", rtol=1e-12, iterations=s["report"].iterations,
                           relres=s["report"].relres, seconds=time.perf_counter() - t0, stride=STRIDE))
    print("tight128", s["report"].iterations, flush=True)


def refsolve(sizes, kind="aniso"):
    for size in sizes:
        nr, nt = (int(v) for v in size.split("x"))
        prob = OS.make_problem(nr, nt, "discontinuous", pin_rotation=True)
        mat = inputs.make_material(MeshView(prob), kind, seed=1)
        tm = {}
        t0 = time.perf_counter()
        s = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-8, itmax=20000,
                            elements=elements(), timing=tm)
        total = time.perf_counter() - t0
        it = np.array(tm["iters"])
        rec = dict(kind=kind, seed=1, rtol=1e-8, schur_pc="lumped", outer=s["report"].iterations,
                   assembly_s=tm["assembly"], setup_s=tm["setup"], iter_mean_s=float(it.mean()),
                   iter_first3_s=float(it[:3].mean()), total_s=total, cores=os.cpu_count(),
                   threads_elements=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
        if size == "128x1024" and kind == "aniso":
            np.savez_compressed(os.path.join(HERE, "ref8_128x1024_aniso.npz"), U_sub=s["U"][::STRIDE],
                                P_sub=s["P"][::STRIDE], stride=STRIDE)
        merge("refsolve", {f"{size}_{kind}": rec})
        print(size, kind, rec, flush=True)


if __name__ == "__main__":
    cmd = sys.argv[1]
    if cmd == "config1":
        config1()
    elif cmd == "tight128":
        tight128()
    elif cmd == "refsolve":
        kind = os.environ.get("KIND", "aniso")
        refsolve(sys.argv[2:], kind)
    else:
        raise SystemExit(__doc__)
