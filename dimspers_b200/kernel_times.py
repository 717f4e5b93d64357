"""Event-timed launches of the kernels around the Stokes solve: the stress
post-processor, the viscosity update, the DEM tensor lookup and the thermal
step (whole step and its element-by-element apply).

    python -m dimspers_b200.kernel_times 128x1024 512x4096

One JSON line per kernel and mesh: the warm (back-to-back) and cold (L2
flushed before each launch) CUDA-event time per launch from
dp_profile_kernel, the algorithmic bytes of one launch, the cold GB/s, and
the wall time of the whole ABI call with host arrays (copies in and out
included; best of 3).  Inputs are seeded synthetic fields of the reference's
shapes and ranges (`inputs_*` below, shared with the CPU baseline in bench.py).
"""
import json
import os
import sys
import time

import numpy as np

from . import StokesContext, inputs
from .fabric import DEM

HERE = os.path.dirname(os.path.abspath(__file__))
DEM_FIXTURE = os.path.join(HERE, "..", "tests", "golden", "dem_1e-3_vol30.npz")


def _line(kernel, size, warm, cold, alg, ok, **extra):
    d = dict(kernel=kernel, size=size, warm_us=1e3 * warm, cold_us=1e3 * cold, alg_MB=alg / 1e6,
             cold_GBs=alg / (cold * 1e-3) / 1e9, finite=bool(ok))
    d.update(extra)
    return d


def _best_ms(fn, reps=3):
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return 1e3 * min(ts)


def inputs_viscosity(mesh, nr, nt, rng):
    """(T, P_vertex, r in m, epsII, tauII, cohesion) of the viscosity-update timing."""
    nel, nn, nv = mesh.nel, mesh.nnod, (nr + 1) * nt
    r = 3.48e6 + (mesh.r - 1.22) * 2.87e6
    return (1300.0 + 1200.0 * rng.random(nn), 2e9 * rng.standard_normal(nv), r,
            np.abs(rng.standard_normal((nel, 7))) * 1e-15, 4e9 * rng.random((nel, 7)),
            np.where(rng.random((nel, 7)) < 0.3, 0.0, 30e6))


def inputs_dem(nel, rng):
    """(vx1, vy1, r1, r2) per IP of the DEM-tensor timing."""
    ang = rng.uniform(-np.pi, np.pi, (nel, 6))
    return np.cos(ang), np.sin(ang), rng.uniform(-0.3, 2.0, (nel, 6)), rng.uniform(-0.3, 2.3, (nel, 6))


def inputs_thermal(mesh, nr, rng):
    """(T, rho, dt): a perturbed conduction profile, diffusion number ~1 per radial cell."""
    th, r = mesh.theta, mesh.r
    T = (4000.0 + (300.0 - 4000.0) * np.log(r / 1.22) / np.log(2.22 / 1.22)
         + 200 * np.sin(3 * th) * np.sin(np.pi * (r - 1.22)))
    rho = 3300.0 * (1 + 0.05 * rng.standard_normal(mesh.nnod))
    h = 1.0 / nr
    return T, rho, h * h * 3300 * 1.2e3 / 3.3


def post_kernels(nr, nt):
    size = "%dx%d" % (nr, nt)
    out = []
    c = StokesContext(nr, nt, "discontinuous")
    m = inputs.make_material(c.mesh, "aniso", seed=1)
    rng = np.random.default_rng(0)
    nel, nn, nv = c.nel, c.nnod, (nr + 1) * nt
    U = rng.standard_normal(2 * nn)
    o = c.stress(U, m.eta_ip, m.C6)
    call = _best_ms(lambda: c.stress(U, m.eta_ip, m.C6))
    out.append(_line("k_stress", size, c.profile_kernel(3, 50), c.profile_kernel(3, 10, True),
                     nel * (7 + 42 + 56) * 8 + nn * 4 * 8, all(np.isfinite(v).all() for v in o.values()),
                     call_ms=call))
    T, P, r, eps, tau, coh = inputs_viscosity(c.mesh, nr, nt, rng)
    eta0 = np.full((nel, 7), 3.3e21)
    eta = c.viscosity_arrhenius(eta0, T, P, r, eps, tau, coh, phi=30.0)
    call = _best_ms(lambda: c.viscosity_arrhenius(eta0, T, P, r, eps, tau, coh, phi=30.0))
    out.append(_line("k_viscosity_arrhenius", size, c.profile_kernel(4, 50), c.profile_kernel(4, 10, True),
                     nel * 7 * 8 * 5 + nn * 2 * 8 + nv * 8, np.isfinite(eta).all(), call_ms=call))
    if os.path.exists(DEM_FIXTURE):
        d = np.load(DEM_FIXTURE)
        dem = DEM(d["C"], d["ax"], 0.02)
        x1, y1, r1, r2 = inputs_dem(nel, rng)
        res = c.anisotropic_tensor(dem, x1, y1, r1, r2)
        call = _best_ms(lambda: c.anisotropic_tensor(dem, x1, y1, r1, r2))
        out.append(_line("k_dem_tensor", size, c.profile_kernel(5, 50), c.profile_kernel(5, 10, True),
                         nel * (24 + 42) * 8, all(np.isfinite(x).all() for x in res), call_ms=call))
    c.close()
    return out


def thermal(nr, nt):
    size = "%dx%d" % (nr, nt)
    c = StokesContext(nr, nt, "continuous")
    T, rho, dt = inputs_thermal(c.mesh, nr, np.random.default_rng(0))
    Tn, it, rel = c.thermal_step(T, rho, dt)
    call = _best_ms(lambda: c.thermal_step(T, rho, dt), reps=5)
    rec = _line("k_th_apply", size, c.profile_kernel(6, 50), c.profile_kernel(6, 10, True),
                c.nel * 21 * 8 + c.nnod * 3 * 8, np.isfinite(Tn).all(), dt=dt, iterations=it, relres=rel,
                step_ms=call, call_ms=call)
    c.close()
    return [rec]


def measure(sizes):
    recs = []
    for size in sizes or ["128x1024"]:
        nr, nt = (int(v) for v in size.split("x"))
        recs += post_kernels(nr, nt) + thermal(nr, nt)
    return recs


def main(argv):
    for rec in measure(argv):
        print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
