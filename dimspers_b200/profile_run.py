"""Launch every kernel family of the library once inside an NVTX range named
"target", for per-kernel ncu captures and launch lists.

    python -m dimspers_b200.profile_run CASE [--nr 256 --nt 2048]

Everything a case needs is set up outside the range (context, material,
assembly or a first solve), so an ncu filter such as

    ncu --nvtx --nvtx-include "target/" --kernel-name-base demangled \\
        -k regex:'k_cheb_step<float>' -c 1 --clock-control none ... \\
        python -m dimspers_b200.profile_run vcycle

captures the first launch of one kernel in the range.  The Stokes cases run on
the fabric workload, by default at 256x2048 (1,048,576 elements: 327 MB of
FP32 / 654 MB of FP64 element blocks, beyond the 126 MB L2, about 3 GB on the
device):

  apply32  one fine-level FP32 element-by-element A-apply
  apply64  one fine-level FP64 A-apply
  vcycle   one FP32 multigrid V-cycle from the fine level (after a solve built
           the hierarchy): Chebyshev steps, restriction, prolongation, dense
           coarsest, the coarse-level applies
  solve32  assembly (FP32 blocks) and one host-driven fast solve of 2 outer
           iterations: Galerkin levels, Gauss-Jordan coarse inverse, the
           FP64 Krylov kernels, G and G^T, the compensated Schur kernels
  solve64  the same in FP64 with the lumped Schur preconditioner
  det      solve32 in deterministic mode: the element-result kernels of the
           applies, right-hand side and diagonal blocks, the per-node gathers,
           the sequential dense coarse assembly
  inner    the graph solve's inner-iteration vector kernels (launched outside
           the graph: ncu cannot look inside conditional graph nodes)
  post     stress post-processor, viscosity update, FSE, DEM tensor lookup,
           thermal step
  cnn      the guess network at 32 channels on the 128x1024 grid (65 x 512),
           batch 8: forward, one training step (backward, Adam)
"""
import sys

import numpy as np


def _range(name):
    import torch
    return torch.cuda.nvtx.range(name)


SIZE = [256, 2048]


def _stokes(precision):
    from . import StokesContext, inputs
    nr, nt = SIZE
    ctx = StokesContext(nr, nt, "discontinuous", pin_rotation=True)
    mat = inputs.make_material(ctx.mesh, "fabric", seed=1)
    ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
    arm = (dict(precision=1, schur_pc=1) if precision == 1 else dict(precision=0, schur_pc=0))
    return ctx, arm


def solve(precision, deterministic=False):
    import torch
    ctx, arm = _stokes(precision)
    if deterministic:
        ctx.set_deterministic(True)
    torch.cuda.synchronize()
    with _range("target"):
        ctx.assemble(arm["precision"])
        ctx.solve(itmax=2, itmin=1, rtol=1e-30, inner_itmax=8, host_loop=1, raise_on_status=False, want_cart=False,
                  **arm)
        torch.cuda.synchronize()
    ctx.close()


def apply(which):
    import torch
    ctx, arm = _stokes(1)
    ctx.assemble(1 if which == 0 else 0)
    torch.cuda.synchronize()
    with _range("target"):
        ctx.profile_kernel(which, reps=1)
        torch.cuda.synchronize()
    ctx.close()


def vcycle():
    import torch
    ctx, arm = _stokes(1)
    ctx.assemble(1)
    ctx.solve(itmax=1, itmin=1, rtol=1e-30, inner_itmax=1, host_loop=1, raise_on_status=False, want_cart=False, **arm)
    torch.cuda.synchronize()
    with _range("target"):
        ctx.profile_kernel(2, reps=1)
        torch.cuda.synchronize()
    ctx.close()


def inner():
    import torch
    ctx, arm = _stokes(1)
    ctx.assemble(1)
    torch.cuda.synchronize()
    with _range("target"):
        ctx.profile_kernel(7, reps=1)
        torch.cuda.synchronize()
    ctx.close()


def post():
    import torch
    from . import StokesContext, inputs
    from . import kernel_times as KT
    from .fabric import DEM
    nr, nt = SIZE
    c = StokesContext(nr, nt, "discontinuous")
    m = inputs.make_material(c.mesh, "aniso", seed=1)
    rng = np.random.default_rng(0)
    U = rng.standard_normal(2 * c.nnod)
    T, P, r, eps, tau, coh = KT.inputs_viscosity(c.mesh, nr, nt, rng)
    eta0 = np.full((c.nel, 7), 3.3e21)
    F = np.eye(2) + 0.3 * rng.standard_normal((c.nel, 6, 2, 2))
    d = np.load(KT.DEM_FIXTURE)
    dem = DEM(d["C"], d["ax"], 0.02)
    x1, y1, r1, r2 = KT.inputs_dem(c.nel, rng)
    ct = StokesContext(nr, nt, "continuous")
    Tt, rho, dt = KT.inputs_thermal(ct.mesh, nr, np.random.default_rng(0))
    torch.cuda.synchronize()
    with _range("target"):
        c.stress(U, m.eta_ip, m.C6)
        c.viscosity_arrhenius(eta0, T, P, r, eps, tau, coh, phi=30.0)
        c.fse(F)
        c.anisotropic_tensor(dem, x1, y1, r1, r2)
        ct.thermal_step(Tt, rho, dt)
        ct.profile_kernel(6, reps=1)     # the thermal apply outside the step's graph
        torch.cuda.synchronize()
    c.close()
    ct.close()


def cnn():
    import torch
    from . import learned
    nrg, ntg = learned.grid_shape(128, 1024)
    net = learned.GuessNet(nrg, ntg, 32, 6, (1, 2, 4, 8, 16, 1), max_batch=8)
    net.init_params(seed=0)
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.randn((8, 4, nrg, ntg), generator=g, device=dev)
    t = torch.randn((8, 1, nrg, ntg), generator=g, device=dev)
    y = torch.empty_like(t)
    torch.cuda.synchronize()
    with _range("target"):
        net.forward(x, y)
        net.train_step(x, t, 1e-3)
        torch.cuda.synchronize()
    net.close()


CASES = {"apply32": lambda: apply(0), "apply64": lambda: apply(1), "vcycle": vcycle, "solve32": lambda: solve(1),
         "solve64": lambda: solve(0), "det": lambda: solve(1, True), "inner": inner, "post": post, "cnn": cnn}

if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--nr", type=int, default=256)
    ap.add_argument("--nt", type=int, default=2048)
    a = ap.parse_args()
    SIZE[:] = [a.nr, a.nt]
    CASES[a.case]()
