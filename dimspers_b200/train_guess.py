"""Train and evaluate the learned initial guess on the GPU.

  python -m dimspers_b200.train_guess --nr 128 --nt 1024 --train 512 --test 64

1. Training data: solves of seeded workloads (3/4 `plumes`, 1/4 `aniso`) with
   the GPU solver (FP32 multigrid / FP64 Krylov, element-block mass Schur
   preconditioner, no guess) to --data-rtol (default 1e-8, the benchmark's
   tolerance); inputs from dp_cnn_inputs, target P/g on the half-resolution
   vertex grid.
2. Training with the library's forward/backward/Adam kernels (dp_cnn_*): BF16
   tensor-core convolutions with FP32 accumulation and FP32 master weights
   (--fp32 for the CUDA-core FP32 path).
3. A/B on the held-out solves at rtol 1e-8: zero guess (use_guess = 0) versus
   learned guess with fallback (use_guess = 2, same absolute stopping target).
Writes the weights (npz) and an evaluation summary (json) next to them.
"""
import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nr", type=int, default=128)
    ap.add_argument("--nt", type=int, default=1024)
    ap.add_argument("--train", type=int, default=512)
    ap.add_argument("--test", type=int, default=64)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--channels", type=int, default=32)
    ap.add_argument("--data-rtol", type=float, default=1e-8)
    ap.add_argument("--fp32", action="store_true", help="FP32 CUDA-core convolutions instead of BF16 tensor cores")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    import torch

    from . import inputs, learned
    from .stokes import StokesContext, build_mesh

    dev = torch.device("cuda", 0)
    mesh = build_mesh(args.nr, args.nt, "discontinuous")
    nrg, ntg = learned.grid_shape(args.nr, args.nt)
    ctx = StokesContext(args.nr, args.nt, "discontinuous")
    # the benchmark's fast arm (relaxation base = the outer target)
    solve_opts = dict(precision=1, schur_pc=1, inner_relax=1e-2, relax_base=1e-8, itmax=20000, raise_on_status=False)
    n = args.train + args.test
    X = torch.empty((n, 4, nrg, ntg), dtype=torch.float32, device=dev)
    Y = torch.empty((n, 1, nrg, ntg), dtype=torch.float32, device=dev)
    mats = []
    t0 = time.time()
    for s in range(n):
        kind = "aniso" if s % 4 == 0 else "plumes"
        mat = inputs.make_material(mesh, kind, seed=1000 + s)
        mats.append(mat if s >= args.train else None)   # only the held-out materials are needed again
        ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
        ctx.assemble(1)
        U, P, _, rep = ctx.solve(rtol=args.data_rtol, want_cart=False, **solve_opts)
        learned.features(ctx, X[s:s + 1])
        Y[s, 0] = torch.from_numpy(learned.vertex_target(mesh, P, mat.g)).to(dev)
    t_data = time.time() - t0
    print(f"data: {n} solves in {t_data:.1f} s", flush=True)

    net = learned.GuessNet(nrg, ntg, args.channels, 6, (1, 2, 4, 8, 16, 1), max_batch=args.batch)
    net.set_math(bf16=not args.fp32)
    net.init_params(seed=0)
    tr = slice(0, args.train)
    xm = X[tr].mean(dim=(0, 2, 3))
    xs = X[tr].std(dim=(0, 2, 3)).clamp_min(1e-6)
    ym, ys = float(Y[tr].mean()), float(Y[tr].std())
    net.x_mean, net.x_std = xm.cpu().numpy(), xs.cpu().numpy()
    net.y_mean, net.y_std = ym, ys
    Xn = ((X - xm.view(1, 4, 1, 1)) / xs.view(1, 4, 1, 1)).contiguous()
    Yn = ((Y - ym) / ys).contiguous()
    rng = np.random.default_rng(0)
    t0 = time.time()
    losses = []
    for it in range(args.steps):
        idx = torch.from_numpy(rng.choice(args.train, args.batch, replace=False)).to(dev)
        xb = Xn.index_select(0, idx).contiguous()
        yb = Yn.index_select(0, idx).contiguous()
        lr = args.lr * 0.5 * (1 + np.cos(np.pi * it / args.steps))
        losses.append(net.train_step(xb, yb, lr))
        if it % 250 == 0 or it == args.steps - 1:
            print(f"step {it} loss {np.mean(losses[-50:]):.4e}", flush=True)
    t_train = time.time() - t0

    # held-out: prediction error and the A/B solve comparison at rtol 1e-8
    y = torch.empty((1, 1, nrg, ntg), dtype=torch.float32, device=dev)
    rel_err, rows = [], []
    guess = learned.LearnedGuess(net, ctx)
    for s in range(args.train, n):
        net.forward(Xn[s:s + 1].contiguous(), y)
        pred = y * ys + ym
        rel_err.append(float(torch.linalg.norm(pred - Y[s:s + 1]) / torch.linalg.norm(Y[s:s + 1])))
        mat = mats[s]
        ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
        ctx.assemble(1)
        ta = time.time()
        _, _, _, r0 = ctx.solve(rtol=1e-8, use_guess=0, want_cart=False, **solve_opts)
        ta = time.time() - ta
        P0 = np.zeros(ctx.npres)
        tb = time.time()
        guess.predict(mat.g, P0.ctypes.data, mem=0)
        _, _, _, r1 = ctx.solve(rtol=1e-8, P0=P0, use_guess=2, want_cart=False, **solve_opts)
        tb = time.time() - tb
        rows.append(dict(seed=1000 + s, zero_outer=r0["iterations"], guess_outer=r1["iterations"],
                         zero_s=ta, guess_s=tb, fallback=r1["fallback_used"], r0=r1["r0"], r0_guess=r1["r0_guess"],
                         status=(r0["status"], r1["status"])))
        print(json.dumps(rows[-1]), flush=True)
    zo = np.array([r["zero_outer"] for r in rows], float)
    go = np.array([r["guess_outer"] for r in rows], float)
    zs = np.array([r["zero_s"] for r in rows])
    gs = np.array([r["guess_s"] for r in rows])
    summary = dict(nr_cells=args.nr, ntheta_cells=args.nt, train=args.train, test=args.test, steps=args.steps,
                   batch=args.batch, channels=args.channels, math="fp32" if args.fp32 else "bf16 tensor cores",
                   data_rtol=args.data_rtol, data_seconds=t_data,
                   train_seconds=t_train, final_loss=float(np.mean(losses[-50:])),
                   heldout_rel_l2_pressure=float(np.mean(rel_err)),
                   mean_outer_zero=float(zo.mean()), mean_outer_guess=float(go.mean()),
                   outer_ratio=float(go.mean() / zo.mean()), mean_seconds_zero=float(zs.mean()),
                   mean_seconds_guess=float(gs.mean()), time_ratio=float(gs.mean() / zs.mean()),
                   fallbacks=int(sum(r["fallback"] for r in rows)),
                   mean_r0_guess_over_r0=float(np.mean([r["r0_guess"] / r["r0"] for r in rows])))
    print(json.dumps(summary), flush=True)
    out = args.out or learned.weights_path(args.nr, args.nt)
    net.save(out, extra=dict(eval=summary))
    with open(out.replace(".npz", "_eval.json"), "w") as f:
        json.dump(dict(summary=summary, heldout=rows), f, indent=1)
    ctx.close()


if __name__ == "__main__":
    main()
