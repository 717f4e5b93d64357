"""The learned-guess network's hand-written CUDA kernels against a torch-CPU
reference of the same network (forward, loss and every parameter gradient),
a training smoke test, and the solver's guess selection / fallback."""
import numpy as np
import pytest

from conftest import rel
from dimspers_b200 import StokesContext, build_mesh, inputs, learned

pytestmark = pytest.mark.gpu


def torch_reference(params, x, t, nrg, ntg, channels, layers, dil):
    import torch
    import torch.nn.functional as F
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    h = torch.tensor(x, dtype=torch.float64)
    off = 0
    for l in range(layers):
        cin = 4 if l == 0 else channels
        cout = 1 if l == layers - 1 else channels
        W = p[off:off + cout * cin * 9].view(cout, cin, 3, 3)
        off += cout * cin * 9
        b = p[off:off + cout]
        off += cout
        d = dil[l]
        hp = F.pad(h, (d, d, 0, 0), mode="circular")        # periodic in theta (last dim)
        hp = F.pad(hp, (0, 0, d, d))                        # zero in r
        h = F.conv2d(hp, W, b, dilation=d)
        if l < layers - 1:
            h = torch.relu(h)
    loss = ((h - torch.tensor(t, dtype=torch.float64)) ** 2).mean()
    loss.backward()
    return h.detach().numpy(), float(loss), p.grad.numpy()


def test_network_gradients_match_torch_cpu():
    import torch
    nrg, ntg, C, L, dil = 6, 16, 8, 4, (1, 2, 3, 1)
    net = learned.GuessNet(nrg, ntg, C, L, dil, max_batch=2)
    net.set_math(bf16=False)           # the FP32 CUDA-core path against FP64 torch
    net.init_params(seed=3)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 4, nrg, ntg)).astype(np.float32)
    t = rng.standard_normal((2, 1, nrg, ntg)).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    yd = torch.empty((2, 1, nrg, ntg), dtype=torch.float32, device="cuda")
    net.forward(xd, yd)
    loss = net.gradients(xd, td)
    params, grads = net.get_params(grads=True)
    y_ref, loss_ref, g_ref = torch_reference(params, x, t, nrg, ntg, C, L, dil)
    assert rel(yd.cpu().numpy(), y_ref) < 1e-5
    assert abs(loss - loss_ref) < 1e-5 * abs(loss_ref)
    assert rel(grads, g_ref) < 1e-4
    net.close()


def _bf16(a):
    import torch
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float64)


def torch_forward_bf16(params, x, channels, layers, dil):
    """The same network with every convolution operand rounded to BF16 (the
    weights, and each layer's input activations) and exact accumulation: what
    the tensor-core path computes, up to its FP32 accumulation order."""
    import torch
    import torch.nn.functional as F
    p = torch.tensor(params, dtype=torch.float64)
    h = torch.tensor(x, dtype=torch.float64)
    off = 0
    for l in range(layers):
        cin = 4 if l == 0 else channels
        cout = 1 if l == layers - 1 else channels
        W = _bf16(p[off:off + cout * cin * 9].view(cout, cin, 3, 3).numpy())
        off += cout * cin * 9
        b = p[off:off + cout]
        off += cout
        d = dil[l]
        hp = F.pad(_bf16(h.numpy()), (d, d, 0, 0), mode="circular")
        hp = F.pad(hp, (0, 0, d, d))
        h = F.conv2d(hp, W, b, dilation=d)
        h = h.to(torch.float32).to(torch.float64)          # FP32 activations between layers
        if l < layers - 1:
            h = torch.relu(h)
    return h.numpy()


@pytest.mark.parametrize("channels", [16, 32])
def test_tensor_core_forward_matches_bf16_reference(channels):
    """BF16 operands, FP32 accumulation (mma.sync m16n8k16).  Two layers, so
    that the only difference from the BF16-rounded reference is the FP32
    accumulation order (plus, rarely, a 1-ulp BF16 re-rounding of an
    activation): a fragment-layout error would show as O(1) differences.  A
    6-layer network then stays within BF16 rounding of the FP32 network."""
    import torch
    nrg, ntg = 9, 48
    rng = np.random.default_rng(2)
    x = rng.standard_normal((2, 4, nrg, ntg)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    for L, dil, bound in ((2, (1, 3), 5e-4), (6, (1, 2, 4, 8, 3, 1), None)):
        net = learned.GuessNet(nrg, ntg, channels, L, dil, max_batch=2)
        net.init_params(seed=5)
        y_tc = torch.empty((2, 1, nrg, ntg), dtype=torch.float32, device="cuda")
        y_32 = torch.empty_like(y_tc)
        net.forward(xd, y_tc)
        net.set_math(bf16=False)
        net.forward(xd, y_32)
        ref = torch_forward_bf16(net.get_params(), x, channels, L, dil)
        a, b = y_tc.cpu().numpy(), y_32.cpu().numpy()
        print(f"C={channels} L={L}: tc vs bf16 reference {rel(a, ref):.2e}, tc vs fp32 {rel(a, b):.2e}")
        if bound is not None:
            assert rel(a, ref) < bound, rel(a, ref)
        assert 1e-5 < rel(a, b) < 5e-2, rel(a, b)
        net.close()


def test_tensor_core_gradients_close_to_fp32():
    """Training gradients with the tensor-core forward and data gradient stay
    within BF16 rounding of the FP32 path's."""
    import torch
    nrg, ntg, C, L, dil = 9, 32, 32, 6, (1, 2, 4, 8, 3, 1)
    net = learned.GuessNet(nrg, ntg, C, L, dil, max_batch=2)
    net.init_params(seed=4)
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.standard_normal((2, 4, nrg, ntg)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((2, 1, nrg, ntg)).astype(np.float32)).cuda()
    loss_tc = net.gradients(x, t)
    g_tc = net.get_params(grads=True)[1]
    net.set_math(bf16=False)
    loss_32 = net.gradients(x, t)
    g_32 = net.get_params(grads=True)[1]
    assert abs(loss_tc - loss_32) < 2e-2 * abs(loss_32)
    assert rel(g_tc, g_32) < 5e-2, rel(g_tc, g_32)
    net.close()


def test_network_trains():
    import torch
    nrg, ntg = 9, 32
    net = learned.GuessNet(nrg, ntg, 8, 4, (1, 2, 1, 1), max_batch=4)
    net.init_params(seed=1)
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.standard_normal((4, 4, nrg, ntg)).astype(np.float32)).cuda()
    t = (0.5 * x[:, :1] - 0.25 * x[:, 1:2]).contiguous()
    first = net.train_step(x, t, 1e-2)
    for _ in range(300):
        last = net.train_step(x, t, 3e-3)
    assert last < 0.2 * first
    net.close()


def test_solver_keeps_a_good_guess_and_rejects_a_bad_one():
    mesh = build_mesh(8, 64, "discontinuous")
    mat = inputs.make_material(mesh, "aniso", seed=5)
    with StokesContext(8, 64, "discontinuous") as ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(1)
        opts = dict(precision=1, rtol=1e-8, itmax=5000)
        U0, P0, _, r0 = ctx.solve(**opts)
        Ptight = ctx.solve(precision=1, rtol=1e-11, itmax=5000)[1]
        # near-exact guess: kept, far fewer iterations, same answer
        _, P1, _, r1 = ctx.solve(P0=Ptight * (1 + 1e-3), use_guess=2, **opts)
        assert r1["fallback_used"] == 0 and r1["iterations"] < r0["iterations"] // 2
        assert abs(r1["r0"] - r0["r0"]) < 1e-9 * r0["r0"]           # tolerance from the zero guess
        assert rel(P1, P0) < 1e-4
        # garbage guess: rejected, identical to the zero-guess solve
        bad = np.random.default_rng(0).standard_normal(ctx.npres) * 1e3 * np.abs(Ptight).max()
        _, P2, _, r2 = ctx.solve(P0=bad, use_guess=2, **opts)
        assert r2["fallback_used"] == 1 and r2["r0_guess"] > r2["r0"]
        # the zero-guess solve again; float atomics reorder sums, so the counts
        # may differ by a few iterations on this ill-conditioned case
        assert abs(r2["iterations"] - r0["iterations"]) <= max(3, r0["iterations"] // 50)
        assert rel(P2, P0) < 1e-5


def test_trained_network_gain_on_held_out_workloads():
    """The committed 128x1024 network (trained by dimspers_b200.train_guess on
    plume/aniso solves with seeds from 1000) on 8 held-out plume workloads with
    seeds it never saw: the fast solve to rtol 1e-8 from the learned guess
    (with the zero-guess fallback) against the same solve from the zero guess.
    What it gains: the initial Schur residual falls by more than 10x on every
    case, and the outer iterations do not grow on average (the slow modes of
    the P2-P1disc Schur complement, which set the count, are element-scale
    pressure modes that a coarse prolongated guess does not resolve)."""
    import os
    path = learned.weights_path(128, 1024)
    if not os.path.exists(path):
        pytest.skip("no trained network")
    mesh = build_mesh(128, 1024, "discontinuous")
    net = learned.GuessNet.load(path, max_batch=1)
    opts = dict(precision=1, schur_pc=1, inner_relax=1e-2, relax_base=1e-8, rtol=1e-8, itmax=20000)
    rows = []
    with StokesContext(128, 1024, "discontinuous") as ctx:
        guess = learned.LearnedGuess(net, ctx)
        for seed in range(5000, 5008):
            mat = inputs.make_material(mesh, "plumes", seed=seed)
            ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
            ctx.assemble(1)
            _, Pz, _, rz = ctx.solve(use_guess=0, want_cart=False, **opts)
            P0 = np.zeros(ctx.npres)
            guess.predict(mat.g, P0.ctypes.data, mem=0)
            _, Pg, _, rg = ctx.solve(P0=P0, use_guess=2, want_cart=False, **opts)
            assert rz["status"] == 0 and rg["status"] == 0
            rows.append((rz["iterations"], rg["iterations"], rg["r0_guess"] / rg["r0"], rg["fallback_used"]))
            print(f"seed {seed}: outer zero {rz['iterations']} guess {rg['iterations']} "
                  f"r0 ratio {rg['r0_guess'] / rg['r0']:.3f} fallback {rg['fallback_used']}")
    zero = np.mean([r[0] for r in rows])
    gss = np.mean([r[1] for r in rows])
    print(f"mean outer: zero {zero:.0f}, guess {gss:.0f} ({gss / zero:.3f})")
    assert all(r[2] < 0.1 and r[3] == 0 for r in rows), rows
    assert gss <= 1.02 * zero, (gss, zero)
    net.close()


def test_guess_pipeline_shapes():
    """features -> network -> prolongation produce finite pressure DOFs."""
    import torch
    mesh = build_mesh(8, 64, "discontinuous")
    mat = inputs.make_material(mesh, "plumes", seed=9)
    nrg, ntg = learned.grid_shape(8, 64)
    net = learned.GuessNet(nrg, ntg, 8, 3, (1, 2, 1), max_batch=1)
    net.init_params(seed=0)
    with StokesContext(8, 64, "discontinuous") as ctx:
        ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
        X = torch.empty((1, 4, nrg, ntg), dtype=torch.float32, device="cuda")
        learned.features(ctx, X)
        Xh = X.cpu().numpy()
        assert np.allclose(Xh[0, 0], mat.rho[np.array([[mesh_vertex(ctx, 2 * i, 2 * j) for j in range(ntg)]
                                                       for i in range(nrg)])], atol=1e-6)
        g = learned.LearnedGuess(net, ctx)
        P0 = np.zeros(ctx.npres)
        g.predict(mat.g, P0.ctypes.data, mem=0)
        assert np.all(np.isfinite(P0)) and np.abs(P0).max() > 0
    net.close()


def mesh_vertex(ctx, ir, it):
    """reference node number of the vertex (ir, it): ir + (ncr + 1) * it"""
    return ir + (ctx.desc.nr_cells + 1) * it
