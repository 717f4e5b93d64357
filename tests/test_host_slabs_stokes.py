"""The Schur-complement Stokes solve sharded over θ-slabs on gloo ranks (no
GPU): each rank holds only its elements' rotated (polar) blocks and its
elements' discontinuous pressure DOFs; the velocity applies are completed by
the neighbour exchange, the reductions by all-reduces.  The result equals
the oracle's StokesPcCG with a direct inner solve, for the discontinuous
pressure (element-local DOFs) and the continuous one (vertex DOFs shared
across slabs like the velocity)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NCR, NCT = 2, 16
RTOL = 1e-10


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(pressure="discontinuous"):
    """Oracle solution and the polar element blocks, in lattice numbering."""
    sys.path.insert(0, ROOT)
    from dimspers_b200.slabs import lattice_element_nodes
    from oracle import assembly as OA
    from oracle import solver as OS
    prob = OS.make_problem(NCR, NCT, pressure, pin_rotation=True)
    gr = prob.gr
    nel = gr.e2n.shape[1]
    A, B = 2 * NCR + 1, 2 * NCT
    lat = lattice_element_nodes(np.arange(nel), NCR, A, B)
    ref2lat = np.full(gr.nnod, -1)
    ref2lat[gr.e2n.T.ravel()] = lat.ravel()
    rng = np.random.default_rng(3)
    eta = 1.0 + 0.5 * rng.random((nel, 7))
    rho = 1.0 + 0.3 * np.cos(3 * gr.theta) * np.sin(np.pi * (gr.r - 1.22))
    g = 10.0
    # the reference solve: assembly, rotation, free slip + pin, StokesPcCG with LU
    Agl = OS.assemble(prob, eta, rho, g)
    U, P, rep = OS.stokes_pcg(Agl["KK"], Agl["MM"], Agl["GG"], Agl["F"], prob.ifree, rtol=RTOL, itmax=5000)
    U_lat = np.zeros(2 * A * B)
    U_lat[(2 * ref2lat[:, None] + np.arange(2)).ravel()] = U
    # element blocks rotated to the polar DOFs with the per-node blocks of TT
    Kp, Ge, Me, Fb = OA.element_matrices(prob.th, prob.r, eta, rho, gr.e2n, g)
    Ke = OA.unpack_sym(Kp, 12, OA.PACK12)                              # (nel, 12, 12) Cartesian
    th = gr.theta[gr.e2n.T]                                            # (nel, 6) node angles
    Te = np.zeros((nel, 12, 12))
    c, s = np.cos(th), np.sin(th)
    for k in range(6):
        Te[:, 2 * k, 2 * k], Te[:, 2 * k, 2 * k + 1] = c[:, k], s[:, k]
        Te[:, 2 * k + 1, 2 * k], Te[:, 2 * k + 1, 2 * k + 1] = -s[:, k], c[:, k]
    Tt = Te.transpose(0, 2, 1)
    Kpol = Tt @ Ke @ Te
    Gpol = Tt @ Ge.T.reshape(nel, 3, 12).transpose(0, 2, 1)           # (nel, 12, 3)
    Fpol = np.einsum("eij,ej->ei", Tt, Fb.T)
    M3 = OA.unpack_sym(Me, 3, OA.PACK3)                                 # (nel, 3, 3)
    pc = 1.0 / M3.sum(axis=2)                                           # lumped mass, element-local
    P_el = P[prob.e2nP.T]                                               # (nel, 3) in element order
    P_lat = np.zeros(A * B)                                             # continuous: on the vertex nodes
    P_lat[lat[:, :3].ravel()] = P_el.ravel()
    return dict(U_lat=U_lat, P_el=P_el, P_lat=P_lat, Kpol=Kpol, Gpol=Gpol, Fpol=Fpol, M3=M3, pc=pc, nel=nel,
                iterations=rep.iterations, pressure=pressure)


def _solve_rank(part, d):
    from dimspers_b200.slabs import ElementPressure, VertexPressure, distributed_stokes_pcg
    el = part.elements
    ln = part.local_element_nodes()
    dofs = torch.as_tensor((ln[:, :, None] * 2 + np.arange(2)).reshape(len(ln), 12))
    K = torch.as_tensor(d["Kpol"][el])
    G = torch.as_tensor(d["Gpol"][el])
    n_u = 2 * part.nloc

    def scatter(v):                                                      # (nel_l, 12) -> partial velocity
        y = torch.zeros(n_u, dtype=torch.float64)
        y.index_add_(0, dofs.reshape(-1), v.reshape(-1))
        return y

    apply_K = lambda u: scatter(torch.einsum("eij,ej->ei", K, u[dofs]))          # noqa: E731
    if d["pressure"] == "discontinuous":
        pspace = ElementPressure(part, 3 * d["nel"])
        apply_G = lambda p: scatter(torch.einsum("eij,ej->ei", G, p.reshape(-1, 3)))  # noqa: E731
        apply_GT = lambda u: torch.einsum("eji,ej->ei", G, u[dofs]).reshape(-1)      # noqa: E731
        pc = torch.as_tensor(d["pc"][el].reshape(-1))
    else:
        pspace = VertexPressure(part)
        v3 = torch.as_tensor(ln[:, :3])

        def apply_G(p):
            return scatter(torch.einsum("eij,ej->ei", G, p[v3]))

        def apply_GT(u):
            y = torch.zeros(part.nloc, dtype=torch.float64)
            y.index_add_(0, v3.reshape(-1), torch.einsum("eji,ej->ei", G, u[dofs]).reshape(-1))
            return y
        rows = torch.zeros(part.nloc, dtype=torch.float64)              # lumped mass: assembled row sums
        rows.index_add_(0, v3.reshape(-1), torch.as_tensor(d["M3"][el].sum(axis=2)).reshape(-1))
        rows = part.exchange_add(rows, 1)
        pc = torch.where(pspace.mask, 1.0 / torch.where(pspace.mask, rows, torch.ones_like(rows)),
                         torch.zeros_like(rows))
    rhs = part.exchange_add(scatter(torch.as_tensor(d["Fpol"][el])), 2)
    diag = part.exchange_add(scatter(torch.diagonal(K, dim1=1, dim2=2).contiguous()), 2)
    gn = part.global_nodes()
    a, b = gn % part.A, gn // part.A
    free = np.ones((part.nloc, 2), dtype=bool)
    free[(a == 0) | (a == 2 * NCR), 1] = False                          # free slip: u_r on both walls
    free[(a == 2 * NCR) & (b == 0), 0] = False                          # the pinned u_theta
    U, P, it, rel = distributed_stokes_pcg(part, apply_K, diag, free.ravel(), apply_G, apply_GT,
                                           lambda r: r * pc, rhs, pspace, rtol=RTOL, itmax=5000,
                                           inner_rtol=1e-12)
    u_ref = d["U_lat"].reshape(-1, 2)[gn].ravel()
    p_ref = d["P_el"][el].ravel() if d["pressure"] == "discontinuous" else d["P_lat"][gn]
    return dict(eu=float(np.abs(U.numpy() - u_ref).max() / np.abs(d["U_lat"]).max()),
                ep=float(np.abs(P.numpy() - p_ref).max() / np.abs(d["P_el"]).max()),
                it=it, rel=rel)


def _rank(rank, world, port, q, pressure):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from dimspers_b200.slabs import SlabPartition
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = _problem(pressure)
        q.put((rank, _solve_rank(SlabPartition(NCR, NCT, world, rank), d), d["iterations"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("pressure", ["discontinuous", "continuous"])
def test_sharded_stokes_single_slab(pressure):
    sys.path.insert(0, ROOT)
    from dimspers_b200.slabs import SlabPartition
    d = _problem(pressure)
    res = _solve_rank(SlabPartition(NCR, NCT, 1, 0), d)
    assert res["eu"] < 1e-6 and res["ep"] < 1e-6, res
    assert abs(res["it"] - d["iterations"]) <= max(2, d["iterations"] // 20), (res, d["iterations"])


@pytest.mark.parametrize("world,pressure", [(2, "discontinuous"), (3, "continuous")])
def test_sharded_stokes_on_gloo_ranks(world, pressure):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, pressure)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    its = {v["it"] for _, v, _ in got}
    assert len(its) == 1                                                   # every rank took the same steps
    for r, v, it_ref in got:
        assert v["eu"] < 1e-6 and v["ep"] < 1e-6, (r, v)
        assert abs(v["it"] - it_ref) <= max(2, it_ref // 20), (v, it_ref)
