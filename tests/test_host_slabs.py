"""θ-slab partition of the multi-rank path on gloo ranks (no GPU): the
element-by-element applies of the thermal (scalar) and Stokes velocity
(2 components) operators, completed by the neighbour exchange, equal the
global assembled operator on every rank's nodes, and the distributed
Jacobi-PCG reaches the global direct solve."""
import os
import socket
import sys

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NCR, NCT = 4, 32


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    """Element blocks in the reference element order and the lattice node
    numbering: thermal (nel, 6, 6) and Stokes velocity (nel, 12, 12)."""
    sys.path.insert(0, ROOT)
    from dimspers_b200.slabs import lattice_element_nodes
    from oracle import assembly as OA
    from oracle import solver as OS
    from oracle import thermal as OT
    prob = OS.make_problem(NCR, NCT, "continuous")
    gr = prob.gr
    nel = gr.e2n.shape[1]
    A, B = 2 * NCR + 1, 2 * NCT
    lat = lattice_element_nodes(np.arange(nel), NCR, A, B)          # (nel, 6)
    ref2lat = np.full(gr.nnod, -1)
    ref2lat[gr.e2n.T.ravel()] = lat.ravel()
    assert np.all(ref2lat >= 0) and np.array_equal(ref2lat[gr.e2n.T], lat)   # same element and local order
    rng = np.random.default_rng(5)
    Ke, Me = OT.element_matrices(prob.th, prob.r, 1.0 + 0.1 * rng.random(gr.nnod), gr.e2n, 2.0, 3.0)
    At = Me + 0.05 * Ke
    eta = np.exp(rng.standard_normal((nel, 7)))
    Kp = OA.element_matrices(prob.th, prob.r, eta, np.ones(gr.nnod), gr.e2n, 1.0)[0]
    Ks = OA.unpack_sym(Kp, 12, OA.PACK12)                             # (nel, 12, 12)
    return lat, At, Ks, A * B


def _global(lat, Ae, ncomp, n):
    dofs = (lat[:, :, None] * ncomp + np.arange(ncomp)).reshape(len(lat), -1)
    rows = np.repeat(dofs, dofs.shape[1], axis=1).ravel()
    cols = np.tile(dofs, (1, dofs.shape[1])).ravel()
    return sp.csr_matrix((Ae.reshape(len(Ae), -1).ravel(), (rows, cols)), shape=(n * ncomp, n * ncomp))


def _local_apply(part, Ae, ncomp):
    ln = part.local_element_nodes()
    dofs = torch.as_tensor((ln[:, :, None] * ncomp + np.arange(ncomp)).reshape(len(ln), -1))
    blocks = torch.as_tensor(Ae[part.elements])

    def apply(x):
        y = torch.zeros_like(x)
        y.index_add_(0, dofs.reshape(-1), torch.einsum("eij,ej->ei", blocks, x[dofs]).reshape(-1))
        return y
    return apply


def _check_rank(part, lat, At, Ks, n):
    from dimspers_b200.slabs import distributed_pcg
    rng = np.random.default_rng(17)
    out = {}
    gl = part.global_nodes()
    for name, Ae, nc in (("thermal", At, 1), ("stokes", Ks, 2)):
        G = _global(lat, Ae, nc, n)
        x = rng.standard_normal(n * nc)                          # same on every rank (same seed)
        y = G @ x
        xl = torch.as_tensor(x.reshape(n, nc)[gl].ravel())
        yl = part.exchange_add(_local_apply(part, Ae, nc)(xl), nc).numpy()
        out[name] = np.abs(yl - y.reshape(n, nc)[gl].ravel()).max() / np.abs(y).max()
    # distributed PCG on the thermal operator with both walls fixed
    G = _global(lat, At, 1, n)
    a = np.arange(n) % (2 * NCR + 1)
    free = (a != 0) & (a != 2 * NCR)
    bg = G @ rng.standard_normal(n)
    xg = np.zeros(n)
    xg[free] = spla.spsolve(G[free][:, free].tocsc(), bg[free])
    x, it, rn = distributed_pcg(part, _local_apply(part, At, 1), torch.as_tensor(bg[gl]),
                                torch.as_tensor(G.diagonal()[gl]), free[gl], 1e-13, 0.0, 2000)
    out["pcg"] = np.abs(x.numpy() - xg[gl]).max() / np.abs(xg).max()
    out["it"] = it
    return out


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from dimspers_b200.slabs import SlabPartition
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lat, At, Ks, n = _problem()
        q.put((rank, _check_rank(SlabPartition(NCR, NCT, world, rank), lat, At, Ks, n)))
    finally:
        dist.destroy_process_group()


def test_partition_covers_the_ring():
    sys.path.insert(0, ROOT)
    from dimspers_b200.slabs import SlabPartition
    for world in (1, 2, 3, 5):
        parts = [SlabPartition(NCR, NCT, world, r) for r in range(world)]
        els = np.concatenate([p.elements for p in parts])
        assert np.array_equal(np.sort(els), np.arange(2 * NCR * NCT))
        owned = np.concatenate([p.global_nodes()[p.owned()] for p in parts])
        assert np.array_equal(np.sort(owned), np.arange((2 * NCR + 1) * 2 * NCT))   # each node counted once
        for p in parts:
            ln = p.local_element_nodes()
            assert ln.min() == 0 and ln.max() == p.nloc - 1
    with pytest.raises(ValueError):
        SlabPartition(NCR, 3, 4, 0)


def test_single_slab_is_the_whole_ring():
    sys.path.insert(0, ROOT)
    from dimspers_b200.slabs import SlabPartition
    res = _check_rank(SlabPartition(NCR, NCT, 1, 0), *_problem())
    assert res["thermal"] < 1e-13 and res["stokes"] < 1e-13 and res["pcg"] < 1e-9


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_on_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, v in res.items():
        assert v["thermal"] < 1e-13 and v["stokes"] < 1e-13, (r, v)
        assert v["pcg"] < 1e-9, (r, v)
    assert len({v["it"] for v in res.values()}) == 1              # every rank took the same steps
