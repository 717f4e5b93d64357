"""θ-slab partition of the annulus for the multi-rank path (host side).

The split-1 annulus of ncr × nct cells is cut into `world` slabs of whole cell
columns (θ ranges); rank k owns the cells of columns [c0, c1) and every
element in them.  A slab's P2 nodes form a local lattice of A = 2 ncr + 1
rows by 2 (c1 - c0) + 1 columns, numbered a + A b like the device lattice
(the global column is (2 c0 + b) mod 2 nct).  Its first and last node columns
are shared with the ring neighbours: after an element-by-element operator
apply each rank holds partial sums there, and `exchange_add` adds the
neighbour's partials so that both copies hold the full value.  Each shared
column is owned by the slab to its right (its column 0) for reductions, so
`dot` counts every node once.  Nothing else crosses ranks: one exchange of
2 · A · ncomp values per neighbour per apply and one all-reduce per dot.

This module is the rank logic only — partition, lattice maps, the exchange,
distributed reductions and a Jacobi-PCG written against them; the local
operator is a callable supplied by the caller (a device kernel on the slab's
elements, or any element-by-element apply).
"""
from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

_TAG_TO_LEFT, _TAG_TO_RIGHT = 11, 12


def lattice_element_nodes(e, ncr, A, B):
    """Lattice (a, b) -> a + A * (b mod B) of the 6 P2 nodes of elements e
    (element e = 2 (ir + ncr it) + t; t = 0: [v1, v2, v4], t = 1: [v2, v3, v4]
    with midpoints 12, 23, 31).  B = None leaves b unwrapped (slab lattices)."""
    e = np.asarray(e, dtype=np.int64)
    q, t = e >> 1, e & 1
    ir, it = q % ncr, q // ncr
    a0, b0 = 2 * ir, 2 * it
    da = np.array([[0, 0, 2, 0, 1, 1], [0, 2, 2, 1, 2, 1]])
    db = np.array([[0, 2, 0, 1, 1, 0], [2, 2, 0, 2, 1, 1]])
    a = a0[:, None] + da[t]
    b = b0[:, None] + db[t]
    if B is not None:
        b = b % B
    return a + A * b


@dataclass
class SlabPartition:
    ncr: int
    nct: int
    world: int
    rank: int

    def __post_init__(self):
        if self.world < 1 or not 0 <= self.rank < self.world:
            raise ValueError("rank must lie in [0, world)")
        if self.nct < self.world:
            raise ValueError("every slab needs at least one cell column (nct >= world)")
        base, extra = divmod(self.nct, self.world)
        self.c0 = self.rank * base + min(self.rank, extra)
        self.ncl = base + (1 if self.rank < extra else 0)
        self.c1 = self.c0 + self.ncl
        self.A = 2 * self.ncr + 1
        self.Bl = 2 * self.ncl + 1                   # local node columns
        self.nloc = self.A * self.Bl
        self.left = (self.rank - 1) % self.world
        self.right = (self.rank + 1) % self.world

    @property
    def elements(self):
        """Global ids of the slab's elements, ascending (its cell columns in order)."""
        cells = np.arange(self.c0 * self.ncr, self.c1 * self.ncr, dtype=np.int64)
        return np.stack([2 * cells, 2 * cells + 1], axis=1).ravel()

    def local_element_nodes(self):
        """(nel_local, 6) local lattice indices of the slab's elements."""
        e = self.elements - 2 * self.c0 * self.ncr      # renumber as if the slab started at column 0
        return lattice_element_nodes(e, self.ncr, self.A, None)

    def global_nodes(self):
        """Global lattice index of every local node (length nloc)."""
        a = np.tile(np.arange(self.A), self.Bl)
        b = (2 * self.c0 + np.repeat(np.arange(self.Bl), self.A)) % (2 * self.nct)
        return a + self.A * b

    def column(self, b):
        return np.arange(self.A) + self.A * b

    def owned(self):
        """Mask of the nodes this rank counts in reductions (all but its last column)."""
        m = np.ones(self.nloc, dtype=bool)
        m[self.column(self.Bl - 1)] = False
        return m

    # ---- communication ------------------------------------------------------
    def exchange_add(self, y, ncomp=1):
        """Completes an element-by-element sum on the shared columns, in place.
        y: local vector (nloc * ncomp, node-major), a torch tensor."""
        lc = _cols(self.column(0), ncomp)
        rc = _cols(self.column(self.Bl - 1), ncomp)
        mine_l, mine_r = y[lc].clone(), y[rc].clone()
        if self.world == 1:                            # the slab is the whole ring
            s = mine_l + mine_r
            y[lc] = s
            y[rc] = s
            return y
        from_l = torch.empty_like(mine_l)
        from_r = torch.empty_like(mine_r)
        ops = [dist.P2POp(dist.isend, mine_l, self.left, tag=_TAG_TO_LEFT),
               dist.P2POp(dist.isend, mine_r, self.right, tag=_TAG_TO_RIGHT),
               dist.P2POp(dist.irecv, from_l, self.left, tag=_TAG_TO_RIGHT),
               dist.P2POp(dist.irecv, from_r, self.right, tag=_TAG_TO_LEFT)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        y[lc] = mine_l + from_l
        y[rc] = mine_r + from_r
        return y

    def dot(self, x, y, ncomp=1):
        """Global x . y over owned nodes (one all-reduce)."""
        m = torch.as_tensor(np.repeat(self.owned(), ncomp), device=x.device)
        s = torch.sum(torch.where(m, x * y, torch.zeros_like(x))).reshape(1)
        if self.world > 1:
            dist.all_reduce(s)
        return s[0]


def _cols(nodes, ncomp):
    return (nodes[:, None] * ncomp + np.arange(ncomp)[None, :]).ravel()


def distributed_pcg(part, apply_local, b, diag, free, rtol, atol, itmax, ncomp=1):
    """Jacobi-PCG on the assembled operator whose element-by-element local
    part is apply_local (x_local -> partial y_local), over the free DOFs.
    b, diag: assembled (exchanged) local vectors; free: local bool mask.
    Stopping test ||r|| <= atol + rtol ||b||.  Returns (x, iterations, ||r||)."""
    fm = torch.as_tensor(free, device=b.device)
    zero = torch.zeros_like(b)
    r = torch.where(fm, b, zero)
    dinv = torch.where(fm, 1.0 / torch.where(fm, diag, torch.ones_like(diag)), zero)
    x = torch.zeros_like(b)
    z = r * dinv
    p = z.clone()
    rz = part.dot(r, z, ncomp)
    tol = atol + rtol * torch.sqrt(part.dot(r, r, ncomp))
    rr = part.dot(r, r, ncomp)
    it = 0
    while it < itmax and torch.sqrt(rr) > tol:
        q = part.exchange_add(apply_local(p), ncomp)
        q = torch.where(fm, q, zero)
        alpha = rz / part.dot(p, q, ncomp)
        x = x + alpha * p
        r = r - alpha * q
        z = r * dinv
        rz_new = part.dot(r, z, ncomp)
        rr = part.dot(r, r, ncomp)
        p = z + (rz_new / rz) * p
        rz = rz_new
        it += 1
    return x, it, float(torch.sqrt(rr))


class ElementPressure:
    """Discontinuous P1: every pressure DOF belongs to one element, so a slab's
    pressure vector (3 per local element) needs no exchange; sums all-reduce."""

    def __init__(self, part, n_global):
        self.part, self.n_global = part, n_global

    def sum(self, v):
        s = torch.sum(v).reshape(1)
        if self.part.world > 1:
            dist.all_reduce(s)
        return s[0]

    def complete(self, v):
        return v

    def remove_mean(self, a):
        return a - self.sum(a) / self.n_global


class VertexPressure:
    """Continuous P1: pressure on the P2 lattice's vertex nodes (even a and b),
    held as a slab-lattice vector that is zero elsewhere; the shared columns
    are vertex columns, completed by the same exchange as the velocity and
    counted once in sums."""

    def __init__(self, part):
        self.part = part
        gn = part.global_nodes()
        a, b = gn % part.A, gn // part.A
        vert = (a % 2 == 0) & (b % 2 == 0)
        self.mask = torch.as_tensor(vert)
        self.owned = torch.as_tensor(vert & part.owned())
        self.n_global = (part.ncr + 1) * part.nct

    def sum(self, v):
        s = torch.sum(torch.where(self.owned, v, torch.zeros_like(v))).reshape(1)
        if self.part.world > 1:
            dist.all_reduce(s)
        return s[0]

    def complete(self, v):
        return self.part.exchange_add(v, 1)

    def remove_mean(self, a):
        return torch.where(self.mask, a - self.sum(a) / self.n_global, a)


def distributed_stokes_pcg(part, apply_K, diag_K, free_u, apply_G, apply_GT, pc_S, rhs_u, pspace,
                           rtol=1e-8, itmax=200, itmin=10, inner_rtol=1e-12, inner_itmax=20000):
    """StokesPcCG (IterativeSolvers.jl:94-168) on slab-local data: the Schur
    PCG on S = G^T K^-1 G with the same step order, Polak-Ribiere beta, mean
    removal and stopping test as the single-GPU solve, an inner Jacobi-PCG on
    K for each K^-1, and only these crossing ranks: the velocity exchange
    after each K or G apply, the pressure exchange after each G^T apply
    (continuous pressure only), and all-reduces for dots, sums and the
    stopping test.

    apply_K(u) / apply_G(p) / apply_GT(u): the slab's partial element sums
    (completed here); pc_S(r): the Schur preconditioner on the slab's
    pressure DOFs; diag_K and rhs_u: assembled (exchanged) local vectors;
    free_u: local mask of the free velocity DOFs; pspace: ElementPressure or
    VertexPressure.  Returns (U, P, outer iterations, relative residual)."""
    def pdot(a, b):
        return pspace.sum(a * b)

    rm0 = pspace.remove_mean                      # rm0space! (IterativeSolvers.jl:172-186)

    def inner(b):
        return distributed_pcg(part, apply_K, b, diag_K, free_u, inner_rtol, 0.0, inner_itmax, ncomp=2)[0]

    U = inner(rhs_u)
    r = rm0(-pspace.complete(apply_GT(U)))
    P = torch.zeros_like(r)
    r0 = torch.sqrt(pdot(r, r))
    tol = r0 * rtol
    d = pc_S(r)
    q = d.clone()
    it = 0
    nr = r0
    for it in range(1, itmax + 1):
        q = rm0(q)
        rd = pdot(r, d)
        z = inner(part.exchange_add(apply_G(q), 2))
        Sq = pspace.complete(apply_GT(z))
        alpha = rd / pdot(q, Sq)
        rlast = r
        P = P + alpha * q
        U = U + alpha * z
        r = rm0(r - alpha * Sq)
        nr = torch.sqrt(pdot(r, r))
        if nr < tol and it >= itmin:
            break
        d = pc_S(r)
        beta = pdot(r - rlast, d) / rd
        q = d + beta * q
    return U, P, it, float(nr / r0) if r0 > 0 else 0.0
