"""Split-1 annulus mesh, midpoint numbering, colouring and velocity BCs (oracle).

All arrays are 0-based but keep the reference's ORDER exactly:
  vertex lattice        src/Grid/mesher.jl:166-172  (node = ir + nr*(itheta-1), theta-major)
  quads / split-1 tris  src/Grid/mesher.jl:174-200  (tri 2q-1 = [1,2,4], tri 2q = [2,3,4])
  element_neighbours    src/Grid/mesher.jl:313-347
  edge_connectivity     src/Grid/mesher.jl:349-392  (midpoints in first-seen order)
  add_midpoints         src/Grid/mesher.jl:394-417  (seam-aware theta average)
  p2top1                src/Grid/mesher.jl:300-311
  point_ids             src/Grid/mesher.jl:419-441
  color_mesh            src/Grid/coloring.jl:5-64
  free_slip / velocity_bcs  src/Setup/boundary_conditions.jl:15-37
  elementcoordinate + fixangles!  src/Utilities.jl:30-61
  rotation_matrix       src/Stokes/StokesSolver.jl:203-245

``Grid_split1`` in the reference calls the 17-field ``Grid`` constructor with
14 arguments (mesher.jl:217-232) and so cannot run as written; this module
restates its topology (mesher.jl:152-213) and returns the fields the Stokes
path reads.  ``nr`` / ``ntheta`` are NODE counts as in the reference
(radial cells = nr-1, angular cells = ntheta).
"""
from dataclasses import dataclass

import numpy as np

R_IN, R_OUT = 1.22, 2.22  # mesher.jl:155-157


def linrange(a, b, n):
    """Julia LinRange(a, b, n) element formula: (1-t)*a + t*b with t = j/(n-1)."""
    j = np.arange(n, dtype=np.float64)
    t = j / (n - 1)
    return (1.0 - t) * a + t * b


@dataclass
class Grid:
    theta: np.ndarray      # (nnod,) node angle
    r: np.ndarray          # (nnod,) node radius
    e2n: np.ndarray        # (6, nel) int64, 0-based, reference order
    e2n_p1: np.ndarray     # (3, 4*nel)
    ntheta: int            # angular nodes (= angular cells)
    nr: int                # radial nodes (= radial cells + 1)
    nel: int
    nnod: int
    nvnod: int

    def e2nP(self, pressure="discontinuous"):
        """Pressure numbering: continuous = EL2NOD[1:3,:] (mesher.jl:213);
        discontinuous = reshape(1:3nel,3,nel) (the commented mesher.jl:212)."""
        if pressure == "continuous":
            return self.e2n[:3].copy()
        return np.arange(3 * self.nel, dtype=np.int64).reshape(self.nel, 3).T.copy()


def _vertices_and_triangles(ntheta, nr, r_in=R_IN, r_out=R_OUT):
    nn = nr * ntheta
    dth = 2 * np.pi / ntheta
    r = np.empty(nn)
    th = np.empty(nn)
    rl = linrange(r_in, r_out, nr)
    for ii in range(ntheta):                         # mesher.jl:168-172
        idx = np.arange(nr) + nr * ii
        r[idx] = rl
        th[idx] = 0.0 + (dth * ii) * 1.0
    nquad = (nr - 1) * ntheta
    quads = np.empty((nquad, 4), dtype=np.int64)
    ir = np.arange(nr - 1)
    for ii in range(ntheta):                         # mesher.jl:176-188
        idx = ir + (nr - 1) * ii
        idx1 = ir + nr * ii
        idx2 = ir + nr * (ii + 1) if ii < ntheta - 1 else ir.copy()
        quads[idx] = np.stack([idx1, idx2, idx2 + 1, idx1 + 1], axis=1)
    tri = np.empty((2 * nquad, 3), dtype=np.int64)    # mesher.jl:191-200
    tri[0::2] = quads[:, [0, 1, 3]]
    tri[1::2] = quads[:, [1, 2, 3]]
    return th, r, tri.T.copy()


def element_neighbours(els):
    """Literal restatement of mesher.jl:313-347 (Python loops; small meshes)."""
    els = els[:3]
    nel = els.shape[1]
    # incidence matrix rows = elements, cols = nodes; nzrange(col) -> ascending elements
    nnod = int(els[2, nel - 1]) + 1                   # nnod = I[end] (mesher.jl:329)
    node_els = [[] for _ in range(int(els.max()) + 1)]
    for j in range(nel):
        for i in range(3):
            node_els[els[i, j]].append(j)
    neighbour = [[] for _ in range(nel)]
    for node in range(nnod):
        el_neighbour = sorted(node_els[node])
        for iel1 in el_neighbour:
            cur = neighbour[iel1]
            for iel2 in el_neighbour:
                if iel1 != iel2 and iel2 not in cur:
                    cur.append(iel2)
    return neighbour


def edge_connectivity(els, neighbours):
    """Literal restatement of mesher.jl:349-392 (Python loops; small meshes)."""
    nel = els.shape[1]
    lm = [(0, 1), (1, 2), (2, 0)]
    el2edge = np.zeros((3, nel), dtype=np.int64)     # 0 = unassigned, ids are 1-based here
    edge2node = []
    gidx = 0
    for iel in range(nel):
        edge = [tuple(sorted((els[a, iel], els[b, iel]))) for a, b in lm]
        nb_edges = [[tuple(sorted((els[a, n], els[b, n]))) for a, b in lm]
                    for n in neighbours[iel]]
        for ie in range(3):
            if el2edge[ie, iel] == 0:
                gidx += 1
                el2edge[ie, iel] = gidx
                edge2node.append(edge[ie])
                for c, ieln in enumerate(neighbours[iel]):
                    for i in range(3):
                        if edge[ie] == nb_edges[c][i]:
                            el2edge[i, ieln] = gidx
                            break
    return el2edge - 1, np.array(edge2node, dtype=np.int64)


def edge_connectivity_firstseen(els):
    """Vectorised equivalent of edge_connectivity for conforming meshes: an edge
    id is created the first time (element, local edge) order meets it."""
    nel = els.shape[1]
    a = els[[0, 1, 2]].T.reshape(-1)
    b = els[[1, 2, 0]].T.reshape(-1)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = lo * (int(els.max()) + 1) + hi
    uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    el2edge = rank[inv].reshape(nel, 3).T.copy()
    edge2node = np.stack([lo[first[order]], hi[first[order]]], axis=1)
    return el2edge, edge2node


def add_midpoints(els, el2edge, edge2node, th, r):
    """mesher.jl:394-417."""
    t1 = th[edge2node[:, 0]].copy()
    t2 = th[edge2node[:, 1]].copy()
    seam = np.abs(t1 - t2) > np.pi
    t1 = np.where(seam & (t1 < np.pi), t1 + 2 * np.pi, t1)
    t2 = np.where(seam & (t2 < np.pi), t2 + 2 * np.pi, t2)
    thmid = 0.5 * (t1 + t2)
    rmid = 0.5 * (r[edge2node[:, 0]] + r[edge2node[:, 1]])
    old = int(els.max()) + 1
    return (np.concatenate([th, thmid]), np.concatenate([r, rmid]),
            np.concatenate([els, el2edge + old], axis=0))


def p2top1(e2n):
    """mesher.jl:300-311: 4 P1 children [1 4 6; 4 2 5; 6 5 3; 4 5 6]."""
    lm = np.array([[0, 3, 5], [3, 1, 4], [5, 4, 2], [3, 4, 5]])
    ch = e2n[lm.reshape(-1)].reshape(4, 3, -1)       # (child, vertex, parent)
    return ch.transpose(1, 2, 0).reshape(3, -1)      # column 4*parent + child


def grid_split1(ntheta, nr, literal=False):
    """Split-1 grid with ntheta angular and nr radial NODES (mesher.jl:152-213)."""
    th, r, els = _vertices_and_triangles(ntheta, nr)
    if literal:
        nb = element_neighbours(els)
        el2edge, edge2node = edge_connectivity(els, nb)
    else:
        el2edge, edge2node = edge_connectivity_firstseen(els)
    th, r, e2n = add_midpoints(els, el2edge, edge2node, th, r)
    nel = e2n.shape[1]
    return Grid(theta=th, r=r, e2n=e2n, e2n_p1=p2top1(e2n), ntheta=ntheta, nr=nr,
                nel=nel, nnod=th.size, nvnod=int(e2n[:3].max()) + 1)


def grid_cells(ncr, nctheta, literal=False):
    """Grid with ncr radial x nctheta angular CELLS (2 triangles per cell)."""
    return grid_split1(nctheta, ncr + 1, literal=literal)


def point_ids(gr):
    """mesher.jl:419-441 -> (top_nodes, bottom_nodes) ascending."""
    rmin, rmax = gr.r.min(), gr.r.max()
    return np.flatnonzero(gr.r == rmax), np.flatnonzero(gr.r == rmin)


def free_slip(gr, pin_rotation=False):
    """boundary_conditions.jl:27-37, :15-25 -> (Omega, ifree) as 0-based DOFs.
    Fixed DOFs are the radial components (1-based 2*node) of wall nodes.
    pin_rotation=True is free_slip(nr, ids) (:180-194): it also fixes the
    tangential DOF 2*nr-1 (1-based), u_theta of node nr (r_out, theta = 0)."""
    top, bot = point_ids(gr)
    nodes = np.concatenate([top, bot])
    omega = 2 * nodes + 1
    if pin_rotation:
        omega = np.concatenate([omega, [2 * gr.nr - 2]])
    mask = np.ones(2 * gr.nnod, dtype=bool)
    mask[omega] = False
    return omega, np.flatnonzero(mask)


def color_mesh(e2n):
    """Greedy first-fit colouring over vertex-sharing neighbours, element order
    (coloring.jl:5-64).  Returns (colors 1-based per element, color_list)."""
    els = e2n[:3]
    nel = els.shape[1]
    node_els = [[] for _ in range(int(els.max()) + 1)]
    for j in range(nel):
        for i in range(3):
            node_els[els[i, j]].append(j)
    colors = np.zeros(nel, dtype=np.int64)
    max_color = 0
    for iel in range(nel):
        occupied = set()
        for i in range(3):
            for n in node_els[els[i, iel]]:
                if n != iel and colors[n] != 0:
                    occupied.add(int(colors[n]))
        free = 0
        for c in range(1, max_color + 1):
            if c not in occupied:
                free = c
                break
        if free == 0:
            max_color += 1
            free = max_color
        colors[iel] = free
    color_list = [np.flatnonzero(colors == c) for c in range(1, max_color + 1)]
    color_list.sort(key=lambda v: tuple(v))           # sort!(color_list)
    return colors, color_list


def element_coordinates(gr):
    """elementcoordinate + fixangles! on the 3 vertices (Utilities.jl:30-61, MAIN.jl:62-66)."""
    th = gr.theta[gr.e2n[:3]].copy()
    r = gr.r[gr.e2n[:3]].copy()
    a = (np.abs(th[0] - th[1]) + np.abs(th[1] - th[2]) + np.abs(th[2] - th[0])) > np.pi
    th = np.where(a[None, :] & (th < np.pi), th + 2 * np.pi, th)
    return th, r


def rotation_blocks(gr):
    """Per-node TT = [c s; -s c] (StokesSolver.jl:203-245); U_cart = TT * U_polar."""
    c, s = np.cos(gr.theta), np.sin(gr.theta)
    return c, s
