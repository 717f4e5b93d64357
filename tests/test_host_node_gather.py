"""Index rule of the deterministic per-node gather (dimspers_b200/csrc/ops.cu,
k_node_gather): a lattice node (a, b) finds every element that contains it,
with the element's local node number, from its parities alone.  Checked here
as the exact inverse of the element -> node rule of the applies (element e =
2 (ir + ncr it) + t, local node k at (2 ir + loc_a, 2 it + loc_b) mod the
periodic theta), on lattices down to one cell, and against the connectivity of
the oracle mesh (the reference's Grid_split1 numbering, src/Grid/mesher.jl)
through the lattice map.  The device kernel itself is checked on the GPU
(tests/test_gpu_deterministic.py)."""
import numpy as np
import pytest

# local node offsets of triangle types 0 and 1 (the order of element_product)
LOC_A = ((0, 0, 2, 0, 1, 1), (0, 2, 2, 1, 2, 1))
LOC_B = ((0, 2, 0, 1, 1, 0), (2, 2, 0, 2, 1, 1))


def element_nodes(e, ncr, nct):
    A, B = 2 * ncr + 1, 2 * nct
    q, t = e >> 1, e & 1
    ir, it = q % ncr, q // ncr
    return [(2 * ir + LOC_A[t][k]) + A * ((2 * it + LOC_B[t][k]) % B) for k in range(6)]


def gather_candidates(n, ncr, nct):
    """(element, local node) pairs of lattice node n, in the kernel's order:
    node (a, b) = (2 i + pa, 2 j + pb); local node k of type t holds it iff
    LOC_A[t][k] has the parity pa and LOC_B[t][k] the parity pb, in cell
    (i + (pa - LOC_A) / 2, j + (pb - LOC_B) / 2), theta periodic."""
    A = 2 * ncr + 1
    b, a = divmod(n, A)
    i, pa = divmod(a, 2)
    j, pb = divmod(b, 2)
    out = []
    for t in (0, 1):
        for k in range(6):
            if LOC_A[t][k] % 2 != pa or LOC_B[t][k] % 2 != pb:
                continue
            ir = i + ((pa - LOC_A[t][k]) >> 1)
            it = j + ((pb - LOC_B[t][k]) >> 1)
            if ir < 0 or ir >= ncr:
                continue
            if it < 0:
                it += nct
            out.append((2 * (ir + ncr * it) + t, k))
    return out


def thread_blocks(ncr, nct):
    """Nodes owned by the kernel's threads (2 x 2 blocks, i <= ncr, j < nct)."""
    A = 2 * ncr + 1
    owned = []
    for q in range((ncr + 1) * nct):
        j, i = divmod(q, ncr + 1)
        for pb in (0, 1):
            for pa in (0, 1):
                if 2 * i + pa <= 2 * ncr:
                    owned.append(2 * i + pa + A * (2 * j + pb))
    return owned


@pytest.mark.parametrize("ncr,nct", [(1, 2), (1, 4), (2, 4), (3, 6), (4, 32), (5, 10)])
def test_gather_is_the_inverse_of_the_element_rule(ncr, nct):
    nel, nnod = 2 * ncr * nct, (2 * ncr + 1) * 2 * nct
    scatter = {n: [] for n in range(nnod)}
    for e in range(nel):
        for k, n in enumerate(element_nodes(e, ncr, nct)):
            scatter[n].append((e, k))
    for n in range(nnod):
        got = gather_candidates(n, ncr, nct)
        assert sorted(got) == sorted(scatter[n]), (n, got, scatter[n])
        assert len(set(got)) == len(got)
    owned = thread_blocks(ncr, nct)
    assert sorted(owned) == list(range(nnod))      # every node written by exactly one thread


def test_gather_matches_the_reference_connectivity():
    """Every (element, local node) of the oracle's Grid_split1 connectivity is
    found by the gather of its node, through the lattice map of the mesh."""
    from oracle import solver as OS
    from conftest import MeshView
    ncr, nct = 4, 32
    prob = OS.make_problem(ncr, nct, "discontinuous", pin_rotation=True)
    m = MeshView(prob)
    A = 2 * ncr + 1
    # lattice position of every reference node from its (theta, r) on the lattice
    th, r = np.asarray(m.theta), np.asarray(m.r)
    rr = np.unique(np.round(r, 12))
    assert rr.size == A
    a = np.searchsorted(rr, np.round(r, 12))
    b = np.rint(np.mod(th, 2 * np.pi) / (2 * np.pi) * 2 * nct).astype(int) % (2 * nct)
    lat = a + A * b
    e2n = np.asarray(m.e2n)                      # (6, nel) reference node ids, 0-based
    seen = set()
    for e in range(e2n.shape[1]):
        nodes = sorted(int(lat[j]) for j in e2n[:, e])
        seen.add(tuple(nodes))
    # the lattice elements' node sets are exactly the reference elements' node sets
    lattice = {tuple(sorted(element_nodes(e, ncr, nct))) for e in range(2 * ncr * nct)}
    assert lattice == seen
