"""Known-answer tests that pin the FP64 oracle (CPU, no GPU).

The reference has no tests, fixtures or golden vectors, and Julia is absent,
so the oracle is pinned by properties its algorithm must satisfy exactly (or to
rounding) plus regression fixtures in tests/golden/ (make_golden.py).
"""
import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT, MeshView, rel
from dimspers_b200 import inputs
from oracle import assembly as OA
from oracle import mesh as OM
from oracle import quadrature as OQ
from oracle import solver as OS

GOLD = os.path.join(ROOT, "tests", "golden")


def test_six_point_rule_is_degree_four_exact():
    """ip_triangle6 (Quadrature.jl:80-107) integrates r^a s^b, a+b <= 4, exactly:
    int_T r^a s^b = a! b! / (a+b+2)!."""
    x, w = OQ.ip_triangle6()
    for a in range(5):
        for b in range(5 - a):
            exact = math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)
            assert abs(np.sum(w * x[:, 0] ** a * x[:, 1] ** b) - exact) < 1e-15


def test_p2_shape_functions():
    nodes = [(0, 0), (1, 0), (0, 1), (0.5, 0), (0.5, 0.5), (0, 0.5)]
    for k, p in enumerate(nodes):
        N = OQ.sf_N_tri6(*p)
        assert np.allclose(N, np.eye(6)[k], atol=1e-15)
    for p in [(0.2, 0.3), (0.7, 0.1)]:
        assert abs(OQ.sf_N_tri6(*p).sum() - 1) < 1e-15
        assert np.allclose(OQ.sf_dN_tri6(*p).sum(axis=1), 0, atol=1e-14)


def test_volume_integral_is_annulus_area():
    """volume_integral(1) (FSE.jl:412-464) = pi (r_out^2 - r_in^2): the
    integrand r is linear in (theta, r) and the geometry is exact there."""
    prob = OS.make_problem(4, 32)
    area = OS.volume_integral(np.ones(prob.gr.nnod), prob.gr.e2n, prob.th, prob.r)
    assert abs(area - math.pi * (2.22 ** 2 - 1.22 ** 2)) < 1e-12


def test_literal_and_vectorised_edge_numbering_agree():
    for ncr, nct in [(3, 7), (4, 32)]:
        a = OM.grid_cells(ncr, nct, literal=True)
        b = OM.grid_cells(ncr, nct, literal=False)
        assert np.array_equal(a.e2n, b.e2n) and np.array_equal(a.theta, b.theta)


def test_colouring_valid():
    g = OM.grid_cells(8, 64)
    colors, lists = OM.color_mesh(g.e2n)
    for ids in lists:
        nodes = g.e2n[:3, ids].ravel()
        assert np.unique(nodes).size == nodes.size


@pytest.mark.parametrize("kind", ["iso", "aniso", "fabric"])
def test_element_matrices_symmetric_psd_translation_null(kind):
    prob = OS.make_problem(4, 32)
    mat = inputs.make_material(MeshView(prob), kind, seed=5)
    Ke, Ge, Me, Fb = OA.element_matrices(prob.th, prob.r, mat.eta_ip, mat.rho, prob.gr.e2n, mat.g, mat.C6)
    full = OA.unpack_sym(Ke, 12, OA.PACK12)
    ev = np.linalg.eigvalsh(full)
    assert ev.min() > -1e-12 * ev.max()
    # Cartesian rigid translations are exactly in the kernel
    t1 = np.zeros(12); t1[0::2] = 1
    t2 = np.zeros(12); t2[1::2] = 1
    scale = np.abs(full).max()
    assert np.abs(full @ t1).max() < 1e-13 * scale and np.abs(full @ t2).max() < 1e-13 * scale
    # two exact zero modes per element: the Cartesian translations (the small
    # rotation (-z, x) is not in P2 on the (theta, r)-mapped element)
    assert np.sum(ev < 1e-12 * ev.max(axis=1, keepdims=True)) >= 2 * prob.gr.nel


def test_isotropic_tensor_is_rotation_invariant():
    """directRotation2D (anisotropy.jl:503-536) with e = (a-h)/2 = 1 leaves the
    isotropic tensor unchanged for any director."""
    phi = np.linspace(0, 2 * np.pi, 17)
    C = inputs.ti_tensor(np.ones_like(phi), np.cos(phi), np.sin(phi))
    ref = (4 / 3, 4 / 3, 1.0, -2 / 3, 0.0, 0.0)
    for c, r in zip(C, ref):
        assert np.allclose(c, r, atol=1e-14)


def test_rotation_matrix_orthogonal():
    g = OM.grid_cells(2, 8)
    TT = OA.rotation_matrix(g.theta).toarray()
    assert np.allclose(TT @ TT.T, np.eye(TT.shape[0]), atol=1e-14)


def test_solution_has_the_forcing_symmetry():
    """Iso material and forcing with 4-fold symmetry (no noise): the converged
    velocity is invariant under a rotation by pi/2 (node permutation)."""
    prob = OS.make_problem(4, 32, "continuous", pin_rotation=False)
    g = prob.gr
    T = np.log(g.r / 2.22) / np.log(1.22 / 2.22) + 0.01 * np.cos(4 * g.theta) * np.sin(np.pi * (g.r - 1.22))
    eta = inputs.eta_from_T(T, g.e2n, 1e3)
    out = OS.solve_stokes(prob, eta, T, 1e5, rtol=1e-12, itmax=2000)
    U = out["U"]
    key = {(round(t, 9) % round(2 * np.pi, 9), round(r, 9)): i for i, (t, r) in enumerate(zip(g.theta, g.r))}
    perm = np.array([key[(round((t + np.pi / 2) % (2 * np.pi), 9) % round(2 * np.pi, 9), round(r, 9))]
                     for t, r in zip(g.theta, g.r)])
    assert rel(U[0::2][perm], U[0::2]) < 1e-6
    assert rel(U[1::2][perm], U[1::2]) < 1e-6


@pytest.mark.parametrize("name", ["iso_4x32_cont", "aniso_4x32_disc", "aniso_8x64_disc_mass", "fabric_8x64_cont"])
def test_oracle_reproduces_golden(name):
    meta = json.load(open(os.path.join(GOLD, "golden.json")))[name]
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    prob = OS.make_problem(meta["nr_cells"], meta["ntheta_cells"], meta["pressure"], pin_rotation=True)
    mat = inputs.make_material(MeshView(prob), meta["kind"], seed=meta["seed"])
    out = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-12, itmax=5000,
                          schur_pc=meta["schur_pc"])
    tol = 1e-10 if meta["pressure"] == "continuous" else 1e-8
    assert rel(out["U"], gold["U"]) < tol and rel(out["P"], gold["P"]) < tol
    assert abs(out["report"].iterations - meta["iterations_rtol12"]) <= 2
    assert rel(out["mats"]["F"], gold["F"]) < 1e-14
    import hashlib
    assert hashlib.sha256(np.ascontiguousarray(prob.gr.e2n).tobytes()).hexdigest() == meta["e2n_sha256"]


def test_stress_rigid_rotation_and_linear_fields_converge_second_order():
    """The post-processor's strain rate of a rigid rotation is 0 and that of a
    linear Cartesian field is its gradient, up to the O(h^2) error of
    interpolating it on (theta, r)-linear elements: the error falls 4x per
    refinement."""
    import oracle.stress as ST
    errs = []
    for n in (4, 8, 16):
        prob = OS.make_problem(n, 8 * n, "discontinuous")
        th, r, e2n = prob.th, prob.r, prob.gr.e2n
        x, z = prob.gr.r * np.sin(prob.gr.theta), prob.gr.r * np.cos(prob.gr.theta)
        one = np.ones((th.shape[1], 7))
        U = np.zeros(2 * x.size)
        U[0::2], U[1::2] = -z, x
        o = ST.stress(U, one, th, r, e2n)
        e_rot = max(np.abs(o[k]).max() for k in ("exx", "ezz", "exz"))
        U[0::2], U[1::2] = 2 * x, -3 * z
        o = ST.stress(U, one, th, r, e2n)
        e_lin = max(np.abs(o["exx"] - 2).max(), np.abs(o["ezz"] + 3).max(), np.abs(o["exz"]).max())
        errs.append((e_rot, e_lin))
    for (a0, b0), (a1, b1) in zip(errs, errs[1:]):
        assert 3.5 < a0 / a1 < 4.5 and 3.5 < b0 / b1 < 4.5
    # invariants and the isotropic stress of the linear field (eta = 1)
    assert np.allclose(o["eII"], np.sqrt(0.5 * (o["exx"] ** 2 + o["ezz"] ** 2) + o["exz"] ** 2))
    assert np.allclose(o["txx"], 4 / 3 * o["exx"] - 2 / 3 * o["ezz"])
    assert np.allclose(o["txz"], 2 * o["exz"])


def test_arrhenius_update_branches_scalar_restatement():
    """The vectorised viscosity update against a scalar per-IP loop written
    straight from getviscosity!(::Arrhenius) (Rheology.jl:348-403) on a few
    elements, with every branch present."""
    from oracle import rheology as RH
    prob = OS.make_problem(4, 16, "continuous")
    e2n, nel = prob.gr.e2n, prob.gr.e2n.shape[1]
    rng = np.random.default_rng(2)
    r = 3.48e6 + (prob.gr.r - 1.22) * 2.87e6
    T = 1300.0 + 1200.0 * rng.random(r.size)
    P = 2e9 * rng.standard_normal(e2n[:3].max() + 1)
    eps = np.abs(rng.standard_normal((nel, 7))) * 1e-15
    eps[::4] = 0.0
    tau = 4e9 * rng.random((nel, 7))
    coh = np.where(rng.random((nel, 7)) < 0.3, 0.0, 30e6)
    prev = np.full((nel, 7), 2e21)
    law = (5e20, 8.314, 100e3, 1e-6, 1600.0, 30.0)
    got = RH.arrhenius_viscosity(prev, T, P, r, e2n, eps, tau, coh, *law)
    eta0, R, Ea, Va, T0, phi = law
    ipx, _ = OQ.ip_triangle7()
    minP, maxr = abs(P.min()), r.max()
    branches = set()
    for e in range(nel):
        for ip in range(7):
            a, b = ipx[ip]
            c = 1.0 - a - b
            N6 = [c * (2 * c - 1), a * (2 * a - 1), b * (2 * b - 1), 4 * a * c, 4 * a * b, 4 * b * c]
            Tip = sum(N6[k] * T[e2n[k, e]] for k in range(6))
            zip_ = sum(N6[k] * r[e2n[k, e]] for k in range(6))
            Pip = c * P[e2n[0, e]] + a * P[e2n[1, e]] + b * P[e2n[2, e]] + minP
            lam = 1e-3 if zip_ < maxr - 2780e3 else (1e0 if zip_ > maxr - 660e3 else 1e1)
            want = min(max(lam * eta0 * math.exp((Ea + Pip * Va) / R / Tip - Ea / R / T0), 1e18), 1e25)
            if coh[e, ip] != 0 and phi != 0 and eps[e, ip] != 0:
                ty = math.cos(math.radians(phi)) * coh[e, ip] + math.sin(math.radians(phi)) * Pip
                if ty < tau[e, ip]:
                    want = max(1e18, min(1e25, ty / (2 * eps[e, ip])))
                    branches.add("yield")
                else:
                    want = prev[e, ip]
                    branches.add("kept")
            else:
                branches.add("creep")
            assert math.isclose(got[e, ip], want, rel_tol=1e-13), (e, ip)
    assert branches == {"yield", "kept", "creep"}


def _dem_fixture(vol=30):
    d = np.load(os.path.join(ROOT, "tests", "golden", "dem_1e-3_vol%d.npz" % vol))
    return d["C"], d["ax"]


def test_dem_tables_of_the_reference_files():
    """getDEM's block structure on the reference's DEM tables (10 blocks of
    10 rows), and the host-side DEM the C ABI receives agrees with the oracle."""
    from oracle import fabric as OF
    from dimspers_b200.fabric import DEM
    for vol in (10, 20, 30):
        C6, ax = _dem_fixture(vol)
        t = OF.dem_tables(C6, ax)
        assert t["sblk"] == 10 and len(t["a1a2_blk"]) == 10 and t["nblk"] == 11
        assert np.all(np.diff(t["a1a2_blk"]) > 0) and np.all(np.diff(t["a2a3_blk"]) > 0)
        assert sorted(t["permutation_blk"]) == list(range(1, 11))
        d = DEM(C6, ax, w=1e-2)
        assert d.sblk == t["sblk"]
        np.testing.assert_array_equal(d.a1a2_blk, t["a1a2_blk"])
        np.testing.assert_array_equal(d.a2a3_blk, t["a2a3_blk"])
        np.testing.assert_array_equal(d.permutation_blk, t["permutation_blk"])


def test_dem_tensor_at_table_points_is_the_table_row():
    """Shapes exactly at table points and an unrotated FSE (vx1 = 1, vy1 = 0)
    return the table row itself: (C11, C33, max(C55, w), C13, 0, 0)."""
    from oracle import fabric as OF
    C6, ax = _dem_fixture()
    t = OF.dem_tables(C6, ax)
    w = 0.02
    rows = [0, 13, 57, 99, 42]
    r1 = np.array([[np.log10(ax[k, 0])] * 6 for k in rows])
    r2 = np.array([[np.log10(1.0 / ax[k, 2])] * 6 for k in rows])
    one, zero = np.ones_like(r1), np.zeros_like(r1)
    out = OF.anisotropic_tensor(one, zero, r1, r2, t, w)
    for j, k in enumerate(rows):
        want = (C6[k, 0], C6[k, 2], max(C6[k, 4], w), C6[k, 7], 0.0, 0.0)
        for f in range(6):
            assert np.allclose(out[f][j], want[f], rtol=0, atol=1e-15), (k, f)
    # argminsorted's first-local-minimum rule, including ties and the last index
    assert OF.argminsorted(np.array([3.0, 2.0, 2.0, 5.0])) == 2
    assert OF.argminsorted(np.array([3.0, 2.0, 1.0])) == 2
    assert OF.argminsorted(np.array([1.0, 2.0, 0.0])) == 0


def test_fse_of_a_rotated_stretch():
    from oracle import fabric as OF
    rng = np.random.default_rng(5)
    ang = rng.uniform(-np.pi, np.pi, (4, 6))
    s1, s2 = rng.uniform(1, 5, (4, 6)), rng.uniform(0.1, 1, (4, 6))
    c, s = np.cos(ang), np.sin(ang)
    R = np.stack([np.stack([c, -s], -1), np.stack([s, c], -1)], -2)
    F = R @ (np.eye(2) * np.stack([s1, s2], -1)[..., None, :])    # R diag(s1, s2): major axis (c, s)
    x1, x2, y1, y2, a1, a2 = OF.fse(F)
    assert np.allclose(a1, s1) and np.allclose(a2, s2)
    assert np.allclose(np.abs(x1 * c + y1 * s), 1.0) and np.allclose(x1 * x2 + y1 * y2, 0.0, atol=1e-12)


def test_thermal_element_blocks():
    """assemble_element! (AssemblerThermal.jl:114-226) restated: constants are
    the conduction block's null space, the mass blocks integrate rho Cp over
    the annulus, both symmetric (K positive semi-definite)."""
    from oracle import thermal as OT
    prob = OS.make_problem(4, 32, "continuous")
    gr = prob.gr
    Ke, Me = OT.element_matrices(prob.th, prob.r, np.full(gr.nnod, 2.0), gr.e2n, 1.7, 3.0)
    assert np.abs(Ke.sum(axis=2)).max() < 1e-12
    assert math.isclose(Me.sum(), 6.0 * math.pi * (2.22 ** 2 - 1.22 ** 2), rel_tol=1e-12)
    assert np.abs(Ke - Ke.transpose(0, 2, 1)).max() < 1e-12 and np.abs(Me - Me.transpose(0, 2, 1)).max() < 1e-14
    assert np.linalg.eigvalsh(Ke).min() > -1e-12


def test_thermal_long_step_converges_to_conduction_profile():
    """A very long backward-Euler step is the steady conduction solution
    T = Tbot + (Ttop - Tbot) ln(r / r_in) / ln(r_out / r_in); the P2 error
    falls by ~8x per refinement."""
    from oracle import thermal as OT
    errs = []
    for nr, nt in ((4, 32), (8, 64)):
        prob = OS.make_problem(nr, nt, "continuous")
        gr = prob.gr
        fixed, tfix = OT.boundary(gr, 300.0, 4000.0)
        T = OT.thermal_step(gr, prob.th, prob.r, np.full(gr.nnod, 1000.0), np.ones(gr.nnod), 1.0, 1.0, 1e9,
                            fixed, tfix)
        exact = 4000.0 + (300.0 - 4000.0) * np.log(gr.r / 1.22) / np.log(2.22 / 1.22)
        errs.append(np.abs(T - exact).max())
    assert errs[1] < errs[0] / 6 and errs[1] < 0.05


@pytest.mark.parametrize("pressure", ["continuous", "discontinuous"])
def test_hydrostatic_balance_converges(pressure):
    """A manufactured solution the radial buoyancy force admits: uniform rho
    and eta give u = 0 and p = g rho r + const.  The discrete velocity vanishes
    and the pressure is linear in r, both to high order under refinement (the
    curved geometry makes neither exact)."""
    errs = []
    for nr, nt in ((4, 32), (8, 64)):
        prob = OS.make_problem(nr, nt, pressure)
        gr = prob.gr
        nel = prob.th.shape[1]
        out = OS.solve_stokes(prob, np.ones((nel, 7)), np.full(gr.nnod, 2.0), 1.5, rtol=1e-12, itmax=2000)
        U, P = out["U"], out["P"]
        rp = np.zeros(len(P))
        rp[prob.e2nP] = gr.r[gr.e2n[:3]]
        A = np.vstack([rp, np.ones(len(P))]).T
        coef = np.linalg.lstsq(A, P, rcond=None)[0]
        errs.append((np.abs(U).max(), np.abs(P - A @ coef).max()))
        assert abs(coef[0] - 3.0) < 1e-5                        # dp/dr = g rho
    assert errs[1][0] < errs[0][0] / 15 and errs[1][0] < 1e-9
    assert errs[1][1] < errs[0][1] / 10 and errs[1][1] < 1e-6


def test_thermal_gmres_restatement_meets_its_stopping_test():
    """The reference's solve (Krylov.jl gmres, full, sqrt(eps) tolerances)
    restated: it stops at ||r|| <= atol + rtol ||b|| with the true residual
    there too, and agrees with the direct solve to kappa * sqrt(eps)."""
    from oracle import thermal as OT
    prob = OS.make_problem(4, 32, "continuous")
    gr = prob.gr
    rng = np.random.default_rng(8)
    Ke, Me = OT.element_matrices(prob.th, prob.r, 1.0 + 0.1 * rng.random(gr.nnod), gr.e2n, 1.0, 1.0)
    A = OT._global(gr.e2n, Me + 1e-3 * Ke, gr.nnod)
    b = rng.standard_normal(gr.nnod)
    x, it, rn = OT.gmres(A, b)
    eps = np.sqrt(np.finfo(float).eps) * (1.0 + np.linalg.norm(b))
    assert 0 < it < gr.nnod and rn <= eps
    assert np.linalg.norm(b - A @ x) <= 1.01 * eps
    xd = spla_solve(A, b)
    assert np.abs(x - xd).max() / np.abs(xd).max() < 1e-5
    fixed, tfix = OT.boundary(gr, 300.0, 4000.0)
    T0 = np.full(gr.nnod, 1000.0)
    Tg = OT.thermal_step(gr, prob.th, prob.r, T0, np.ones(gr.nnod), 1.0, 1.0, 1e-2, fixed, tfix, solver="gmres")
    Td = OT.thermal_step(gr, prob.th, prob.r, T0, np.ones(gr.nnod), 1.0, 1.0, 1e-2, fixed, tfix)
    assert np.abs(Tg - Td).max() / np.abs(Td).max() < 1e-6


def spla_solve(A, b):
    import scipy.sparse.linalg as spla
    return spla.spsolve(A.tocsc(), b)


@pytest.mark.parametrize("kind", ["iso", "aniso"])
def test_c_and_numpy_element_restatements_agree(kind):
    """Two independent restatements of the Stokes element blocks (NumPy,
    oracle/assembly.py; plain C with OpenMP, oracle/stokes_elements.c) agree
    to round-off on every packed entry."""
    from oracle import c_elements as OC
    prob = OS.make_problem(8, 64, "discontinuous")
    mat = inputs.make_material(MeshView(prob), kind, seed=9)
    ref = OA.element_matrices(prob.th, prob.r, mat.eta_ip, mat.rho, prob.gr.e2n, mat.g, mat.C6)
    got = OC.element_matrices(prob.th, prob.r, mat.eta_ip, mat.rho, prob.gr.e2n, mat.g, mat.C6)
    for a, b in zip(got, ref):
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_c_and_python_dem_lookups_agree():
    """The DEM tensor lookup restated twice (per-IP Python loop,
    oracle/fabric.py; plain C, oracle/fabric_lookup.c) on the reference's
    table: the same rows everywhere, round-off in the rotation only."""
    from oracle import c_elements as OC
    from oracle import fabric as OF
    C6, ax = _dem_fixture()
    t = OF.dem_tables(C6, ax)
    rng = np.random.default_rng(4)
    nel = 300
    ang = rng.uniform(-np.pi, np.pi, (nel, 6))
    args = (np.cos(ang), np.sin(ang), rng.uniform(-0.3, 2.0, (nel, 6)), rng.uniform(-0.3, 2.3, (nel, 6)))
    ref = OF.anisotropic_tensor(*args, t, 0.02)
    got = OC.anisotropic_tensor(*args, t, 0.02)
    for a, b in zip(got, ref):
        assert np.abs(a - b).max() < 1e-14
