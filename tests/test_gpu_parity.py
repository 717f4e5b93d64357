"""GPU parity of the CUDA path against the FP64 oracle, through the C ABI.

Tolerances (written here, as the contract asks):
  element blocks (Ke, Ge, Me, Fb), Cartesian, FP64 path   <= 1e-12 relative (norm-wise)
  operator applies K, G, G^T and the assembled RHS / pc   <= 1e-12 relative
  converged U (rotation removed) and P, FP64 path:
      continuous pressure (Taylor-Hood)                   <= 1e-9 relative L2
      discontinuous pressure                              <= 1e-8 relative L2
  FP32-refined path U, P                                  <= 1e-7 relative L2
The solve comparisons run both sides to rtol 1e-12 with the rigid rotation
pinned, so that the two solutions are the same discrete solution.  The
Schur complement of P2-P1disc on this mesh is ill-conditioned (its smallest
non-zero eigenvalue falls with h), so two solutions that both meet
||r|| <= 1e-12 ||r0|| differ by up to kappa(S) * 1e-12 ~ 1e-9..1e-8.
"""
import numpy as np
import pytest

from conftest import MeshView, rel
from dimspers_b200 import StokesContext, inputs
from oracle import assembly as OA
from oracle import solver as OS

pytestmark = pytest.mark.gpu


def _setup(ncr, nct, pressure, kind, pin=True, seed=3):
    prob = OS.make_problem(ncr, nct, pressure, pin_rotation=pin)
    mat = inputs.make_material(MeshView(prob), kind, seed=seed)
    ctx = StokesContext(ncr, nct, pressure, pin_rotation=pin)
    return prob, mat, ctx


@pytest.mark.parametrize("kind", ["iso", "aniso"])
def test_element_matrices(kind):
    prob, mat, ctx = _setup(4, 32, "discontinuous", kind)
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(0)
        Ke, Ge, Me, Fb = ctx.element_matrices()
    oKe, oGe, oMe, oFb = OA.element_matrices(prob.th, prob.r, mat.eta_ip, mat.rho, prob.gr.e2n, mat.g, mat.C6)
    assert rel(Ke, oKe) < 1e-12
    assert rel(Ge, oGe) < 1e-12
    assert rel(Me, oMe) < 1e-12
    assert rel(Fb, oFb) < 1e-12


def test_ti_material_matches_full_tensor():
    prob, mat, ctx = _setup(4, 32, "discontinuous", "aniso")
    with ctx:
        ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
        ctx.assemble(0)
        Ke_ti = ctx.element_matrices()[0]
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(0)
        Ke_full = ctx.element_matrices()[0]
    assert rel(Ke_ti, Ke_full) < 1e-13


@pytest.mark.parametrize("pressure", ["continuous", "discontinuous"])
def test_operator_applies(pressure):
    prob, mat, ctx = _setup(8, 64, pressure, "aniso")
    A = OS.assemble(prob, mat.eta_ip, mat.rho, mat.g, mat.C6)
    f = prob.ifree
    rng = np.random.default_rng(0)
    x = np.zeros(2 * prob.gr.nnod)
    x[f] = rng.standard_normal(f.size)
    p = rng.standard_normal(prob.npres)
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(0)
        y = ctx.apply_K(x)
        yg = ctx.apply_G(p)
        pg = ctx.apply_GT(x)
        F, pc = ctx.rhs()
    Kf = A["KK"][f][:, f]
    assert rel(y[f], Kf @ x[f]) < 1e-12
    assert np.all(y[prob.omega] == 0)
    assert rel(yg[f], (A["GG"] @ p)[f]) < 1e-12
    assert rel(pg, A["GG"].T @ x) < 1e-12
    assert rel(F[f], A["F"][f]) < 1e-12
    assert rel(pc, OS.lumped_pc(A["MM"])) < 1e-12


@pytest.mark.parametrize("pressure,kind,size", [("continuous", "iso", (8, 64)),
                                                ("discontinuous", "aniso", (8, 64)),
                                                ("continuous", "aniso", (32, 256))])
def test_solve_fp64_matches_oracle(pressure, kind, size):
    prob, mat, ctx = _setup(*size, pressure, kind)
    ref = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-12, itmax=5000)
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(0)
        U, P, Uc, rep = ctx.solve(rtol=1e-12, itmax=5000, inner_rtol=1e-13, inner_itmax=2000)
    assert rep["status"] == 0, rep
    tol = 1e-9 if pressure == "continuous" else 1e-8
    assert rel(U, ref["U"]) < tol, (rel(U, ref["U"]), rep)
    assert rel(P, ref["P"]) < tol, (rel(P, ref["P"]), rep)
    c, s = np.cos(prob.gr.theta), np.sin(prob.gr.theta)
    assert rel(Uc[0::2], c * U[0::2] + s * U[1::2]) < 1e-14


def test_solve_reference_tolerance_iterations():
    """At the reference's rtol 1e-8 / itmin 10 the outer iteration count of
    the exact-inner-solve oracle is reproduced within a few iterations."""
    prob, mat, ctx = _setup(8, 64, "continuous", "iso")
    ref = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6)
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(0)
        U, P, Uc, rep = ctx.solve(inner_rtol=1e-12)
    assert rep["status"] == 0
    assert abs(rep["iterations"] - ref["report"].iterations) <= 2
    assert rel(U, ref["U"]) < 1e-6
    assert rel(P, ref["P"]) < 1e-6


@pytest.mark.parametrize("pressure,precision", [("continuous", 1), ("discontinuous", 1),
                                                ("continuous", 2), ("discontinuous", 2)])
def test_solve_fp32_refined(pressure, precision):
    """FP32 element matrices / FP32 multigrid with FP64 residuals (precision 1)
    and classic FP32 iterative refinement (precision 2) against the FP64 oracle."""
    prob, mat, ctx = _setup(8, 64, pressure, "aniso")
    ref = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-12, itmax=5000)
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(precision)
        U, P, Uc, rep = ctx.solve(precision=precision, rtol=1e-11, itmax=5000, inner_rtol=1e-12)
    assert rep["status"] == 0, rep
    assert rel(U, ref["U"]) < 1e-7, rel(U, ref["U"])
    assert rel(P, ref["P"]) < 1e-7, rel(P, ref["P"])


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_graph_matches_host_loop(precision):
    """The single-graph solve (device-side loop control) and the host-driven
    loops run the same kernels in the same order."""
    prob, mat, ctx = _setup(8, 64, "discontinuous", "aniso")
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(precision)
        U0, P0, _, r0 = ctx.solve(precision=precision, host_loop=1, itmax=5000, rtol=1e-11, inner_rtol=1e-12)
        U1, P1, _, r1 = ctx.solve(precision=precision, itmax=5000, rtol=1e-11, inner_rtol=1e-12)
    assert r0["status"] == 0 and r1["status"] == 0
    assert abs(r0["iterations"] - r1["iterations"]) <= max(3, r0["iterations"] // 50)
    assert rel(U1, U0) < 1e-7 and rel(P1, P0) < 1e-7
    assert r1["kernel_launches"] > 0


def test_jacobi_inner_matches_mg():
    prob, mat, ctx = _setup(4, 32, "continuous", "iso")
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(0)
        U1, P1, _, r1 = ctx.solve(rtol=1e-12, itmax=1000, inner_rtol=1e-13, inner_itmax=20000)
        U2, P2, _, r2 = ctx.solve(rtol=1e-12, itmax=1000, inner_rtol=1e-13, inner_itmax=20000, inner_pc=1)
    assert r1["status"] == 0 and r2["status"] == 0
    assert rel(U1, U2) < 1e-9 and rel(P1, P2) < 1e-9
    assert r2["inner_iterations"] > r1["inner_iterations"]


def test_fse_director_kernel():
    prob, mat, ctx = _setup(4, 32, "discontinuous", "iso")
    rng = np.random.default_rng(1)
    F = np.eye(2)[None] + 0.5 * rng.standard_normal((prob.gr.nel, 2, 2))
    with ctx:
        dx, dy = ctx.fse_director(F)
    L = F @ F.transpose(0, 2, 1)
    w, v = np.linalg.eigh(L)
    vmax = v[:, :, 1]
    # sign is arbitrary: compare the projector
    assert np.allclose(np.abs(dx * vmax[:, 0] + dy * vmax[:, 1]), 1.0, atol=1e-10)


def test_mass_schur_preconditioner_matches_oracle():
    """schur_pc = 1 (element-block M^-1, discontinuous pressure) against the
    oracle's StokesPcCG with the same preconditioner: same solution, fewer
    outer iterations than the lumped mass."""
    prob, mat, ctx = _setup(8, 64, "discontinuous", "aniso")
    ref = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-12, itmax=5000, schur_pc="mass")
    ref8 = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-8, itmax=5000, schur_pc="mass")
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(1)
        U, P, _, rep = ctx.solve(precision=1, schur_pc=1, rtol=1e-12, itmax=5000, inner_rtol=1e-13)
        _, _, _, rep8 = ctx.solve(precision=1, schur_pc=1, rtol=1e-8, itmax=5000, inner_rtol=1e-12)
        _, _, _, rep_l = ctx.solve(precision=1, schur_pc=0, rtol=1e-8, itmax=5000, inner_rtol=1e-12)
    assert rep["status"] == 0
    assert rel(U, ref["U"]) < 1e-8 and rel(P, ref["P"]) < 1e-8
    assert abs(rep8["iterations"] - ref8["report"].iterations) <= 3
    assert rep8["iterations"] < 0.8 * rep_l["iterations"]


def test_relaxed_inner_tolerance_accuracy():
    """The relaxed inner tolerance keeps U, P within 1e-7 of the fixed-tolerance
    solve on a well-conditioned (Taylor-Hood) case while doing less inner work."""
    prob, mat, ctx = _setup(32, 256, "continuous", "aniso")
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(1)
        U0, P0, _, r0 = ctx.solve(precision=1, inner_rtol=1e-12)
        U1, P1, _, r1 = ctx.solve(precision=1, inner_rtol=1e-10, inner_relax=1e-6)
    assert r1["status"] == 0
    assert rel(U1, U0) < 1e-7 and rel(P1, P0) < 1e-7
    assert r1["inner_iterations"] < r0["inner_iterations"]


@pytest.mark.parametrize("pressure,kind", [("discontinuous", "aniso"), ("continuous", "fabric")])
def test_matrix_free_apply_matches_packed_matrices(pressure, kind):
    """The matrix-free fine-level apply (rotated tensors + per-ring reference
    derivatives) is the operator of the packed element matrices."""
    prob, mat, ctx = _setup(8, 64, pressure, kind)
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(1)
        x = np.random.default_rng(5).standard_normal(2 * ctx.nnod)
        ys = {}
        for mf in (0, 1):
            ctx.solve(want_cart=False, raise_on_status=False, itmax=1, itmin=1, precision=1, matrix_free=mf)
            ys[mf] = ctx.apply_K(x)
        assert rel(ys[1], ys[0]) < 1e-13, rel(ys[1], ys[0])
        out = [ctx.solve(want_cart=False, precision=p, matrix_free=mf, itmax=5000, rtol=1e-11, inner_rtol=1e-12)
               for p in (0, 1) for mf in (0, 1)]
    for U, P, _, r in out:
        assert r["status"] == 0
    for U, P, _, r in out[1:]:
        assert rel(U, out[0][0]) < 1e-7 and rel(P, out[0][1]) < 1e-7


def test_true_residual_restart_with_relaxed_inner_solves():
    """Loose inner solves (inner_relax = 1e-2): the outer loop is restarted
    until the TRUE Schur residual meets rtol, and U = K^-1 (F + G P) holds to
    the tight inner tolerance at the end."""
    prob, mat, ctx = _setup(16, 128, "discontinuous", "aniso")
    with ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(1)
        common = dict(want_cart=False, precision=1, schur_pc=1, rtol=1e-8, itmax=5000)
        _, _, _, r1 = ctx.solve(inner_relax=1e-2, true_residual=1, **common)
        _, _, _, r0 = ctx.solve(inner_relax=1e-2, true_residual=0, **common)
        Ut, Pt, _, rt = ctx.solve(want_cart=False, precision=1, schur_pc=1, rtol=1e-11, inner_rtol=1e-12, itmax=5000)
        U1, P1, _, _ = ctx.solve(inner_relax=1e-2, true_residual=1, **common)
    assert r1["status"] == 0 and r1["restarts"] >= 1
    assert r1["div_residual"] < 1e-8          # the true residual, not the recursive one
    assert r1["mom_residual"] < 1e-8          # U solves the momentum equation for the final P
    assert r0["mom_residual"] > 10 * r1["mom_residual"]
    assert rel(U1, Ut) < 1e-4 and rel(P1, Pt) < 1e-2   # a 1e-8 solution of this P2-P1disc problem
