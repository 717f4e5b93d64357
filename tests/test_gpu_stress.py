"""The strain-rate / stress post-processor (dp_stress) against the oracle's
restatement of stress! (src/Stress/StressCalculation.jl:23-249)."""
import numpy as np
import pytest

from conftest import MeshView, rel

import oracle.solver as OS
import oracle.stress as ST

pytestmark = pytest.mark.gpu


def _max_rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("kind", ["iso", "aniso"])
def test_stress_matches_oracle_on_a_smooth_field(kind):
    from dimspers_b200 import StokesContext, inputs
    prob = OS.make_problem(8, 64, "discontinuous")
    mat = inputs.make_material(MeshView(prob), kind, seed=4)
    th, r = prob.gr.theta, prob.gr.r
    x, z = r * np.sin(th), r * np.cos(th)
    U = np.zeros(2 * th.size)
    U[0::2] = np.sin(3 * th) * (r - 1.22) + 0.3 * z
    U[1::2] = np.cos(2 * th) * (2.22 - r) ** 2 - 0.1 * x
    with StokesContext(8, 64, "discontinuous") as ctx:
        got = ctx.stress(U, mat.eta_ip, mat.C6)
    ref = ST.stress(U, mat.eta_ip, prob.th, prob.r, prob.gr.e2n, mat.C6)
    for k in ST.NAMES:
        assert _max_rel(got[k], ref[k]) < 1e-12, (k, _max_rel(got[k], ref[k]))


def test_stress_of_a_solve_matches_oracle():
    """The post-processor on the solver's own Cartesian velocity (MAIN.jl:241-243)."""
    from dimspers_b200 import StokesContext, inputs
    prob = OS.make_problem(8, 64, "discontinuous")
    mat = inputs.make_material(MeshView(prob), "aniso", seed=6)
    with StokesContext(8, 64, "discontinuous") as ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(1)
        U, P, Ucart, rep = ctx.solve(precision=1, schur_pc=1, rtol=1e-10, itmax=5000)
        got = ctx.stress(Ucart, mat.eta_ip, mat.C6)
    assert rep["status"] == 0
    ref = ST.stress(Ucart, mat.eta_ip, prob.th, prob.r, prob.gr.e2n, mat.C6)
    for k in ST.NAMES:
        assert _max_rel(got[k], ref[k]) < 1e-12, k
    assert np.all(got["eII"] >= 0) and np.all(got["tII"] >= 0)


def test_arrhenius_viscosity_update_matches_oracle():
    """getviscosity!(::Arrhenius) on dimensional inputs: every branch (depth
    zones, clamps, plastic yield, plastic-but-not-yielding kept, no cohesion)."""
    from dimspers_b200 import StokesContext
    import oracle.rheology as RH
    prob = OS.make_problem(8, 64, "continuous")
    nel, nn = prob.th.shape[1], prob.gr.r.size
    nv = 9 * 64
    rng = np.random.default_rng(11)
    r = 3.48e6 + (prob.gr.r - 1.22) * 2.87e6           # radius in m: all three depth zones
    T = 1300.0 + 1200.0 * rng.random(nn)
    P = 2e9 * rng.standard_normal(nv)
    eps = np.abs(rng.standard_normal((nel, 7))) * 1e-15
    eps[::5] = 0.0                                     # no strain rate: the non-plastic branch
    tau = 4e9 * rng.random((nel, 7))
    coh = np.where(rng.random((nel, 7)) < 0.3, 0.0, 30e6)
    eta0 = np.full((nel, 7), 3.3e21)
    law = dict(eta0=5e20, R=8.314, Ea=100e3, Va=1e-6, T0=1600.0, phi=30.0)
    ref = RH.arrhenius_viscosity(eta0, T, P, r, prob.gr.e2n, eps, tau, coh, law["eta0"], law["R"], law["Ea"],
                                 law["Va"], law["T0"], law["phi"])
    with StokesContext(8, 64, "continuous") as ctx:
        got = ctx.viscosity_arrhenius(eta0, T, P, r, eps, tau, coh, **law)
    assert np.abs(got / ref - 1).max() < 1e-12
    kept = ref == 3.3e21
    assert kept.any() and (ref == 1e18).any() and (~kept & (ref > 1e18)).any()


def test_stress_properties_at_128x1024():
    """Size-independent properties at the benchmark mesh: a rigid rotation
    (u = omega x r) has no strain rate and a Cartesian-linear field has its
    constant strain rate and stress, up to the second-order error of the P2
    space on elements straight in (theta, r) (6.1e-4 and 1.3e-3 at 8x64, 4x
    less per refinement: ~2.4e-6 and 5e-6 here)."""
    from dimspers_b200 import StokesContext, build_mesh
    mesh = build_mesh(128, 1024, "discontinuous", colors=False)
    x, z = mesh.r * np.sin(mesh.theta), mesh.r * np.cos(mesh.theta)
    eta = np.full((mesh.nel, 7), 2.0)
    with StokesContext(128, 1024, "discontinuous") as ctx:
        U = np.zeros(2 * mesh.nnod)
        U[0::2], U[1::2] = 0.7 * z, -0.7 * x                   # rigid rotation
        rot = ctx.stress(U, eta)
        U[0::2], U[1::2] = 0.3 * x + 0.2 * z, 0.5 * x - 0.3 * z  # exx = 0.3, ezz = -0.3, exz = 0.35
        lin = ctx.stress(U, eta)
    assert max(np.abs(rot[k]).max() for k in ("exx", "ezz", "exz", "eII")) < 1e-5
    for k, v in (("exx", 0.3), ("ezz", -0.3), ("exz", 0.35)):
        assert np.abs(lin[k] - v).max() < 1e-5, k
    assert np.abs(lin["txx"] - 2.0 * (4 / 3 * 0.3 + 2 / 3 * 0.3)).max() < 2e-5
    assert np.abs(lin["txz"] - 2.0 * 2 * 0.35).max() < 2e-5
