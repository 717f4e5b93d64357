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
