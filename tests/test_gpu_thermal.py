"""The thermal diffusion step (dp_thermal_step) against the oracle's
restatement of solveDiffusion_threaded (src/ThermalDiffusion/
AssemblerThermal.jl:1-57) with a direct solve."""
import numpy as np
import pytest

import oracle.solver as OS
import oracle.thermal as OT

pytestmark = pytest.mark.gpu


def _case(nr, nt, seed):
    prob = OS.make_problem(nr, nt, "continuous")
    gr = prob.gr
    rng = np.random.default_rng(seed)
    cond = 4000.0 + (300.0 - 4000.0) * np.log(gr.r / 1.22) / np.log(2.22 / 1.22)
    T = cond + 200.0 * np.sin(3 * gr.theta) * np.sin(np.pi * (gr.r - 1.22)) + 20.0 * rng.standard_normal(gr.nnod)
    rho = 3300.0 * (1.0 + 0.05 * rng.standard_normal(gr.nnod))
    return prob, T, rho


@pytest.mark.parametrize("heated", [1, 0])
def test_thermal_step_matches_oracle(heated):
    from dimspers_b200 import StokesContext
    prob, T, rho = _case(8, 64, 3 + heated)
    gr = prob.gr
    K, Cp, dt = 3.3, 1.2e3, 2e6
    fixed, tfix = OT.boundary(gr, 300.0, 4000.0, heated=bool(heated))
    ref = OT.thermal_step(gr, prob.th, prob.r, T, rho, K, Cp, dt, fixed, tfix)
    with StokesContext(8, 64, "continuous") as ctx:
        got, it, rel = ctx.thermal_step(T, rho, dt, K=K, Cp=Cp, heated=heated, rtol=1e-14, atol=0.0)
        loose, it2, rel2 = ctx.thermal_step(T, rho, dt, K=K, Cp=Cp, heated=heated)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-11
    assert np.array_equal(got[fixed], tfix)
    # the reference's default stopping test: ||r|| <= sqrt(eps) (1 + ||b||)
    assert 0 < it2 < it and rel2 <= 1.5e-8
    assert np.abs(loose - ref).max() / np.abs(ref).max() < 1e-5


def test_thermal_step_repeats_and_reports():
    from dimspers_b200 import StokesContext
    prob, T, rho = _case(16, 64, 9)
    with StokesContext(16, 64, "continuous") as ctx:
        a = ctx.thermal_step(T, rho, 1e6)
        b = ctx.thermal_step(T, rho, 1e6)
        # the element-by-element sums use atomics, so repeats agree to round-off, not bitwise
        assert np.abs(a[0] - b[0]).max() / np.abs(a[0]).max() < 1e-12 and abs(a[1] - b[1]) <= 1
        with pytest.raises(Exception):
            ctx.thermal_step(T, rho, 1e6, itmax=2)            # not converged
        with pytest.raises(Exception):
            ctx.thermal_step(T, rho, -1.0)                     # negative dt
        # dt = 0: the mass system returns T_old inside and the wall values on the walls
        T0, _, _ = ctx.thermal_step(T, rho, 0.0, rtol=1e-14, atol=0.0)
    fixed, tfix = OT.boundary(prob.gr, 300.0, 4000.0)
    inside = np.setdiff1d(np.arange(prob.gr.nnod), fixed)
    assert np.abs(T0[inside] - T[inside]).max() / np.abs(T).max() < 1e-2


def test_thermal_long_step_at_128x1024():
    """At the benchmark mesh a very long step is the steady conduction profile
    (the P2 error falls as h^4: 1.7e-5 K at 32x256, ~1e-7 K here; the bound
    leaves room for the solver's kappa * rtol), and the walls hold their values."""
    from dimspers_b200 import StokesContext
    with StokesContext(128, 1024, "continuous") as ctx:
        r = ctx.mesh.r
        T0 = np.full(ctx.nnod, 1000.0)
        T, it, rel = ctx.thermal_step(T0, np.ones(ctx.nnod), 1e9, K=1.0, Cp=1.0, rtol=1e-13, atol=0.0,
                                      itmax=200000)
    exact = 4000.0 + (300.0 - 4000.0) * np.log(r / 1.22) / np.log(2.22 / 1.22)
    assert np.abs(T - exact).max() < 5e-3
    assert np.all(T[r == r.max()] == 300.0) and np.all(T[r == r.min()] == 4000.0)
