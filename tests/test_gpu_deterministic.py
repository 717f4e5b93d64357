"""Deterministic mode (dp_set_deterministic): the scatters of the solve path
run as per-element results summed per node in a fixed order, so repeated
solves of the same inputs are identical bit for bit, iteration counts
included.  Against the atomic scatter the operators agree to rounding
(<= 1e-14 relative) and the converged solutions to the solve tolerance.
The reference's threaded assembly gets race freedom from element colouring
(src/Grid/coloring.jl:5-64, src/Stokes/AssemblerStokes.jl:94-96)."""
import numpy as np
import pytest

from conftest import rel
from dimspers_b200 import StokesContext, inputs

pytestmark = pytest.mark.gpu

FAST = dict(precision=1, cheb_degree=3, cheb_lo=0.05, inner_rtol=1e-10, inner_relax=1e-2, relax_base=1e-8,
            schur_pc=1)


def _ctx(nr, nt, kind="aniso", pressure="discontinuous", seed=3):
    ctx = StokesContext(nr, nt, pressure, pin_rotation=True)
    mat = inputs.make_material(ctx.mesh, kind, seed=seed)
    ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
    return ctx


def test_operators_match_the_atomic_scatter():
    with _ctx(16, 128) as ctx:
        ctx.assemble(1)
        rng = np.random.default_rng(7)
        x, p = rng.standard_normal(2 * ctx.nnod), rng.standard_normal(ctx.npres)
        ref = (ctx.apply_K(x), ctx.apply_G(p), ctx.rhs()[0])
        ctx.set_deterministic(True)
        ctx.assemble(1)
        got = (ctx.apply_K(x), ctx.apply_G(p), ctx.rhs()[0])
        again = (ctx.apply_K(x), ctx.apply_G(p))
    for name, a, b in zip(("K x", "G p", "F"), ref, got):
        assert rel(b, a) < 1e-14, (name, rel(b, a))
    assert np.array_equal(again[0], got[0]) and np.array_equal(again[1], got[1])


@pytest.mark.parametrize("opts", [dict(FAST), dict(precision=0, schur_pc=0, inner_rtol=1e-10)],
                         ids=["fast", "fp64"])
def test_repeated_solves_are_bit_identical(opts):
    runs = []
    with _ctx(32, 256) as ctx:
        ctx.set_deterministic(True)
        for _ in range(2):
            ctx.assemble(opts["precision"])
            U, P, _, r = ctx.solve(want_cart=False, rtol=1e-8, itmax=20000, **opts)
            runs.append((U, P, r))
    (U0, P0, r0), (U1, P1, r1) = runs
    assert r0["status"] == 0 and r1["status"] == 0
    assert r0["iterations"] == r1["iterations"] and r0["inner_iterations"] == r1["inner_iterations"]
    assert np.array_equal(U0, U1) and np.array_equal(P0, P1)


def test_deterministic_solution_matches_the_atomic_one():
    out = []
    with _ctx(32, 256) as ctx:
        for det in (False, True):
            ctx.set_deterministic(det)
            ctx.assemble(1)
            U, P, _, r = ctx.solve(want_cart=False, rtol=1e-11, inner_rtol=1e-12, itmax=20000, precision=1,
                                   schur_pc=1)
            assert r["status"] == 0
            out.append((U, P))
    assert rel(out[1][0], out[0][0]) < 1e-7 and rel(out[1][1], out[0][1]) < 1e-6


def test_refusals():
    with _ctx(8, 64, pressure="continuous") as ctx:
        with pytest.raises(Exception, match="discontinuous"):
            ctx.set_deterministic(True)
    with _ctx(8, 64) as ctx:
        ctx.set_deterministic(True)
        with pytest.raises(Exception, match="dp_assemble"):
            ctx.solve(want_cart=False)           # switching the mode on discards the assembly
        ctx.assemble(1)
        with pytest.raises(Exception, match="matrix_free"):
            ctx.solve(want_cart=False, precision=1, matrix_free=1)
        ctx.set_deterministic(False)
        _, _, _, r = ctx.solve(want_cart=False, precision=1, matrix_free=1, itmax=5000)
        assert r["status"] == 0
