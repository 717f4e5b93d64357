"""Size-independent properties at the benchmark's full size (512x4096 cells:
4,194,304 elements, 16,793,600 velocity DOF, 12,582,912 pressure DOF), where
the oracle cannot run: the assembled operator is symmetric, G and G^T are
adjoint to each other, and the hydrostatic manufactured state (uniform rho
and eta under the radial body force: u = 0, p = g rho r + const; the oracle
KAT checks it converges at high order, tests/test_oracle_kat.py) comes out of
the fast solve.  All through the C ABI."""
import numpy as np
import pytest

from dimspers_b200 import StokesContext, inputs

pytestmark = pytest.mark.gpu

NR, NT = 512, 4096


@pytest.fixture(scope="module")
def fabric_ctx():
    ctx = StokesContext(NR, NT, "discontinuous", pin_rotation=True)
    mat = inputs.make_material(ctx.mesh, "fabric", seed=1)
    ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
    ctx.assemble(0)
    yield ctx
    ctx.close()


def test_full_size_operator_is_symmetric(fabric_ctx):
    ctx = fabric_ctx
    rng = np.random.default_rng(0)
    x, y = rng.standard_normal(2 * ctx.nnod), rng.standard_normal(2 * ctx.nnod)
    Kx, Ky = ctx.apply_K(x), ctx.apply_K(y)
    a, b = float(x @ Ky), float(y @ Kx)
    scale = np.linalg.norm(x) * np.linalg.norm(Ky)
    assert abs(a - b) <= 1e-12 * scale, (a, b, scale)


def test_full_size_G_and_GT_are_adjoint(fabric_ctx):
    ctx = fabric_ctx
    rng = np.random.default_rng(1)
    y, p = rng.standard_normal(2 * ctx.nnod), rng.standard_normal(ctx.npres)
    Gp, GTy = ctx.apply_G(p), ctx.apply_GT(y)
    a, b = float(y @ Gp), float(p @ GTy)
    scale = np.linalg.norm(y) * np.linalg.norm(Gp)
    assert abs(a - b) <= 1e-12 * scale, (a, b, scale)


def test_full_size_hydrostatic_state():
    g, rho = 1.5, 2.0
    with StokesContext(NR, NT, "discontinuous", pin_rotation=True) as ctx:
        ctx.set_material(np.ones((ctx.nel, 7)), np.full(ctx.nnod, rho), g, None)
        ctx.assemble(1)
        U, P, _, rep = ctx.solve(precision=1, schur_pc=1, inner_relax=1e-2, relax_base=1e-12, rtol=1e-12,
                                 inner_rtol=1e-13, itmax=20000, want_cart=False)
        assert rep["status"] == 0, rep
        m = ctx.mesh
        rp = m.r[m.e2n[:3]].T.ravel()          # r of the vertex of each discontinuous P DOF (3e + k)
    A = np.vstack([rp, np.ones_like(rp)]).T
    coef = np.linalg.lstsq(A, P, rcond=None)[0]
    print(f"512x4096 hydrostatic: outer {rep['iterations']}, max|U| {np.abs(U).max():.2e}, dp/dr {coef[0]:.10f}, "
          f"max|P - fit| {np.abs(P - A @ coef).max():.2e}")
    assert abs(coef[0] - g * rho) < 1e-7 * g * rho
    assert np.abs(P - A @ coef).max() < 1e-6 * np.abs(P).max()
    assert np.abs(U).max() < 1e-7 * g * rho
