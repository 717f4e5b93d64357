"""The benchmark workloads themselves against one yardstick: the FP64 oracle
(the reference's StokesPcCG with a direct LU inner solve) converged to rtol
1e-12, committed by tests/golden/make_tight.py.

Config 1 (32x256 isotropic, contrast 1e3, Ra 1e5, discontinuous P1, the
reference's temperature formula with seeded noise) and the 128x1024
anisotropic workload (contrast 1e5, delta ~ U[1,10], 8-mode director) are
solved on the GPU through the C ABI with
  * the plain FP64 path (the reference's algorithm: lumped-mass Schur
    preconditioner, inner solves to 1e-10 instead of LU), and
  * the fast path exactly as benchmarked (FP32 element data and multigrid
    under an FP64 Krylov, compensated Schur dots, element-mass Schur
    preconditioner, relaxed inner solves with true-residual restarts),
and each is compared with the yardstick.

What the oracle itself achieves sets the bars (tests/golden/tight.json):
  * two rtol-1e-8 oracle solves that differ only in the LU column ordering
    differ by ~7e-6 (U) and ~3e-6 (P) on config 1, and each is ~5e-6 (U) /
    ~1.3e-5 (P) from the rtol-1e-12 solution: at the reference's stopping
    rule the answer is only defined to ~1e-5 (the Schur complement of
    P2-P1disc on this mesh is ill-conditioned);
  * at rtol 1e-12 the same two orderings differ by 4.3e-10 (U), 1.3e-11 (P).
Tolerances:
  FP64 path, rtol 1e-12 vs yardstick   U, P <= 2e-9          (oracle floor 4.3e-10)
  either path, rtol 1e-8 vs yardstick  <= 3 x the oracle's own rtol-1e-8 error
                                       (config 1: ~5e-6 U, ~1.5e-5 P; 128x1024: 3.9e-5 U,
                                       9.0e-4 P)
  fast path, rtol 1e-11 vs yardstick   U, P <= 1e-7 on config 1 (the fast-path bar); at
                                       128x1024 U <= 1e-7 and P within 3x of FP64 with the
                                       same algorithm at the same tolerance
"""
import json
import os

import numpy as np
import pytest

from conftest import MeshView, rel
from dimspers_b200 import StokesContext, inputs
from oracle import solver as OS

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
META = json.load(open(os.path.join(GOLD, "tight.json")))

PLAIN = dict(precision=0, schur_pc=0, inner_rtol=1e-10, inner_relax=0.0)
FAST = dict(precision=1, schur_pc=1, inner_rtol=1e-10, inner_relax=1e-2, relax_base=1e-8, true_residual=1)


def _config1_ctx():
    prob = OS.make_problem(32, 256, "discontinuous", pin_rotation=True)
    mat = inputs.make_material(MeshView(prob), "iso", seed=1)
    ctx = StokesContext(32, 256, "discontinuous", pin_rotation=True)
    ctx.set_material(mat.eta_ip, mat.rho, mat.g, None)
    return ctx


@pytest.fixture(scope="module")
def config1():
    fx = np.load(os.path.join(GOLD, "config1_32x256_iso_disc.npz"))
    ctx = _config1_ctx()
    yield ctx, fx, META["config1"]
    ctx.close()


def _solve(ctx, arm, **kw):
    ctx.assemble(arm["precision"])
    U, P, _, rep = ctx.solve(**dict(arm, **kw), itmax=20000, want_cart=False)
    assert rep["status"] == 0, rep
    return U, P, rep


def test_config1_fp64_tight_matches_yardstick(config1):
    ctx, fx, meta = config1
    U, P, rep = _solve(ctx, PLAIN, rtol=1e-12, inner_rtol=1e-13)
    eu, ep = rel(U, fx["U"]), rel(P, fx["P"])
    print(f"config1 FP64 rtol1e-12: U {eu:.2e} P {ep:.2e} (oracle floor U {meta['noise_floor_rtol1e-12']['u']:.1e}"
          f" P {meta['noise_floor_rtol1e-12']['p']:.1e}), outer {rep['iterations']}")
    assert eu <= 2e-9 and ep <= 2e-9, (eu, ep)


def test_config1_fp64_at_reference_rule(config1):
    ctx, fx, meta = config1
    U, P, rep = _solve(ctx, PLAIN, rtol=1e-8)
    bu = 3 * max(meta["MMD_AT_PLUS_A_rtol1e-08"]["u_vs_tight"], meta["COLAMD_rtol1e-08"]["u_vs_tight"])
    bp = 3 * max(meta["MMD_AT_PLUS_A_rtol1e-08"]["p_vs_tight"], meta["COLAMD_rtol1e-08"]["p_vs_tight"])
    eu, ep = rel(U, fx["U"]), rel(P, fx["P"])
    print(f"config1 FP64 rtol1e-8: U {eu:.2e} P {ep:.2e} (bars {bu:.1e} {bp:.1e}); outer {rep['iterations']} "
          f"vs oracle {meta['MMD_AT_PLUS_A_rtol1e-08']['iterations']}")
    assert eu <= bu and ep <= bp, (eu, ep, bu, bp)
    # same algorithm, same stopping rule: the outer count within 5 % of the oracle's
    n_or = meta["MMD_AT_PLUS_A_rtol1e-08"]["iterations"]
    assert abs(rep["iterations"] - n_or) <= 0.05 * n_or, (rep["iterations"], n_or)


def test_config1_fast_at_reference_rule(config1):
    ctx, fx, meta = config1
    U, P, rep = _solve(ctx, FAST, rtol=1e-8)
    bu = 3 * max(meta["MMD_AT_PLUS_A_rtol1e-08"]["u_vs_tight"], meta["COLAMD_rtol1e-08"]["u_vs_tight"])
    bp = 3 * max(meta["MMD_AT_PLUS_A_rtol1e-08"]["p_vs_tight"], meta["COLAMD_rtol1e-08"]["p_vs_tight"])
    eu, ep = rel(U, fx["U"]), rel(P, fx["P"])
    print(f"config1 fast rtol1e-8: U {eu:.2e} P {ep:.2e} (bars {bu:.1e} {bp:.1e}); outer {rep['iterations']}")
    assert eu <= bu and ep <= bp, (eu, ep, bu, bp)


def test_config1_fast_tight_meets_1e7(config1):
    ctx, fx, meta = config1
    U, P, rep = _solve(ctx, FAST, rtol=1e-11, inner_rtol=1e-13, relax_base=1e-11)
    eu, ep = rel(U, fx["U"]), rel(P, fx["P"])
    print(f"config1 fast rtol1e-11: U {eu:.2e} P {ep:.2e}; outer {rep['iterations']}")
    assert eu <= 1e-7 and ep <= 1e-7, (eu, ep)


# ---- 128x1024 anisotropic (the secondary bench workload) -----------------------------
T128 = os.path.join(GOLD, "tight_128x1024_aniso.npz")


@pytest.fixture(scope="module")
def aniso128():
    if not os.path.exists(T128):
        pytest.skip("128x1024 yardstick not generated")
    fx = np.load(T128)
    mesh_ctx = StokesContext(128, 1024, "discontinuous", pin_rotation=True)
    mat = inputs.make_material(mesh_ctx.mesh, "aniso", seed=1)
    mesh_ctx.set_material_ti(mat.eta_ip, mat.rho, mat.g, mat.delta, mat.dir_x, mat.dir_y)
    yield mesh_ctx, fx
    mesh_ctx.close()


def _err_sub(U, P, fx):
    st = int(fx["stride"])
    return rel(U[::st], fx["U_sub"]), rel(P[::st], fx["P_sub"])


def test_aniso128_both_arms_at_reference_rule(aniso128):
    """At rtol 1e-8 the plain FP64 arm sits ~1e-5 from the yardstick (the
    problem's own floor, as on config 1); the fast arm is no further off."""
    ctx, fx = aniso128
    own = META["tight128"]["oracle_rtol1e-8_lumped_vs_tight"]   # the oracle's own rtol-1e-8 error
    U, P, rep = _solve(ctx, PLAIN, rtol=1e-8)
    eu64, ep64 = _err_sub(U, P, fx)
    print(f"128x1024 FP64 rtol1e-8: U {eu64:.2e} P {ep64:.2e} (oracle at rtol 1e-8: U {own['u']:.1e} "
          f"P {own['p']:.1e}); outer {rep['iterations']}")
    assert eu64 <= 3 * own["u"] and ep64 <= 3 * own["p"], (eu64, ep64, own)
    U, P, rep = _solve(ctx, FAST, rtol=1e-8)
    eu, ep = _err_sub(U, P, fx)
    print(f"128x1024 fast rtol1e-8: U {eu:.2e} P {ep:.2e}; outer {rep['iterations']}")
    assert eu <= 3 * eu64 + 1e-7 and ep <= 3 * ep64 + 1e-7, (eu, ep, eu64, ep64)


def test_aniso128_fast_tight_as_accurate_as_fp64(aniso128):
    """At rtol 1e-11 the fast path's U is within 1e-7 of the yardstick.  Its P
    is as close as FP64 with the same algorithm at the same tolerance gets: at
    128x1024 the pressure error is conditioning-limited (~1e5 x rtol for the
    oracle itself, 9.0e-4 at rtol 1e-8), so the bar for P is the FP64 solve's
    own error, not a fixed number."""
    ctx, fx = aniso128
    tight = dict(rtol=1e-11, inner_rtol=1e-13, relax_base=1e-11)
    U, P, rep = _solve(ctx, FAST, **tight)
    eu, ep = _err_sub(U, P, fx)
    U64, P64, rep64 = _solve(ctx, dict(FAST, precision=0), **tight)
    eu64, ep64 = _err_sub(U64, P64, fx)
    print(f"128x1024 rtol1e-11: fast U {eu:.2e} P {ep:.2e} (outer {rep['iterations']}); "
          f"FP64 same algorithm U {eu64:.2e} P {ep64:.2e} (outer {rep64['iterations']})")
    assert eu <= 1e-7, eu
    assert ep <= 3 * ep64 + 1e-7, (ep, ep64)
