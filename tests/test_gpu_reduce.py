"""The Schur-complement loop's compensated reductions (dp_reduce ops 1 and 3)
against exact sums.

The reference's mydot / mynorm (src/Algebra/Algebra.jl:104-113) and vmean
(src/IterativeSolvers.jl:172-186) are plain FP64 sums; the fast path keeps
these Schur-complement reductions in FP64 with double-double (TwoSum /
TwoProduct) accumulation.  The vectors below cancel heavily: pairs of products
of ~1e19 that annihilate, around a small remainder.  Every product a_i*b_i is
exact in FP64 (26-bit by 20-bit integer mantissas), so math.fsum of the
products is the correctly rounded exact dot."""
import math

import numpy as np
import pytest

from dimspers_b200 import StokesContext

pytestmark = pytest.mark.gpu


def _cancelling(n_pairs, n_small, seed):
    rng = np.random.default_rng(seed)
    big_a = rng.integers(1, 2 ** 26, n_pairs).astype(np.float64) * 2.0 ** 20
    big_b = rng.integers(1, 2 ** 20, n_pairs).astype(np.float64)
    sm_a = rng.integers(-2 ** 20, 2 ** 20, n_small).astype(np.float64) * 2.0 ** -30
    sm_b = rng.integers(1, 1000, n_small).astype(np.float64)
    a = np.concatenate([big_a, big_a, sm_a])
    b = np.concatenate([big_b, -big_b, sm_b])
    perm = rng.permutation(a.size)
    return a[perm], b[perm]


@pytest.fixture(scope="module")
def ctx():
    with StokesContext(4, 32, "discontinuous") as c:
        yield c


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_compensated_dot_is_exact_under_cancellation(ctx, seed):
    a, b = _cancelling(60_000, 5_000, seed)
    exact = math.fsum(a * b)            # every product is exact in FP64
    comp = ctx.reduce(a, b, compensated=True)
    plain = ctx.reduce(a, b, compensated=False)
    err_c = abs(comp - exact) / abs(exact)
    err_p = abs(plain - exact) / abs(exact)
    assert err_c <= 1e-14, (comp, exact, err_c)
    assert err_p > 1e3 * max(err_c, 1e-16), (err_p, err_c)   # the plain sum does lose it
    assert ctx.reduce(a, b, compensated=True) == comp      # bitwise reproducible


def test_compensated_sum_matches_fsum_over_16_decades(ctx):
    rng = np.random.default_rng(7)
    mags = 10.0 ** rng.uniform(-8, 8, 200_000)
    x = mags * rng.choice([-1.0, 1.0], mags.size)
    x = np.concatenate([x, -x[:150_000], [math.pi]])
    x = x[rng.permutation(x.size)]
    exact = math.fsum(x)
    comp = ctx.reduce(x, compensated=True)
    assert abs(comp - exact) <= 1e-14 * abs(exact), (comp, exact)


def test_compensated_and_plain_agree_on_benign_vectors(ctx):
    rng = np.random.default_rng(11)
    a, b = rng.standard_normal(1_000_003), rng.uniform(0.5, 1.5, 1_000_003)
    exact = math.fsum(np.concatenate([a * b, np.array([0.0])]))
    comp = ctx.reduce(a, b)
    plain = ctx.reduce(a, b, compensated=False)
    scale = np.abs(a * b).sum()
    assert abs(comp - plain) <= 1e-13 * scale
    assert abs(comp - exact) <= 1e-15 * scale
    assert ctx.reduce(np.zeros(0)) == 0.0
