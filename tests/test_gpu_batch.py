"""Batched solves (several contexts in one graph launch) against the same
problems solved one call each, the tile shapes of the element-by-element
apply, and the autotuner's record/replay."""
import json

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

TIGHT = dict(rtol=1e-11, inner_rtol=1e-12, itmax=5000)


def _ctx(nr, nt, pressure, kind, seed):
    from dimspers_b200 import StokesContext, inputs
    c = StokesContext(nr, nt, pressure)
    m = inputs.make_material(c.mesh, kind, seed=seed)
    if m.C6 is None:
        c.set_material(m.eta_ip, m.rho, m.g)
    else:
        c.set_material_ti(m.eta_ip, m.rho, m.g, m.delta, m.dir_x, m.dir_y)
    c.assemble(0)
    return c


def test_apply_tiles_agree():
    """Every tile shape (linear and theta-stacked CTAs) computes the same K x."""
    c = _ctx(32, 128, "discontinuous", "aniso", 3)
    with c:
        x = np.random.default_rng(0).standard_normal(2 * c.nnod)
        ys = []
        for w, wt in ((4, 1), (1, 1), (2, 2), (4, 4), (8, 2), (8, 8)):
            # a one-iteration solve sets the context's apply tile
            c.solve(want_cart=False, raise_on_status=False, itmax=1, itmin=1, apply_warps=w, apply_warps_t=wt)
            ys.append(c.apply_K(x))
        for y in ys[1:]:
            assert rel(y, ys[0]) < 1e-13


def test_tiled_solves_agree():
    c = _ctx(32, 128, "discontinuous", "aniso", 4)
    with c:
        out = [c.solve(want_cart=False, precision=1, schur_pc=1, apply_warps=w, apply_warps_t=wt, **TIGHT)
               for w, wt in ((4, 1), (4, 4), (8, 2))]
    for U, P, _, r in out:
        assert r["status"] == 0
    for U, P, _, r in out[1:]:
        assert rel(U, out[0][0]) < 1e-7 and rel(P, out[0][1]) < 1e-7


def _problems():
    return [(_ctx(8, 64, "discontinuous", "aniso", 11), dict(precision=1, schur_pc=1, **TIGHT)),
            (_ctx(32, 128, "discontinuous", "plumes", 12),
             dict(precision=1, schur_pc=1, apply_warps=4, apply_warps_t=4, cheb_degree=2, **TIGHT)),
            (_ctx(16, 64, "continuous", "iso", 13), dict(precision=0, coarse_max=256, **TIGHT))]


def _individual(probs):
    return [c.solve(want_cart=False, **o) for c, o in probs]


def _check(batch_out, ref, reports, done):
    for (U, P), (U0, P0, _, r0), rb in zip(batch_out, ref, reports):
        assert rb["status"] == 0 and r0["status"] == 0
        assert abs(rb["iterations"] - r0["iterations"]) <= max(3, r0["iterations"] // 50)
        assert rel(U, U0) < 1e-7 and rel(P, P0) < 1e-7
    assert np.all(done > 0)


def _run(b, probs, guesses=None):
    U = [np.zeros(2 * c.nnod) for c, _ in probs]
    P = [np.zeros(c.npres) for c, _ in probs]
    reps, done = b.run(guesses, U, P)
    return list(zip(U, P)), reps, done


def test_batch_matches_individual_solves():
    from dimspers_b200.batch import SolveBatch
    probs = _problems()
    ref = _individual(probs)
    with SolveBatch([c for c, _ in probs], [o for _, o in probs]) as b:
        for _ in range(2):  # the second launch reuses the instantiated graph
            out, reps, done = _run(b, probs)
            _check(out, ref, reps, done)
            assert all(r["kernel_launches"] > 0 for r in reps)
    for c, _ in probs:
        c.close()


def test_batch_follows_reassembly_and_reallocation():
    """New material on one problem, and a solve with another coarse size on
    another (which reallocates its hierarchy) between two batch launches."""
    from dimspers_b200 import inputs
    from dimspers_b200.batch import SolveBatch
    probs = _problems()
    with SolveBatch([c for c, _ in probs], [o for _, o in probs]) as b:
        _run(b, probs)
        c0 = probs[0][0]
        m = inputs.make_material(c0.mesh, "aniso", seed=99)
        c0.set_material_ti(m.eta_ip, m.rho, m.g, m.delta, m.dir_x, m.dir_y)
        c0.assemble(0)
        probs[1][0].solve(want_cart=False, raise_on_status=False, precision=1, coarse_max=64, rtol=1e-4, itmax=50)
        out, reps, done = _run(b, probs)
        ref = _individual(probs)
        _check(out, ref, reps, done)
    for c, _ in probs:
        c.close()


def test_batch_guess_and_bad_args():
    from dimspers_b200._lib import check, lib
    from dimspers_b200.batch import SolveBatch
    probs = _problems()
    # guesses: solutions of a looser solve; the reference is the individual
    # solve from the same guess (same stopping test relative to that start)
    guesses = [c.solve(want_cart=False, **dict(o, rtol=1e-4))[1] for c, o in probs]
    ref = [c.solve(want_cart=False, P0=g, **o) for (c, o), g in zip(probs, guesses)]
    opts = [dict(o, use_guess=1) for _, o in probs]
    with SolveBatch([c for c, _ in probs], opts) as b:
        out, reps, done = _run(b, probs, guesses)
    _check(out, ref, reps, done)
    with pytest.raises(Exception):
        SolveBatch([probs[0][0], probs[0][0]])          # a context twice
    with pytest.raises(Exception):
        SolveBatch([probs[0][0]], [dict(host_loop=1)])  # host loops are not batched
    with pytest.raises(Exception):
        with SolveBatch([probs[0][0]], [dict(use_guess=1)]) as b:
            b.run(None, None, None)                     # guess missing
    for c, _ in probs:
        c.close()


def test_autotune_records_and_replays(tmp_path):
    from dimspers_b200 import batch
    c = _ctx(32, 256, "discontinuous", "aniso", 21)
    space = dict(apply=((4, 1), (4, 4)), cheb_degree=(2, 3), coarse_max=(1024,))
    path = str(tmp_path / "tune.json")
    with c:
        table = batch.tune_all([c], path, outer_its=5, reps=1, space=space)
        key = batch.tuning_key(c)
        assert key == "32x256/discontinuous" and table[key]["trials"] == 4
        assert json.load(open(path)) == table
        o = batch.tuned_opts(c, batch.load_tuning(path))
        assert (o["apply_warps"], o["apply_warps_t"], o["cheb_degree"]) == \
            (table[key]["apply_warps"], table[key]["apply_warps_t"], table[key]["cheb_degree"])
        U, P, _, r = c.solve(want_cart=False, itmax=5000, **o)
        assert r["status"] == 0


@pytest.mark.parametrize("precision", [0, 1])
def test_cluster_tail_matches_separate_levels(precision):
    """The V-cycle's small levels as one cluster kernel (mg_tail) give the
    solve of the separate level kernels."""
    c = _ctx(32, 128, "discontinuous", "aniso", 7)
    with c:
        U0, P0, _, r0 = c.solve(want_cart=False, precision=precision, schur_pc=1, **TIGHT)
        for tail in (1024, 16384):
            U1, P1, _, r1 = c.solve(want_cart=False, precision=precision, schur_pc=1, mg_tail=tail, **TIGHT)
            assert r1["status"] == 0
            assert abs(r1["iterations"] - r0["iterations"]) <= max(3, r0["iterations"] // 50)
            assert rel(U1, U0) < 1e-7 and rel(P1, P0) < 1e-7
