"""The reference arm's cost model (oracle/refmodel.py) against oracle solves
that ran to completion (tests/golden/tight.json, "refsolve": the reference's
StokesPcCG with a SuperLU inner solve, lumped Schur preconditioner, rtol 1e-8,
on the seeded anisotropic workload at 32x256, 64x512 and 128x1024)."""
import json
import os

import pytest

from conftest import ROOT
from oracle import refmodel

GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def records():
    return json.load(open(os.path.join(GOLD, "tight.json")))["refsolve"]


def test_model_predicts_a_completed_solve_within_15_percent(records):
    v = refmodel.validate(records, "32x256_aniso", "64x512_aniso", "128x1024_aniso")
    assert abs(v["rel_error"]) <= 0.15, v


def test_per_iteration_cost_is_steady(records):
    """The model times a few outer iterations; over a whole solve the mean
    iteration time stays within 25 % of the first ones'."""
    for key, r in records.items():
        assert abs(r["iter_mean_s"] / r["iter_first3_s"] - 1.0) <= 0.25, (key, r)


def test_gpu_plain_path_takes_the_oracle_outer_count(records):
    """The outer count the model uses at sizes the oracle cannot finish is the
    plain FP64 GPU path's (the same algorithm); where both ran to completion
    the counts agree within 3 %."""
    gpu = json.load(open(os.path.join(GOLD, "outer_iterations.json")))
    ora = records["128x1024_aniso"]["outer"]
    assert abs(gpu["128x1024_discontinuous_aniso"] - ora) <= 0.03 * ora


def test_fit_and_predict_are_power_laws():
    a = dict(nr=8, nt=64, dof=refmodel._dof(8, 64), asm=1.0, setup=2.0, iter=0.1)
    b = dict(nr=16, nt=128, dof=refmodel._dof(16, 128), asm=2.0, setup=8.0, iter=0.2)
    f = refmodel.fit(a, b)
    p = refmodel.predict(f, 16, 128, 10)
    assert p["total"] == pytest.approx(2.0 + 8.0 + 10 * 0.2)
    q = refmodel.predict(f, 32, 256, 10)
    x = refmodel._dof(32, 256) / refmodel._dof(16, 128)
    assert q["setup"] == pytest.approx(8.0 * x ** f["p_setup"])
