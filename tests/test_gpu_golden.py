"""The CUDA path against the committed golden fixtures of the oracle (no oracle
run needed): U and P of small seeded cases solved to rtol 1e-12."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, rel
from dimspers_b200 import StokesContext, build_mesh, inputs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden")
META = json.load(open(os.path.join(GOLD, "golden.json")))


@pytest.mark.parametrize("name", sorted(META))
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_matches_golden(name, precision):
    m = META[name]
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    mesh = build_mesh(m["nr_cells"], m["ntheta_cells"], m["pressure"], pin_rotation=True)
    mat = inputs.make_material(mesh, m["kind"], seed=m["seed"])
    with StokesContext(m["nr_cells"], m["ntheta_cells"], m["pressure"], pin_rotation=True) as ctx:
        ctx.set_material(mat.eta_ip, mat.rho, mat.g, mat.C6)
        ctx.assemble(precision)
        U, P, _, rep = ctx.solve(precision=precision, rtol=1e-12, itmax=5000, inner_rtol=1e-13,
                                 schur_pc=1 if m["schur_pc"] == "mass" else 0)
    assert rep["status"] == 0, rep
    tol = (1e-9 if m["pressure"] == "continuous" else 1e-8) if precision == 0 else 1e-7
    assert rel(U, gold["U"]) < tol, rel(U, gold["U"])
    assert rel(P, gold["P"]) < tol, rel(P, gold["P"])
    assert abs(rep["iterations"] - m["iterations_rtol12"]) <= max(3, m["iterations_rtol12"] // 20)
