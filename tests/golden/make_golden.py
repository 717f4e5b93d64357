"""Generate the golden fixtures of the oracle (test infrastructure).

The reference ships no tests or golden vectors (parity is unpinned), so these
fixtures pin the FP64 oracle against regressions and let the GPU tests check
the CUDA path without re-running the oracle.  Each fixture is one small
seeded case solved with the oracle's StokesPcCG restatement to rtol 1e-12.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dimspers_b200 import inputs  # noqa: E402
from oracle import mesh as OM  # noqa: E402
from oracle import solver as OS  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, ncr, nct, pressure, material kind, seed, schur preconditioner
    ("iso_4x32_cont", 4, 32, "continuous", "iso", 11, "lumped"),
    ("aniso_4x32_disc", 4, 32, "discontinuous", "aniso", 12, "lumped"),
    ("aniso_8x64_disc_mass", 8, 64, "discontinuous", "aniso", 13, "mass"),
    ("fabric_8x64_cont", 8, 64, "continuous", "fabric", 14, "lumped"),
]


class MeshView:
    def __init__(self, prob):
        self.theta, self.r, self.e2n = prob.gr.theta, prob.gr.r, prob.gr.e2n
        self.th_el, self.r_el = prob.th, prob.r


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    meta = {}
    for name, ncr, nct, pressure, kind, seed, spc in CASES:
        prob = OS.make_problem(ncr, nct, pressure, literal=True, pin_rotation=True)
        mat = inputs.make_material(MeshView(prob), kind, seed=seed)
        out = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-12, itmax=5000, schur_pc=spc)
        out8 = OS.solve_stokes(prob, mat.eta_ip, mat.rho, mat.g, mat.C6, rtol=1e-8, itmax=5000, schur_pc=spc)
        colors, _ = OM.color_mesh(prob.gr.e2n)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), U=out["U"], P=out["P"], U_raw=out["U_raw"],
                            omega=out["omega"], Ke0=out["mats"]["Ke"][:, :8], F=out["mats"]["F"])
        meta[name] = dict(nr_cells=ncr, ntheta_cells=nct, pressure=pressure, kind=kind, seed=seed, schur_pc=spc,
                          iterations_rtol12=out["report"].iterations, iterations_rtol8=out8["report"].iterations,
                          e2n_sha256=digest(prob.gr.e2n), colors_sha256=digest(colors.astype(np.int64)),
                          ncolors=int(colors.max()))
        print(name, meta[name]["iterations_rtol12"], meta[name]["iterations_rtol8"], flush=True)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
