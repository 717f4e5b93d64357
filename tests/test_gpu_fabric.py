"""Per-IP finite-strain ellipsoid (dp_fse) and DEM viscous tensor
(dp_anisotropic_tensor) against the oracle's restatements of _FSE
(src/Stress/FSE.jl:143-161) and anisotropic_tensor (src/Rheology/
anisotropy.jl:140-285), on the reference's own DEM tables."""
import os

import numpy as np
import pytest

from conftest import ROOT

import oracle.fabric as OF

pytestmark = pytest.mark.gpu

NR, NT = 8, 64


def _dem(vol=30):
    d = np.load(os.path.join(ROOT, "tests", "golden", "dem_1e-3_vol%d.npz" % vol))
    return d["C"], d["ax"]


def _deformation(nel, seed):
    """Seeded F per IP: rotations of stretches, a few identities and shears."""
    rng = np.random.default_rng(seed)
    ang = rng.uniform(-np.pi, np.pi, (nel, 6))
    s1 = np.exp(rng.uniform(0, 4, (nel, 6)))
    s2 = np.exp(-rng.uniform(0, 2, (nel, 6)))
    c, s = np.cos(ang), np.sin(ang)
    R = np.stack([np.stack([c, -s], -1), np.stack([s, c], -1)], -2)
    F = R @ (np.eye(2) * np.stack([s1, s2], -1)[..., None, :])
    F[::17] = np.eye(2)                                       # undeformed
    F[5::23] = np.array([[1.0, 3.0], [0.0, 1.0]])             # simple shear
    return F


def test_fse_matches_oracle():
    from dimspers_b200 import StokesContext
    with StokesContext(NR, NT, "continuous") as ctx:
        F = _deformation(ctx.nel, 1)
        got = ctx.fse(F)
    x1, x2, y1, y2, a1, a2 = OF.fse(F)
    assert np.abs(got["a1"] / a1 - 1).max() < 1e-12
    assert np.abs(got["a2"] / a2 - 1).max() < 1e-9          # minor axis of stretches up to e^6
    # eigenvectors agree up to sign
    assert np.abs(np.abs(got["vx1"] * x1 + got["vy1"] * y1) - 1).max() < 1e-12
    assert np.abs(np.abs(got["vx2"] * x2 + got["vy2"] * y2) - 1).max() < 1e-12
    und = np.all(F == np.eye(2), axis=(-2, -1))                # the undeformed IPs
    assert und.any()
    assert np.all(got["vx1"][und] == 1.0) and np.all(got["vy1"][und] == 0.0)


@pytest.mark.parametrize("vol", [10, 30])
def test_dem_tensor_matches_oracle(vol):
    from dimspers_b200 import StokesContext
    from dimspers_b200.fabric import DEM
    C6, ax = _dem(vol)
    w = 0.02
    dem = DEM(C6, ax, w)
    t = OF.dem_tables(C6, ax)
    with StokesContext(NR, NT, "continuous") as ctx:
        nel = ctx.nel
        rng = np.random.default_rng(vol)
        # shapes over and beyond the table's range (both ends clamp to a row)
        r1 = rng.uniform(-0.3, 2.0, (nel, 6))
        r2 = rng.uniform(-0.3, 2.3, (nel, 6))
        r1[::7, 0] = t["a1a2_blk"][3]                          # exactly on table points
        r2[::7, 0] = t["a2a3_blk"][5]
        F = _deformation(nel, 2)
        fse = ctx.fse(F)
        got = ctx.anisotropic_tensor(dem, fse["vx1"], fse["vy1"], r1, r2)
    ref = OF.anisotropic_tensor(fse["vx1"], fse["vy1"], r1, r2, t, w)
    for f in range(6):
        scale = np.abs(ref[f]).max()
        assert np.abs(got[f] - ref[f]).max() < 1e-13 * max(scale, 1.0), f
    assert np.all(got[2] >= w)


def test_dem_tensor_rejects_bad_tables():
    from dimspers_b200 import StokesContext
    from dimspers_b200.fabric import DEM
    C6, ax = _dem()
    z = np.zeros((NR * NT * 2, 6))
    with StokesContext(NR, NT, "continuous") as ctx:
        bad = DEM(C6, ax, 0.02)
        bad.permutation_blk = bad.permutation_blk.copy()
        bad.permutation_blk[3] = 11                             # outside 1..sblk
        with pytest.raises(Exception):
            ctx.anisotropic_tensor(bad, z + 1, z, z, z)
        short = DEM(C6[:50], ax[:50], 0.02)
        short.a1a2_blk = np.ascontiguousarray(np.linspace(0, 1, 10))   # 10 blocks of 10 > 50 rows
        with pytest.raises(Exception):
            ctx.anisotropic_tensor(short, z + 1, z, z, z)
