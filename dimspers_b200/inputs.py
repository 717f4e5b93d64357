"""Seeded synthetic material inputs for the annulus Stokes workloads.

The reference draws its perturbations from Julia's unseeded ``rand()``
(src/Setup/Setup.jl:86-88), which cannot be reproduced.  These generators use
one counter-based SplitMix64 stream instead, so the oracle and the CUDA path
receive bit-identical arrays.  Arrays follow the reference's layouts:

  eta_ip  (nel, 7) float64, element-fastest (``eta.ip``, Rheology.jl:352-359);
          the 6 Stokes IPs are columns 0..5, column 6 holds the centroid value
  C6      tuple of six (nel, 7) arrays in StiffnessTensor order
          (C11, C33, C55, C13, C15, C35)  (anisotropy.jl:1-8)
  rho     (nnod,) nodal density; body force g*rho*r_hat (StokesSolver.jl:838-845)

Workloads (all on r in [1.22, 2.22], free slip, rotation removed):
  iso      T = conductive + 0.01 cos(4 theta) sin(pi (r - r_in)) + U(+-1e-3);
           eta = exp(-ln(contrast) T), contrast 1e3, Ra = 1e5 (rho = T, g = Ra)
  aniso    same T, contrast 1e5; transversely isotropic tensor with weak-plane
           shear viscosity 1/delta, delta ~ U[1, 10] per element; director angle
           = sum of 8 Fourier modes in (theta, r) with seeded phases
  fabric   contrast 1e6; director = major eigenvector of F F^T per element,
           F = I + 0.5 G, G a seeded smooth 2x2 field (8 modes per component)
  plumes   training workload of the learned guess: conductive profile plus
           1-16 Gaussian plumes (radius 0.05-0.2, amplitude +-0.3, random
           centres), Ra log-uniform in [1e5, 1e7], contrast 1e5, delta and
           director as `aniso`
"""
from dataclasses import dataclass

import numpy as np

R_IN, R_OUT = 1.22, 2.22
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    """SplitMix64 finaliser on a uint64 array (Steele, Lea, Flood 2014)."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def uniform(seed, stream, n):
    """n uniforms in [0, 1): counter c -> splitmix64(seed * 2^32 + stream * 2^48 + c)."""
    base = (np.uint64(seed) << np.uint64(32)) ^ (np.uint64(stream) << np.uint64(48))
    c = np.arange(n, dtype=np.uint64) + base
    return (splitmix64(c) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


# 6-point rule (same formulas as the Stokes assembly) + centroid, for T -> eta at IPs
def _ip7():
    g1 = (8.0 - np.sqrt(10.0) + np.sqrt(38.0 - 44.0 * np.sqrt(2.0 / 5.0))) / 18.0
    g2 = (8.0 - np.sqrt(10.0) - np.sqrt(38.0 - 44.0 * np.sqrt(2.0 / 5.0))) / 18.0
    return np.array([[1 - 2 * g1, g1], [g1, 1 - 2 * g1], [g1, g1],
                     [1 - 2 * g2, g2], [g2, 1 - 2 * g2], [g2, g2], [1 / 3, 1 / 3]])


def _p2(r, s):
    t = 1.0 - r - s
    return np.array([t * (2 * t - 1), r * (2 * r - 1), s * (2 * s - 1), 4 * r * t, 4 * r * s, 4 * s * t])


N7 = np.stack([_p2(*p) for p in _ip7()])        # (7, 6)
N3_7 = np.stack([[1 - p[0] - p[1], p[0], p[1]] for p in _ip7()])


@dataclass
class Material:
    eta_ip: np.ndarray
    rho: np.ndarray
    g: float
    C6: tuple = None          # full tensor fields, or None (isotropic)
    delta: np.ndarray = None  # per element (transversely isotropic form)
    dir_x: np.ndarray = None
    dir_y: np.ndarray = None
    T: np.ndarray = None


def temperature(theta, r, seed, amp_noise=1e-3):
    T = np.log(r / R_OUT) / np.log(R_IN / R_OUT) + 0.01 * np.cos(4 * theta) * np.sin(np.pi * (r - R_IN))
    T = T + amp_noise * (2.0 * uniform(seed, 1, theta.size) - 1.0)
    return T


def plume_temperature(theta, r, seed):
    u = uniform(seed, 5, 1 + 5 * 16)
    nplume = 1 + int(u[0] * 16)
    T = np.log(r / R_OUT) / np.log(R_IN / R_OUT)
    x, z = r * np.sin(theta), r * np.cos(theta)
    for k in range(nplume):
        a, b, c, d, e = u[1 + 5 * k: 6 + 5 * k]
        th_c = 2 * np.pi * a
        r_c = R_IN + 0.1 + 0.8 * b
        rad = 0.05 + 0.15 * c
        amp = 0.3 * (2 * d - 1)
        xc, zc = r_c * np.sin(th_c), r_c * np.cos(th_c)
        T = T + amp * np.exp(-((x - xc) ** 2 + (z - zc) ** 2) / (rad * rad))
    return T


def eta_from_T(T, e2n, contrast):
    Tip = N7 @ T[e2n[:6]]                       # (7, nel)
    return np.ascontiguousarray(np.exp(-np.log(contrast) * Tip).T)


def centroids(th_el, r_el):
    return th_el.mean(axis=0), r_el.mean(axis=0)


def fourier_field(theta, r, seed, stream, nmodes=8):
    """sum_m (1/m) cos(m theta + (1 + m mod 3) pi rho + 2 pi u_m), rho = (r-r_in)/(r_out-r_in)."""
    ph = uniform(seed, stream, nmodes)
    rho = (r - R_IN) / (R_OUT - R_IN)
    f = np.zeros_like(theta)
    for m in range(1, nmodes + 1):
        f += np.cos(m * theta + (1 + m % 3) * np.pi * rho + 2 * np.pi * ph[m - 1]) / m
    return f


def ti_tensor(delta, dir_x, dir_y):
    """Transversely isotropic viscous tensor: frame a = c = 4/3, h = -2/3,
    e = 1/delta, rotated by the director with the 2D fourth-order tensor
    rotation of src/Rheology/anisotropy.jl:503-536 (rotmatrix :287-292)."""
    a = c = 4.0 / 3.0
    h = -2.0 / 3.0
    e = 1.0 / delta
    inv = 1.0 / np.sqrt(dir_y * dir_y + dir_x * dir_x)
    cs, sn = dir_x * inv, dir_y * inv
    x1 = y2 = cs
    x2 = sn
    y1 = -sn
    x1x1, x2x2, y1y1, y2y2 = x1 * x1, x2 * x2, y1 * y1, y2 * y2
    n11 = (c * x2x2 + h * x1x1 + 4 * e * x1x1) * x2x2 + (a * x1x1 + h * x2x2) * x1x1
    n33 = (c * y2y2 + h * y1y1 + 4 * e * y1y1) * y2y2 + (a * y1y1 + h * y2y2) * y1y1
    n55 = ((c * x2 * y2 + h * x1 * y1) * x2 * y2 + (x1 * y2 + x2 * y1) * (x1 * y2 + x2 * y1) * e
           + (a * x1 * y1 + h * x2 * y2) * x1 * y1)
    n13 = ((c * x2x2 + h * x1x1) * y2 + 4 * e * x1 * x2 * y1) * y2 + (a * x1x1 + h * x2x2) * y1y1
    n15 = ((c * x2x2 + h * x1x1) * y2 + 2 * (x1 * y2 + x2 * y1) * e * x1) * x2 + (a * x1x1 + h * x2x2) * x1 * y1
    n35 = ((c * y2y2 + h * y1y1) * x2 + 2 * (x1 * y2 + x2 * y1) * e * y1) * y2 + (a * y1y1 + h * y2y2) * x1 * y1
    return n11, n33, n55, n13, n15, n35


def _tile7(v):
    return np.ascontiguousarray(np.repeat(v[:, None], 7, axis=1))


def make_material(mesh, kind="iso", seed=1, Ra=1e5, contrast=None):
    """mesh: object with theta, r (nodal), e2n (6, nel) 0-based, th_el, r_el (3, nel)."""
    if kind == "plumes":
        T = plume_temperature(mesh.theta, mesh.r, seed)
        Ra = float(10.0 ** (5.0 + 2.0 * uniform(seed, 6, 1)[0]))
    else:
        T = temperature(mesh.theta, mesh.r, seed)
    nel = mesh.e2n.shape[1]
    if kind == "iso":
        eta = eta_from_T(T, mesh.e2n, contrast or 1e3)
        return Material(eta_ip=eta, rho=T.copy(), g=Ra, T=T)
    thc, rc = centroids(mesh.th_el, mesh.r_el)
    delta = 1.0 + 9.0 * uniform(seed, 2, nel)
    if kind in ("aniso", "plumes"):
        eta = eta_from_T(T, mesh.e2n, contrast or 1e5)
        phi = fourier_field(thc, rc, seed, 3)
        dx, dy = np.cos(phi), np.sin(phi)
    elif kind == "fabric":
        eta = eta_from_T(T, mesh.e2n, contrast or 1e6)
        G = [fourier_field(thc, rc, seed, 4 + k) for k in range(4)]
        F = np.stack([1.0 + 0.5 * G[0], 0.5 * G[1], 0.5 * G[2], 1.0 + 0.5 * G[3]])  # F11 F12 F21 F22
        dx, dy = major_eigvec_FFt(F)
    else:
        raise ValueError(kind)
    C = ti_tensor(delta, dx, dy)
    return Material(eta_ip=eta, rho=T.copy(), g=Ra, C6=tuple(_tile7(c) for c in C),
                    delta=delta, dir_x=dx, dir_y=dy, T=T)


def major_eigvec_FFt(F):
    """Unit eigenvector of the larger eigenvalue of L = F F^T per element
    (src/Stress/FSE.jl:143-161, eigval_order :189).  F rows: F11, F12, F21, F22."""
    f11, f12, f21, f22 = F
    l11 = f11 * f11 + f12 * f12
    l12 = f11 * f21 + f12 * f22
    l22 = f21 * f21 + f22 * f22
    half_tr = 0.5 * (l11 + l22)
    disc = np.sqrt(0.25 * (l11 - l22) ** 2 + l12 * l12)
    lmax = half_tr + disc
    # eigenvector from the better-conditioned row of (L - lmax I)
    ax, ay = l12, lmax - l11
    bx, by = lmax - l22, l12
    use_a = (ax * ax + ay * ay) >= (bx * bx + by * by)
    vx = np.where(use_a, ax, bx)
    vy = np.where(use_a, ay, by)
    nrm = np.sqrt(vx * vx + vy * vy)
    iso = nrm == 0
    vx = np.where(iso, 1.0, vx / np.where(iso, 1.0, nrm))
    vy = np.where(iso, 0.0, vy / np.where(iso, 1.0, nrm))
    return vx, vy
