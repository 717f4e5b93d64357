"""Strain-rate / stress post-processor (FP64 restatement; test infrastructure).

Follows src/Stress/StressCalculation.jl:
  _stress! (isotropic)    :23-127   per element and 7-point IP: curved inverse
                                    Jacobian, dN/dx, dN/dz (the same geometry as
                                    the Stokes assembly), strain rate of the
                                    Cartesian velocity, eII, deviatoric stress, tII
  _stress! (anisotropic)  :129-242  the stress from the rotated tensor, with the
                                    reference's own factors (tau_xx and tau_xz
                                    take eta * e_xz, tau_zz takes 2 eta * e_xz)
  stress!                 :244-249  loop over elements; MAIN.jl:241-243 calls it
                                    with Ucart, nip = 7 (MAIN.jl:94, :164)
Shape functions: ip_triangle7 (Quadrature.jl:109-138), sf_dN_tri6 at those
points, linear N3 (stress_shape_functions, AssemblerStokes.jl:303-311).
"""
import numpy as np

from .quadrature import DN3DS, ip_triangle7, sf_dN_tri6, sf_N_tri3

NAMES = ("exx", "ezz", "exz", "eII", "txx", "tzz", "txz", "tII")


def stress(Ucart, eta_ip, th, r, e2n, C6=None):
    """Ucart (2*nnod,) interleaved [ux, uz] per node (reference numbering);
    eta_ip (nel, >=7); th, r (3, nel) seam-fixed vertex coordinates; e2n (6,
    nel) 0-based; C6: None (isotropic) or six (nel, >=7) fields in
    StiffnessTensor order (C11, C33, C55, C13, C15, C35).
    Returns {name: (nel, 7)} for NAMES."""
    ipx, _ = ip_triangle7()
    nel = th.shape[1]
    ux = Ucart[0::2][e2n]                          # (6, nel)
    uz = Ucart[1::2][e2n]
    J_th = th.T @ DN3DS.T
    J_r = r.T @ DN3DS.T
    detJ = J_th[:, 0] * J_r[:, 1] - J_th[:, 1] * J_r[:, 0]
    invdet = 1.0 / detJ
    R21, R31 = r[1] - r[0], r[2] - r[0]
    T31, T21 = th[2] - th[0], th[1] - th[0]
    out = {k: np.zeros((nel, 7)) for k in NAMES}
    for ip in range(7):
        N3 = sf_N_tri3(*ipx[ip])
        dN = sf_dN_tri6(*ipx[ip])                  # (2, 6)
        th_ip = N3 @ th
        r_ip = N3 @ r
        s, c = np.sin(th_ip), np.cos(th_ip)
        cr, sr = c / r_ip, s / r_ip
        a11 = R31 * cr - T31 * s
        a12 = -R21 * cr + T21 * s
        a21 = -R31 * sr - T31 * c
        a22 = R21 * sr + T21 * c
        dx = (a11[:, None] * dN[0][None, :] + a12[:, None] * dN[1][None, :]) * invdet[:, None]   # (nel, 6)
        dz = (a21[:, None] * dN[0][None, :] + a22[:, None] * dN[1][None, :]) * invdet[:, None]
        exx = np.einsum("ek,ke->e", dx, ux)
        ezz = np.einsum("ek,ke->e", dz, uz)
        duxdz = np.einsum("ek,ke->e", dz, ux)
        duzdx = np.einsum("ek,ke->e", dx, uz)
        exz = 0.5 * (duxdz + duzdx)
        eta = eta_ip[:, ip]
        if C6 is None:
            txx = eta * (4.0 / 3.0 * exx - 2.0 / 3.0 * ezz)
            tzz = eta * (-2.0 / 3.0 * exx + 4.0 / 3.0 * ezz)
            txz = eta * 2.0 * exz
        else:
            c11, c33, c55, c13, c15, c35 = [np.asarray(f)[:, ip] * eta for f in C6]
            a = -exx / 3.0 + 2.0 * ezz / 3.0
            b = 2.0 * exx / 3.0 - ezz / 3.0
            txx = c13 * a + c11 * b + c15 * exz
            tzz = c33 * a + c13 * b + c35 * 2.0 * exz
            txz = c35 * a + c15 * b + c55 * exz
        out["exx"][:, ip], out["ezz"][:, ip], out["exz"][:, ip] = exx, ezz, exz
        out["eII"][:, ip] = np.sqrt(0.5 * (exx * exx + ezz * ezz) + exz * exz)
        out["txx"][:, ip], out["tzz"][:, ip], out["txz"][:, ip] = txx, tzz, txz
        out["tII"][:, ip] = np.sqrt(0.5 * (txx * txx + tzz * tzz) + txz * txz)
    return out
