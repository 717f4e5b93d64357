"""Per-IP viscosity update of the Arrhenius law with Drucker-Prager plasticity
(FP64 restatement; test infrastructure).

Follows src/Rheology/Rheology.jl:
  getviscosity!(::Arrhenius, T, P, epsII, tauII, e2n, r)  :348-403
      per element and 7-point IP: T_ip and z_ip = r_ip by the P2 shape functions,
      P_ip by the linear ones at the vertices plus |min P|; depth factor lambda
      (1e1 between maxr - 2780 km and maxr - 660 km, 1e-3 below, 1e0 above);
      eta_TP = clamp(lambda * eta(T_ip, P_ip), 1e18, 1e25); where cohesion,
      friction angle and epsII are all non-zero the plastic branch applies:
      yield stress tau_y = cosd(phi) C + sind(phi) P_ip (druckerPrager :338-344)
      and, if tau_y < tauII, eta = clamp(tau_y / (2 epsII), 1e18, 1e25) -- and
      otherwise the previous eta is kept (the reference does not fall back to
      eta_TP there)
  getviscosity(::Arrhenius, T, P)  :171-173  eta0 exp((Ea + P Va) / (R T) - Ea / (R T0))
Shape functions at ip_triangle7 (Quadrature.jl:109-138), via _get_SF.
"""
import numpy as np

from .quadrature import ip_triangle7, sf_N_tri3, sf_N_tri6


def arrhenius_viscosity(eta_prev, T, P, r, e2n, epsII, tauII, C, eta0, R, Ea, Va, T0, phi):
    """eta_prev, epsII, tauII, C: (nel, 7); T, r: (nnod,) nodal; P: vertex
    values (P[e2n[k]] for the 3 vertices); e2n (6, nel) 0-based; phi in
    degrees.  Returns the updated (nel, 7) viscosity."""
    ipx, _ = ip_triangle7()
    eta = np.array(eta_prev, dtype=np.float64, copy=True)
    minP = abs(np.min(P))
    maxr = np.max(r)
    Tel, rel_, Pel = T[e2n], r[e2n], P[e2n[:3]]
    sphi, cphi = np.sin(np.deg2rad(phi)), np.cos(np.deg2rad(phi))
    for ip in range(7):
        N = sf_N_tri6(*ipx[ip])
        N3 = sf_N_tri3(*ipx[ip])
        T_ip = N @ Tel
        z_ip = N @ rel_
        P_ip = N3 @ Pel + minP
        lam = np.where(z_ip < maxr - 2780e3, 1e-3, np.where(z_ip > maxr - 660e3, 1e0, 1e1))
        etaTP = np.minimum(np.maximum(lam * eta0 * np.exp((Ea + P_ip * Va) / R / T_ip - Ea / R / T0), 1e18), 1e25)
        e2 = epsII[:, ip]
        plastic = (C[:, ip] > 0) & (phi > 0) & (e2 != 0.0)
        tau_y = cphi * C[:, ip] + sphi * P_ip
        yielded = plastic & (tau_y < tauII[:, ip])
        safe_e2 = np.where(e2 != 0.0, e2, 1.0)
        eta_y = np.maximum(1e18, np.minimum(1e25, 0.5 * tau_y / safe_e2))
        eta[:, ip] = np.where(plastic, np.where(yielded, eta_y, eta[:, ip]), etaTP)
    return eta
