"""6-point triangle quadrature and P2 / P1 shape functions (FP64 restatement;
test infrastructure).

Follows src/Algebra/Quadrature.jl:
  ip_triangle6      :80-107   (weights carry the x0.5 reference-triangle area)
  sf_N_tri6         :264-285  (local node order 1,2,3 vertices; 4=mid(1,2),
                               5=mid(2,3), 6=mid(3,1))
  sf_dN_tri6        :287-307
  sf_N_tri3/dN_tri3 :166-199  (linear N3 and P1 pressure NP)
  _get_SF           :35-49
  ip_triangle7      :109-138  (the stress post-processor's rule, centroid first)
"""
import numpy as np


def ip_triangle6():
    """Integration points (6x2: r, s) and weights (6,) -- Quadrature.jl:80-107."""
    g1 = (8.0 - np.sqrt(10.0) + np.sqrt(38.0 - 44.0 * np.sqrt(2.0 / 5.0))) / 18.0
    g2 = (8.0 - np.sqrt(10.0) - np.sqrt(38.0 - 44.0 * np.sqrt(2.0 / 5.0))) / 18.0
    ipx = np.array([
        [1.0 - 2.0 * g1, g1],
        [g1, 1.0 - 2.0 * g1],
        [g1, g1],
        [1.0 - 2.0 * g2, g2],
        [g2, 1.0 - 2.0 * g2],
        [g2, g2],
    ])
    w1 = (620.0 + np.sqrt(213125.0 - 53320.0 * np.sqrt(10.0))) / 3720.0
    w2 = (620.0 - np.sqrt(213125.0 - 53320.0 * np.sqrt(10.0))) / 3720.0
    ipw = np.array([w1, w1, w1, w2, w2, w2])
    return ipx, 0.5 * ipw


def ip_triangle7():
    """7-point rule (7x2: r, s) and weights -- Quadrature.jl:109-138."""
    g1 = (6.0 - np.sqrt(15.0)) / 21.0
    g2 = (6.0 + np.sqrt(15.0)) / 21.0
    ipx = np.array([
        [1.0 / 3.0, 1.0 / 3.0],
        [1.0 - 2.0 * g1, g1],
        [g1, 1.0 - 2.0 * g1],
        [g1, g1],
        [1.0 - 2.0 * g2, g2],
        [g2, 1.0 - 2.0 * g2],
        [g2, g2],
    ])
    w1 = (155.0 - np.sqrt(15.0)) / 1200.0
    w2 = (155.0 + np.sqrt(15.0)) / 1200.0
    ipw = np.array([0.225, w1, w1, w1, w2, w2, w2])
    return ipx, 0.5 * ipw


def sf_N_tri6(r, s):
    """P2 shape functions at local (r, s) -- Quadrature.jl:264-285."""
    t = 1.0 - r - s
    return np.array([t * (2.0 * t - 1.0), r * (2.0 * r - 1.0), s * (2.0 * s - 1.0),
                     4.0 * r * t, 4.0 * r * s, 4.0 * s * t])


def sf_dN_tri6(r, s):
    """P2 derivatives (2x6: d/dr, d/ds) -- Quadrature.jl:287-307."""
    t = 1.0 - r - s
    return np.array([
        [-(4.0 * t - 1.0), 4.0 * r - 1.0, 0.0, 4.0 * (t - r), 4.0 * s, -4.0 * s],
        [-(4.0 * t - 1.0), 0.0, 4.0 * s - 1.0, -4.0 * r, 4.0 * r, 4.0 * (t - s)],
    ])


def sf_N_tri3(r, s):
    """Linear shape functions [t r s] -- Quadrature.jl:166-180."""
    return np.array([1.0 - r - s, r, s])


DN3DS = np.array([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]])  # Quadrature.jl:41-44


def stokes_shape_functions():
    """(N 6x6, dNds 6x2x6, N3 6x3, NP 6x3, w 6) at the 6 IPs -- _get_SF :35-49."""
    ipx, w = ip_triangle6()
    N = np.stack([sf_N_tri6(*p) for p in ipx])
    dNds = np.stack([sf_dN_tri6(*p) for p in ipx])
    N3 = np.stack([sf_N_tri3(*p) for p in ipx])
    return N, dNds, N3, N3.copy(), w
