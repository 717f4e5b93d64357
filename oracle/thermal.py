"""Thermal diffusion step on the P2 annulus (FP64 restatement; test
infrastructure).

Follows the reference's threaded path, the one MAIN.jl calls (:272-291):
  solveDiffusion_threaded  src/ThermalDiffusion/AssemblerThermal.jl:1-57
      assembly_threaded! -> KT (conduction), MT (rho Cp mass), FT;
      _prepare_matrices!(MT, FT, KT, T, dt) (ThermalSolver.jl:55-65, alpha = 1):
          FT += MT T;  MT += dt KT          (backward Euler)
      _apply_bcs!(T, MT, FT, dOmega, tfix) (ThermalSolver.jl:38-41):
          T[dOmega] = tfix;  FT -= MT[:, dOmega] tfix
      T[tfree] = gmres(MT[tfree, tfree], FT[tfree])   (Krylov.jl, no preconditioner)
  assemble_element!  AssemblerThermal.jl:114-226, with nip = 7 (diffusion_immutables
      is called with nip = 7, MAIN.jl:167-169): per IP the curved inverse Jacobian
      [R31 cos/r - T31 sin, -R21 cos/r + T21 sin; -R31 sin/r - T31 cos, R21 sin/r + T21 cos]
      / detJ, omega = r_ip detJ w_ip, Ke += dNdx' K dNdx omega, Me += N' N omega rho_ip Cp
      (rho_ip from the three vertex values and the linear N3).
      The element force vector is never added: the function returns from
      update_stiffness_matrix! before update_force_vector! (:219-225), so FT
      starts at zero.
  heated_bottom (src/Setup/boundary_conditions.jl:77-93): T fixed to Ttop on
      the outer wall and Tbot on the inner one; insulated_bottom (:95-): the
      outer wall only.
Here the linear system is solved directly (SuperLU): the GPU's PCG and the
reference's GMRES both stop at a relative residual of sqrt(eps).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .quadrature import ip_triangle7, sf_dN_tri6, sf_N_tri3, sf_N_tri6

DN3DS = np.array([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]])


def element_matrices(th, r, rho_node, e2n, K, Cp):
    """Ke, Me: (nel, 6, 6) conduction and rho Cp mass blocks.  th, r: (3, nel)
    seam-fixed vertex coordinates; rho_node nodal (vertices read)."""
    ipx, w = ip_triangle7()
    J_th = th.T @ DN3DS.T
    J_r = r.T @ DN3DS.T
    detJ = J_th[:, 0] * J_r[:, 1] - J_th[:, 1] * J_r[:, 0]
    R21, R31 = r[1] - r[0], r[2] - r[0]
    T31, T21 = th[2] - th[0], th[1] - th[0]
    rho_v = rho_node[e2n[:3]]
    nel = th.shape[1]
    Ke = np.zeros((nel, 6, 6))
    Me = np.zeros((nel, 6, 6))
    for ip in range(7):
        N = sf_N_tri6(*ipx[ip])
        dN = sf_dN_tri6(*ipx[ip])
        N3 = sf_N_tri3(*ipx[ip])
        th_ip = th.T @ N3
        r_ip = r.T @ N3
        s, c = np.sin(th_ip), np.cos(th_ip)
        rho_ip = rho_v.T @ N3
        a11 = R31 * c / r_ip - T31 * s
        a12 = -R21 * c / r_ip + T21 * s
        a21 = -R31 * s / r_ip - T31 * c
        a22 = R21 * s / r_ip + T21 * c
        dNdx = (a11[:, None] * dN[0][None, :] + a12[:, None] * dN[1][None, :]) / detJ[:, None]
        dNdz = (a21[:, None] * dN[0][None, :] + a22[:, None] * dN[1][None, :]) / detJ[:, None]
        om = r_ip * detJ * w[ip]
        Ke += K * om[:, None, None] * (dNdx[:, :, None] * dNdx[:, None, :] + dNdz[:, :, None] * dNdz[:, None, :])
        Me += (om * rho_ip * Cp)[:, None, None] * np.outer(N, N)[None]
    return Ke, Me


def _global(e2n, Ae, nnod):
    rows = np.repeat(e2n.T, 6, axis=1).ravel()
    cols = np.tile(e2n.T, (1, 6)).ravel()
    return sp.csr_matrix((Ae.reshape(len(Ae), 36).ravel(), (rows, cols)), shape=(nnod, nnod))


def boundary(gr, Ttop, Tbot, heated=True):
    """(fixed nodes, their values), 0-based: outer wall first, then inner."""
    rmax, rmin = gr.r.max(), gr.r.min()
    top = np.flatnonzero(gr.r == rmax)
    nodes, vals = [top], [np.full(top.size, Ttop)]
    if heated:
        bot = np.flatnonzero(gr.r == rmin)
        nodes.append(bot)
        vals.append(np.full(bot.size, Tbot))
    return np.concatenate(nodes), np.concatenate(vals)


def thermal_step(gr, th, r, T, rho_node, K, Cp, dt, fixed, tfix):
    """One solveDiffusion_threaded step: returns the new nodal T."""
    Ke, Me = element_matrices(th, r, rho_node, gr.e2n, K, Cp)
    MT = _global(gr.e2n, Me, gr.nnod)
    KT = _global(gr.e2n, Ke, gr.nnod)
    F = MT @ T
    A = (MT + dt * KT).tocsc()
    Tn = np.array(T, dtype=np.float64, copy=True)
    Tn[fixed] = tfix
    F = F - A[:, fixed] @ tfix
    free = np.setdiff1d(np.arange(gr.nnod), fixed)
    Tn[free] = spla.spsolve(A[free][:, free].tocsc(), F[free])
    return Tn
