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
The linear system is solved directly (SuperLU) by default; solver="gmres"
restates the reference's call instead: Krylov.jl's gmres with its defaults
(restart = false, i.e. full GMRES; atol = rtol = sqrt(eps); itmax = 2n; no
preconditioner), modified Gram-Schmidt Arnoldi with Givens rotations, stopping
when the residual norm falls to atol + rtol ||b||.  The GPU's PCG stops at the
same test.
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


def gmres(A, b, atol=np.sqrt(np.finfo(float).eps), rtol=np.sqrt(np.finfo(float).eps), itmax=None):
    """Full GMRES from x0 = 0 (Krylov.jl gmres defaults); returns (x, iterations, ||r||)."""
    n = b.size
    itmax = 2 * n if itmax is None else itmax
    beta = np.linalg.norm(b)
    eps = atol + rtol * beta
    if beta <= eps:
        return np.zeros(n), 0, beta
    V = [b / beta]
    H = []                                   # columns of the Hessenberg matrix after the rotations
    cs, sn = [], []
    g = [beta]
    k = 0
    rnorm = beta
    while rnorm > eps and k < itmax:
        w = A @ V[k]
        h = np.zeros(k + 2)
        for i in range(k + 1):               # modified Gram-Schmidt
            h[i] = V[i] @ w
            w = w - h[i] * V[i]
        h[k + 1] = wn = np.linalg.norm(w)
        for i in range(k):                   # previous rotations
            t = cs[i] * h[i] + sn[i] * h[i + 1]
            h[i + 1] = -sn[i] * h[i] + cs[i] * h[i + 1]
            h[i] = t
        d = np.hypot(h[k], h[k + 1])
        c, s = h[k] / d, h[k + 1] / d
        cs.append(c)
        sn.append(s)
        h[k] = d
        h[k + 1] = 0.0
        g.append(-s * g[k])
        g[k] = c * g[k]
        H.append(h[:k + 1].copy())
        rnorm = abs(g[k + 1])
        k += 1
        if wn == 0.0:                        # lucky breakdown: the Krylov space holds the solution
            break
        V.append(w / wn)
    R = np.zeros((k, k))
    for j in range(k):
        R[:j + 1, j] = H[j]
    y = np.linalg.solve(np.triu(R), np.array(g[:k]))
    x = np.column_stack(V[:k]) @ y
    return x, k, rnorm


def thermal_step(gr, th, r, T, rho_node, K, Cp, dt, fixed, tfix, solver="direct"):
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
    Aff = A[free][:, free].tocsc()
    if solver == "gmres":
        Tn[free] = gmres(Aff.tocsr(), F[free])[0]
    else:
        Tn[free] = spla.spsolve(Aff, F[free])
    return Tn
