"""FP64 element assembly of the Stokes blocks on the annulus (oracle).

Restates src/Stokes/StokesSolver.jl:
  assembly_stokes_cylindric  :247-404  (vectorised over all elements instead of
                                        1200-element blocks; per-entry IP
                                        accumulation order 1..6 is unchanged)
  _fill_R_J!                 :522-541
  _ip_loop!                  :587-638  (eta read at the 6 Stokes IPs, :608)
  _derivative_weights!       :641-686  (curved inverse Jacobian, omega = r*detJ*w)
  _fill_Kblk! iso / aniso    :688-742 / :744-810  (no [1e18,1e25] clamp, as in
                                        the src/src copy; see module note)
  _fill_Gblk! / _fill_Mblk! / _fill_Fbblk!  :812-845
  _element_density           :1017-1038
  _create_stokes_matrices    :488-520 with the triplet patterns of
                             src/Algebra/Sparsity.jl:31-103
  _prepare_matrices          :192-201
  _apply_bcs                 :186-190

Packed layouts (same as the reference):
  Ke 78 = lower triangle of the 12x12 element matrix, column-major, DOF order
          [ux1, uz1, ..., ux6, uz6]
  Ge 36 = 12x3 column-major (row 2k-1: omega*NP_i*dN_k/dx, row 2k: .../dz)
  Me  6 = lower triangle of 3x3, column-major
  Fb 12 = [x1, z1, ..., x6, z6]

D matrix (Voigt xx, zz, xz): isotropic eta*[4/3 -2/3 0; -2/3 4/3 0; 0 0 1]
(StokesSolver.jl:691-692, AssemblerStokes.jl:321-325); anisotropic
eta*[C11 C13 C15; C13 C33 C35; C15 C35 C55] (StokesSolver.jl:749-754,
AssemblerStokes.jl:313-319).
"""
import numpy as np
import scipy.sparse as sp

from .quadrature import stokes_shape_functions, DN3DS


def packed_pairs(n=12):
    """(row, col) of the lower column-major packing, in the exact order the
    reference loops emit them (StokesSolver.jl:696-741)."""
    pairs = []
    nn = n // 2
    for i in range(nn):
        for j in range(i, nn):
            pairs.append((2 * j, 2 * i))
            pairs.append((2 * j + 1, 2 * i))
        for j in range(i, nn):
            if j > i:
                pairs.append((2 * j, 2 * i + 1))
            pairs.append((2 * j + 1, 2 * i + 1))
    return np.array(pairs, dtype=np.int64)


PACK12 = packed_pairs(12)          # (78, 2)
PACK3 = np.array([(0, 0), (1, 0), (2, 0), (1, 1), (2, 1), (2, 2)], dtype=np.int64)


def unpack_sym(packed, n, pairs):
    """(npk, nel) packed lower -> (nel, n, n) full symmetric."""
    nel = packed.shape[1]
    full = np.zeros((nel, n, n))
    full[:, pairs[:, 0], pairs[:, 1]] = packed.T
    full[:, pairs[:, 1], pairs[:, 0]] = packed.T
    return full


def d_matrices(eta_ip, C6=None):
    """Per element per IP 3x3 D: (nel, 6, 3, 3).  C6 = (C11, C33, C55, C13, C15, C35),
    each (nel, >=6), following StiffnessTensor field order (anisotropy.jl:1-8)."""
    nel = eta_ip.shape[0]
    eta = eta_ip[:, :6]
    D = np.zeros((nel, 6, 3, 3))
    if C6 is None:
        D[..., 0, 0] = 4.0 / 3.0
        D[..., 1, 1] = 4.0 / 3.0
        D[..., 0, 1] = D[..., 1, 0] = -2.0 / 3.0
        D[..., 2, 2] = 1.0
    else:
        c11, c33, c55, c13, c15, c35 = [np.asarray(c)[:, :6] for c in C6]
        D[..., 0, 0] = c11
        D[..., 1, 1] = c33
        D[..., 2, 2] = c55
        D[..., 0, 1] = D[..., 1, 0] = c13
        D[..., 0, 2] = D[..., 2, 0] = c15
        D[..., 1, 2] = D[..., 2, 1] = c35
    return D * eta[:, :, None, None]


def element_matrices(th, r, eta_ip, rho_node, e2n, g, C6=None):
    """Element blocks in CARTESIAN DOFs: Ke (78,nel), Ge (36,nel), Me (6,nel), Fb (12,nel).

    th, r: (3, nel) seam-fixed vertex coordinates; eta_ip: (nel, >=6);
    rho_node: (nnod,) nodal density (vertices read, :1021-1022)."""
    N, dNds, N3, NP, w = stokes_shape_functions()
    nel = th.shape[1]
    D = d_matrices(eta_ip, C6)
    # _fill_R_J! (:522-541) with J = VCOORD' * dN3ds'
    J_th = th.T @ DN3DS.T
    J_r = r.T @ DN3DS.T
    detJ = J_th[:, 0] * J_r[:, 1] - J_th[:, 1] * J_r[:, 0]
    R31, R21 = r[2] - r[0], r[1] - r[0]
    T31, T21 = th[2] - th[0], th[1] - th[0]
    Kp = np.zeros((78, nel))
    Ge = np.zeros((nel, 36))
    Me = np.zeros((nel, 6))
    Fb = np.zeros((nel, 12))
    rho_v = rho_node[e2n[:3]]                       # (3, nel)
    for ip in range(6):
        th_ip = th.T @ N3[ip]
        r_ip = r.T @ N3[ip]
        dens = rho_v.T @ NP[ip]
        visc = eta_ip[:, ip]
        fg = g * dens
        s, c = np.sin(th_ip), np.cos(th_ip)
        inv = 1.0 / r_ip / detJ
        ix0 = (R31 * c - T31 * s * r_ip) * inv
        ix1 = (-R21 * c + T21 * s * r_ip) * inv
        iz0 = (-R31 * s - T31 * c * r_ip) * inv
        iz1 = (R21 * s + T21 * c * r_ip) * inv
        om = r_ip * detJ * w[ip]
        dNdx = ix0[:, None] * dNds[ip, 0][None, :] + ix1[:, None] * dNds[ip, 1][None, :]
        dNdz = iz0[:, None] * dNds[ip, 0][None, :] + iz1[:, None] * dNds[ip, 1][None, :]
        _fill_K(Kp, D[:, ip], om, dNdx, dNdz)
        # _fill_Gblk! (:812-823)
        for i in range(3):
            t = om * NP[ip, i]
            Ge[:, i * 12 + 0:i * 12 + 12:2] += t[:, None] * dNdx
            Ge[:, i * 12 + 1:i * 12 + 12:2] += t[:, None] * dNdz
        # _fill_Mblk! (:825-836)
        w3 = om / visc
        for k, (a, b) in enumerate(PACK3):
            Me[:, k] += w3 * NP[ip, a] * NP[ip, b]
        # _fill_Fbblk! (:838-845)
        cte = (om * fg)[:, None] * N[ip][None, :]
        Fb[:, 0::2] += s[:, None] * cte
        Fb[:, 1::2] += c[:, None] * cte
    return Kp, Ge.T.copy(), Me.T.copy(), Fb.T.copy()


def _fill_K(Kp, D, om, dx, dz):
    """One IP of _fill_Kblk! (StokesSolver.jl:744-810, C = 1, no clamp): the
    78 packed entries in the reference's loop order, vectorised over elements.
    D (nel, 3, 3) already includes eta; isotropic D gives :688-742."""
    e11, e13, e15 = D[:, 0, 0], D[:, 0, 1], D[:, 0, 2]
    e33, e35, e55 = D[:, 1, 1], D[:, 1, 2], D[:, 2, 2]
    idx = 0
    for i in range(6):
        xi, zi = dx[:, i], dz[:, i]
        for j in range(i, 6):
            xj, zj = dx[:, j], dz[:, j]
            Kp[idx] += om * (xi * (e11 * xj + e15 * zj) + zi * (e15 * xj + e55 * zj))
            idx += 1
            Kp[idx] += om * (xi * (e13 * zj + e15 * xj) + zi * (e35 * zj + e55 * xj))
            idx += 1
        for j in range(i, 6):
            xj, zj = dx[:, j], dz[:, j]
            if j > i:
                Kp[idx] += om * (xi * (e15 * xj + e55 * zj) + zi * (e13 * xj + e35 * zj))
                idx += 1
            Kp[idx] += om * (xi * (e35 * zj + e55 * xj) + zi * (e33 * zj + e35 * xj))
            idx += 1


def el2dof(e2n):
    """EL2DOF (StokesSolver.jl:508-510), 0-based: 2*node, 2*node+1."""
    nel = e2n.shape[1]
    d = np.empty((12, nel), dtype=np.int64)
    d[0::2] = 2 * e2n
    d[1::2] = 2 * e2n + 1
    return d


def global_matrices(e2n, e2nP, Ke, Ge, Me, Fb, nnod, npres):
    """Triplets -> CSC with duplicate summation (StokesSolver.jl:488-520,
    Sparsity.jl:31-103).  Returns KK (lower), GG, MM (lower), Fb."""
    nU = 2 * nnod
    dof = el2dof(e2n)
    Ki = dof[PACK12[:, 0]]
    Kj = dof[PACK12[:, 1]]
    lo = np.maximum(Ki, Kj)
    hi = np.minimum(Ki, Kj)
    KK = sp.coo_matrix((Ke.ravel(), (lo.ravel(), hi.ravel())), shape=(nU, nU)).tocsc()
    Gi = np.tile(dof, (3, 1))
    Gj = e2nP[np.repeat(np.arange(3), 12)]
    GG = sp.coo_matrix((Ge.ravel(), (Gi.ravel(), Gj.ravel())), shape=(nU, npres)).tocsc()
    Mi = e2nP[PACK3[:, 0]]
    Mj = e2nP[PACK3[:, 1]]
    MM = sp.coo_matrix((Me.ravel(), (np.maximum(Mi, Mj).ravel(), np.minimum(Mi, Mj).ravel())),
                       shape=(npres, npres)).tocsc()
    F = np.bincount(dof.ravel(), weights=Fb.ravel(), minlength=nU)   # accumarray
    return KK, GG, MM, F


def rotation_matrix(theta):
    """Sparse TT with per-node blocks [c s; -s c] (StokesSolver.jl:203-245)."""
    n = theta.size
    c, s = np.cos(theta), np.sin(theta)
    i0 = 2 * np.arange(n)
    rows = np.concatenate([i0, i0 + 1, i0, i0 + 1])
    cols = np.concatenate([i0, i0 + 1, i0 + 1, i0])
    vals = np.concatenate([c, c, s, -s])
    return sp.csc_matrix((vals, (rows, cols)), shape=(2 * n, 2 * n))


def sym_lower(A):
    """SparseMatrixCSC(Symmetric(A, :L))."""
    L = sp.tril(A)
    return (L + sp.tril(L, -1).T).tocsc()


def prepare_matrices(KK, GG, F, TT):
    """_prepare_matrices (StokesSolver.jl:192-201)."""
    KK = sym_lower(KK)
    KK.eliminate_zeros()
    GG = GG.copy()
    GG.eliminate_zeros()
    KK = (TT.T @ KK @ TT).tocsc()
    GG = (TT.T @ GG).tocsc()
    F = TT.T @ F
    KK = sym_lower(KK)
    return KK, GG, F
