"""Finite-strain ellipsoid and DEM viscous-tensor update per integration
point (FP64 restatement; test infrastructure).

Follows the reference:
  src/Stress/FSE.jl
    _FSE :143-161       L = F F^T; FSE = major/minor eigenvectors (vx1, vy1),
                        (vx2, vy2) and semi-axes a1 = sqrt|lmax|, a2 = sqrt|lmin|
    eigval_order :189   imax = 2 only if eigval[2] > eigval[1]
  src/Rheology/anisotropy.jl
    getDEM :64-95       a1a2 = log10(ax1 / 1), a2a3 = log10(1 / ax3);
                        a1a2_blk = a1a2 at the block starts, a2a3_blk = the
                        first block's a2a3 sorted, with its permutation
    get_stride :97-103, sort_axes :105-113
    argminsorted :110-118   first i with v[i] < v[i+1], else the last index
    anisotropic_tensor :140-221   IPs 1..6 by get_tensor_and_rotate!, IP 7 =
                        the mean of IPs 1..6
    get_tensor_and_rotate! :249-285   row im = sblk (i1 - 1) + perm[i2] of the
                        table, C55 floored at the cut-off w, rotated by
                        rotmatrix(vx1, vy1), eta55 floored at w again
    rotmatrix :287-292, directRotation2D :503-536
fabric_shape(a1, 1, parameterization), which maps the FSE's a1 to the
inclusion shape (r1, r2) = (log10 a1/a2, log10 a2/a3), and the cut-off
weakening(d_eta, phi) come from the Fabrics.jl dependency (0.1.0, git-tree
e9bb32545533e62b6900689f853e0461fe0ac17c), which is not part of the reference
tree: both are inputs here.
"""
import numpy as np


def dem_tables(C, ax):
    """getDEM's processing of the loaded table: C (n, 9), ax (n, 3)."""
    a1a2 = np.log10(ax[:, 0] / 1.0)
    a2a3 = np.log10(1.0 / ax[:, 2])
    sblk = 1
    while a1a2[sblk - 1] == a1a2[sblk]:
        sblk += 1
    first = a2a3[:sblk]
    perm = np.argsort(first, kind="stable") + 1          # 1-based, as sortperm
    return dict(C=np.asarray(C, dtype=np.float64), a1a2_blk=a1a2[::sblk].copy(), a2a3_blk=np.sort(first),
                permutation_blk=perm.astype(np.int64), sblk=int(sblk), nblk=len(a2a3) // sblk + 1)


def argminsorted(v):
    """0-based index of argminsorted (1-based in the reference)."""
    for i in range(len(v) - 1):
        if v[i] < v[i + 1]:
            return i
    return len(v) - 1


def direct_rotation_2d(cosa, sina, a, c, e, h):
    x1 = y2 = cosa
    x2 = sina
    y1 = -sina
    x1x1, x2x2, y1y1, y2y2 = x1 * x1, x2 * x2, y1 * y1, y2 * y2
    m = x1 * y2 + x2 * y1
    n11 = (c * x2x2 + h * x1x1 + 4 * e * x1x1) * x2x2 + (a * x1x1 + h * x2x2) * x1x1
    n33 = (c * y2y2 + h * y1y1 + 4 * e * y1y1) * y2y2 + (a * y1y1 + h * y2y2) * y1y1
    n55 = (c * x2 * y2 + h * x1 * y1) * x2 * y2 + m * m * e + (a * x1 * y1 + h * x2 * y2) * x1 * y1
    n13 = ((c * x2x2 + h * x1x1) * y2 + 4 * e * x1 * x2 * y1) * y2 + (a * x1x1 + h * x2x2) * y1y1
    n15 = ((c * x2x2 + h * x1x1) * y2 + 2 * m * e * x1) * x2 + (a * x1x1 + h * x2x2) * x1 * y1
    n35 = ((c * y2y2 + h * y1y1) * x2 + 2 * m * e * y1) * y2 + (a * y1y1 + h * y2y2) * x1 * y1
    return n11, n33, n55, n13, n15, n35


def anisotropic_tensor(x1, y1, r1, r2, dem, w):
    """x1, y1 (FSE major axis), r1, r2 (fabric shape): (nel, 6).  Returns the
    six StiffnessTensor fields (C11, C33, C55, C13, C15, C35), each (nel, 7)."""
    nel = x1.shape[0]
    out = np.zeros((6, nel, 7))
    T, b1, b2, perm, sblk = dem["C"], dem["a1a2_blk"], dem["a2a3_blk"], dem["permutation_blk"], dem["sblk"]
    for e in range(nel):
        for ip in range(6):
            i1 = argminsorted(np.abs(r1[e, ip] - b1))
            i2 = perm[argminsorted(np.abs(r2[e, ip] - b2))]      # 1-based
            row = sblk * i1 + i2 - 1
            a, c, ee, h = T[row, 0], T[row, 2], max(T[row, 4], w), T[row, 7]
            hh = 1.0 / np.sqrt(y1[e, ip] * y1[e, ip] + x1[e, ip] * x1[e, ip])
            n = direct_rotation_2d(x1[e, ip] * hh, y1[e, ip] * hh, a, c, ee, h)
            out[:, e, ip] = n
            out[2, e, ip] = max(n[2], w)
    out[:, :, 6] = out[:, :, :6].sum(axis=2) * (1.0 / 6.0)
    return tuple(out)


def fse(F):
    """F: (nel, 6, 2, 2).  Returns (x1, x2, y1, y2, a1, a2), each (nel, 6);
    eigenvector signs are those of LAPACK here and are not significant."""
    L = np.einsum("...ik,...jk->...ij", F, F)
    lam, vec = np.linalg.eigh(L)                 # ascending
    imax = np.where(lam[..., 1] > lam[..., 0], 1, 0)      # eigval_order: ties keep the first
    imin = 1 - imax
    take = lambda a, i: np.take_along_axis(a, i[..., None], axis=-1)[..., 0]  # noqa: E731
    x1 = take(vec[..., 0, :], imax)
    y1 = take(vec[..., 1, :], imax)
    x2 = take(vec[..., 0, :], imin)
    y2 = take(vec[..., 1, :], imin)
    return x1, x2, y1, y2, np.sqrt(np.abs(take(lam, imax))), np.sqrt(np.abs(take(lam, imin)))
