"""The DEM viscous-tensor table of the fabric update (host side).

getDEM (src/Rheology/anisotropy.jl:64-95) minus the file read: from the table
C (n, 9) = [C11 C22 C33 C44 C55 C66 C12 C13 C23] and the inclusion semi-axes
ax (n, 3), a1a2 = log10(ax1 / 1) and a2a3 = log10(1 / ax3); the rows come in
blocks of `sblk` sharing a1a2 (get_stride :97-103); a1a2_blk holds one value
per block, a2a3_blk the first block's values sorted, permutation_blk the
1-based sorting permutation (sort_axes :105-113).  The viscosity cut-off w is
Fabrics.jl's weakening(d_eta, phi), passed in by the caller.
"""
import ctypes as C

import numpy as np

from ._lib import Dem


class DEM:
    def __init__(self, C_table, ax, w):
        self.C = np.asfortranarray(C_table, dtype=np.float64)
        ax = np.asarray(ax, dtype=np.float64)
        if self.C.ndim != 2 or self.C.shape[1] != 9 or ax.shape != (self.C.shape[0], 3):
            raise ValueError("C must be (n, 9) and ax (n, 3)")
        a1a2 = np.log10(ax[:, 0] / 1.0)
        a2a3 = np.log10(1.0 / ax[:, 2])
        sblk = 1
        while sblk < len(a1a2) and a1a2[sblk - 1] == a1a2[sblk]:
            sblk += 1
        self.sblk = sblk
        self.nblk = len(a2a3) // sblk + 1
        self.a1a2_blk = np.ascontiguousarray(a1a2[::sblk])
        self.a2a3_blk = np.ascontiguousarray(np.sort(a2a3[:sblk]))
        self.permutation_blk = np.ascontiguousarray(np.argsort(a2a3[:sblk], kind="stable") + 1, dtype=np.int64)
        self.w = float(w)

    @classmethod
    def load(cls, path, w):
        """From an .npz holding C and ax (the arrays of the reference's DEM files)."""
        d = np.load(path)
        return cls(d["C"], d["ax"], w)

    def struct(self):
        return Dem(self.C.ctypes.data, self.C.shape[0], self.a1a2_blk.ctypes.data, len(self.a1a2_blk),
                   self.a2a3_blk.ctypes.data, self.permutation_blk.ctypes.data, self.sblk, self.w)
