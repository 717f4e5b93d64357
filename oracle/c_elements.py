"""ctypes bindings of the oracle's plain-C restatements (test
infrastructure), threaded with OpenMP: the Stokes element blocks
(oracle/stokes_elements.c) and the DEM viscous-tensor lookup
(oracle/fabric_lookup.c).  `build()` compiles them in place with gcc."""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "stokes_elements.c")
LIB = os.path.join(HERE, "libstokes_elements.so")
SRC_FABRIC = os.path.join(HERE, "fabric_lookup.c")
LIB_FABRIC = os.path.join(HERE, "libfabric_lookup.so")
_lib = None
_flib = None


def _compile(src, out, force):
    if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", out, src, "-lm"])
    return out


def build(force=False):
    _compile(SRC_FABRIC, LIB_FABRIC, force)
    return _compile(SRC, LIB, force)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(_compile(SRC, LIB, False))
        P = C.c_void_p
        _lib.dpo_element_matrices.restype = C.c_int
        _lib.dpo_element_matrices.argtypes = [C.c_int64, P, P, P, C.c_int64, C.POINTER(P), C.c_int64, P,
                                              C.c_double, P, P, P, P]
    return _lib


def element_matrices(th, r, eta_ip, rho_node, e2n, g, C6=None):
    """Same contract as oracle.assembly.element_matrices: Cartesian Ke (78, nel),
    Ge (36, nel), Me (6, nel), Fb (12, nel)."""
    th = np.ascontiguousarray(th, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    nel = th.shape[1]
    eta = np.asfortranarray(eta_ip, dtype=np.float64)
    rho_v = np.ascontiguousarray(np.asarray(rho_node, dtype=np.float64)[e2n[:3]])
    keep = []
    fields = None
    ldc = 0
    if C6 is not None:
        keep = [np.asfortranarray(c, dtype=np.float64) for c in C6]
        fields = (C.c_void_p * 6)(*[c.ctypes.data for c in keep])
        ldc = keep[0].shape[0]
    out = [np.empty((n, nel)) for n in (78, 36, 6, 12)]
    st = lib().dpo_element_matrices(nel, th.ctypes.data, r.ctypes.data, eta.ctypes.data, eta.shape[0], fields, ldc,
                                    rho_v.ctypes.data, float(g), *[o.ctypes.data for o in out])
    if st != 0:
        raise ValueError("bad leading dimensions")
    return tuple(out)


def fabric_lib():
    global _flib
    if _flib is None:
        _flib = C.CDLL(_compile(SRC_FABRIC, LIB_FABRIC, False))
        P = C.c_void_p
        _flib.dpo_anisotropic_tensor.restype = C.c_int
        _flib.dpo_anisotropic_tensor.argtypes = [C.c_int64, P, P, P, P, P, C.c_int64, P, C.c_int64, P, P, C.c_int64,
                                                 C.c_double, C.POINTER(P), C.c_int]
    return _flib


def anisotropic_tensor(x1, y1, r1, r2, dem, w, nthreads=0):
    """Same contract as oracle.fabric.anisotropic_tensor (dem from
    oracle.fabric.dem_tables); nthreads = 0 uses OpenMP's default."""
    ins = [np.asfortranarray(a, dtype=np.float64) for a in (x1, y1, r1, r2)]
    nel = ins[0].shape[0]
    Ct = np.asfortranarray(dem["C"], dtype=np.float64)
    b1 = np.ascontiguousarray(dem["a1a2_blk"], dtype=np.float64)
    b2 = np.ascontiguousarray(dem["a2a3_blk"], dtype=np.float64)
    perm = np.ascontiguousarray(dem["permutation_blk"], dtype=np.int64)
    outs = [np.empty((nel, 7), order="F") for _ in range(6)]
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in outs])
    st = fabric_lib().dpo_anisotropic_tensor(nel, *[a.ctypes.data for a in ins], Ct.ctypes.data, Ct.shape[0],
                                             b1.ctypes.data, b1.size, b2.ctypes.data, perm.ctypes.data, dem["sblk"],
                                             float(w), ptrs, int(nthreads))
    if st != 0:
        raise ValueError("inconsistent DEM table")
    return tuple(outs)
