"""ctypes binding of the plain-C element assembly (oracle/stokes_elements.c;
test infrastructure): the second restatement of the Stokes element blocks,
threaded with OpenMP.  `build()` compiles it in place with gcc."""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "stokes_elements.c")
LIB = os.path.join(HERE, "libstokes_elements.so")
_lib = None


def build(force=False):
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", LIB, SRC, "-lm"])
    return LIB


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
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
