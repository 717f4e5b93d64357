"""Host-side mirror of the reference's Stokes interface over the C ABI.

Reference call being replaced (src/Stokes/StokesSolver.jl:7-54)::

    Ucartesian, Upolar, U, Ucart, P, to = solveStokes(U, P, T, gr, Ucartesian, Upolar, g, rho,
        eta, C, epsII, coordinates, RotationMatrices, PhaseID, UBC, KKidx, GGidx, MMidx, to;
        solver=:suitesparse)

Here ``StokesContext`` owns the device side of one annulus mesh (mesh,
lattice permutation, element blocks, multigrid hierarchy).  ``solve_stokes``
is the one-call equivalent of ``solveStokes``: assembly
(assembly_stokes_cylindric), rotation/BCs (_prepare_matrices, _apply_bcs),
the Schur PCG (StokesPcCG) and the rigid-rotation removal (updatevelocity2).
Arrays use the reference layouts (1-based indices are converted at the ABI):
U interleaved [u_theta, u_r] per node, P continuous (vertex) or
discontinuous (3 per element), eta.ip (nel, 7), tensor fields (nel, 7).
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (DP_MEM_DEVICE, DP_MEM_HOST, DP_PRESSURE_CONTINUOUS, DP_PRESSURE_DISCONTINUOUS, MeshDesc,
                   SolveOpts, SolveReport, check, lib)

R_IN, R_OUT = 1.22, 2.22
PRESSURE = {"continuous": DP_PRESSURE_CONTINUOUS, "discontinuous": DP_PRESSURE_DISCONTINUOUS}


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def mesh_desc(nr_cells, ntheta_cells, pressure="discontinuous", device=0, pin_rotation=True,
              r_in=R_IN, r_out=R_OUT):
    return MeshDesc(int(nr_cells), int(ntheta_cells), float(r_in), float(r_out), PRESSURE[pressure],
                    int(device), 1 if pin_rotation else 0)


@dataclass
class Mesh:
    """Host copy of the split-1 annulus mesh in the reference numbering
    (Grid_split1, mesher.jl:152-233; color_mesh, coloring.jl:5-64)."""
    nr_cells: int
    ntheta_cells: int
    pressure: str
    pin_rotation: bool
    e2n: np.ndarray      # (6, nel) 0-based
    theta: np.ndarray    # (nnod,)
    r: np.ndarray
    colors: np.ndarray   # (nel,) 1-based
    ncolors: int
    omega: np.ndarray    # fixed DOFs, 0-based
    nel: int
    nnod: int
    npres: int

    @property
    def th_el(self):
        return self.element_coordinates()[0]

    @property
    def r_el(self):
        return self.element_coordinates()[1]

    def element_coordinates(self):
        """Seam-fixed vertex coordinates (elementcoordinate + fixangles!,
        Utilities.jl:30-61)."""
        if not hasattr(self, "_elc"):
            th = self.theta[self.e2n[:3]].copy()
            r = self.r[self.e2n[:3]].copy()
            a = (np.abs(th[0] - th[1]) + np.abs(th[1] - th[2]) + np.abs(th[2] - th[0])) > np.pi
            th = np.where(a[None, :] & (th < np.pi), th + 2 * np.pi, th)
            object.__setattr__(self, "_elc", (th, r))
        return self._elc

    @property
    def ifree(self):
        m = np.ones(2 * self.nnod, dtype=bool)
        m[self.omega] = False
        return np.flatnonzero(m)


def build_mesh(nr_cells, ntheta_cells, pressure="discontinuous", pin_rotation=True, colors=True):
    d = mesh_desc(nr_cells, ntheta_cells, pressure, pin_rotation=pin_rotation)
    L = lib()
    nel, nnod, npres, nfix = (C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64())
    check(L.dp_mesh_sizes(C.byref(d), C.byref(nel), C.byref(nnod), C.byref(npres), C.byref(nfix)))
    e2n = np.empty((nel.value, 6), dtype=np.int64)
    th = np.empty(nnod.value)
    r = np.empty(nnod.value)
    col = np.empty(nel.value, dtype=np.int32)
    ncol = C.c_int32(0)
    check(L.dp_mesh_build(C.byref(d), e2n.ctypes.data_as(_lib._I64), th.ctypes.data_as(_lib._D),
                          r.ctypes.data_as(_lib._D), col.ctypes.data_as(_lib._I32) if colors else None,
                          C.byref(ncol) if colors else None))
    om = np.empty(nfix.value, dtype=np.int64)
    nom = C.c_int64(0)
    check(L.dp_mesh_free_slip(C.byref(d), om.ctypes.data_as(_lib._I64), C.byref(nom)))
    return Mesh(int(nr_cells), int(ntheta_cells), pressure, bool(pin_rotation), e2n.T - 1, th, r, col,
                int(ncol.value), om[:nom.value] - 1, int(nel.value), int(nnod.value), int(npres.value))


def default_opts(**kw):
    o = SolveOpts()
    lib().dp_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class StokesContext:
    """Device context for one annulus mesh (dp_ctx)."""

    def __init__(self, nr_cells, ntheta_cells, pressure="discontinuous", device=0, pin_rotation=True):
        self.desc = mesh_desc(nr_cells, ntheta_cells, pressure, device, pin_rotation)
        self.h = C.c_void_p()
        check(lib().dp_ctx_create(C.byref(self.desc), C.byref(self.h)))
        self.mesh = build_mesh(nr_cells, ntheta_cells, pressure, pin_rotation, colors=False)
        self.nel, self.nnod, self.npres = self.mesh.nel, self.mesh.nnod, self.mesh.npres

    def close(self):
        if self.h:
            lib().dp_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self):
        return lib().dp_ctx_stream(self.h)

    def _chk(self, st):
        check(st, self.h)

    def connectivity(self):
        e2n = np.empty((self.nel, 6), dtype=np.int64)
        col = np.empty(self.nel, dtype=np.int32)
        self._chk(lib().dp_get_connectivity(self.h, e2n.ctypes.data_as(_lib._I64), col.ctypes.data_as(_lib._I32)))
        return e2n.T - 1, col

    # ---- material -----------------------------------------------------------
    def set_material(self, eta_ip, rho, g, C6=None):
        """eta_ip (nel, >=6) Fortran-or-C layout handled; C6 six (nel, >=6)."""
        eta = np.asfortranarray(eta_ip, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        fields = None
        keep = [eta, rho]
        ldc = 0
        if C6 is not None:
            cs = [np.asfortranarray(c, dtype=np.float64) for c in C6]
            keep += cs
            fields = (C.c_void_p * 6)(*[c.ctypes.data for c in cs])
            ldc = cs[0].shape[0]
        self._chk(lib().dp_set_material(self.h, _ptr(eta), eta.shape[0], fields, ldc, _ptr(rho), float(g),
                                        DP_MEM_HOST))

    def set_material_ti(self, eta_ip, rho, g, delta, dir_x, dir_y):
        eta = np.asfortranarray(eta_ip, dtype=np.float64)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (delta, dir_x, dir_y, rho)]
        self._chk(lib().dp_set_material_ti(self.h, _ptr(eta), eta.shape[0], _ptr(arrs[0]), _ptr(arrs[1]),
                                           _ptr(arrs[2]), _ptr(arrs[3]), float(g), DP_MEM_HOST))

    def fse_director(self, F):
        """F: (nel, 2, 2) per-element deformation gradient -> (dir_x, dir_y)."""
        Fj = np.ascontiguousarray(np.asarray(F, dtype=np.float64).transpose(0, 2, 1).reshape(self.nel, 4))
        dx = np.empty(self.nel)
        dy = np.empty(self.nel)
        self._chk(lib().dp_fse_director(self.h, _ptr(Fj), _ptr(dx), _ptr(dy), DP_MEM_HOST))
        return dx, dy

    # ---- assembly & operators -------------------------------------------------
    def assemble(self, precision=0):
        self._chk(lib().dp_assemble(self.h, int(precision)))

    def set_deterministic(self, on=True):
        """Scatter without atomics (fixed-order per-node sums), so repeated
        solves are bit-identical; discards the assembly when switched on."""
        self._chk(lib().dp_set_deterministic(self.h, 1 if on else 0))

    def element_matrices(self):
        Ke = np.empty((self.nel, 78))
        Ge = np.empty((self.nel, 36))
        Me = np.empty((self.nel, 6))
        Fb = np.empty((self.nel, 12))
        self._chk(lib().dp_get_element_matrices(self.h, _ptr(Ke), _ptr(Ge), _ptr(Me), _ptr(Fb)))
        return Ke.T, Ge.T, Me.T, Fb.T

    def apply_K(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(2 * self.nnod)
        self._chk(lib().dp_apply_K(self.h, _ptr(x), _ptr(y), DP_MEM_HOST))
        return y

    def reduce(self, a, b=None, compensated=True):
        """The solver's deterministic reduction of host vectors: sum a_i b_i
        (b given) or sum a_i, compensated (the Schur loop's) or plain."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        op = (0 if b is not None else 2) + (1 if compensated else 0)
        bp = None
        if b is not None:
            b = np.ascontiguousarray(b, dtype=np.float64)
            bp = _ptr(b)
        out = C.c_double(0.0)
        self._chk(lib().dp_reduce(self.h, _ptr(a), bp, a.size, op, C.byref(out), DP_MEM_HOST))
        return out.value

    def apply_G(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        y = np.empty(2 * self.nnod)
        self._chk(lib().dp_apply_G(self.h, _ptr(p), _ptr(y), DP_MEM_HOST))
        return y

    def apply_GT(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = np.empty(self.npres)
        self._chk(lib().dp_apply_GT(self.h, _ptr(x), _ptr(p), DP_MEM_HOST))
        return p

    def stress(self, Ucart, eta_ip, C6=None):
        """stress! (src/Stress/StressCalculation.jl:244-249) for the Cartesian
        velocity Ucart (2*nnod, reference numbering): dict of (nel, 7) arrays
        exx, ezz, exz, eII, txx, tzz, txz, tII at the 7-point IPs."""
        U = np.ascontiguousarray(Ucart, dtype=np.float64)
        eta = np.asfortranarray(eta_ip, dtype=np.float64)
        if eta.shape[1] < 7:
            raise ValueError("eta_ip needs 7 IP columns")
        fields, keep, ldc = None, [], 0
        if C6 is not None:
            keep = [np.asfortranarray(f, dtype=np.float64) for f in C6]
            fields = (C.c_void_p * 6)(*[f.ctypes.data for f in keep])
            ldc = keep[0].shape[0]
        out = np.empty(8 * 7 * self.nel)
        self._chk(lib().dp_stress(self.h, _ptr(U), _ptr(eta), eta.shape[0],
                                  C.cast(fields, C.POINTER(C.c_void_p)) if fields is not None else None, ldc,
                                  _ptr(out), DP_MEM_HOST))
        names = ("exx", "ezz", "exz", "eII", "txx", "tzz", "txz", "tII")
        blocks = out.reshape(8, 7, self.nel)
        return {n: blocks[i].T.copy() for i, n in enumerate(names)}

    def viscosity_arrhenius(self, eta_ip, T, P_vertex, r, epsII, tauII, cohesion, eta0=5e20, R=8.314, Ea=100e3,
                            Va=1e-6, T0=1600.0, phi=1.0):
        """getviscosity!(::Arrhenius, ...) (src/Rheology/Rheology.jl:348-403):
        the updated (nel, 7) eta.ip from nodal T and r (reference numbering),
        vertex pressure, and the (nel, 7) epsII, tauII and cohesion."""
        law = _lib.Arrhenius(eta0, R, Ea, Va, T0, phi)
        eta = np.asfortranarray(eta_ip, dtype=np.float64).copy(order="F")
        mats = [np.asfortranarray(a, dtype=np.float64) for a in (epsII, tauII, cohesion)]
        for a in [eta] + mats:
            if a.shape != (self.nel, 7):
                raise ValueError("IP arrays must be (nel, 7)")
        vec = [np.ascontiguousarray(a, dtype=np.float64) for a in (T, P_vertex, r)]
        self._chk(lib().dp_viscosity_arrhenius(self.h, C.byref(law), _ptr(vec[0]), _ptr(vec[1]), vec[1].size,
                                               _ptr(vec[2]), _ptr(mats[0]), _ptr(mats[1]), _ptr(mats[2]),
                                               _ptr(eta), DP_MEM_HOST))
        return np.array(eta)

    def thermal_step(self, T, rho_node, dt, raise_on_status=True, **opts):
        """solveDiffusion_threaded (AssemblerThermal.jl:1-57): one backward-Euler
        step of the nodal temperature T (reference numbering).  opts: K, Cp,
        Ttop, Tbot, heated, rtol, atol, itmax (defaults: dp_default_thermal_opts).
        Returns (T_new, iterations, relres); with raise_on_status=False a step
        that stopped at itmax (DP_NOT_CONVERGED) returns its last iterate."""
        o = _lib.ThermalOpts()
        lib().dp_default_thermal_opts(C.byref(o))
        o.dt = float(dt)
        for k, v in opts.items():
            if not hasattr(o, k):
                raise KeyError(k)
            setattr(o, k, v)
        Tn = np.array(T, dtype=np.float64, copy=True)
        rho = np.ascontiguousarray(rho_node, dtype=np.float64)
        if Tn.shape != (self.nnod,) or rho.shape != (self.nnod,):
            raise ValueError("T and rho_node must hold nnod values")
        it = C.c_int32(0)
        rel = C.c_double(0.0)
        st = lib().dp_thermal_step(self.h, C.byref(o), _ptr(rho), _ptr(Tn), C.byref(it), C.byref(rel), DP_MEM_HOST)
        if st != 0 and (raise_on_status or st >= 2):
            self._chk(st)
        return Tn, it.value, rel.value

    def fse(self, F):
        """getFSE (src/Stress/FSE.jl:131-161) per IP.  F: (nel, 6, 2, 2).
        Returns dict vx1, vx2, vy1, vy2, a1, a2 of (nel, 6) arrays."""
        F = np.asarray(F, dtype=np.float64)
        if F.shape != (self.nel, 6, 2, 2):
            raise ValueError("F must be (nel, 6, 2, 2)")
        # Julia memory order: IP-major over elements, each 2x2 column-major
        Fj = np.ascontiguousarray(F.transpose(1, 0, 3, 2))
        outs = [np.empty((self.nel, 6), order="F") for _ in range(6)]
        ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in outs])
        self._chk(lib().dp_fse(self.h, _ptr(Fj), ptrs, self.nel, DP_MEM_HOST))
        return dict(zip(("vx1", "vx2", "vy1", "vy2", "a1", "a2"), outs))

    def anisotropic_tensor(self, dem, vx1, vy1, r1, r2):
        """anisotropic_tensor (src/Rheology/anisotropy.jl:140-285) from the FSE
        major axis and the fabric shape (r1, r2) per IP, (nel, 6) each, with
        the DEM table `dem` (`dimspers_b200.fabric.DEM`).  Returns the six
        StiffnessTensor fields, (nel, 7) each."""
        ins = [np.asfortranarray(a, dtype=np.float64) for a in (vx1, vy1, r1, r2)]
        for a in ins:
            if a.shape != (self.nel, 6):
                raise ValueError("inputs must be (nel, 6)")
        outs = [np.empty((self.nel, 7), order="F") for _ in range(6)]
        ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in outs])
        d = dem.struct()
        self._chk(lib().dp_anisotropic_tensor(self.h, C.byref(d), *[_ptr(a) for a in ins], self.nel, ptrs, self.nel,
                                              DP_MEM_HOST))
        return tuple(outs)

    def rhs(self):
        F = np.empty(2 * self.nnod)
        pc = np.empty(self.npres)
        self._chk(lib().dp_get_rhs(self.h, _ptr(F), _ptr(pc)))
        return F, pc

    # ---- solve ----------------------------------------------------------------
    def solve(self, P0=None, want_cart=True, raise_on_status=True, **opts):
        """StokesPcCG + updatevelocity2 -> (U, P, Ucart, report dict)."""
        o = default_opts(**opts)
        U = np.zeros(2 * self.nnod)
        P = np.zeros(self.npres) if P0 is None else np.array(P0, dtype=np.float64)
        if P0 is not None and o.use_guess == 0:
            o.use_guess = 1
        Uc = np.zeros(2 * self.nnod) if want_cart else None
        rep = SolveReport()
        st = lib().dp_solve(self.h, _ptr(U), _ptr(P), _ptr(Uc), C.byref(o), C.byref(rep), DP_MEM_HOST)
        if st != 0 and (raise_on_status or st >= 3):
            self._chk(st)
        return U, P, Uc, rep.as_dict()

    def solve_device(self, U_ptr, P_ptr, Uc_ptr=None, **opts):
        """Same as solve() on device pointers (ints); returns the report dict."""
        o = default_opts(**opts)
        rep = SolveReport()
        st = lib().dp_solve(self.h, C.c_void_p(U_ptr), C.c_void_p(P_ptr),
                            C.c_void_p(Uc_ptr) if Uc_ptr else None, C.byref(o), C.byref(rep), DP_MEM_DEVICE)
        if st >= 3:
            self._chk(st)
        return rep.as_dict()

    def profile_kernel(self, which, reps=50, flush_l2=False):
        """Average ms per launch: 0 FP32 A-apply, 1 FP64 A-apply, 2 V-cycle,
        3 stress post-processor, 4 viscosity update, 5 DEM tensor lookup, 6
        thermal apply (last call's inputs), 7 the graph solve's inner-iteration
        vector kernels launched outside the graph (for profilers);
        flush_l2 times each launch alone after overwriting 256 MB (cold L2)."""
        ms = C.c_double(0.0)
        self._chk(lib().dp_profile_kernel(self.h, int(which), int(reps), 1 if flush_l2 else 0, C.byref(ms)))
        return ms.value

    def set_material_device(self, eta_ptr, ld_eta, rho_ptr, g, C6_ptrs=None, ld_C=0):
        fields = (C.c_void_p * 6)(*C6_ptrs) if C6_ptrs is not None else None
        self._chk(lib().dp_set_material(self.h, C.c_void_p(eta_ptr), int(ld_eta), fields, int(ld_C),
                                        C.c_void_p(rho_ptr), float(g), DP_MEM_DEVICE))

    def set_material_ti_device(self, eta_ptr, ld_eta, rho_ptr, g, delta_ptr, dx_ptr, dy_ptr):
        self._chk(lib().dp_set_material_ti(self.h, C.c_void_p(eta_ptr), int(ld_eta), C.c_void_p(delta_ptr),
                                           C.c_void_p(dx_ptr), C.c_void_p(dy_ptr), C.c_void_p(rho_ptr), float(g),
                                           DP_MEM_DEVICE))


def solve_stokes(ctx, eta_ip, rho, g, C6=None, precision=0, P0=None, **opts):
    """solveStokes (StokesSolver.jl:7-54) on a StokesContext: set material,
    assemble, Schur PCG, rigid-rotation removal.  Returns (U, P, Ucart, report)."""
    ctx.set_material(eta_ip, rho, g, C6)
    ctx.assemble(precision)
    return ctx.solve(P0=P0, precision=precision, **opts)
