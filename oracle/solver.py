"""Schur-complement PCG and the full solveStokes pipeline (FP64 oracle).

Restates:
  solveStokes            src/Stokes/StokesSolver.jl:7-54 (solver=:suitesparse branch)
  StokesPcCG             src/IterativeSolvers.jl:94-168
  rm0space! / vmean      src/IterativeSolvers.jl:172-186
  _preconditioner(:jacobi) -> lumpedpreconditioner  :189-217, :238-240
  _updatesolution!       :246-259
  xpy!                   src/Algebra/Algebra.jl:61-65
  _CholeskyFactorizationSolve / _CholeskyWithFactorization!
                         src/PardisoSolvers.jl:247-256, :274-278.  The reference
                         calls UMFPACK ``lu`` (SuiteSparse, Julia 1.6.5 stdlib);
                         here SciPy's SuperLU ``splu`` stands in for it: both are
                         direct sparse LU solves of the same K[ifree, ifree].
  updatevelocity2        src/Stokes/StokesSolver.jl:170-184
  volume_integral        src/Stress/FSE.jl:412-464
"""
import time
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import mesh as M
from .assembly import element_matrices, global_matrices, rotation_matrix, prepare_matrices
from .quadrature import stokes_shape_functions, DN3DS


@dataclass
class PcgReport:
    iterations: int = 0
    relres: float = 0.0
    history: list = field(default_factory=list)


def rm0space(a):
    return a - a.sum() / a.size


def lumped_pc(MM):
    """MM = MM + tril(MM,-1)'; pc = 1 ./ rowsum  (IterativeSolvers.jl:190, :238-240)."""
    Ms = MM + sp.tril(MM, -1).T
    return 1.0 / np.asarray(Ms.sum(axis=1)).ravel()


def stokes_pcg(KK, MM, GG, Rhs, ifree, rtol=1e-8, itmax=200, itmin=10, permc="MMD_AT_PLUS_A",
               schur_pc="lumped", timing=None):
    """StokesPcCG (IterativeSolvers.jl:94-168); returns U, P, report.

    schur_pc="lumped" is the reference's StokesPcCG (:jacobi -> 1/rowsum M);
    "mass" applies M^-1 with a direct factorisation of the symmetrised M, the
    `d = pc \\ r` of StokesPcCG_pardiso (:32-34, :82) whose incomplete LDL^T
    (lldl) is exact for block-diagonal M (discontinuous pressure).
    timing: optional dict; receives "setup" (s, factorisation and first
    solve) and "iters" (s per outer iteration, the whole loop body)."""
    t_start = time.perf_counter()
    nU = Rhs.size
    U = np.zeros(nU)
    P = np.zeros(GG.shape[1])
    z = np.zeros(nU)
    Rhs = Rhs + GG @ P
    Kf = KK[ifree][:, ifree].tocsc()
    lu = spla.splu(Kf, permc_spec=permc)
    U[ifree] = lu.solve(Rhs[ifree])
    GT = GG.T.tocsr()
    r = rm0space(-(GT @ U))
    tol = np.sqrt(r @ r) * rtol
    if schur_pc == "lumped":
        pc = lumped_pc(MM)
        prec = lambda v: v * pc  # noqa: E731
    else:
        Mlu = spla.splu((MM + sp.tril(MM, -1).T).tocsc())
        prec = Mlu.solve
    d = prec(r)
    q = d.copy()
    rep = PcgReport()
    t_last = time.perf_counter()
    if timing is not None:
        timing["setup"] = t_last - t_start
        timing["iters"] = []
    for it in range(1, itmax + 1):
        q = rm0space(q)
        rd = r @ d
        y = GG @ q
        z[ifree] = lu.solve(y[ifree])
        Sq = GT @ z
        qSq = q @ Sq
        rlast = r.copy()
        alpha = rd / qSq
        P += alpha * q
        U += alpha * z
        r = r - alpha * Sq
        r = rm0space(r)
        nr = np.sqrt(r @ r)
        rep.history.append(nr)
        rep.iterations = it
        if nr < tol and it >= itmin:
            if timing is not None:
                timing["iters"].append(time.perf_counter() - t_last)
            break
        d = prec(r)
        beta = ((r - rlast) @ d) / rd
        q = d + beta * q
        if timing is not None:
            t = time.perf_counter()
            timing["iters"].append(t - t_last)
            t_last = t
    rep.relres = rep.history[-1] / (tol / rtol) if tol > 0 else 0.0
    return U, P, rep


def volume_integral(V, e2n, th, r):
    """FSE.jl:412-464: sum_e sum_ip (N.V_el) * r_ip * detJ * w_ip."""
    N, _, N3, _, w = stokes_shape_functions()
    J = np.einsum("ak,ke->ea", DN3DS, th), np.einsum("ak,ke->ea", DN3DS, r)
    detJ = J[0][:, 0] * J[1][:, 1] - J[0][:, 1] * J[1][:, 0]
    Vel = V[e2n[:6]]                                 # (6, nel)
    tot = np.zeros(th.shape[1])
    for ip in range(6):
        r_ip = r.T @ N3[ip]
        tot += (Vel.T @ N[ip]) * (r_ip * detJ * w[ip])
    return tot.sum()


def update_velocity2(U, rho_node, gr, th, r):
    """Rigid-rotation removal (StokesSolver.jl:170-184) -> (U, Ucart)."""
    U = U.copy()
    Uth = U[0::2]
    am = volume_integral(Uth * rho_node, gr.e2n, th, r)
    mom = volume_integral(gr.r * rho_node, gr.e2n, th, r)
    om = am / mom
    U[0::2] -= om * gr.r
    TT = rotation_matrix(gr.theta)
    return U, TT @ U, om


@dataclass
class StokesProblem:
    gr: M.Grid
    pressure: str
    e2nP: np.ndarray
    th: np.ndarray
    r: np.ndarray
    omega: np.ndarray
    ifree: np.ndarray

    @property
    def npres(self):
        return int(self.e2nP.max()) + 1


def make_problem(ncr, nctheta, pressure="discontinuous", literal=False, pin_rotation=True):
    gr = M.grid_cells(ncr, nctheta, literal=literal)
    th, r = M.element_coordinates(gr)
    omega, ifree = M.free_slip(gr, pin_rotation)
    return StokesProblem(gr=gr, pressure=pressure, e2nP=gr.e2nP(pressure), th=th, r=r,
                         omega=omega, ifree=ifree)


def assemble(prob, eta_ip, rho_node, g, C6=None, elements=None):
    """assembly_stokes_cylindric + _prepare_matrices + _apply_bcs (vfix = 0).
    elements: the element-block restatement to use (default the NumPy one;
    oracle.c_elements.element_matrices is the threaded C one)."""
    gr = prob.gr
    Ke, Ge, Me, Fb = (elements or element_matrices)(prob.th, prob.r, eta_ip, rho_node, gr.e2n, g, C6)
    KK, GG, MM, F = global_matrices(gr.e2n, prob.e2nP, Ke, Ge, Me, Fb, gr.nnod, prob.npres)
    TT = rotation_matrix(gr.theta)
    KK, GG, F = prepare_matrices(KK, GG, F, TT)
    return dict(Ke=Ke, Ge=Ge, Me=Me, Fb=Fb, KK=KK, GG=GG, MM=MM, F=F)


def solve_stokes(prob, eta_ip, rho_node, g, C6=None, rtol=1e-8, itmax=200, itmin=10,
                 remove_rotation=True, schur_pc="lumped", permc="MMD_AT_PLUS_A", elements=None, timing=None):
    """solveStokes (StokesSolver.jl:7-54), solver=:suitesparse.
    timing: optional dict, filled with "assembly" (s) and stokes_pcg's fields."""
    t0 = time.perf_counter()
    A = assemble(prob, eta_ip, rho_node, g, C6, elements=elements)
    if timing is not None:
        timing["assembly"] = time.perf_counter() - t0
    U, P, rep = stokes_pcg(A["KK"], A["MM"], A["GG"], A["F"], prob.ifree, rtol, itmax, itmin,
                           permc=permc, schur_pc=schur_pc, timing=timing)
    Upol = U
    om = 0.0
    if remove_rotation:
        Upol, _, om = update_velocity2(U, rho_node, prob.gr, prob.th, prob.r)
    return dict(U_raw=U, U=Upol, P=P, report=rep, omega=om, mats=A)
