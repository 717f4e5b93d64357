"""dimspers_b200 -- B200-native Stokes hot path of DimsPers (Persephone).

P2-P1 element assembly on the 2D annulus with an anisotropic viscosity
tensor and the Schur-complement PCG that solves it, as hand-written CUDA
kernels for sm_100a behind a C ABI (include/dimspers_b200.h).  This package
holds the ctypes binding, a host-side mirror of the reference's Stokes
interface and the seeded synthetic input generators.
"""
from ._lib import LIB_PATH, DPError, lib  # noqa: F401
from .stokes import Mesh, StokesContext, build_mesh, default_opts, solve_stokes  # noqa: F401
