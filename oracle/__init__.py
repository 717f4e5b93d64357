"""FP64 CPU oracle for the DimsPers Stokes hot path -- TEST INFRASTRUCTURE ONLY.

This package is a plain NumPy/SciPy restatement of the reference's Stokes
assembly and Schur-complement PCG (Julia package ``Persephone``) and of the
steps around it, with two plain-C restatements for cross-checks and the CPU
baseline.  Every
function cites the reference file:line it follows.  It is the checker for the
CUDA path: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.
The product package ``dimspers_b200`` never imports it.

Parity status: UNPINNED.  The reference ships no tests, fixtures or golden
vectors for this path, and it cannot run here (no Julia toolchain).  The
oracle is instead pinned by mathematical known-answer tests (quadrature
exactness, rigid-body kernels, annulus area, rotation invariance, colouring
validity) and by committed golden outputs of this oracle at small sizes.

Modules
-------
quadrature  6-point rule and P2/P1 shape functions   (src/Algebra/Quadrature.jl)
mesh        split-1 annulus mesh, edge numbering, colouring, BCs
            (src/Grid/mesher.jl, src/Grid/coloring.jl, src/Setup/boundary_conditions.jl,
             src/Utilities.jl)
assembly    blocked element assembly, sparse assembly, rotation
            (src/Stokes/StokesSolver.jl, src/Algebra/Sparsity.jl)
solver      StokesPcCG with a sparse LU inner solve, rigid-rotation removal
            (src/IterativeSolvers.jl, src/PardisoSolvers.jl, src/Stress/FSE.jl)
stress      strain rates and stresses at the 7-point IPs (src/Stress/StressCalculation.jl)
rheology    Arrhenius viscosity with Drucker-Prager yield (src/Rheology/Rheology.jl)
fabric      finite-strain ellipsoid and DEM viscous tensor
            (src/Stress/FSE.jl, src/Rheology/anisotropy.jl)
thermal     thermal diffusion step, direct and GMRES solves
            (src/ThermalDiffusion/AssemblerThermal.jl, ThermalSolver.jl)
c_elements  ctypes bindings of stokes_elements.c (element blocks) and
            fabric_lookup.c (DEM lookup), plain C with OpenMP
"""
