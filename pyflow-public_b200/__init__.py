"""pyflow_b200: a B200-native drop-in for PyFlow's time-advance hot path.

The staggered-grid RK4 predictor, divergence, pressure Poisson solve (BiCGStab
and Jacobi on the 7-point Laplacian), pressure-gradient projection and SGS
closure run as hand-written sm_100a CUDA kernels behind a C-ABI shared library
(``libpyflow_b200.so``, declared in ``include/pyflow_b200.h``).  The Python
modules mirror the reference's driver and module interfaces
(``PyFlow.run(inputConfig)``, ``advancer.RK4``, ``pressure.solver_bicgstab``,
...) so that reference drivers run unchanged.  There is no CPU fallback: if the
CUDA library is missing, the product path raises.
"""
__version__ = "0.1.0"
