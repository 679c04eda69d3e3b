"""B200-native (sm_100a) implementation of the mguso implicit IPC step.

Python side of the C ABI in ``include/mguso_cuda.h``: a mirror of the reference engine's
solver API (scene build -> step -> readback, and its ``LinearSolver`` seam) plus the
operator entry points (BSR SpMV, Schwarz, LBVH). Everything computes on the GPU through
``nguo-3d_b200/lib/libmguso_cuda.so``; there is no CPU fallback.
"""
from ._lib import MgusoError, load  # noqa: F401
from .linsolve import Bsr, Context, CsrMatrix, CudaLinearSolver, LinearStats, Schwarz  # noqa: F401
from .solver import ImplicitBatch, ImplicitSolver  # noqa: F401,E402
from .adjoint import AdjointDrape  # noqa: F401,E402
from . import arrange, bridge, capture, garment, metrics, patterns, seams, sewing, triangulate  # noqa: F401,E402
