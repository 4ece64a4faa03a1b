"""fvb200: B200 implementation of the finite-volumes crate's assemble + Krylov
hot path, behind the C ABI of include/fv_b200.h.

The names mirror the reference crate (fvm::assembly::assemble,
linalg::{DistributedMatrix, DistributedVector}, preconditioners::{
IncompleteCholesky, IncompleteLowerUpper, DiagonalPreconditioner}, solvers::{conjugate_gradient,
bi_conjugate_gradient_stab, LinearSolverOptions, LinearSolverInfo}).
"""
from ._lib import FvError, lib  # noqa: F401
from .linalg import (  # noqa: F401
    DiagonalPreconditioner, DistributedMatrix, DistributedVector, IdentityPreconditioner, IncompleteCholesky,
    IncompleteLowerUpper,
    LinearSolverInfo, LinearSolverOptions, assemble, bi_conjugate_gradient_stab, compute_gradients,
    PermutedSystem, conjugate_gradient, merge_orders, order_boxes, order_boxes_host,
)
from .bcs import FaceConstraints  # noqa: F401
from .mesh import DeviceMesh, Mesh  # noqa: F401
from .terms import (  # noqa: F401
    Backward, Corrected, Euler, Orthogonal, Upwind, convection, divergence, laplacian, linear_source, source, time,
)
