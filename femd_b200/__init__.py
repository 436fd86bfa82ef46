"""femd_b200: FEMd's 2D Lagrange P_k assembly + Jacobi-PCG path on NVIDIA B200 (sm_100a).

The compute runs in libfemd_cuda.so (hand-written CUDA, C ABI in include/femd_cuda.h); this
package is the host-side mirror of the reference's interface for that path.  Importing it
loads the library and fails if it is missing -- there is no CPU fallback.
"""
from .core import (Cache2D, Coef, Context, CSRMatrix, ILU0Preconditioner, JacobiPreconditioner,  # noqa: F401
                   LagrangeSpace2D, Mesh2D, SSORPreconditioner, SparsityPattern, assemble_matrix_2d, assemble_vector_2d, cell_pattern, cg_solve, cg_solve_host,
                   context, quad_degree, rectangle_mesh, scatter_map_2d)
from .krylov import KrylovInfo, cg  # noqa: F401
from ._native import FemdError, lib  # noqa: F401

__version__ = "0.1.0"
from .batch import Batch  # noqa: F401,E402
