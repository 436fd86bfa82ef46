"""fd.cg on the GPU: the reference's Python entry point (python/femd/krylov.py:178-202) with A a
femd_b200 CSRMatrix and M None or a JacobiPreconditioner."""
from __future__ import annotations

import warnings
from dataclasses import dataclass

from .core import cg_solve


@dataclass
class KrylovInfo:
    converged: bool
    iterations: int
    residual: float            # ||b - A x|| / ||b||
    precond_residual: float    # reported as residual, as the reference's cg does
    method: str

    def __repr__(self):
        state = "converged" if self.converged else "NOT converged"
        return (f"KrylovInfo({self.method} {state} in {self.iterations} iterations, residual {self.residual:.2e}, "
                f"preconditioned {self.precond_residual:.2e})")


def cg(A, b, M=None, x0=None, *, maxiter=None, tol=1e-10, warn=True, mixed=False):
    """Solve A x = b by Jacobi-preconditioned CG on the GPU.  Returns (x, KrylovInfo); x is a
    float64 CUDA tensor.  maxiter defaults to max(1000, 10 n) and x0 to zero (krylov.py:190-193)."""
    n = A.nrows
    maxiter = int(maxiter if maxiter is not None else max(1000, 10 * n))
    x, conv, its, res, breakdown = cg_solve(A, M, b, x0, maxiter, float(tol), mixed=mixed)
    info = KrylovInfo(bool(conv), int(its), float(res), float(res), "cg")
    if warn and breakdown:
        warnings.warn("cg broke down (p^T A p <= 0 or r^T M^{-1} r <= 0): A or the preconditioner is not "
                      "symmetric positive definite; use gmres", RuntimeWarning, stacklevel=2)
    elif warn and not info.converged:
        warnings.warn(f"cg did not converge in {info.iterations} iterations (residual {info.residual:.2e}, "
                      f"tol {tol:.1e}); raise maxiter or improve the preconditioner", RuntimeWarning, stacklevel=2)
    return x, info
