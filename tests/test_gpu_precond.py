"""The stronger preconditioners on the GPU (f4): ILU(0) and SSOR on the natural ordering and CG
preconditioned by them, against the reference's fixtures (ILU0Preconditioner,
SSORPreconditioner and krylov::cg run by the reference driver with --pc).

Tolerances.  The factorization and each application do every row's arithmetic exactly as the
reference does (same operations, same order, no contraction), so they are compared bit for bit:
ILU(0)'s smallest pivot and the application to the fixture's fixed vector.  CG: converged, the
iteration count within 2 % (+2) of the reference's (the dot products are summed in another fixed
order), the solution within 1e-8 relative of the reference's FP64 Cholesky solution.
"""
import numpy as np
import pytest

from conftest import PC_CASES, golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


def _matrix(fb, z):
    n = z["indptr"].size - 1
    return fb.CSRMatrix.from_arrays(n, n, z["indptr"], z["indices"], z["data"])


@pytest.mark.parametrize("name", PC_CASES)
def test_preconditioners_bit_exact(fb, name):
    z, meta = golden(name)
    K = _matrix(fb, z)
    n = K.nrows
    xs = 1.0 + 0.5 * np.sin(1.0 + 0.7 * np.arange(n))
    ilu = fb.ILU0Preconditioner(K)
    assert ilu.min_pivot() == float(meta["ilu0_min_pivot"])
    assert np.array_equal(ilu.apply(xs).cpu().numpy(), z["ilu0_apply_y"])
    ssor = fb.SSORPreconditioner(K, 1.0)
    assert np.array_equal(ssor.apply(xs).cpu().numpy(), z["ssor_apply_y"])
    assert ilu.levels[0] >= 1 and ilu.levels[1] >= 1


@pytest.mark.parametrize("name", PC_CASES)
@pytest.mark.parametrize("kind", ["ilu0", "ssor"])
def test_cg_with_preconditioner(fb, name, kind):
    z, meta = golden(name)
    K = _matrix(fb, z)
    M = fb.ILU0Preconditioner(K) if kind == "ilu0" else fb.SSORPreconditioner(K)
    n = K.nrows
    x, conv, its, res, brk = fb.cg_solve(K, M, z["rhs"], None, max(1000, 10 * n), 1e-10)
    ref_its = int(meta[f"{kind}_iterations"])
    assert conv and not brk and res <= 1e-9
    assert abs(its - ref_its) <= 0.02 * ref_its + 2, (its, ref_its)
    xc = z["x_chol"]
    assert np.linalg.norm(x.cpu().numpy() - xc) <= 1e-8 * np.linalg.norm(xc)
    # the reference's own preconditioned solution (its iterates) agrees as closely
    assert np.linalg.norm(x.cpu().numpy() - z[f"x_{kind}"]) <= 1e-8 * np.linalg.norm(xc)


def test_sparse_solver_cg_defaults_to_ilu0(fb):
    """A.solver("cg") takes the reference's default M="ilu0" (python/femd/sparse.py:440-446);
    M="ssor" and M="jacobi" too; the fused loop ('cuda-cg') refuses ILU(0)."""
    from femd_b200.forms import SparseSolver
    z, meta = golden("p2_poisson_pc_n16")
    K = _matrix(fb, z)
    S = SparseSolver(K, "cg")
    assert isinstance(S._M, fb.ILU0Preconditioner)
    x = S.solve(z["rhs"]).cpu().numpy()
    assert S.info.converged and abs(S.info.iterations - int(meta["ilu0_iterations"])) <= 3
    assert np.linalg.norm(x - z["x_chol"]) <= 1e-8 * np.linalg.norm(z["x_chol"])
    S2 = SparseSolver(K, "cg", M="ssor")
    S2.solve(z["rhs"])
    assert S2.info.converged and abs(S2.info.iterations - int(meta["ssor_iterations"])) <= 3
    with pytest.raises(ValueError, match="Jacobi-preconditioned"):
        SparseSolver(K, "cuda-cg", M="ilu0")


def test_preconditioner_errors(fb):
    """The reference's errors: a zero diagonal entry (ValueError), SSOR's omega range, a zero
    pivot (RuntimeError) and a solve on another pattern."""
    ip = np.array([0, 2, 4], dtype=np.int32)
    ix = np.array([0, 1, 0, 1], dtype=np.int32)
    Z = fb.CSRMatrix.from_arrays(2, 2, ip, ix, np.array([0.0, 1.0, 1.0, 2.0]))
    with pytest.raises(ValueError, match="ILU\\(0\\): zero diagonal entry in row 0"):
        fb.ILU0Preconditioner(Z)
    with pytest.raises(ValueError, match="SSOR: zero diagonal entry in row 0"):
        fb.SSORPreconditioner(Z)
    A = fb.CSRMatrix.from_arrays(2, 2, ip, ix, np.array([1.0, 1.0, 1.0, 1.0]))
    with pytest.raises(ValueError, match="omega must lie in"):
        fb.SSORPreconditioner(A, 2.0)
    with pytest.raises(RuntimeError, match="ILU\\(0\\): zero pivot in row 1"):
        fb.ILU0Preconditioner(A)
    z, _ = golden("p2_poisson_pc_n16")
    K1, K2 = _matrix(fb, z), _matrix(fb, z)
    with pytest.raises(ValueError, match="another matrix pattern"):
        fb.cg_solve(K1, fb.ILU0Preconditioner(K2), z["rhs"], None, 100, 1e-10)
