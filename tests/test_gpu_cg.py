"""K5 / K6: SpMV and Jacobi-PCG on the GPU against the reference.

Tolerances.  SpMV: each y_i within 1e-14 (sum_j |a_ij x_j|) of the reference (a different
summation order).  CG: converged with the reference's stopping rule; the iteration count
within 2 % (+2) of the reference's (the reductions are deterministic but ordered differently);
the solution within 1e-8 relative of the reference's FP64 Cholesky solution.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden
from gpu_problems import build
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


SOLVE_CASES = [n for n in GOLDEN_CASES if "heat" not in n]


def _from_golden(fb, z):
    n = z["indptr"].size - 1
    return fb.CSRMatrix.from_arrays(n, n, z["indptr"], z["indices"], z["data"])


@pytest.mark.parametrize("name", SOLVE_CASES)
def test_spmv_matches_reference(fb, name):
    z, meta = golden(name)
    K = _from_golden(fb, z)
    n = K.nrows
    xs = 1.0 + 0.5 * np.sin(1.0 + 0.7 * np.arange(n))
    y = K.matvec(xs).cpu().numpy()
    scale = O.spmv(z["indptr"], z["indices"], np.abs(z["data"]), np.abs(xs))
    assert np.all(np.abs(y - z["spmv_y"]) <= 1e-14 * scale)


@pytest.mark.parametrize("name", SOLVE_CASES)
def test_cg_jacobi_matches_reference(fb, name):
    z, meta = golden(name)
    K = _from_golden(fb, z)
    M = fb.JacobiPreconditioner(K)
    assert np.array_equal(M.inverse_diagonal(), z["inv_diag"])
    n = K.nrows
    x, conv, its, res, brk = fb.cg_solve(K, M, z["rhs"], None, max(1000, 10 * n), 1e-10)
    ref_its = int(meta["cg_iterations"])
    assert conv and not brk
    assert abs(its - ref_its) <= 0.02 * ref_its + 2
    assert res <= 10 * 1e-10
    xc = z["x_chol"]
    assert np.linalg.norm(x.cpu().numpy() - xc) / np.linalg.norm(xc) <= 1e-8


@pytest.mark.parametrize("name", ["c1_p3_poisson_n32", "p2_varcoef_n16"])
def test_cg_solve_host_drop_in(fb, name):
    """The reference binding's data (host CSR arrays, the Jacobi inverse diagonal, numpy b)."""
    z, meta = golden(name)
    x, conv, its, res, brk = fb.cg_solve_host(z["indptr"], z["indices"], z["data"], z["inv_diag"], z["rhs"])
    assert conv and not brk and res <= 1e-9
    assert abs(its - int(meta["cg_iterations"])) <= 0.02 * int(meta["cg_iterations"]) + 2
    assert np.linalg.norm(x - z["x_chol"]) / np.linalg.norm(z["x_chol"]) <= 1e-8
    # M = None: plain CG
    x2, conv2, its2, res2, _ = fb.cg_solve_host(z["indptr"], z["indices"], z["data"], None, z["rhs"])
    x3, _ = O.cg_jacobi(z["indptr"], z["indices"], z["data"], np.ones(x.size), z["rhs"])
    assert conv2 and np.linalg.norm(x2 - z["x_chol"]) / np.linalg.norm(z["x_chol"]) <= 1e-8


def test_cg_edge_cases(fb):
    z, meta = golden("p2_helmholtz_n6")
    K = _from_golden(fb, z)
    M = fb.JacobiPreconditioner(K)
    n = K.nrows
    # zero right-hand side: x = 0, converged, 0 iterations (cg.hpp:306)
    x, conv, its, res, brk = fb.cg_solve(K, M, np.zeros(n), np.ones(n), 100, 1e-10)
    assert conv and its == 0 and not np.any(x.cpu().numpy())
    # x0 already the solution: 0 iterations (cg.hpp:312)
    x, conv, its, res, brk = fb.cg_solve(K, M, z["rhs"], z["x_chol"], 100, 1e-6)
    assert conv and its == 0
    # max_iter reached: not converged, the reported residual is the true one
    x, conv, its, res, brk = fb.cg_solve(K, M, z["rhs"], None, 3, 1e-14)
    assert its == 3 and not conv and res > 1e-6
    xo, info = O.cg_jacobi(z["indptr"], z["indices"], z["data"], z["inv_diag"], z["rhs"], max_iter=3, tol=1e-14)
    assert res == pytest.approx(info["residual"], rel=1e-6)
    # an indefinite matrix breaks down (p^T A p <= 0)
    K2 = fb.CSRMatrix.from_arrays(n, n, z["indptr"], z["indices"], -z["data"])
    x, conv, its, res, brk = fb.cg_solve(K2, None, z["rhs"], None, 100, 1e-10)
    assert brk and not conv
    # shape errors are ValueErrors, as in the reference
    with pytest.raises(ValueError):
        fb.cg_solve(K, M, np.ones(n + 1), None, 10, 1e-10)


def test_cg_deterministic(fb):
    z, _ = golden("c1_p3_poisson_n32")
    K = _from_golden(fb, z)
    M = fb.JacobiPreconditioner(K)
    x1 = fb.cg_solve(K, M, z["rhs"], None, 100000, 1e-10)[0].cpu().numpy()
    x2 = fb.cg_solve(K, M, z["rhs"], None, 100000, 1e-10)[0].cpu().numpy()
    assert np.array_equal(x1, x2)


@pytest.mark.parametrize("name", ["c1_p3_poisson_n32", "p2_varcoef_n16", "p2_helmholtz_n6"])
def test_mixed_precision_matches_cholesky(fb, name):
    z, meta = golden(name)
    K = _from_golden(fb, z)
    M = fb.JacobiPreconditioner(K)
    x, conv, its, res, brk = fb.cg_solve(K, M, z["rhs"], None, 100000, 1e-10, mixed=True)
    assert conv and not brk and res <= 1e-9
    xc = z["x_chol"]
    assert np.linalg.norm(x.cpu().numpy() - xc) / np.linalg.norm(xc) <= 1e-8


def test_assembled_solve_end_to_end(fb):
    """Config 1 through the product path: GPU pattern, assembly, Jacobi, CG; vs the reference's
    Cholesky solution."""
    z, meta = golden("c1_p3_poisson_n32")
    pr = build(fb, "poisson_sin", 32, 3)
    M = fb.JacobiPreconditioner(pr["K"])
    x, conv, its, res, brk = fb.cg_solve(pr["K"], M, pr["rhs"], None, 100000, 1e-10)
    assert conv
    assert abs(its - 228) <= 7
    xc = z["x_chol"]
    assert np.linalg.norm(x.cpu().numpy() - xc) / np.linalg.norm(xc) <= 1e-8


def test_preconditioned_solves_refuse_a_matrix_without_inverse_diagonal(fb):
    """A matrix whose inverse diagonal was never written (no JacobiPreconditioner, no assembly
    with want_inv): the C ABI's preconditioned solves return FEMD_EINVAL instead of reading
    uninitialised memory; the unpreconditioned solve runs.  femd_cuda_matrix_set_inv_diag gives
    it the preconditioner of another matrix, as cg_solve(A, M) with M of another matrix does."""
    import ctypes as C

    import torch
    z, _ = golden("p2_varcoef_n16")
    K = _from_golden(fb, z)
    n = K.nrows
    b = torch.as_tensor(z["rhs"]).cuda()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res = fb._native.femd_cg_result()
    args = (C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1000, 1e-10, C.byref(res))
    torch.cuda.synchronize()
    for fn in (fb.lib.femd_cuda_cg_jacobi, fb.lib.femd_cuda_cg_jacobi_noalloc):
        assert fn(K.ctx.h, K.h, 1, *args) == 1
        assert b"call JacobiPreconditioner first" in fb.lib.femd_cuda_last_error()
    assert fb.lib.femd_cuda_pcg_mixed(K.ctx.h, K.h, *args) == 1
    bh = C.c_void_p()
    assert fb.lib.femd_cuda_batch_create(K.ctx.h, 0, None, 0, C.byref(bh)) == 0
    mid = C.c_int()
    assert fb.lib.femd_cuda_batch_add(bh, K.h, C.byref(mid)) == 1
    fb.lib.femd_cuda_release(bh)
    assert fb.lib.femd_cuda_cg_jacobi(K.ctx.h, K.h, 0, *args) == 0 and res.converged
    # the preconditioner of another matrix with the same values
    K2 = _from_golden(fb, z)
    M2 = fb.JacobiPreconditioner(K2)
    xg, conv, its, r, brk = fb.cg_solve(K, M2, z["rhs"], None, 1000, 1e-10)
    assert conv
    x2, conv2, its2, *_ = fb.cg_solve(K2, M2, z["rhs"], None, 1000, 1e-10)
    assert its == its2 and torch.equal(xg, x2)
