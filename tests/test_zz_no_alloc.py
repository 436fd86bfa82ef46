"""The allocation-free Jacobi-PCG entry point, femd_cuda_cg_jacobi_noalloc.

It exists for callers that cannot call cudaMalloc while they solve (a solver inside a program
whose allocator already owns the device memory, or a latency-bound loop that must not
allocate).  Its work vectors live in one fixed static device array shared by every call.  This
test calls it through the C ABI twice in a row on the same system and checks each result
against femd_cuda_cg_jacobi (the allocating entry point): the same iteration count, and the
solution within 1e-12 relative (the kernels are the same, so the two normally agree bit for
bit).  The second call also shows that the array's leftover contents from the first call do not
leak into the next solve.  The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _solve(fb, fn, K, b, n, tol=1e-10, jac=1, max_iter=None):
    import torch
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res = fb._native.femd_cg_result()
    torch.cuda.synchronize()
    mi = max(1000, 10 * n) if max_iter is None else max_iter
    st = fn(K.ctx.h, K.h, jac, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), mi, tol, C.byref(res))
    assert st == 0, fb.lib.femd_cuda_last_error()
    return x.cpu().numpy(), res


@pytest.mark.parametrize("name", ["c1_p3_poisson_n32", "p2_varcoef_n16"])
def test_noalloc_matches_allocating_cg_twice(name):
    import torch

    import femd_b200 as fb
    z, _ = golden(name)
    n = z["indptr"].size - 1
    K = fb.CSRMatrix.from_arrays(n, n, z["indptr"], z["indices"], z["data"])
    fb.JacobiPreconditioner(K)
    b = torch.as_tensor(z["rhs"]).cuda()
    x_ref, r_ref = _solve(fb, fb.lib.femd_cuda_cg_jacobi, K, b, n)
    assert r_ref.converged
    for _ in range(2):
        x, r = _solve(fb, fb.lib.femd_cuda_cg_jacobi_noalloc, K, b, n)
        assert r.converged and not r.breakdown
        assert r.iterations == r_ref.iterations
        assert abs(r.residual - r_ref.residual) <= 1e-12 * r_ref.residual
        assert np.linalg.norm(x - x_ref) <= 1e-12 * np.linalg.norm(x_ref)


@pytest.mark.parametrize("jac", [0, 1])
@pytest.mark.parametrize("max_iter", [5, 17, None])
def test_noalloc_same_bits_as_allocating_cg(jac, max_iter):
    """Both branches (Jacobi or no preconditioner) and runs stopped by max_iter: the same
    iterations, residual, converged flag and solution bits as femd_cuda_cg_jacobi, whose loop
    runs in captured chunks of another length."""
    import torch

    import femd_b200 as fb
    z, _ = golden("p2_varcoef_n16")
    n = z["indptr"].size - 1
    K = fb.CSRMatrix.from_arrays(n, n, z["indptr"], z["indices"], z["data"])
    fb.JacobiPreconditioner(K)
    b = torch.as_tensor(z["rhs"]).cuda()
    x_ref, r_ref = _solve(fb, fb.lib.femd_cuda_cg_jacobi, K, b, n, jac=jac, max_iter=max_iter)
    for _ in range(2):
        x, r = _solve(fb, fb.lib.femd_cuda_cg_jacobi_noalloc, K, b, n, jac=jac, max_iter=max_iter)
        assert (r.iterations, r.converged, r.breakdown) == (r_ref.iterations, r_ref.converged, r_ref.breakdown)
        assert r.residual == r_ref.residual
        assert np.array_equal(x, x_ref)
    if max_iter is not None:
        assert r.iterations == max_iter and not r.converged


def test_noalloc_rejects_overlapping_b_and_x():
    """The solve updates x in place while it reads b: one vector passed as both is refused."""
    import torch

    import femd_b200 as fb
    z, _ = golden("p2_varcoef_n16")
    n = z["indptr"].size - 1
    K = fb.CSRMatrix.from_arrays(n, n, z["indptr"], z["indices"], z["data"])
    fb.JacobiPreconditioner(K)
    v = torch.as_tensor(z["rhs"]).cuda()
    res = fb._native.femd_cg_result()
    st = fb.lib.femd_cuda_cg_jacobi_noalloc(K.ctx.h, K.h, 1, C.c_void_p(v.data_ptr()), C.c_void_p(v.data_ptr()), 100,
                                            1e-10, C.byref(res))
    assert st == 1
    assert b"overlap" in fb.lib.femd_cuda_last_error()


def test_noalloc_rejects_systems_beyond_its_scratch():
    import torch

    import femd_b200 as fb
    n = (1 << 20) + 1
    indptr = np.arange(n + 1, dtype=np.int32)
    indices = np.arange(n, dtype=np.int32)
    K = fb.CSRMatrix.from_arrays(n, n, indptr, indices, np.full(n, 2.0))
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res = fb._native.femd_cg_result()
    st = fb.lib.femd_cuda_cg_jacobi_noalloc(K.ctx.h, K.h, 0, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 10, 1e-10,
                                            C.byref(res))
    assert st == 1
    assert b"exceed the fixed scratch" in fb.lib.femd_cuda_last_error()


def test_noalloc_refuses_a_capturing_stream():
    """The solve synchronizes between chunks, so it cannot be captured: on a stream that is being
    captured it returns FEMD_EINVAL before it enqueues anything (the capture is then ended)."""
    import torch

    import femd_b200 as fb
    z, _ = golden("p2_varcoef_n16")
    n = z["indptr"].size - 1
    K = fb.CSRMatrix.from_arrays(n, n, z["indptr"], z["indices"], z["data"])
    fb.JacobiPreconditioner(K)
    b = torch.as_tensor(z["rhs"]).cuda()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rt = C.CDLL("libcudart.so.12")                   # the runtime the library is linked against
    s = C.c_void_p(fb.lib.femd_cuda_ctx_stream(K.ctx.h))
    assert rt.cudaStreamBeginCapture(s, 1) == 0      # cudaStreamCaptureModeThreadLocal
    res = fb._native.femd_cg_result()
    try:
        st = fb.lib.femd_cuda_cg_jacobi_noalloc(K.ctx.h, K.h, 1, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 100,
                                                1e-10, C.byref(res))
        err = fb.lib.femd_cuda_last_error()
    finally:
        g = C.c_void_p()
        rt.cudaStreamEndCapture(s, C.byref(g))
        if g.value:
            rt.cudaGraphDestroy(g)
    assert st == 1 and b"cannot be captured" in err
    # the context still solves afterwards
    st = fb.lib.femd_cuda_cg_jacobi_noalloc(K.ctx.h, K.h, 1, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 100000,
                                            1e-10, C.byref(res))
    assert st == 0 and res.converged
