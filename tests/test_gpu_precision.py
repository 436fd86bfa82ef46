"""Precision at full size: -div(k grad u) = f on rectangle_mesh 512 x 512, P2 (1,046,529
unknowns), k = 1 + 0.5 sin(2 pi x) sin(2 pi y), f i.i.d. N(0, 1) at the dofs (seed 0).  The FP32
inner / FP64 reliable-update PCG (single solve and batched) and the FP64 PCG are checked against
the reference's own FP64 sparse Cholesky solution (oracle/_ref, run here on the host cores); the
errors are printed for every result.  Skipped where the reference build is absent."""
import math
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "femd_ref_omp")
N, K = 512, 2
ERR_CONTRACT = 1e-8       # relative error of every solution against the FP64 Cholesky oracle


@pytest.fixture(scope="module")
def case():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref is not built")
    import torch
    import femd_b200 as fb
    n = (K * N - 1) ** 2
    f = np.random.default_rng(0).standard_normal(n)
    with tempfile.TemporaryDirectory() as d:
        f.tofile(os.path.join(d, "f.bin"))
        subprocess.run([REF, "varcoef_field", str(N), str(K), d, "--f", os.path.join(d, "f.bin"), "--chol", "--nocg"],
                       check=True, capture_output=True)
        x_chol = np.fromfile(os.path.join(d, "x_chol.bin"))
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, K, bc="dirichlet")
    Qa = V.cache(fb.quad_degree("varcoef", K))
    Qf = V.cache(fb.quad_degree("rhs_field", K))
    A = fb.CSRMatrix(V.pattern())
    kc = fb.Coef.sinsin(1.0, 0.5, 2 * math.pi, 2 * math.pi)
    fb.assemble_matrix_2d(Qa, Qa, [1, 2], [1, 2], [kc, kc], A)
    fd = torch.as_tensor(f).cuda()
    b = fb.assemble_vector_2d(Qf, [0], [fb.Coef.field(fd)])
    return fb, torch, A, b, x_chol


def rel(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


@pytest.mark.parametrize("tol", [1e-10, 1e-12])
def test_config3_against_cholesky(case, tol):
    fb, torch, A, b, x_chol = case
    M = fb.JacobiPreconditioner(A)
    out = {}
    for mixed in (False, True):
        x, conv, its, res, brk = fb.cg_solve(A, M, b, None, 100000, tol, mixed=mixed)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        x, conv, its, res, brk = fb.cg_solve(A, M, b, None, 100000, tol, mixed=mixed)
        t1.record()
        t1.synchronize()
        assert conv and not brk
        out["mixed" if mixed else "fp64"] = (rel(x.cpu().numpy(), x_chol), its, fb.core.cg_solve.last.outer,
                                             t0.elapsed_time(t1))
    B = fb.Batch([A])
    xs, res = B.solve([b], tol=tol, mixed=True)
    xs, res = B.solve([b], tol=tol, mixed=True)
    assert res[0]["converged"]
    out["batched_mixed"] = (rel(xs[0].cpu().numpy(), x_chol), res[0]["iterations"], res[0]["reliable_updates"],
                            res[0]["seconds"] * 1e3)
    for k, (err, its, outer, ms) in out.items():
        print(f"config 3, tol {tol:g}, {k}: relative error vs FP64 Cholesky {err:.2e}, {its} iterations, "
              f"{outer} reliable updates, {ms:.1f} ms")
    # the contract of the mixed-precision path: every result within 1e-8 relative of the FP64
    # Cholesky oracle (the error of a solve to relative residual tol is about kappa tol, and at
    # tol 1e-10 it is 1e-9 here); FP32 inner iteration with FP64 reliable updates reaches the
    # accuracy of the FP64 solve
    for err, *_ in out.values():
        assert err <= ERR_CONTRACT
    assert out["mixed"][0] <= 10 * out["fp64"][0] + 1e-13


def test_mixed_precision_falls_back_to_fp64_on_stagnation():
    """-Lap u + u = f on 512 x 512 P2 with the smooth f = (2 pi^2 + 1) sin(pi x) sin(pi y): the
    solution is the slowest mode, which the FP32 matrix copy resolves poorly, so the FP32
    recurrence stagnates.  The mixed solves detect it (two reliable updates in a row that cut the
    true residual by less than 2x) and finish in FP64: converged, within the FP64 solve's
    accuracy, single and batched."""
    import torch
    import femd_b200 as fb
    n = 512
    m = fb.rectangle_mesh(0, 0, 1, 1, n, n)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    Qa = V.cache(fb.quad_degree("helmholtz", 2))
    Qf = V.cache(fb.quad_degree("rhs_data", 2))
    K = fb.CSRMatrix(V.pattern())
    fb.assemble_matrix_2d(Qa, Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], K)
    b = fb.assemble_vector_2d(Qf, [0], [fb.Coef.helmholtz_sinsin(2 * math.pi ** 2, math.pi, math.pi)], V.pattern())
    M = fb.JacobiPreconditioner(K)
    x64, conv, its64, res, brk = fb.cg_solve(K, M, b, None, 100000, 1e-10)
    assert conv
    x32, conv, its32, res, brk = fb.cg_solve(K, M, b, None, 100000, 1e-10, mixed=True)
    assert conv and not brk and its32 < 10 * its64
    xs, rr = fb.Batch([K]).solve([b], tol=1e-10, mixed=True)
    assert rr[0]["converged"] and rr[0]["iterations"] < 10 * its64
    ref = x64.cpu().numpy()
    for x in (x32.cpu().numpy(), xs[0].cpu().numpy()):
        assert np.linalg.norm(x - ref) <= 1e-7 * np.linalg.norm(ref)
