"""Run one kernel of the path on one synthetic workload a few times, for an ncu capture.

    python -m femd_b200.profile_kernels spmv --n 640 --k 2 --reps 3
    python -m femd_b200.profile_kernels assemble --n 640 --k 2 --reps 3
    python -m femd_b200.profile_kernels cg --n 640 --k 2

Workload: -Lap u + u = f on rectangle_mesh(0, 0, 1, 1, n, n), P_k, zero Dirichlet (the form of
the config-2 benchmark at another size).  Prints the sizes and a CUDA-event time per launch.
"""
from __future__ import annotations

import argparse
import math

PI = math.pi


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("kernel", choices=["spmv", "assemble", "rhs", "cg", "cg_mixed", "pattern"])
    ap.add_argument("--n", type=int, default=640)
    ap.add_argument("--k", type=int, default=2)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    import torch

    import femd_b200 as fb
    from femd_b200.core import _ptr

    m = fb.rectangle_mesh(0, 0, 1, 1, a.n, a.n)
    V = fb.LagrangeSpace2D(m, a.k, bc="dirichlet")
    Qa = V.cache(fb.quad_degree("helmholtz", a.k))
    Qf = V.cache(fb.quad_degree("rhs_data", a.k))
    P = V.pattern()
    K = fb.CSRMatrix(P)
    fb.assemble_matrix_2d(Qa, Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], K)
    b = fb.assemble_vector_2d(Qf, [0], [fb.Coef.helmholtz_sinsin(2 * PI * PI, PI, PI)], P)
    ctx = fb.context()
    s = ctx.stream
    x = torch.ones(V.dim, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)

    def run():
        if a.kernel == "spmv":
            fb.lib.femd_cuda_spmv(ctx.h, K.h, _ptr(x), _ptr(y))
        elif a.kernel == "assemble":
            fb.assemble_matrix_2d(Qa, Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], K)
        elif a.kernel == "rhs":
            fb.assemble_vector_2d(Qf, [0], [fb.Coef.helmholtz_sinsin(2 * PI * PI, PI, PI)], P, out=y)
        elif a.kernel == "pattern":
            fb.cell_pattern(V, V)
        elif a.kernel in ("cg", "cg_mixed"):
            M = fb.JacobiPreconditioner(K)
            fb.cg_solve(K, M, b, None, 100000, 1e-10, mixed=a.kernel == "cg_mixed")

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(a.reps):
        run()
    e1.record(s)
    e1.synchronize()
    print(f"{a.kernel}: n {V.dim} nnz {P.nnz} ncells {m.ncells}: {e0.elapsed_time(e1) / a.reps * 1e3:.1f} us per call")


if __name__ == "__main__":
    main()
