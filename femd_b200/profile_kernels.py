"""Run one kernel of the path on one synthetic workload a few times, for an ncu capture.

    python -m femd_b200.profile_kernels spmv --n 640 --k 2 --reps 3
    python -m femd_b200.profile_kernels assemble --n 640 --k 2 --reps 3
    python -m femd_b200.profile_kernels cg --n 640 --k 2
    python -m femd_b200.profile_kernels batch --nmin 150 --nmax 256 --nprob 24 --iters 100 --mixed
    python -m femd_b200.profile_kernels lockstep --nmin 0 --kmin 1 --nprob 16 --iters 0 --reps 1
    python -m femd_b200.profile_kernels lockstep --nmin 0 --kmin 1 --nprob 16 --iters 120 --reps 1 --mixed
    python -m femd_b200.profile_kernels numbering --n 512 --k 2 --reps 3
    python -m femd_b200.profile_kernels forms --n 512 --k 2 --reps 3
    python -m femd_b200.profile_kernels facets --n 512 --k 2 --reps 3
    python -m femd_b200.profile_kernels precond --n 128 --k 2 --reps 3

Workload: -Lap u + u = f on rectangle_mesh(0, 0, 1, 1, n, n), P_k, zero Dirichlet (the form of
the config-2 benchmark at another size).  Prints the sizes and a CUDA-event time per launch.
batch: the problems of the config-4 stream (seed 0) with N in [nmin, nmax] and k >= kmin, the
first nprob of them, solved together by the batched PCG capped at iters iterations; prints the
launch time and its algorithmic bytes (femd_b200.workloads.batch_bytes).  lockstep: the same
problems solved by the lockstep engine (iters 0: to convergence); prints the solve time and its
algorithmic bytes.  numbering: the device dof numbering of the space; forms: a coefficient
program on the cells' points and a P_k field with its derivatives there; facets: the ds matrix and
load on every exterior facet of the free space; precond: ILU(0) and SSOR built and applied.
"""
from __future__ import annotations

import argparse
import math

PI = math.pi


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("kernel", choices=["spmv", "assemble", "assemble_values", "rhs", "cg", "cg_mixed", "pattern", "batch",
                                       "lockstep", "numbering", "forms", "facets", "precond"])
    ap.add_argument("--n", type=int, default=640)
    ap.add_argument("--k", type=int, default=2)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--nprob", type=int, default=24)
    ap.add_argument("--nmin", type=int, default=150)
    ap.add_argument("--nmax", type=int, default=256)
    ap.add_argument("--kmin", type=int, default=2)
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--nnz-per-entry", type=int, default=0, help="lockstep: nonzeros per table entry (0: the default)")
    a = ap.parse_args()
    if a.kernel in ("batch", "lockstep"):
        return batch(a)
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
    extra = {}
    if a.kernel == "forms":
        from femd_b200.forms import Integrand, eval_field
        extra["prog"], extra["eval_field"] = Integrand.varcoef(2 * PI), eval_field
        extra["c"] = torch.randn(V.dim, dtype=torch.float64, device="cuda")
    elif a.kernel == "facets":
        from femd_b200.lift import FacetCache2D, assemble_facet_matrix, assemble_facet_vector
        Vf = fb.LagrangeSpace2D(m, a.k, bc="free")
        Kf = fb.CSRMatrix(Vf.pattern())
        extra.update(F=FacetCache2D(Vf, 2 * a.k), Kf=Kf, mat=assemble_facet_matrix, vec=assemble_facet_vector,
                     bf=torch.zeros(Vf.dim, dtype=torch.float64, device="cuda"))

    def run():
        if a.kernel == "spmv":
            fb.lib.femd_cuda_spmv(ctx.h, K.h, _ptr(x), _ptr(y))
        elif a.kernel == "assemble":
            fb.assemble_matrix_2d(Qa, Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], K)
        elif a.kernel == "assemble_values":
            fb.assemble_matrix_2d(Qa, Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], K, jacobi=False)
        elif a.kernel == "rhs":
            fb.assemble_vector_2d(Qf, [0], [fb.Coef.helmholtz_sinsin(2 * PI * PI, PI, PI)], P, out=y)
        elif a.kernel == "pattern":
            fb.cell_pattern(V, V)
        elif a.kernel in ("cg", "cg_mixed"):
            M = fb.JacobiPreconditioner(K)
            fb.cg_solve(K, M, b, None, 100000, 1e-10, mixed=a.kernel == "cg_mixed")
        elif a.kernel == "numbering":
            fb.LagrangeSpace2D(m, a.k, bc="dirichlet", numbering="device")
        elif a.kernel == "forms":
            extra["prog"].evaluate_cells(Qa, [], [1.0, 0.5, 2 * PI])
            extra["eval_field"](Qa, extra["c"], [0, 1, 2])
        elif a.kernel == "facets":
            extra["mat"](extra["F"], [0], [0], [1.0], extra["Kf"])
            extra["vec"](extra["F"], [0], [fb.Coef.const(1.0)], extra["bf"])
        elif a.kernel == "precond":
            for pc in (fb.ILU0Preconditioner(K), fb.SSORPreconditioner(K)):
                pc.apply(b)

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(a.reps):
        run()
    e1.record(s)
    e1.synchronize()
    print(f"{a.kernel}: n {V.dim} nnz {P.nnz} ncells {m.ncells}: {e0.elapsed_time(e1) / a.reps * 1e3:.1f} us per call")


def batch(a):
    import femd_b200 as fb
    from femd_b200 import workloads as W
    spec = [s for s in W.poisson_batch_spec(seed=0, nprob=256) if a.nmin <= s["N"] <= a.nmax and s["k"] >= a.kmin]
    spec = spec[:a.nprob]
    cache = W.SpaceCache()
    probs = [W.build_poisson(s, cache) for s in spec]
    B = fb.Batch([K for K, _ in probs])
    if a.nnz_per_entry:
        B.configure_lockstep(nnz_per_entry=a.nnz_per_entry)
    bs = [b for _, b in probs]
    engine = "lockstep" if a.kernel == "lockstep" else "persistent"
    for _ in range(a.reps):
        xs, res = B.solve(bs, tol=1e-10, max_iter=a.iters, mixed=a.mixed, engine=engine)
    sizes = [(K.nrows, K.nnz) for K, _ in probs]
    compact = engine == "lockstep" and a.mixed and B.lockstep_stats()["plain"] == 0
    alg = W.batch_bytes(sizes, res, a.mixed, compact)
    t = res[0]["seconds"]
    if engine == "lockstep":
        its = [r["iterations"] for r in res]
        n_all, z_all = sum(n for n, _ in sizes), sum(z for _, z in sizes)
        print(f"lockstep ({'mixed' if a.mixed else 'fp64'}): {len(probs)} problems, n {n_all} nnz {z_all}, iterations "
              f"max {max(its)} sum {sum(its)}: {t * 1e3:.3f} ms, algorithmic {alg} B = {alg / t / 1e9:.1f} GB/s; "
              f"layout {B.lockstep_stats()}")
        # one launch of each kernel while every member runs (what an ncu capture of an early launch sees)
        st = B.lockstep_stats()
        if a.mixed and st["compact"] == len(probs):
            spmv = 6 * z_all + 4 * (n_all + len(probs)) + 16 * n_all
            upd = 32 * n_all
            print(f"per launch, every member running: k_ls_spmv<true> (compact) {spmv} B (6 B / nonzero: value and 16-bit "
                  f"offset; 4 B / row pointer; z and the previous direction read, the direction and A p written: "
                  f"16 B / row), k_ls_update<true> {upd} B (r, A p, inv, d, p read; r, z, d written: 32 B / row)")
        return
    pr = B.profile()
    print(f"batch ({'mixed' if a.mixed else 'fp64'}): {len(probs)} problems, n {sum(n for n, _ in sizes)} "
          f"nnz {sum(z for _, z in sizes)}, {B.info()['slots']} team slots on a grid of {B.info()['grid']}: "
          f"{t * 1e3:.3f} ms per launch, algorithmic {alg} B = {alg / t / 1e9:.1f} GB/s; team-barrier wait "
          f"{pr['team_wait'] / pr['block']:.3f}, chunk-barrier wait {pr['chunk_sync'] / pr['block']:.3f} of block cycles")


if __name__ == "__main__":
    main()
