"""Benchmark of the FEMd 2D P_k assembly + Jacobi-PCG path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-cpu]
                    [--workload c4s|c2]

Default workload (c4s), the metric's "served + mixed vs plain GPU": the stream of 256 independent
Poisson problems -c Lap u = f on rectangle_mesh(0,0,1,1,N,N), N uniform in {16..256}, P_k with k
uniform in {1,2,3}, c log-uniform in [0.1, 10], load-vector dof values N(0,1), all from seed 0
(30.5M unknowns, 448M nonzeros in all), served by femd_b200.serve.Server: every problem is a
request (all arriving at once), assembled in FP64 on its cached pattern and solved by the
batched persistent Jacobi-PCG -- FP32 inner iteration on an FP32 matrix copy with FP64 reliable
updates -- to relative residual 1e-10.  One step = serving the whole stream.  The metric is
solves/s; p50 / p99 request latency, the plain FP64 GPU path on the same stream (one assembly +
cg_solve per request, first come first served) and the largest relative difference between the
served and the plain FP64 solutions are reported beside it.  The working set (4+ GB) is larger
than L2, so no flush is needed between steps.

value      device-resident: meshes, spaces and patterns built, load vectors in HBM
e2e        through the public API from host buffers: each step copies every load vector from
           pinned host memory to the device and every solution back to pinned host memory
roofline   the dominant kernel, the batched PCG launch (k_batch_pcg), timed with CUDA events on
           the library's stream; algorithmic bytes from each member's iterations and reliable
           updates (batch_bytes below)
cpu_baseline / --impl reference: the reference's own C++ (oracle/_ref/femd_ref_omp, OpenMP,
           every host thread) on a stratified sample of 8 of the 256 problems (the midpoints of
           8 strata of equal count by size): assembly + Jacobi-PCG; solves/s on the sample
Workload c2 (the plain method at scale): -Lap u + u = f on rectangle_mesh 1024x1024, P2,
           FP64 assembly + FP64 Jacobi-PCG to 1e-10, one solve per step.
Multi-GPU (torchrun): replicas only -- every rank serves its own copy of the stream, no
collective on the data path; value = all ranks' solves / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s (FP64 assembly + Jacobi-PCG to 1e-10), rectangle 1024x1024 P2"
METRIC_C4 = ("solves/s of the served config-4 stream (256 Poisson problems, FP64 assembly + FP32-inner/FP64-refined "
             "batched Jacobi-PCG to 1e-10), with p99 latency and the plain FP64 GPU path beside it")
UNIT = "solves/s"
NPROB, SEED, NSAMPLE, CG_SAMPLE = 256, 0, 8, 40
N_MESH, DEGREE, TOL = 1024, 2, 1e-10
PI = 3.141592653589793


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _ref_binary():
    for name in ("femd_ref_omp", "femd_ref"):
        p = os.path.join(ROOT, "oracle", "_ref", name)
        if os.path.exists(p):
            return p
    return None


def run_reference(reps, sample, full_first=True, threads=None):
    """Run the reference's C++ on the workload; returns (per-step list of (t_asm, t_cg, its), meta)."""
    exe = _ref_binary()
    if exe is None:
        return None, {"error": "oracle/_ref is not built (make -C oracle ref where the reference tree is)"}
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads or os.cpu_count())
    env["OPENBLAS_NUM_THREADS"] = "1"
    args = [exe, "helmholtz_sin", str(N_MESH), str(DEGREE), "-", "--nodump", "--nocg", "--time", str(reps),
            "--cg-sample", str(sample)]
    if full_first:
        args.append("--full-first")
    out = subprocess.run(args, capture_output=True, text=True, env=env, check=True).stdout
    steps, meta = [], {}
    for line in out.splitlines():
        parts = line.split()
        if not parts:
            continue
        if parts[0] == "step":
            steps.append((float(parts[1]), float(parts[2]), int(parts[3])))
        else:
            meta[parts[0]] = parts[1]
    meta["exe"] = os.path.basename(exe)
    return steps, meta


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax = float(c[2])
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- our arm ---------------------------------------------------------------------------------
class Problem:
    """The workload on the GPU, set up once: mesh, space, caches, pattern, matrix."""

    def __init__(self, fb, torch, N=N_MESH, k=DEGREE):
        t0 = time.time()
        self.fb, self.torch = fb, torch
        self.ctx = fb.context()
        self.mesh = fb.rectangle_mesh(0, 0, 1, 1, N, N)
        self.V = fb.LagrangeSpace2D(self.mesh, k, bc="dirichlet")
        self.Qa = self.V.cache(fb.quad_degree("helmholtz", k))
        self.Qf = self.V.cache(fb.quad_degree("rhs_data", k))
        self.P = self.V.pattern()
        self.K = fb.CSRMatrix(self.P)
        self.b = torch.empty(self.V.dim, dtype=torch.float64, device="cuda")
        fb.scatter_map_2d(self.P)
        self.coef_f = fb.Coef.helmholtz_sinsin(2.0 * PI * PI, PI, PI)
        # one assembly, then the project autotuner picks the SpMV launch shape for this matrix
        fb.assemble_matrix_2d(self.Qa, self.Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], self.K)
        shape, _ = self.K.autotune_spmv(True)
        self.spmv_shape = f"{shape & 0xff} lanes/row, {max(shape >> 8, 1)} loads/lane"
        self.setup_s = time.time() - t0
        self.n, self.nnz = self.V.dim, self.P.nnz

    def step(self, phases=None):
        fb, torch = self.fb, self.torch
        s = self.ctx.stream
        if phases is not None:
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(s)
        fb.assemble_matrix_2d(self.Qa, self.Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], self.K)
        fb.assemble_vector_2d(self.Qf, [0], [self.coef_f], self.P, out=self.b)
        M = fb.JacobiPreconditioner(self.K)
        if phases is not None:
            ev[1].record(s)
        x, conv, its, res, brk = fb.cg_solve(self.K, M, self.b, None, max(1000, 10 * self.n), TOL)
        if phases is not None:
            ev[2].record(s)
            ev[2].synchronize()
            phases.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), fb.core.cg_solve.last.seconds * 1e3))
        if not conv:
            raise RuntimeError(f"CG did not converge: {its} iterations, residual {res:.2e}")
        return x, its, res


def event_time(torch, stream, fn, reps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    e0.record(stream)
    out = None
    for _ in range(reps):
        out = fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, out


def ours_c2(args, rank, world, dist):
    import torch
    import femd_b200 as fb
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pr = Problem(fb, torch)
    ctx = pr.ctx
    s = ctx.stream
    hbm, peak_kind = peaks()
    # warm-up
    its = None
    for _ in range(args.warmup):
        _, its, res = pr.step()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timed region
    barrier()
    clk = Clocks(local)
    l0 = fb.lib.femd_cuda_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    phases = []
    e0.record(s)
    for _ in range(args.steps):
        x, its, res = pr.step(phases)
    e1.record(s)
    e1.synchronize()
    barrier()
    clocks = clk.stop()
    launches = (fb.lib.femd_cuda_kernel_launches() - l0) // args.steps
    t = e0.elapsed_time(e1) / 1e3
    t_all = _max_over_ranks(torch, dist, t)
    value = world * args.steps / t_all
    phase_ms = {"assembly_ms": round(sum(p[0] for p in phases) / len(phases), 3),
                "solve_ms": round(sum(p[1] for p in phases) / len(phases), 3),
                "cg_device_ms": round(sum(p[2] for p in phases) / len(phases), 3)}

    # ---- end to end: host buffers through the public API
    pts_host = torch.from_numpy(pr.mesh.points).pin_memory()
    pts_dev = torch.empty(pts_host.shape, dtype=torch.float64, device="cuda")
    x_host = torch.empty(pr.n, dtype=torch.float64).pin_memory()

    def e2e_step():
        with torch.cuda.stream(s):
            pts_dev.copy_(pts_host, non_blocking=True)
        pr.mesh.set_points(pts_dev)
        x, its_, _ = pr.step()
        with torch.cuda.stream(s):
            x_host.copy_(x, non_blocking=True)
        return its_

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    barrier()
    te, _ = event_time(torch, s, e2e_step, args.steps)
    te_all = _max_over_ranks(torch, dist, te)
    e2e_value = world * args.steps / te_all

    # ---- the dominant kernel: CSR SpMV, timed alone on the library stream
    xv = torch.ones(pr.n, dtype=torch.float64, device="cuda")
    yv = torch.empty_like(xv)
    for _ in range(3):
        pr.K.matvec(xv)
    reps = 50

    def spmv():
        fb.lib.femd_cuda_spmv(ctx.h, pr.K.h, fb.core._ptr(xv), fb.core._ptr(yv))
    t_spmv, _ = event_time(torch, s, spmv, reps)
    t_launch = t_spmv / reps
    alg_bytes = 12 * pr.nnz + 4 * (pr.n + 1) + 8 * pr.n + 8 * pr.n
    achieved = alg_bytes / t_launch / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "k_spmv_c2_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_all / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded closed-form rhs)",
        "config": {"workload": "rectangle_mesh 1024x1024, P2, -Lap u + u = f (2 pi^2+1) sin sin, FP64 assembly + "
                               "Jacobi-PCG tol 1e-10", "n": pr.n, "nnz": pr.nnz, "cg_iterations": its,
                   "final_residual": res, "l2": "inputs larger than L2 (CSR 0.58 GB), no flush",
                   "parallelism": f"replicas x{world}", "setup_s": round(pr.setup_s, 2),
                   "spmv_shape": pr.spmv_shape, "phases": phase_ms},
        "e2e": {"value": round(e2e_value, 4), "unit": UNIT, "h2d_bytes_per_step": int(pr.mesh.points.nbytes),
                "d2h_bytes_per_step": int(8 * pr.n)},
        "roofline": {"kernel": "k_spmv (FP64 CSR SpMV of the CG loop)", "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "traffic": traffic, "algorithmic_bytes": alg_bytes, "launch_us": round(t_launch * 1e6, 2)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(its)
    return line


def _max_over_ranks(torch, dist, t):
    from femd_b200.replicas import max_over_ranks
    return max_over_ranks(t, dist, "cuda")


def cpu_baseline(gpu_its):
    sample = 40
    steps, meta = run_reference(2, sample, full_first=False)
    if steps is None:
        return {"value": None, "unit": UNIT, "error": meta.get("error")}
    t_asm = min(s[0] for s in steps)
    t_it = min(s[1] / s[2] for s in steps)
    its_full = gpu_its
    t_solve = t_asm + t_it * its_full
    return {"value": round(1.0 / t_solve, 5), "unit": UNIT, "cores": int(meta.get("threads", 1)), "kind": "reference",
            "sample": f"reference C++ ({meta['exe']}, {cpu_model()}): best of 2 steps of assembly + {sample} CG "
                      f"iterations, extrapolated to {its_full} iterations (the GPU solve's count); "
                      f"per-iteration {t_it * 1e3:.2f} ms, assembly {t_asm:.3f} s; setup (space, pattern, map) "
                      f"{float(meta.get('t_space', 0)) + float(meta.get('t_pattern', 0)) + float(meta.get('t_map', 0)):.2f} s"}


# ---- reference arm ---------------------------------------------------------------------------
def reference_c2(args, rank, world):
    if rank != 0:
        return None
    sample = 40
    steps, meta = run_reference(args.warmup + args.steps, sample, full_first=True)
    if steps is None:
        return {"impl": "reference", "unavailable": meta.get("error")}
    its_full = steps[0][2]
    timed = steps[args.warmup:]
    per = [sa + (sc / si) * its_full for (sa, sc, si) in timed]
    t = sum(per)
    value = len(per) / t
    cores = int(meta.get("threads", 1))
    sample_txt = (f"reference C++ ({meta['exe']}, OpenMP, {cores} threads, {cpu_model()}): per step assembly + "
                  f"{sample} Jacobi-PCG iterations extrapolated to {its_full} (the count of its own full solve in the "
                  f"first warm-up step)")
    return {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": len(per), "warmup": args.warmup, "ms_per_step": round(t / len(per) * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded closed-form rhs)",
            "config": {"workload": "rectangle_mesh 1024x1024, P2, -Lap u + u = f (2 pi^2+1) sin sin, FP64 assembly + "
                                   "Jacobi-PCG tol 1e-10", "n": int(meta.get("dim", 0)), "nnz": int(meta.get("nnz", 0)),
                       "cg_iterations": its_full, "parallelism": "OpenMP (host)"},
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample_txt},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}



# ---- the served config-4 stream ----------------------------------------------------------------
def c4_spec():
    from femd_b200 import workloads as W
    return W.poisson_batch_spec(seed=SEED, nprob=NPROB)


def c4_sample(spec, m=NSAMPLE):
    """A stratified sample: the problems sorted by size (n x iterations ~ (kN)^3), cut into m
    strata of equal count, the middle problem of each."""
    work = [(s["k"] * s["N"]) ** 3 for s in spec]
    order = sorted(range(len(spec)), key=lambda i: (work[i], i))
    return [order[(2 * j + 1) * len(order) // (2 * m)] for j in range(m)]


def c4_rhs(spec):
    """The load vectors (float64 numpy), from each problem's seed."""
    import numpy as np
    from femd_b200 import serve
    out = []
    for s in spec:
        n = serve.SpaceLibrary.dim(s["N"], s["k"])
        out.append(np.random.default_rng(s["seed"]).standard_normal(n))
    return out


def batch_bytes(reqs, lib, mixed=True):
    """Algorithmic HBM bytes of the batched launch that served these requests
    (femd_b200.workloads.batch_bytes)."""
    from femd_b200.workloads import batch_bytes as bb
    sizes = [(lib.get(r.N, r.k)["n"], lib.get(r.N, r.k)["nnz"]) for r in reqs]
    return bb(sizes, [dict(iterations=r.iterations, reliable_updates=r.outer) for r in reqs], mixed)


def ours_c4(args, rank, world, dist):
    import numpy as np
    import torch
    import femd_b200 as fb
    from femd_b200 import serve
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    hbm, peak_kind = peaks()
    t_setup = time.time()
    spec = c4_spec()
    lib = serve.SpaceLibrary()
    for sp in spec:
        lib.get(sp["N"], sp["k"])
    rhs = c4_rhs(spec)
    b_dev = [torch.as_tensor(b).cuda() for b in rhs]
    b_host = [torch.as_tensor(b).pin_memory() for b in rhs]
    x_host = [torch.empty(b.size, dtype=torch.float64).pin_memory() for b in rhs]
    srv = serve.Server(lib, [], mixed=True, iters=1 << 30, keep_solutions=False, engine=args.engine)
    setup_s = time.time() - t_setup
    ctx = fb.context()
    s = ctx.stream

    def reqs(host=False, keep=False):
        return [serve.Request(i, 0.0, "poisson", N=sp["N"], k=sp["k"], c=sp["c"], seed=sp["seed"],
                              b=(b_host[i] if host else b_dev[i]), out=(x_host[i] if host else None))
                for i, sp in enumerate(spec)]

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        srv.run(reqs(), realtime=False)
    # ---- device-resident timed region
    barrier()
    clk = Clocks(local)
    l0 = fb.lib.femd_cuda_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    stats, launch_s, last = [], [], None
    for _ in range(args.steps):
        last = reqs()
        stats.append(srv.run(last, realtime=False))
        launch_s.append(srv.last_launch_s)
    e1.record(s)
    e1.synchronize()
    barrier()
    clocks = clk.stop()
    launches = (fb.lib.femd_cuda_kernel_launches() - l0) // args.steps
    t = e0.elapsed_time(e1) / 1e3
    t_all = _max_over_ranks(torch, dist, t)
    value = world * args.steps * NPROB / t_all
    st = stats[-1]
    # ---- end to end: load vectors from pinned host memory, solutions back to pinned host memory
    srv.run(reqs(host=True), realtime=False)
    barrier()
    e0.record(s)
    for _ in range(args.steps):
        srv.run(reqs(host=True), realtime=False)
    e1.record(s)
    e1.synchronize()
    te = _max_over_ranks(torch, dist, e0.elapsed_time(e1) / 1e3)
    e2e_value = world * args.steps * NPROB / te
    # ---- the plain FP64 GPU path on the same stream (one pass), and the served-vs-plain error
    served = reqs()
    srv_keep = serve.Server(lib, [], mixed=True, iters=1 << 30, keep_solutions=True, engine=args.engine)
    srv_keep.run(served, realtime=False)
    xs_served = {r.rid: r.x for r in served}
    plain = reqs()
    pst = serve.run_plain(lib, [], plain, tol=1e-10, realtime=False, keep_solutions=True)
    err = 0.0
    for r in plain:
        a = xs_served[r.rid]
        err = max(err, float(torch.linalg.norm(a - r.x) / torch.linalg.norm(r.x)))
        r.x = None
    xs_served.clear()
    # ---- roofline of the batched launch of the last timed step
    alg = batch_bytes(last, lib, mixed=True)
    t_launch = launch_s[-1]
    achieved = alg / t_launch / 1e9
    traffic = None
    lockstep = args.engine == "lockstep"
    tp = os.path.join(ROOT, "profiles", "k_ls_spmv_traffic.json" if lockstep else "k_batch_pcg_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = int(json.load(open(tp))["dram_over_algorithmic"] * alg)
        except Exception:
            traffic = None
    nnz = sum(lib.get(sp["N"], sp["k"])["nnz"] for sp in spec)
    n = sum(lib.get(sp["N"], sp["k"])["n"] for sp in spec)
    line = {
        "metric": METRIC_C4, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_all / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (FP32 inner PCG, FP64 assembly/residual/update)",
        "data": "synthetic (seeded: meshes, coefficients, N(0,1) load vectors)",
        "config": {"workload": "config-4 stream: 256 Poisson problems, rectangle N x N (N in 16..256), P1-P3, "
                               "c log-uniform [0.1,10], served (all arrive at t=0: one wave of the batched "
                               f"solver, {args.engine} engine), FP32-inner / FP64-refined Jacobi-PCG to 1e-10",
                   "problems": NPROB, "n_total": n, "nnz_total": nnz, "arrivals": "burst at t=0",
                   "p50_ms": round(st["p50_ms"], 2), "p99_ms": round(st["p99_ms"], 2),
                   "mean_iterations": round(st["mean_iterations"], 1), "all_converged": st["all_converged"],
                   "max_rel_diff_vs_plain_fp64": err,
                   "plain_fp64_gpu": {"solves_per_s": round(pst["solves_per_s"], 3), "p50_ms": round(pst["p50_ms"], 2),
                                      "p99_ms": round(pst["p99_ms"], 2), "mean_iterations": round(pst["mean_iterations"], 1),
                                      "path": "per request: FP64 assembly + cg_solve (CUDA-graph CG), FIFO"},
                   "engine": args.engine,
                   "batch_shape": srv.batch.params() if not lockstep else {"nnz_per_entry": 16384, "chunk": 8,
                                                                          "spmv": "row groups"},
                   "l2": "working set > 4 GB, larger than L2; no flush",
                   "parallelism": f"replicas x{world}", "setup_s": round(setup_s, 2)},
        "e2e": {"value": round(e2e_value, 4), "unit": UNIT, "h2d_bytes_per_step": int(sum(b.nbytes for b in rhs)),
                "d2h_bytes_per_step": int(sum(b.nbytes for b in rhs))},
        "roofline": {"kernel": ("lockstep solve: k_ls_spmv / k_ls_update / k_ls_flush / k_ls_resid over the wave, "
                                "bytes and time of the whole solve" if lockstep else
                                "k_batch_pcg (batched persistent Jacobi-PCG, mixed)"), "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": traffic, "algorithmic_bytes": alg,
                     "launch_ms": round(t_launch * 1e3, 3)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        its = {r.rid: r.iterations for r in plain}
        line["cpu_baseline"] = cpu_baseline_c4(spec, rhs, its)
    return line


def run_reference_c4(spec, rhs, idx, reps, sample, full_first):
    """The reference's C++ on the sampled problems (poisson_vec: c grad.grad, the load vector read
    from a file); per problem a list of (t_asm, t_cg, its) per rep."""
    import numpy as np
    exe = _ref_binary()
    if exe is None:
        return None, {"error": "oracle/_ref is not built (make -C oracle ref where the reference tree is)"}
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(os.cpu_count())
    out, meta = {}, {}
    with tempfile.TemporaryDirectory() as d:
        for i in idx:
            sp = spec[i]
            bp = os.path.join(d, f"b{i}.bin")
            np.asarray(rhs[i], dtype=np.float64).tofile(bp)
            a = [exe, "poisson_vec", str(sp["N"]), str(sp["k"]), "-", "--c", repr(sp["c"]), "--b", bp, "--nodump",
                 "--nocg", "--time", str(reps), "--cg-sample", str(sample)]
            if full_first:
                a.append("--full-first")
            txt = subprocess.run(a, capture_output=True, text=True, env=env, check=True).stdout
            steps = []
            for line in txt.splitlines():
                p = line.split()
                if p and p[0] == "step":
                    steps.append((float(p[1]), float(p[2]), int(p[3])))
                elif len(p) == 2:
                    meta[p[0]] = p[1]
            out[i] = steps
    meta["exe"] = os.path.basename(exe)
    return out, meta


def cpu_baseline_c4(spec, rhs, gpu_its):
    idx = c4_sample(spec)
    steps, meta = run_reference_c4(spec, rhs, idx, 2, CG_SAMPLE, False)
    if steps is None:
        return {"value": None, "unit": UNIT, "error": meta.get("error")}
    t = 0.0
    for i in idx:
        t_asm = min(a for a, _, _ in steps[i])
        t_it = min(c / k for _, c, k in steps[i])
        t += t_asm + t_it * gpu_its[i]
    return {"value": round(len(idx) / t, 5), "unit": UNIT, "cores": int(meta.get("threads", 1)), "kind": "reference",
            "sample": f"reference C++ ({meta['exe']}, {cpu_model()}) on {len(idx)} of the 256 problems (stratified by "
                      f"size: {[(spec[i]['N'], spec[i]['k']) for i in idx]}): best of 2 steps of assembly + {CG_SAMPLE} "
                      f"Jacobi-PCG iterations, extrapolated to each problem's FP64 iteration count on the GPU; "
                      f"solves/s = {len(idx)} / the summed solve times"}


def reference_c4(args, rank, world):
    if rank != 0:
        return None
    spec = c4_spec()
    rhs = c4_rhs(spec)
    idx = c4_sample(spec)
    steps, meta = run_reference_c4(spec, rhs, idx, args.warmup + args.steps, CG_SAMPLE, True)
    if steps is None:
        return {"impl": "reference", "unavailable": meta.get("error")}
    per = []
    for rep in range(args.warmup, args.warmup + args.steps):
        t = 0.0
        for i in idx:
            its_full = steps[i][0][2]
            sa, sc, si = steps[i][rep]
            t += sa + (sc / si) * its_full
        per.append(t)
    t = sum(per)
    value = len(per) * len(idx) / t
    cores = int(meta.get("threads", 1))
    sample_txt = (f"reference C++ ({meta['exe']}, OpenMP, {cores} threads, {cpu_model()}) on {len(idx)} of the 256 "
                  f"problems (stratified by size: {[(spec[i]['N'], spec[i]['k']) for i in idx]}): per step and problem "
                  f"assembly + {CG_SAMPLE} Jacobi-PCG iterations extrapolated to the count of its own full solve (first "
                  f"warm-up step); solves/s = problems / summed solve times")
    return {"impl": "reference", "metric": METRIC_C4, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": len(per), "warmup": args.warmup, "ms_per_step": round(t / len(per) * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded: meshes, coefficients, N(0,1) load vectors)",
            "config": {"workload": "config-4 stream: 256 Poisson problems (stratified sample of 8 on the host), FP64 "
                                   "assembly + Jacobi-PCG to 1e-10", "parallelism": "OpenMP (host)"},
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample_txt},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--engine", default="lockstep", choices=["lockstep", "persistent"],
                    help="batched engine of the config-4 stream")
    ap.add_argument("--workload", default="c4s", choices=["c4s", "c2"],
                    help="c4s: the served config-4 stream (default); c2: one P2 solve on 1024x1024")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        line = (reference_c4 if args.workload == "c4s" else reference_c2)(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist = None
    if world > 1:
        import torch
        from femd_b200 import replicas
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist = replicas.init("nccl", 120.0)
    line = (ours_c4 if args.workload == "c4s" else ours_c2)(args, rank, world, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        from femd_b200 import replicas
        replicas.finish(dist)


if __name__ == "__main__":
    main()
