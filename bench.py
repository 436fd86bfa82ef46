"""Benchmark of the FEMd 2D P_k assembly + Jacobi-PCG path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-cpu]
                    [--workload c4s|c2|c5] [--engine lockstep|persistent] [--no-c5]

Default workload (c4s), the metric's "served + mixed vs plain GPU": the stream of 256 independent
Poisson problems -c Lap u = f on rectangle_mesh(0,0,1,1,N,N), N uniform in {16..256}, P_k with k
uniform in {1,2,3}, c log-uniform in [0.1, 10], load-vector dof values N(0,1), all from seed 0
(30.5M unknowns, 448M nonzeros in all), served by femd_b200.serve.Server: every problem is a
request (all arriving at once), assembled in FP64 on its cached pattern and solved by the
batched Jacobi-PCG -- FP32 inner iteration on an FP32 matrix copy with FP64 reliable updates --
to relative residual 1e-10.  One step = serving the whole stream.  The metric is solves/s;
p50 / p99 request latency, the plain FP64 GPU path on the same stream (one assembly + cg_solve
per request, first come first served) and the largest relative difference between the served
and the plain FP64 solutions are reported beside it.  The working set (4+ GB) is larger than
L2, so no flush is needed between steps.

value      device-resident: meshes, spaces and patterns built, load vectors in HBM
e2e        through the public API from host buffers: each step copies every load vector from
           pinned host memory to the device and every solution back to pinned host memory
roofline   the batched solve (all its kernels), timed with CUDA events on the library's stream;
           algorithmic bytes from each member's iterations and reliable updates
kernels    K3 (FP64 assembly), K5 (SpMV + p.Ap) and K6 (the fused CG update) at config-2 size
           (rectangle 1024 x 1024, P2), CUDA events, against the measured HBM peak
checker    (outside every timed region) the served mixed and plain FP64 solutions of 8 problems
           of the stream (one per size stratum) against the reference's own FP64 sparse Cholesky
           solution (oracle/_ref), relative error each
c5         the config-5 serving sweep (Poisson arrivals at lambda = 100, 1,000, 10,000 req/s;
           backward-Euler heat steps and fresh Poisson solves 70/30), served vs plain
cpu_baseline / --impl reference: the reference's own C++ (oracle/_ref/femd_ref_omp, OpenMP,
           every host thread): full solves (assembly + Jacobi-PCG to 1e-10) of the 8 stratum
           problems; solves/s = 8 / the sum of their mean solve times
Workload c2 (the plain method at scale): -Lap u + u = f on rectangle_mesh 1024x1024, P2,
           FP64 assembly + FP64 Jacobi-PCG to 1e-10, one solve per step.
Multi-GPU (torchrun): replicas only -- every rank serves its own copy of the stream, no
collective on the data path; value = all ranks' solves / the slowest rank's time.

The workload spec below is plain numpy: the reference arm never imports femd_b200.
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
METRIC_C5 = "solves/s and p99 latency of the config-5 serving sweep (heat steps + Poisson solves), served vs plain"
UNIT = "solves/s"
NPROB, SEED, NSAMPLE = 256, 0, 8
N_MESH, DEGREE, TOL = 1024, 2, 1e-10
LAMBDAS = (100.0, 1000.0, 10000.0)
PI = 3.141592653589793


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ---- the workloads (plain numpy) ---------------------------------------------------------------
def c4_spec(seed=SEED, nprob=NPROB, nmin=16, nmax=256):
    """The config-4 stream: N uniform in {nmin..nmax}, k uniform in {1,2,3}, c log-uniform in
    [0.1, 10], and each problem's load-vector seed (the same draws as
    femd_b200.workloads.poisson_batch_spec)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    N = rng.integers(nmin, nmax + 1, nprob)
    k = rng.integers(1, 4, nprob)
    c = np.exp(rng.uniform(np.log(0.1), np.log(10.0), nprob))
    return [dict(N=int(N[i]), k=int(k[i]), c=float(c[i]), seed=int(seed) * 100003 + i) for i in range(nprob)]


def c4_dim(N, k):
    """Unknowns of P_k on rectangle_mesh N x N with every exterior node Dirichlet."""
    return (k * N - 1) ** 2


def c4_rhs(spec):
    """The load vectors (float64 numpy), from each problem's seed."""
    import numpy as np
    return [np.random.default_rng(s["seed"]).standard_normal(c4_dim(s["N"], s["k"])) for s in spec]


def c4_sample(spec, m=NSAMPLE):
    """A stratified sample, in increasing size: the problems sorted by work (n x iterations ~
    (kN)^3), cut into m strata of equal count, the middle problem of each."""
    work = [(s["k"] * s["N"]) ** 3 for s in spec]
    order = sorted(range(len(spec)), key=lambda i: (work[i], i))
    return [order[(2 * j + 1) * len(order) // (2 * m)] for j in range(m)]


# ---- the reference's own CPU build (oracle/_ref) -------------------------------------------------
def _ref_binary():
    for name in ("femd_ref_omp", "femd_ref"):
        p = os.path.join(ROOT, "oracle", "_ref", name)
        if os.path.exists(p):
            return p
    return None


def _ref_env(threads=None):
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads or os.cpu_count())
    env["OPENBLAS_NUM_THREADS"] = "1"
    return env


def _parse(txt):
    steps, meta = [], {}
    for line in txt.splitlines():
        p = line.split()
        if not p:
            continue
        if p[0] == "step":
            steps.append((float(p[1]), float(p[2]), int(p[3])))
        elif len(p) == 2:
            meta[p[0]] = p[1]
    return steps, meta


def ref_full_solve(sp, b, d, threads=None):
    """One full solve of a stream problem by the reference's C++: FP64 assembly + cg_jacobi to
    1e-10 (the driver times assembly and solve, not its setup).  Returns (t_asm, t_cg, its, meta)."""
    import numpy as np
    exe = _ref_binary()
    bp = os.path.join(d, "b.bin")
    np.asarray(b, dtype=np.float64).tofile(bp)
    a = [exe, "poisson_vec", str(sp["N"]), str(sp["k"]), "-", "--c", repr(sp["c"]), "--b", bp, "--nodump", "--nocg",
         "--time", "1", "--cg-sample", "0"]
    steps, meta = _parse(subprocess.run(a, capture_output=True, text=True, env=_ref_env(threads), check=True).stdout)
    ta, tc, its = steps[0]
    return ta, tc, its, meta


def ref_cholesky(sp, b, d, threads=None):
    """The reference's FP64 sparse Cholesky solution of a stream problem (SparseCholesky::apply,
    include/femd/sparse/cholesky.hpp:212)."""
    import numpy as np
    exe = _ref_binary()
    bp = os.path.join(d, "b.bin")
    np.asarray(b, dtype=np.float64).tofile(bp)
    out = os.path.join(d, "chol")
    os.makedirs(out, exist_ok=True)
    subprocess.run([exe, "poisson_vec", str(sp["N"]), str(sp["k"]), out, "--c", repr(sp["c"]), "--b", bp, "--chol",
                    "--nocg", "--nodump"], capture_output=True, text=True, env=_ref_env(threads), check=True)
    return np.fromfile(os.path.join(out, "x_chol.bin"))


def ref_sample_solves(spec, rhs, order, threads=None):
    """Full reference solves of the problems `order` (indices into spec), one each, in that order;
    returns [(i, seconds, iterations)] and the driver's meta."""
    out, meta = [], {}
    with tempfile.TemporaryDirectory() as d:
        for i in order:
            ta, tc, its, meta = ref_full_solve(spec[i], rhs[i], d, threads)
            out.append((i, ta + tc, its))
    return out, meta


def sample_rate(solves, idx):
    """solves/s of the stratified sample: len(idx) / the sum over its problems of each problem's
    mean solve time (every problem solved at least once; else problems / summed time)."""
    per = {}
    for i, t, _ in solves:
        per.setdefault(i, []).append(t)
    if all(i in per for i in idx):
        return len(idx) / sum(sum(per[i]) / len(per[i]) for i in idx)
    return len(solves) / sum(t for _, t, _ in solves)


def cpu_baseline_c4(spec, rhs):
    idx = c4_sample(spec)
    if _ref_binary() is None:
        return {"value": None, "unit": UNIT, "error": "oracle/_ref is not built (make -C oracle ref where the "
                                                      "reference tree is)"}
    solves, meta = ref_sample_solves(spec, rhs, idx)
    v = sample_rate(solves, idx)
    return {"value": round(v, 5), "unit": UNIT, "cores": int(meta.get("threads", os.cpu_count())), "kind": "reference",
            "sample": f"reference C++ ({os.path.basename(_ref_binary())}, OpenMP, {cpu_model()}): one full solve "
                      f"(FP64 assembly + Jacobi-PCG to 1e-10) of each of the 8 stratum problems of the stream "
                      f"{[(spec[i]['N'], spec[i]['k']) for i in idx]}, iterations {[s[2] for s in solves]}; "
                      f"solves/s = 8 / the summed solve times ({sum(s[1] for s in solves):.1f} s)"}


# ---- reference arm -----------------------------------------------------------------------------
def reference_c4(args, rank, world):
    """The reference's CPU implementation on the config-4 stream: each step is one full solve of
    every one of the 8 stratum problems of the stream (a bounded, size-stratified sample of the
    256), every host thread; value = 8 / the sum of the problems' mean solve times, so any number
    of steps measures the same sample."""
    if rank != 0:
        return None
    if _ref_binary() is None:
        return {"impl": "reference", "unavailable": "oracle/_ref is not built (the reference tree was absent where "
                                                    "the bench was built)"}
    spec = c4_spec()
    idx = c4_sample(spec)
    rhs_all = c4_rhs([spec[i] for i in idx])
    rhs = {i: b for i, b in zip(idx, rhs_all)}
    t_wall0 = time.time()
    with tempfile.TemporaryDirectory() as d:
        for j in range(args.warmup):
            for i in idx:
                ref_full_solve(spec[i], rhs[i], d)
        solves, meta = [], {}
        tw = 0.0
        for j in range(args.steps):
            t0 = time.time()
            for i in idx:
                ta, tc, its, meta = ref_full_solve(spec[i], rhs[i], d)
                solves.append((i, ta + tc, its))
            tw += time.time() - t0
    value = sample_rate(solves, idx)
    cores = int(meta.get("threads", os.cpu_count()))
    t_solve = sum(t for _, t, _ in solves)
    sample_txt = (f"reference C++ ({os.path.basename(_ref_binary())}, OpenMP, {cores} threads, {cpu_model()}): each step "
                  f"= one full solve (FP64 assembly + Jacobi-PCG to 1e-10, timed by the driver) of each of the 8 stratum "
                  f"problems of the stream {[(spec[i]['N'], spec[i]['k']) for i in idx]}; solves/s = 8 / the sum of the "
                  f"problems' mean solve times")
    return {"impl": "reference", "metric": METRIC_C4, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tw / max(1, args.steps) * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded: meshes, coefficients, N(0,1) load vectors)",
            "config": {"workload": "config-4 stream: the 8 stratum problems of the 256 (each solved in full once per "
                                   "step), FP64 assembly + Jacobi-PCG to 1e-10 on the host cores",
                       "sample": [(spec[i]["N"], spec[i]["k"]) for i in idx], "parallelism": "OpenMP (host)",
                       "solve_seconds_total": round(t_solve, 3), "wall_seconds": round(time.time() - t_wall0, 2)},
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample_txt},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_c2(args, rank, world):
    if rank != 0:
        return None
    exe = _ref_binary()
    if exe is None:
        return {"impl": "reference", "unavailable": "oracle/_ref is not built"}
    a = [exe, "helmholtz_sin", str(N_MESH), str(DEGREE), "-", "--nodump", "--nocg", "--time",
         str(args.warmup + args.steps), "--cg-sample", "0"]
    steps, meta = _parse(subprocess.run(a, capture_output=True, text=True, env=_ref_env(), check=True).stdout)
    timed = steps[args.warmup:]
    t = sum(sa + sc for sa, sc, _ in timed)
    value = len(timed) / t
    cores = int(meta.get("threads", 1))
    sample_txt = (f"reference C++ ({os.path.basename(exe)}, OpenMP, {cores} threads, {cpu_model()}): per step FP64 "
                  f"assembly + a full Jacobi-PCG solve to 1e-10 ({timed[-1][2]} iterations)")
    return {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": len(timed), "warmup": args.warmup, "ms_per_step": round(t / len(timed) * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded closed-form rhs)",
            "config": {"workload": "rectangle_mesh 1024x1024, P2, -Lap u + u = f (2 pi^2+1) sin sin, FP64 assembly + "
                                   "Jacobi-PCG tol 1e-10", "n": int(meta.get("dim", 0)), "nnz": int(meta.get("nnz", 0)),
                       "cg_iterations": timed[-1][2], "parallelism": "OpenMP (host)"},
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample_txt},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


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


def _max_over_ranks(torch, dist, t):
    from femd_b200.replicas import max_over_ranks
    return max_over_ranks(t, dist, "cuda")


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


# ---- config 2: the plain method at scale ---------------------------------------------------------
class Problem:
    """-Lap u + u = f on rectangle_mesh N x N, P_k, set up once on the GPU: mesh, space (device
    numbering), caches, pattern, matrix."""

    def __init__(self, fb, torch, N=N_MESH, k=DEGREE, tune=True):
        t0 = time.time()
        self.fb, self.torch = fb, torch
        self.ctx = fb.context()
        self.mesh = fb.rectangle_mesh(0, 0, 1, 1, N, N)
        self.V = fb.LagrangeSpace2D(self.mesh, k, bc="dirichlet", numbering="device")
        self.Qa = self.V.cache(fb.quad_degree("helmholtz", k))
        self.Qf = self.V.cache(fb.quad_degree("rhs_data", k))
        self.P = self.V.pattern()
        self.K = fb.CSRMatrix(self.P)
        self.b = torch.empty(self.V.dim, dtype=torch.float64, device="cuda")
        fb.scatter_map_2d(self.P)
        self.coef_f = fb.Coef.helmholtz_sinsin(2.0 * PI * PI, PI, PI)
        fb.assemble_matrix_2d(self.Qa, self.Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], self.K)
        self.spmv_shape = None
        if tune:
            # the project autotuner picks the SpMV launch shape for this matrix
            shape, _ = self.K.autotune_spmv(True)
            self.spmv_shape = f"{shape & 0xff} lanes/row, {max(shape >> 8, 1)} loads/lane"
        self.setup_s = time.time() - t0
        self.n, self.nnz = self.V.dim, self.P.nnz

    def assemble(self, jacobi=True):
        self.fb.assemble_matrix_2d(self.Qa, self.Qa, [1, 2, 0], [1, 2, 0], [1.0, 1.0, 1.0], self.K, jacobi=jacobi)

    def step(self, phases=None):
        fb, torch = self.fb, self.torch
        s = self.ctx.stream
        if phases is not None:
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(s)
        self.assemble()
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


def kernel_rates(fb, torch, pr, hbm):
    """K3, K5 and K6 at the problem's size: CUDA-event time per launch, algorithmic bytes per
    launch, achieved GB/s and the fraction of the measured HBM peak."""
    import ctypes as C
    ctx, s = pr.ctx, pr.ctx.stream
    n, nnz = pr.n, pr.nnz
    nv, ne, nl = pr.mesh.nverts, pr.mesh.ncells, pr.V.nloc
    out = []
    # K3: the FP64 assembly (per-cell factors + the row kernel), values only
    for _ in range(3):
        pr.assemble(jacobi=False)
    reps = 20
    t, _ = event_time(torch, s, lambda: pr.assemble(jacobi=False), reps)
    alg3 = 16 * nv + 12 * ne + 4 * ne * nl * nl + 8 * nnz
    out.append(("K3 assembly (k_elem_factors + k_assemble_rows_off), FP64 values", t / reps, alg3,
                "16 nv (coordinates) + 12 ne (triangles) + 4 ne nloc^2 (map) + 8 nnz (values written)"))
    pr.assemble(jacobi=True)
    us = C.c_double()
    for kern, name, alg, txt in (
            (0, "K5 k_spmv (FP64 SpMV fused with p.Ap)", 12 * nnz + 4 * (n + 1) + 16 * n,
             "12 nnz + 4 (n+1) + 8 n (p, counted once) + 8 n (Ap)"),
            (1, "K6 k_cg_update (x += a p, r -= a Ap, ||r||^2, r.D^-1 r)", 56 * n, "40 n read + 16 n written")):
        fb.core.check(fb.lib.femd_cuda_kernel_time(ctx.h, pr.K.h, kern, 50, C.byref(us)))
        out.append((name, us.value * 1e-6, alg, txt))
    rows = []
    for name, sec, alg, txt in out:
        gbs = alg / sec / 1e9
        rows.append({"kernel": name, "us_per_launch": round(sec * 1e6, 2), "algorithmic_bytes": int(alg),
                     "bytes_model": txt, "achieved_gbs": round(gbs, 1), "frac_of_measured_hbm": round(gbs / hbm, 4)})
    return rows


def ours_c2(args, rank, world, dist):
    import torch
    import femd_b200 as fb
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pr = Problem(fb, torch)
    ctx = pr.ctx
    s = ctx.stream
    hbm, peak_kind = peaks()
    its = None
    for _ in range(args.warmup):
        _, its, res = pr.step()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

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
    # end to end: the mesh coordinates from pinned host memory in, the solution out, every step
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
    kern = kernel_rates(fb, torch, pr, hbm)
    k5 = kern[1]
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
        "roofline": {"kernel": k5["kernel"], "bound": "hbm", "achieved": k5["achieved_gbs"], "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": k5["frac_of_measured_hbm"],
                     "traffic": _traffic("k_spmv_c2_traffic.json", k5["algorithmic_bytes"]),
                     "algorithmic_bytes": k5["algorithmic_bytes"], "launch_us": k5["us_per_launch"]},
        "kernels": kern,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_c2()
    return line


def cpu_baseline_c2():
    exe = _ref_binary()
    if exe is None:
        return {"value": None, "unit": UNIT, "error": "oracle/_ref is not built"}
    a = [exe, "helmholtz_sin", str(N_MESH), str(DEGREE), "-", "--nodump", "--nocg", "--time", "1", "--cg-sample", "0"]
    steps, meta = _parse(subprocess.run(a, capture_output=True, text=True, env=_ref_env(), check=True).stdout)
    ta, tc, its = steps[0]
    return {"value": round(1.0 / (ta + tc), 5), "unit": UNIT, "cores": int(meta.get("threads", 1)), "kind": "reference",
            "sample": f"reference C++ ({os.path.basename(exe)}, {cpu_model()}): one full solve (FP64 assembly + "
                      f"Jacobi-PCG to 1e-10, {its} iterations): assembly {ta:.3f} s, CG {tc:.2f} s"}


def _traffic(name, alg):
    """DRAM bytes per launch from an ncu capture's measured DRAM / algorithmic ratio (profiles/)."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    try:
        return int(json.load(open(p))["dram_over_algorithmic"] * alg)
    except Exception:
        return None


# ---- config 4: the served stream ---------------------------------------------------------------
def batch_bytes(reqs, lib, mixed=True, compact=False):
    """Algorithmic HBM bytes of the batched solve that served these requests
    (femd_b200.workloads.batch_bytes)."""
    from femd_b200.workloads import batch_bytes as bb
    sizes = [(lib.get(r.N, r.k)["n"], lib.get(r.N, r.k)["nnz"]) for r in reqs]
    return bb(sizes, [dict(iterations=r.iterations, reliable_updates=r.outer) for r in reqs], mixed, compact)


def checker(spec, rhs, served, plain):
    """The served and plain solutions of the stratum problems against the reference's FP64
    sparse Cholesky solution (outside every timed region)."""
    import numpy as np
    idx = c4_sample(spec)
    if _ref_binary() is None:
        return {"error": "oracle/_ref is not built"}
    rows, es, ep = [], [], []
    with tempfile.TemporaryDirectory() as d:
        for i in idx:
            xc = ref_cholesky(spec[i], rhs[i], d)
            nc = np.linalg.norm(xc)
            e_s = float(np.linalg.norm(served[i] - xc) / nc)
            e_p = float(np.linalg.norm(plain[i] - xc) / nc)
            es.append(e_s)
            ep.append(e_p)
            rows.append({"N": spec[i]["N"], "k": spec[i]["k"], "n": int(xc.size), "served_mixed": e_s, "plain_fp64": e_p})
    return {"oracle": "reference SparseCholesky (FP64, AMD), oracle/_ref", "problems": rows,
            "err_vs_cholesky_max_served_mixed": max(es), "err_vs_cholesky_max_plain_fp64": max(ep),
            "contract": 1e-8, "within_contract": bool(max(es) <= 1e-8 and max(ep) <= 1e-8)}


def ours_c4(args, rank, world, dist):
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
    # the lockstep launch shape (nonzeros per block), autotuned before the clock on every 8th
    # problem of the stream
    tuned, tune_times = None, {}
    if args.engine in ("lockstep", "continuous"):
        sample = range(0, NPROB, 8)
        tb = fb.Batch([serve.stiffness(lib, spec[i]["N"], spec[i]["k"], spec[i]["c"]) for i in sample])
        tuned, tune_times = tb.tune_lockstep([b_dev[i] for i in sample])
        del tb
        srv.batch.configure_lockstep(nnz_per_entry=tuned)
    setup_s = time.time() - t_setup
    ctx = fb.context()
    s = ctx.stream

    def reqs(host=False):
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
    # ---- the plain FP64 GPU path on the same stream (one pass), the served-vs-plain difference,
    # and both against the reference's Cholesky on the stratum problems (outside the timed regions)
    served = reqs()
    srv_keep = serve.Server(lib, [], mixed=True, iters=1 << 30, keep_solutions=True, engine=args.engine)
    if tuned:
        srv_keep.batch.configure_lockstep(nnz_per_entry=tuned)
    srv_keep.run(served, realtime=False)
    xs_served = {r.rid: r.x for r in served}
    plain = reqs()
    pst = serve.run_plain(lib, [], plain, tol=1e-10, realtime=False, keep_solutions=True)
    err = 0.0
    idx = set(c4_sample(spec))
    keep_s, keep_p = {}, {}
    for r in plain:
        a = xs_served[r.rid]
        err = max(err, float(torch.linalg.norm(a - r.x) / torch.linalg.norm(r.x)))
        if r.rid in idx:
            keep_s[r.rid] = a.cpu().numpy()
            keep_p[r.rid] = r.x.cpu().numpy()
        r.x = None
    xs_served.clear()
    chk = checker(spec, rhs, keep_s, keep_p) if rank == 0 else None
    # ---- roofline of the batched solve of the last timed step
    lst = srv.batch.lockstep_stats() if args.engine != "persistent" else {"compact": 0, "plain": 1}
    all_compact = lst["compact"] > 0 and lst["plain"] == 0
    alg = batch_bytes(last, lib, mixed=True, compact=all_compact)
    t_launch = launch_s[-1]
    achieved = alg / t_launch / 1e9
    lockstep = args.engine in ("lockstep", "continuous")
    traffic = _traffic("k_ls_spmv_mixed_traffic.json" if lockstep else "k_batch_pcg_traffic.json", alg)
    nnz = sum(lib.get(sp["N"], sp["k"])["nnz"] for sp in spec)
    n = sum(lib.get(sp["N"], sp["k"])["n"] for sp in spec)
    line = {
        "metric": METRIC_C4, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_all / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (FP32 inner PCG, FP64 assembly/residual/update)",
        "data": "synthetic (seeded: meshes, coefficients, N(0,1) load vectors)",
        "config": {"workload": "config-4 stream: 256 Poisson problems, rectangle N x N (N in 16..256), P1-P3, "
                               "c log-uniform [0.1,10], served (all arrive at t=0), FP64 assembly per request + "
                               f"FP32-inner / FP64-refined batched Jacobi-PCG to 1e-10 ({args.engine} engine)",
                   "problems": NPROB, "n_total": n, "nnz_total": nnz, "arrivals": "burst at t=0",
                   "p50_ms": round(st["p50_ms"], 2), "p99_ms": round(st["p99_ms"], 2),
                   "mean_iterations": round(st["mean_iterations"], 1), "max_iterations": st["max_iterations"],
                   "slowest": [[r.N, r.k, r.iterations, r.outer] for r in sorted(last, key=lambda r: -r.iterations)[:4]],
                   "all_converged": st["all_converged"],
                   "max_rel_diff_vs_plain_fp64": err,
                   "plain_fp64_gpu": {"solves_per_s": round(pst["solves_per_s"], 3), "p50_ms": round(pst["p50_ms"], 2),
                                      "p99_ms": round(pst["p99_ms"], 2), "mean_iterations": round(pst["mean_iterations"], 1),
                                      "max_iterations": pst["max_iterations"],
                                      "path": "per request: FP64 assembly + cg_solve (CUDA-graph CG), FIFO"},
                   "served_over_plain": round(value / pst["solves_per_s"], 3),
                   "checker": chk,
                   "engine": args.engine,
                   "batch_shape": srv.batch.params() if not lockstep else dict(srv.batch.lockstep_params(),
                                                                               **srv.batch.lockstep_stats()),
                   "lockstep_tuning": ({"chosen_nnz_per_entry": tuned, "sample": "every 8th problem, 48 iterations",
                                        "seconds": {str(c): round(t, 5) for c, t in tune_times.items()}}
                                       if tuned else None),
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
    # the per-kernel rates of the plain path's kernels at config-2 size (outside the timed regions)
    pr = Problem(fb, torch, tune=False)
    line["kernels"] = kernel_rates(fb, torch, pr, hbm)
    line["kernels_case"] = (f"rectangle_mesh 1024x1024, P2, -Lap u + u (n {pr.n}, nnz {pr.nnz}); default SpMV "
                            f"shape; CUDA events on the library stream, mean of back-to-back launches")
    del pr
    if not args.no_c5:
        line["c5"] = c5_sweep(fb, torch, nreq=args.c5_requests)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_c4(spec, rhs)
    return line


# ---- config 5: the serving sweep ---------------------------------------------------------------
C5_BIG_NNZ = 1_000_000


def c5_sweep(fb, torch, nreq=120, nsessions=16, seed=21, lambdas=LAMBDAS, big_nnz=C5_BIG_NNZ):
    """Served (mixed precision: continuous batching, and requests of at least big_nnz nonzeros
    one at a time on the whole GPU by the single mixed solve) and plain FP64 on the same seeded
    trace at each lambda: solves/s, p50 / p99 latency; the simulations are reset between the two
    paths."""
    from femd_b200 import serve
    lib = serve.SpaceLibrary()
    sessions = serve.make_sessions(lib, seed, nsessions)
    rows = []
    for lam in lambdas:
        row = {"lambda_req_s": lam, "requests": nreq}
        for path in ("plain", "served"):
            for S in sessions:
                S.reset()
            trace = serve.make_trace(seed + int(lam), lam, nreq, nsessions)
            if path == "plain":
                st = serve.run_plain(lib, sessions, trace, tol=TOL, realtime=True)
            else:
                srv = serve.Server(lib, sessions, mixed=True, engine="continuous", big_nnz=big_nnz, big_mixed=True)
                st = srv.run(trace, realtime=True)
                del srv
            row[path] = {"solves_per_s": round(st["solves_per_s"], 3), "p50_ms": round(st["p50_ms"], 1),
                         "p99_ms": round(st["p99_ms"], 1), "all_converged": st["all_converged"]}
        rows.append(row)
    return {"workload": f"config 5: {nsessions} resident heat sessions (N log-uniform on a 2^(1/3) grid in [16, 1024], "
                        f"k in {{1, 2}}, dt log-uniform in [1e-4, 1e-1]), {nreq} requests per lambda (70% "
                        "backward-Euler steps, 30% fresh Poisson), Poisson arrivals in real time; served: "
                        f"requests under {big_nnz} nonzeros batched (continuous lockstep engine), the others solved one "
                        "at a time on the whole GPU (single-system PCG) between batch steps, all in FP32-inner / "
                        "FP64-refined mixed precision",
            "sweep": rows}


def ours_c5(args, rank, world, dist):
    import torch
    import femd_b200 as fb
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.time()
    c5 = c5_sweep(fb, torch, nreq=args.c5_requests)
    served = [r["served"] for r in c5["sweep"]]
    total = sum(r["requests"] for r in c5["sweep"])
    secs = sum(r["requests"] / s["solves_per_s"] for r, s in zip(c5["sweep"], served))
    return {"metric": METRIC_C5, "value": round(total / secs, 4), "unit": UNIT, "n_gpus": world, "steps": 1,
            "warmup": 0, "ms_per_step": round(secs * 1e3, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded trace)",
            "config": {"workload": c5["workload"], "sweep": c5["sweep"], "wall_s": round(time.time() - t0, 1)}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-c5", action="store_true", help="skip the config-5 serving sweep leg of the c4s line")
    ap.add_argument("--c5-requests", type=int, default=120, help="requests per lambda of the config-5 sweep")
    ap.add_argument("--engine", default="continuous", choices=["continuous", "lockstep", "persistent"],
                    help="batched engine of the config-4 stream (continuous: the lockstep engine, resumable)")
    ap.add_argument("--workload", default="c4s", choices=["c4s", "c2", "c5"],
                    help="c4s: the served config-4 stream (default); c2: one P2 solve on 1024x1024; c5: the serving sweep")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        fn = {"c4s": reference_c4, "c2": reference_c2}.get(args.workload)
        line = fn(args, rank, world) if fn else (
            {"impl": "reference", "unavailable": "the reference has no serving loop (config 5 is GPU-side only)"}
            if rank == 0 else None)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist = None
    if world > 1:
        import torch
        from femd_b200 import replicas
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist = replicas.init("nccl", 120.0)
    fn = {"c4s": ours_c4, "c2": ours_c2, "c5": ours_c5}[args.workload]
    line = fn(args, rank, world, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        from femd_b200 import replicas
        replicas.finish(dist)


if __name__ == "__main__":
    main()
