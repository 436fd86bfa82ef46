"""Benchmark of the FEMd 2D P_k assembly + Jacobi-PCG path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-cpu]

Workload (the plain method at scale on one GPU): -Lap u + u = f on rectangle_mesh 1024 x 1024
(2,097,152 triangles), P2 Lagrange (4,190,209 unknowns, 48,136,245 nonzeros), zero Dirichlet,
f = 2 pi^2 sin(pi x) sin(pi y) + sin(pi x) sin(pi y); FP64 assembly of A and b into CSR on the
cached pattern, then FP64 Jacobi-PCG to relative residual 1e-10.  One step = one solve
(assemble A and b, Jacobi, CG).  The metric is solves/s.  Inputs (the CSR matrix, 0.58 GB) are
larger than L2 (126 MB), so no L2 flush is needed between steps.

value      device-resident: mesh, pattern and scatter map already in HBM
e2e        through the public API from host buffers: each step copies the mesh coordinates
           from pinned host memory to the device, assembles, solves and copies x back
roofline   the dominant kernel, the CSR SpMV of the CG loop (k_spmv), timed with CUDA events
           on the library's stream: algorithmic bytes 12 nnz + 4 (n+1) + 8 n + 8 n per launch
cpu_baseline / --impl reference: the reference's own C++ (oracle/_ref/femd_ref_omp, OpenMP,
           every host thread) on the same problem: assembly + Jacobi-PCG, a bounded sample of
           CG iterations per step extrapolated to the full iteration count
Multi-GPU (torchrun): replicas only -- every rank solves its own copy, no collective on the
data path; value = all ranks' solves / the slowest rank's time.
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
UNIT = "solves/s"
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


def ours(args, rank, world, dist):
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
    if dist is None:
        return t
    v = torch.tensor([t], dtype=torch.float64, device="cuda")
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return float(v.item())


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
def reference(args, rank, world):
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        line = reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as D
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = D
    line = ours(args, rank, world, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
