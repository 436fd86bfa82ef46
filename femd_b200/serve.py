"""Serving: a request loop of Poisson solves and backward-Euler heat steps of mixed mesh size and
degree, continuously batched into one persistent Jacobi-PCG launch (femd_b200.batch).

Requests arrive on a seeded Poisson process.  A heat step advances a resident simulation by
one step of (M + dt K) u^{n+1} = M u^n (the loop of the reference's example13, there with a
factored matrix); a fresh Poisson request assembles c (grad u, grad v) on a mesh from the
library and solves it for a random load vector.  The server admits arrived requests while free
HBM allows (in arrival order, skipping ones that do not fit or whose simulation is busy), arms
them in the batch, and advances every armed solve by a bounded number of iterations per launch:
requests that arrive while others are on the GPU join at the next launch, and their work
overlaps on the device.  The baseline is the plain FP64 GPU path serving the same trace first
come, first served, one cg_solve at a time.

Every mesh, space, pattern and simulation is built before the clock starts (the library of a
server); what a request costs -- assembly of a fresh matrix, M u, the solve -- is timed.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass

import numpy as np

from . import core as fb
from .batch import Batch

# N log-uniform in [16, 1024] on a geometric grid of ratio 2^(1/3), so that meshes are reused
SIZES = [int(round(16 * 2 ** (j / 3))) for j in range(19)]


def _torch():
    import torch
    return torch


class SpaceLibrary:
    """Meshes, spaces, patterns and quadrature caches on rectangle_mesh(0,0,1,1,N,N) per (N, k)."""

    def __init__(self):
        self.spaces = {}

    @staticmethod
    def dim(N, k):
        """Unknowns of P_k with every exterior node Dirichlet: the interior nodes of the lattice."""
        return (k * N - 1) ** 2

    def get(self, N, k):
        s = self.spaces.get((N, k))
        if s is None:
            m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
            V = fb.LagrangeSpace2D(m, k, bc="dirichlet")
            P = V.pattern()
            P.batch_layout()                        # the batched engine's layout, before any clock
            s = self.spaces[(N, k)] = dict(mesh=m, V=V, P=P, Qk=V.cache(fb.quad_degree("gradgrad", k)),
                                           Qm=V.cache(fb.quad_degree("mass", k)), n=V.dim, nnz=P.nnz)
        return s


def stiffness(lib, N, k, c=1.0, into=None):
    """c (grad u, grad v) on the library's (N, k) space, with its Jacobi inverse diagonal (into: a
    CSRMatrix on that space's pattern to overwrite instead of a new one)."""
    s = lib.get(N, k)
    K = into if into is not None else fb.CSRMatrix(s["P"], symmetric=True)
    fb.assemble_matrix_2d(s["Qk"], s["Qk"], [1, 2], [1, 2], [c, c], K)
    return K


def mass(lib, N, k):
    """(u, v) on the library's (N, k) space."""
    s = lib.get(N, k)
    M = fb.CSRMatrix(s["P"], symmetric=True)
    fb.assemble_matrix_2d(s["Qm"], s["Qm"], [0], [0], [1.0], M)
    return M


class HeatSession:
    """A resident backward-Euler simulation on (N, k) with step dt: M, A = M + dt K with its
    Jacobi inverse, and the state u (float64, on the device)."""

    def __init__(self, lib, N, k, dt, u0=None, seed=0):
        torch = _torch()
        self.N, self.k, self.dt = int(N), int(k), float(dt)
        self.M = mass(lib, N, k)
        K = stiffness(lib, N, k)
        self.A = self.M.combine(K, 1.0, self.dt)
        fb.JacobiPreconditioner(self.A)
        del K
        self.n = self.A.nrows
        if u0 is None:
            u0 = torch.as_tensor(np.random.default_rng(seed).standard_normal(self.n)).cuda()
        self.u0 = u0.clone()
        self.u = u0.clone()
        self.busy = False
        self.member = None

    def reset(self):
        self.u = self.u0.clone()
        self.busy = False


@dataclass
class Request:
    rid: int
    t: float                      # arrival, seconds from the start of the trace
    kind: str                     # "heat" | "poisson"
    session: int = -1             # heat: the simulation it advances
    N: int = 0                    # poisson: mesh and degree, coefficient, load-vector seed
    k: int = 1
    c: float = 1.0
    seed: int = 0
    t_admit: float = math.nan
    t_done: float = math.nan
    iterations: int = 0
    converged: bool = False
    residual: float = math.nan
    status: int = 0
    outer: int = 0                # reliable updates (mixed precision)
    x: object = None              # the solution (kept when the server is asked to)
    b: object = None              # poisson: the load vector (device, or pinned host: copied in), else seeded
    out: object = None            # a host tensor that receives the solution

    @property
    def latency(self):
        return self.t_done - self.t


def make_sessions(lib, seed, nsessions, sizes=SIZES, degrees=(1, 2), dt_range=(1e-4, 1e-1)):
    rng = np.random.default_rng(seed)
    out = []
    for s in range(nsessions):
        N = int(rng.choice(sizes))
        k = int(rng.choice(degrees))
        dt = float(np.exp(rng.uniform(np.log(dt_range[0]), np.log(dt_range[1]))))
        out.append(HeatSession(lib, N, k, dt, seed=seed * 7919 + s))
    return out


def make_trace(seed, lam, nreq, nsessions, heat_frac=0.7, sizes=SIZES, degrees=(1, 2)):
    """A seeded request stream: Poisson arrivals at rate lam (requests/s), heat steps (uniform
    over the simulations) and fresh Poisson solves split heat_frac / 1 - heat_frac."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / lam, nreq))
    t -= t[0]
    heat = rng.random(nreq) < heat_frac
    out = []
    for i in range(nreq):
        if heat[i] and nsessions > 0:
            out.append(Request(i, float(t[i]), "heat", session=int(rng.integers(nsessions))))
        else:
            out.append(Request(i, float(t[i]), "poisson", N=int(rng.choice(sizes)), k=int(rng.choice(degrees)),
                               c=float(np.exp(rng.uniform(np.log(0.1), np.log(10.0)))), seed=int(seed) * 1000003 + i))
    return out


def poisson_rhs(n, seed):
    torch = _torch()
    return torch.as_tensor(np.random.default_rng(seed).standard_normal(n)).cuda()


def request_bytes(lib, r, sessions):
    """Device memory a request holds while it is served (the simulations' own is resident)."""
    if r.kind == "heat":
        return 16 * sessions[r.session].n
    s = lib.get(r.N, r.k)
    return 12 * s["nnz"] + 60 * s["n"]


def summarize(trace, elapsed):
    done = [r for r in trace if not math.isnan(r.t_done)]
    lat = np.array([r.latency for r in done]) if done else np.zeros(1)
    return dict(requests=len(trace), completed=len(done), elapsed_s=elapsed,
                solves_per_s=len(done) / elapsed if elapsed > 0 else 0.0,
                p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
                mean_iterations=float(np.mean([r.iterations for r in done])) if done else 0.0,
                max_iterations=int(max([r.iterations for r in done])) if done else 0,
                all_converged=all(r.converged for r in done))


class Server:
    """Continuous batching over one Batch.  mixed: FP32 inner iteration with FP64 reliable
    updates (True) or FP64 Jacobi-PCG; iters: iterations per member per launch.  Admission: the
    device's free memory (free_memory(), default cudaMemGetInfo through torch) less
    reserve_bytes, and, when hbm_budget is given, that budget less what the requests in flight
    hold.  big_nnz: requests whose matrix has at least that many nonzeros are solved one at a time
    on the whole GPU between batch launches (femd_b200.cg_solve: the fused FP64 Jacobi-PCG, or
    the single mixed solve when big_mixed) -- a large system streams HBM better through the
    single-solve kernels than as many table entries among other members.  engine:
    "continuous" (the lockstep engine, resumable: requests join at the next chunk boundary
    after they are admitted, every request in flight advances by about iters iterations per
    step, finished ones leave), "persistent" (members join and leave between cooperative launches
    of at most iters iterations) or "lockstep" (the admitted requests are solved together to
    completion, one wave at a time; requests that arrive meanwhile wait for the next wave)."""

    def __init__(self, lib, sessions=(), *, mixed=True, iters=64, tol=1e-10, reserve_bytes=2 << 30, free_memory=None,
                 hbm_budget=None, max_members=1024, keep_solutions=False, shape=None, big_nnz=None,
                 big_mixed=False, engine="continuous"):
        torch = _torch()
        if engine not in ("persistent", "lockstep", "continuous"):
            raise ValueError(f"serve: unknown engine {engine!r}")
        self.engine = engine
        self.lib, self.sessions = lib, list(sessions)
        self.mixed, self.iters, self.tol = bool(mixed), int(iters), float(tol)
        self.reserve = int(reserve_bytes)
        self.free_memory = free_memory or (lambda: torch.cuda.mem_get_info()[0])
        self.hbm_budget = hbm_budget
        self.max_members = int(max_members)
        self.keep = keep_solutions
        self.big_nnz = big_nnz
        self.big_mixed = bool(big_mixed)
        self.batch = Batch()
        if shape:
            self.batch.configure(*shape)
        for S in self.sessions:
            S.member = None if self._big(S.A.nnz) else self.batch.add(S.A)
        self.launches = 0
        self.active = {}
        self.direct = collections.deque()           # admitted requests for the whole-GPU path
        self.last_launch_s = 0.0
        # finished Poisson requests leave their matrix and batch member here, per (N, k), for the
        # next request on that space: in steady state a request allocates nothing
        self._pool = collections.defaultdict(list)

    def _big(self, nnz):
        return self.big_nnz is not None and nnz >= self.big_nnz

    def _admit(self, r, budget):
        """Set the request up and arm it; the bytes it takes, or None when it has to wait."""
        torch = _torch()
        need = request_bytes(self.lib, r, self.sessions)
        if need > budget:
            return None
        if r.kind == "heat":
            S = self.sessions[r.session]
            if S.busy:
                return None
            S.busy = True
            b = S.M.matvec(S.u)
            x = S.u.clone()
            if S.member is None:
                self.direct.append((r, S, S.A, b, x, need))
            else:
                self.batch.arm(S.member, b, x, tol=self.tol)
                self.active[S.member] = (r, S, None, b, x, need)
        else:
            pool = self._pool[(r.N, r.k)]
            K, mid = pool.pop() if pool else (None, None)
            K = stiffness(self.lib, r.N, r.k, r.c, into=K)
            b = _rhs(r, K.nrows)
            x = torch.zeros(K.nrows, dtype=torch.float64, device=b.device)
            if self._big(K.nnz):
                self.direct.append((r, None, K, b, x, need))
            else:
                if mid is None:
                    mid = self.batch.add(K)
                self.batch.arm(mid, b, x, tol=self.tol)
                self.active[mid] = (r, None, K, b, x, need)
        return need

    def _finish(self, r, S, x, res, t_done):
        r.t_done = t_done
        r.iterations, r.converged = res["iterations"], res["converged"]
        r.residual, r.status, r.outer = res["residual"], res["status"], res["reliable_updates"]
        if self.keep:
            r.x = x
        if r.out is not None:
            r.out.copy_(x, non_blocking=True)
        if S is not None:
            S.u = x
            S.busy = False

    def _solve_direct(self, t0):
        """One request of the whole-GPU path."""
        r, S, K, b, x, _ = self.direct.popleft()
        x, conv, its, res, brk = fb.cg_solve(K, fb.JacobiPreconditioner(K), b, x, max(1000, 10 * K.nrows), self.tol,
                                             mixed=self.mixed and self.big_mixed)
        last = fb.cg_solve.last
        self._finish(r, S, x, dict(iterations=its, converged=conv, residual=res, status=0,
                                   reliable_updates=int(last.outer)), time.perf_counter() - t0)

    def run(self, trace, *, realtime=True, max_seconds=600.0):
        """Serve the trace (arrivals in real time from now, or all at once); returns the summary
        and fills the requests' timing and result fields."""
        torch = _torch()
        for S in self.sessions:
            S.busy = False
        for r in trace:
            if r.kind == "poisson":
                self.lib.get(r.N, r.k)              # the mesh library is set up before the clock
        pending = collections.deque(sorted(trace, key=lambda r: r.t))
        queue = []
        self.active = {}
        self.direct.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: math.inf)
        while pending or queue or self.active or self.direct:
            now = clock()
            while pending and pending[0].t <= now:
                queue.append(pending.popleft())
            if queue:
                budget = self.free_memory() - self.reserve
                if self.hbm_budget is not None:
                    held = sum(a[5] for a in self.active.values()) + sum(a[5] for a in self.direct)
                    budget = min(budget, self.hbm_budget - held)
                keep = []
                for i, r in enumerate(queue):
                    if len(self.active) >= self.max_members or len(keep) >= 256:
                        keep.extend(queue[i:])
                        break
                    need = self._admit(r, budget)
                    if need is None:
                        keep.append(r)
                    else:
                        r.t_admit = time.perf_counter() - t0
                        budget -= need
                queue = keep
            if self.active:
                fin = self.batch.step(self.iters, mixed=self.mixed, engine=self.engine)
                self.launches += 1
                t_done = time.perf_counter() - t0
                for mid, res in fin:
                    r, S, K, b, x, _ = self.active.pop(mid)
                    self.last_launch_s = res["seconds"]
                    self._finish(r, S, x, res, t_done)
                    if S is None:
                        self._pool[(r.N, r.k)].append((K, mid))
                if self.batch.last_status != 0:
                    raise RuntimeError(f"serve: batch launch failed with status {self.batch.last_status}")
            if self.direct:
                self._solve_direct(t0)
            elif not self.active and pending:
                wait = pending[0].t - clock()
                if wait > 2e-3:
                    time.sleep(wait - 1e-3)
            if time.perf_counter() - t0 > max_seconds:
                break
        torch.cuda.synchronize()                    # results copied out to host buffers
        return summarize(trace, time.perf_counter() - t0)


def run_plain(lib, sessions, trace, *, tol=1e-10, realtime=True, keep_solutions=False, mixed=False):
    """The plain FP64 GPU path on the same trace: first come, first served, one cg_solve at a time.
    A Poisson request re-assembles into its (N, k) space's matrix (one per space, kept across
    requests, as a caller of cg_solve would), so the solver's workspace and captured graphs are
    reused; a heat step solves with its simulation's resident matrix."""
    torch = _torch()
    for S in sessions:
        S.busy = False
    for r in trace:
        if r.kind == "poisson":
            lib.get(r.N, r.k)
    order = sorted(trace, key=lambda r: r.t)
    mats = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in order:
        if realtime:
            wait = r.t - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        r.t_admit = time.perf_counter() - t0
        if r.kind == "heat":
            S = sessions[r.session]
            b = S.M.matvec(S.u)
            x, conv, its, res, brk = fb.cg_solve(S.A, fb.JacobiPreconditioner(S.A), b, S.u, max(1000, 10 * S.n), tol,
                                                 mixed=mixed)
            S.u = x
        else:
            K = mats[(r.N, r.k)] = stiffness(lib, r.N, r.k, r.c, into=mats.get((r.N, r.k)))
            b = _rhs(r, K.nrows)
            x, conv, its, res, brk = fb.cg_solve(K, fb.JacobiPreconditioner(K), b, None, max(1000, 10 * K.nrows), tol,
                                                 mixed=mixed)
        torch.cuda.synchronize()
        r.t_done = time.perf_counter() - t0
        r.iterations, r.converged, r.residual = its, conv, res
        if keep_solutions:
            r.x = x
        if r.out is not None:
            r.out.copy_(x, non_blocking=True)
            torch.cuda.synchronize()
    return summarize(trace, time.perf_counter() - t0)


def _rhs(r, n):
    """The request's load vector on the device: its own (copied in from pinned host memory when
    it is there) or the seeded N(0, 1) one."""
    if r.b is None:
        return poisson_rhs(n, r.seed)
    if r.b.numel() != n:
        raise ValueError("serve: load vector length differs from the problem")
    return r.b if r.b.is_cuda else r.b.to("cuda", non_blocking=True)
