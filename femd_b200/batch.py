"""Batched Jacobi-PCG: many independent systems solved together (femd_cuda_batch_*).

A Batch holds member systems (CSR matrices with their Jacobi inverse diagonals) and two engines.
The persistent engine runs every member in one cooperative launch (teams of blocks per member);
arm() / step() advance armed members a bounded number of iterations per launch, so members can
join and leave between launches (the continuous batching of femd_b200.serve).  The lockstep
engine runs each iteration as a few whole-GPU kernels over every member still running, to
completion (solve(..., engine="lockstep"), or step(engine="lockstep") for a wave of armed
members).  In either engine a member's iterates depend on the member and the engine's shape
alone: the same bits alone or in any mix.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import _native as N
from .core import CSRMatrix, _as_device, _torch, check, context, lib


def _result(r: N.femd_cg_result) -> dict:
    return dict(converged=bool(r.converged), iterations=int(r.iterations), residual=float(r.residual),
                breakdown=bool(r.breakdown), status=int(r.status), reliable_updates=int(r.outer),
                seconds=float(r.seconds))


class Batch:
    """Member systems solved together, FP64 or mixed precision (FP32 inner iteration, FP64
    reliable updates)."""

    def __init__(self, mats: list[CSRMatrix] = (), nnz_per_block: int = 0, ctx=None):
        from .core import JacobiPreconditioner
        self.ctx = ctx or context()
        mats = list(mats)
        for K in mats:
            JacobiPreconditioner(K)             # the inverse diagonal, checked (zero diagonal -> ValueError)
        arr = (C.c_void_p * max(len(mats), 1))(*[K.h.value for K in mats])
        h = C.c_void_p()
        check(lib.femd_cuda_batch_create(self.ctx.h, len(mats), arr, int(nnz_per_block), C.byref(h)))
        self.h = h
        self.members = {i: K for i, K in enumerate(mats)}   # id -> matrix (kept alive while a member)
        self.mats = mats
        self.last_status = N.FEMD_OK
        self._armed = {}                                    # id -> (b, x) kept alive while armed
        self._ls_shape = dict(nnz_per_entry=16384, chunk=8, spmv="row groups", compact=True)

    def __del__(self):
        try:
            if self.h and not sys.is_finalizing():
                lib.femd_cuda_release(self.h)
                self.h = None
        except Exception:
            pass

    # ---- shape -------------------------------------------------------------------------
    def info(self):
        n, g, s = C.c_int(), C.c_int(), C.c_int()
        teams = np.empty(max(len(self.members), 1), dtype=np.int32)
        check(lib.femd_cuda_batch_info(self.h, C.byref(n), C.byref(g), C.byref(s), teams.ctypes.data_as(C.POINTER(C.c_int))))
        return dict(nprob=n.value, grid=g.value, slots=s.value, teams=teams[:n.value])

    def configure(self, block=256, nnz_per_block=65536, nnz_per_thread=4):
        """Set the launch shape (femd_cuda_batch_configure)."""
        check(lib.femd_cuda_batch_configure(self.h, int(block), int(nnz_per_block), int(nnz_per_thread)))

    def configure_lockstep(self, nnz_per_entry=0, chunk=0, windows=None, compact=None):
        """Shape of the lockstep engine (femd_cuda_batch_lockstep_configure; 0 / None keep a
        value).  windows: SpMV by windows of whole rows (True) or by row groups (False); compact:
        in mixed precision, the reordered layout (SELL-32 slices of length-sorted RCM rows, one
        lane per row, 16-bit column offsets, the direction read from shared memory; True, the
        default) or the plain layout (False).  Row groups and windows are the FP64 and plain FP32
        layouts' SpMV forms."""
        w = -1 if windows is None else int(bool(windows))
        cp = -1 if compact is None else int(bool(compact))
        check(lib.femd_cuda_batch_lockstep_configure(self.h, int(nnz_per_entry), int(chunk), w, cp))
        if nnz_per_entry:
            self._ls_shape["nnz_per_entry"] = int(nnz_per_entry)
        if chunk:
            self._ls_shape["chunk"] = int(chunk)
        if windows is not None:
            self._ls_shape["spmv"] = "windows" if windows else "row groups"
        if compact is not None:
            self._ls_shape["compact"] = bool(compact)

    def lockstep_stats(self):
        """The last lockstep solve's layout (femd_cuda_batch_lockstep_stats): members in the compact
        and in the plain layout, the widest shared-memory window, the table entries."""
        out = (C.c_longlong * 4)()
        check(lib.femd_cuda_batch_lockstep_stats(self.h, out))
        return dict(compact=out[0], plain=out[1], widest_window=out[2], entries=out[3])

    def lockstep_params(self):
        """The lockstep engine's shape as configured (nonzeros per table entry, iterations per
        chunk, SpMV form)."""
        return dict(self._ls_shape)

    def params(self):
        b, n, t, g = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib.femd_cuda_batch_params(self.h, C.byref(b), C.byref(n), C.byref(t), C.byref(g)))
        return dict(block=b.value, nnz_per_block=n.value, nnz_per_thread=t.value, graph=g.value)

    # ---- fixed batch -------------------------------------------------------------------
    def _vectors(self, bs, xs):
        torch = _torch()
        mats = [self.members[i] for i in sorted(self.members)]
        bs = [_as_device(b, self.ctx) for b in bs]
        if len(bs) != len(mats):
            raise ValueError("batch: one right-hand side per member")
        if xs is None:
            xs = [torch.zeros(K.nrows, dtype=torch.float64, device=b.device) for K, b in zip(mats, bs)]
        for K, b, x in zip(mats, bs, xs):
            if b.numel() != K.nrows or x.numel() != K.nrows:
                raise ValueError("batch: vector length differs from its matrix")
        bp = (C.c_void_p * len(bs))(*[b.data_ptr() for b in bs])
        xp = (C.c_void_p * len(xs))(*[x.data_ptr() for x in xs])
        return bs, xs, bp, xp

    def tune(self, bs, *, tol=1e-10, max_iter=0, mixed=True):
        """Autotune the launch shape on these right-hand sides (femd_cuda_batch_tune); returns the
        chosen params and the best time in seconds."""
        bs, xs, bp, xp = self._vectors(bs, None)
        best = (C.c_int * 3)()
        sec = C.c_double()
        self.ctx.enter()
        st = lib.femd_cuda_batch_tune(self.ctx.h, self.h, bp, xp, int(max_iter), float(tol), int(bool(mixed)), best,
                                      C.byref(sec))
        self.ctx.leave()
        check(st)
        return self.params(), sec.value

    def tune_lockstep(self, bs, *, candidates=(8192, 16384, 32768, 65536), iters=48, reps=2, mixed=True):
        """Autotune the lockstep engine's launch shape: the nonzeros per table entry, that is the
        rows one block of 256 threads takes (8 warps, each a slice of 32 rows in the compact
        layout). Each candidate runs `iters` iterations of every member on these right-hand
        sides (on scratch solutions, no member stops early), `reps` times; the fastest device
        time wins and stays configured. Returns (best, {candidate: seconds})."""
        if not candidates or iters < 1 or reps < 1:
            raise ValueError("tune_lockstep: needs candidates, iters >= 1 and reps >= 1")
        times = {}
        for c in candidates:
            self.configure_lockstep(nnz_per_entry=int(c))
            best = float("inf")
            for _ in range(reps):
                _, res = self.solve(bs, None, tol=1e-300, max_iter=int(iters), mixed=mixed, engine="lockstep")
                best = min(best, max(r["seconds"] for r in res))
            times[int(c)] = best
        pick = min(times, key=times.get)
        self.configure_lockstep(nnz_per_entry=pick)
        return pick, times

    def solve(self, bs, xs=None, *, tol=1e-10, max_iter=0, mixed=True, engine="persistent"):
        """Solve every member (in id order) to completion.  bs: right-hand sides; xs: initial
        guesses (default 0), overwritten.  engine "persistent": one cooperative launch (teams of
        blocks per member); "lockstep": a few whole-GPU kernels per iteration over all the members
        still running.  Returns (xs, results) with one dict per member (converged, iterations,
        residual, breakdown, status, reliable_updates, seconds)."""
        if engine not in ("persistent", "lockstep"):
            raise ValueError(f"batch: unknown engine {engine!r}")
        bs, xs, bp, xp = self._vectors(bs, xs)
        res = (N.femd_cg_result * len(bs))()
        fn = lib.femd_cuda_batch_solve if engine == "persistent" else lib.femd_cuda_batch_solve_lockstep
        self.ctx.enter()
        st = fn(self.ctx.h, self.h, bp, xp, int(max_iter), float(tol), int(bool(mixed)), res)
        self.ctx.leave()
        self.last_status = st
        if st not in (N.FEMD_OK, N.FEMD_ETIMEOUT, N.FEMD_EABORT):
            check(st)
        return xs, [_result(r) for r in res]

    # ---- dynamic membership --------------------------------------------------------------
    def add(self, K: CSRMatrix) -> int:
        """Add a member; returns its id."""
        from .core import JacobiPreconditioner
        JacobiPreconditioner(K)
        i = C.c_int()
        check(lib.femd_cuda_batch_add(self.h, K.h, C.byref(i)))
        self.members[i.value] = K
        return i.value

    def remove(self, i: int):
        check(lib.femd_cuda_batch_remove(self.h, int(i)))
        self.members.pop(i, None)
        self._armed.pop(i, None)

    def arm(self, i: int, b, x, *, tol=1e-10, max_iter=0):
        """Start a solve of member i on the next steps (b, x: float64 device tensors; x holds the
        initial guess and receives the solution)."""
        K = self.members[i]
        if b.numel() != K.nrows or x.numel() != K.nrows:
            raise ValueError("batch: vector length differs from its matrix")
        self.ctx.enter()
        st = lib.femd_cuda_batch_arm(self.h, int(i), b.data_ptr(), x.data_ptr(), int(max_iter), float(tol))
        self.ctx.leave()
        check(st)
        self._armed[i] = (b, x)

    def step(self, iters: int, *, mixed=True, engine="persistent"):
        """Advance the armed members.  engine "persistent": one launch, every armed member by at
        most iters iterations; "lockstep": every armed member to completion (one wave; iters
        unused); "continuous": the lockstep engine resumable -- members armed since the last step
        join, every member in flight advances by about iters iterations (whole chunks), the ones
        done leave.  Returns [(id, result dict)] of the members that finished."""
        if engine not in ("persistent", "lockstep", "continuous"):
            raise ValueError(f"batch: unknown engine {engine!r}")
        n = max(len(self._armed), 1)
        ids = (C.c_int * n)()
        res = (N.femd_cg_result * n)()
        nf = C.c_int()
        self.ctx.enter()
        if engine == "persistent":
            st = lib.femd_cuda_batch_step(self.ctx.h, self.h, int(iters), int(bool(mixed)), C.byref(nf), ids, res)
        elif engine == "continuous":
            chunks = max(1, int(iters) // max(1, self._ls_shape["chunk"]))
            st = lib.femd_cuda_batch_advance_lockstep(self.ctx.h, self.h, int(bool(mixed)), chunks, C.byref(nf), ids, res)
        else:
            st = lib.femd_cuda_batch_step_lockstep(self.ctx.h, self.h, int(bool(mixed)), C.byref(nf), ids, res)
        self.ctx.leave()
        self.last_status = st
        if st not in (N.FEMD_OK, N.FEMD_ETIMEOUT, N.FEMD_EABORT):
            check(st)
        out = [(int(ids[k]), _result(res[k])) for k in range(nf.value)]
        for i, _ in out:
            self._armed.pop(i, None)
        return out

    # ---- control -----------------------------------------------------------------------
    def abort(self):
        lib.femd_cuda_batch_abort(self.h)

    def profile(self):
        """Cycle counters of the last launch summed over blocks: kernel, team-barrier waits,
        SpMV chunk-barrier waits (femd_cuda_batch_profile)."""
        out = (C.c_longlong * 7)()
        check(lib.femd_cuda_batch_profile(self.h, out))
        return dict(block=out[0], team_wait=out[1], chunk_sync=out[2], fail_where=out[3], fail_at=out[4],
                    fail_team=out[5], fail_seen=out[6])

    def debug(self, ghost_problem=-1, spin_limit=0):
        check(lib.femd_cuda_batch_debug(self.h, int(ghost_problem), int(spin_limit)))
