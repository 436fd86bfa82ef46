"""Batched Jacobi-PCG: many independent systems in one persistent launch (femd_cuda_batch_*)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .core import CSRMatrix, _as_device, _torch, check, context, lib


class Batch:
    """A fixed set of matrices (each with its Jacobi inverse diagonal) solved together.

    solve() runs every system's Jacobi-PCG in one cooperative launch, FP64 or mixed precision
    (FP32 inner iteration, FP64 reliable updates).  A system's result does not depend on the
    other systems of the batch."""

    def __init__(self, mats: list[CSRMatrix], nnz_per_block: int = 0, ctx=None):
        from .core import JacobiPreconditioner
        self.ctx = ctx or context()
        self.mats = list(mats)
        for K in self.mats:
            JacobiPreconditioner(K)             # the inverse diagonal, checked (zero diagonal -> ValueError)
        arr = (C.c_void_p * len(mats))(*[K.h.value for K in self.mats])
        h = C.c_void_p()
        check(lib.femd_cuda_batch_create(self.ctx.h, len(mats), arr, int(nnz_per_block), C.byref(h)))
        self.h = h

    def __del__(self):
        try:
            if self.h:
                lib.femd_cuda_release(self.h)
                self.h = None
        except Exception:
            pass

    def info(self):
        n, g, s = C.c_int(), C.c_int(), C.c_int()
        teams = np.empty(len(self.mats), dtype=np.int32)
        check(lib.femd_cuda_batch_info(self.h, C.byref(n), C.byref(g), C.byref(s), teams.ctypes.data_as(C.POINTER(C.c_int))))
        return dict(nprob=n.value, grid=g.value, slots=s.value, teams=teams)

    def solve(self, bs, xs=None, *, tol=1e-10, max_iter=0, mixed=True):
        """bs: right-hand sides (device tensors or arrays); xs: initial guesses (default 0), overwritten.
        Returns (xs, results), results a list of dicts (converged, iterations, residual, breakdown,
        status, reliable_updates) and the launch time."""
        torch = _torch()
        bs = [_as_device(b, self.ctx) for b in bs]
        if len(bs) != len(self.mats):
            raise ValueError("batch: one right-hand side per matrix")
        if xs is None:
            xs = [torch.zeros(K.nrows, dtype=torch.float64, device=b.device) for K, b in zip(self.mats, bs)]
        for K, b, x in zip(self.mats, bs, xs):
            if b.numel() != K.nrows or x.numel() != K.nrows:
                raise ValueError("batch: vector length differs from its matrix")
        bp = (C.c_void_p * len(bs))(*[b.data_ptr() for b in bs])
        xp = (C.c_void_p * len(xs))(*[x.data_ptr() for x in xs])
        res = (N.femd_cg_result * len(bs))()
        self.ctx.enter()
        st = lib.femd_cuda_batch_solve(self.ctx.h, self.h, bp, xp, int(max_iter), float(tol), int(bool(mixed)), res)
        self.ctx.leave()
        out = [dict(converged=bool(r.converged), iterations=int(r.iterations), residual=float(r.residual),
                    breakdown=bool(r.breakdown), status=int(r.status), reliable_updates=int(r.outer),
                    seconds=float(r.seconds)) for r in res]
        self.last_status = st
        if st not in (N.FEMD_OK, N.FEMD_ETIMEOUT, N.FEMD_EABORT):
            check(st)
        return xs, out

    def abort(self):
        lib.femd_cuda_batch_abort(self.h)

    def debug(self, ghost_problem=-1, spin_limit=0):
        check(lib.femd_cuda_batch_debug(self.h, int(ghost_problem), int(spin_limit)))
