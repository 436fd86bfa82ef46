"""The host-side mirror of FEMd's 2D hot path, over libfemd_cuda's C ABI.

Names, argument meaning and errors follow the reference's nanobind module `_femd`
(python/src/femd_bindings*.cpp) and its Python callers:

    rectangle_mesh            python/femd/mesh2d.py:687          -> Mesh2D
    LagrangeSpace2D           python/femd/spaces2d.py:113        (bc="dirichlet" / "free")
    V.cache(degree)           Cache2D(V, degree), include/femd/fe/cache_2d.hpp:67
    cell_pattern(V, V)        femd_bindings_2d.cpp:762           -> SparsityPattern (device)
    CSRMatrix(pattern)        femd_bindings_2d.cpp:101           (values in HBM)
    scatter_map_2d            include/femd/forms/assembly_2d.hpp:136
    assemble_matrix_2d        femd_bindings_2d.cpp:810
    assemble_vector_2d        femd_bindings_2d.cpp:817
    JacobiPreconditioner      femd_bindings_2d.cpp:183
    cg_solve                  femd_bindings.cpp:799              -> (x, converged, iterations, residual, breakdown)

Device arrays are torch CUDA tensors (torch is only the allocator and stream plumbing here);
every computation runs in libfemd_cuda's kernels.  Nothing falls back to the CPU: without the
library or a CUDA device these calls raise.
"""
from __future__ import annotations

import ctypes as C
import math
import sys
import threading

import numpy as np

from . import _native as N
from ._native import check, lib

PI = math.pi


def _torch():
    import torch
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _np_ptr(a):
    return C.c_void_p(a.ctypes.data)


# ---- context ---------------------------------------------------------------------------------
class Context:
    """One device and one stream of libfemd_cuda (femd_ctx)."""

    def __init__(self, device: int = 0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("femd_b200 needs a CUDA device (B200); none is visible")
        torch.cuda.set_device(device)
        h = C.c_void_p()
        check(lib.femd_cuda_ctx_create(int(device), C.byref(h)), "ctx_create")
        self.h = h
        self.device = device
        self._stream = torch.cuda.ExternalStream(lib.femd_cuda_ctx_stream(h), device=f"cuda:{device}")

    @property
    def stream(self):
        """The context's stream as a torch stream (for ordering torch work around library calls)."""
        return self._stream

    def sync(self):
        check(lib.femd_cuda_ctx_sync(self.h))

    def enter(self):
        """Order the library's stream after the work torch has queued (inputs made by torch)."""
        torch = _torch()
        self._stream.wait_stream(torch.cuda.current_stream())

    def leave(self):
        """Order torch's current stream after the library's work (outputs read by torch)."""
        torch = _torch()
        torch.cuda.current_stream().wait_stream(self._stream)

    def close(self):
        if self.h:
            lib.femd_cuda_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            if not sys.is_finalizing():     # at exit the process frees everything
                self.close()
        except Exception:
            pass


_default = {}
_default_lock = threading.Lock()


def context(device: int | None = None) -> Context:
    """The default context of a device (one per device and host thread)."""
    torch = _torch()
    dev = torch.cuda.current_device() if device is None else device
    key = (dev, threading.get_ident())
    with _default_lock:
        c = _default.get(key)
        if c is None:
            c = _default[key] = Context(dev)
    return c


class _Handle:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        try:
            if self.h and not sys.is_finalizing():
                lib.femd_cuda_release(self.h)
                self.h = None
        except Exception:
            pass


# ---- mesh, space, cache (host setup) ---------------------------------------------------------
class Mesh2D:
    """A triangle mesh: points (nverts, 2) float64 and triangles (ncells, 3) int32, counter-clockwise."""

    def __init__(self, points, tris):
        self.points = np.ascontiguousarray(points, dtype=np.float64)
        self.tris = np.ascontiguousarray(tris, dtype=np.int32)
        self._dev = None

    @property
    def nverts(self):
        return self.points.shape[0]

    @property
    def ncells(self):
        return self.tris.shape[0]

    def device(self, ctx: Context | None = None):
        """(points, tris) as device tensors (uploaded once)."""
        if self._dev is None:
            torch = _torch()
            ctx = ctx or context()
            with torch.cuda.stream(ctx.stream):
                self._dev = (torch.from_numpy(self.points).to(f"cuda:{ctx.device}", non_blocking=False),
                             torch.from_numpy(self.tris).to(f"cuda:{ctx.device}", non_blocking=False))
            ctx.stream.synchronize()
        return self._dev

    def set_points(self, points_dev):
        """Replace the vertex coordinates by a device tensor (same topology)."""
        _, tris = self.device()
        self._dev = (points_dev, tris)

    def c_struct(self, ctx=None):
        pts, tris = self.device(ctx)
        return N.femd_mesh2d(self.nverts, self.ncells, pts.data_ptr(), tris.data_ptr())


def rectangle_mesh(x0, y0, x1, y1, nx, ny, *, diagonal="right"):
    """Structured mesh of [x0, x1] x [y0, y1], nx x ny cells split by the "/" diagonal
    (python/femd/mesh2d.py:687, include/femd/mesh/structured.hpp:338)."""
    if diagonal != "right":
        raise ValueError("rectangle_mesh: only diagonal='right' is implemented on this path")
    nx, ny = int(nx), int(ny)
    if nx < 1 or ny < 1:
        raise ValueError("rectangle_mesh: need nx, ny >= 1")
    pts = np.empty(((nx + 1) * (ny + 1), 2))
    tris = np.empty((2 * nx * ny, 3), dtype=np.int32)
    check(lib.femd_host_rectangle_mesh(float(x0), float(y0), float(x1), float(y1), nx, ny, _np_ptr(pts), _np_ptr(tris)))
    return Mesh2D(pts, tris)


def quad_degree(form: str, k: int) -> int:
    """The quadrature degree the reference's form compiler infers (python/femd/forms.py:2487-2500)
    for the forms of this path: sum of argument degrees (k minus derivative order) plus the
    coefficient's degree, a non-polynomial coefficient of the data counting as k + 1."""
    d = {"gradgrad": 2 * (k - 1), "helmholtz": 2 * k, "varcoef": 2 * (k - 1) + (k + 1), "rhs_data": 2 * k + 1,
         "rhs_field": 2 * k, "mass": 2 * k, "heat": 2 * k}[form]
    return max(d, 1)


class Cache2D:
    """A quadrature rule on the reference triangle with the basis tabulated at its points
    (Cache2D, include/femd/fe/cache_2d.hpp:67-121).  Per-point geometry is not stored: the
    kernels form it from the mesh."""

    def __init__(self, space: "LagrangeSpace2D", degree: int):
        self.space = space
        self.degree = int(degree)
        xi, eta, w = np.empty(64), np.empty(64), np.empty(64)
        nq = lib.femd_host_triangle_quadrature(self.degree, _np_ptr(xi), _np_ptr(eta), _np_ptr(w))
        if nq < 0:
            check(-nq)
        self.xi, self.eta, self.w = xi[:nq].copy(), eta[:nq].copy(), w[:nq].copy()
        k = space.degree
        self.ref = np.empty((nq, 3, space.nloc))
        r = lib.femd_host_tabulate(k, nq, _np_ptr(self.xi), _np_ptr(self.eta), _np_ptr(self.ref))
        if r < 0:
            check(-r)

    @property
    def nq(self):
        return self.xi.size

    def with_tables(self, ref):
        """A copy of this rule with another tabulation (for instance the reference's own)."""
        c = object.__new__(Cache2D)
        c.__dict__.update(self.__dict__)
        c.ref = np.ascontiguousarray(ref, dtype=np.float64).reshape(self.ref.shape)
        return c

    def c_struct(self):
        return N.femd_rule(self.space.degree, self.space.nloc, self.nq, self.ref.ctypes.data, self.xi.ctypes.data,
                           self.eta.ctypes.data, self.w.ctypes.data)


class LagrangeSpace2D:
    """Continuous P_k on a triangle mesh; bc="dirichlet" eliminates every exterior node
    (python/femd/spaces2d.py:113-152, include/femd/fe/space_2d.hpp:390-526)."""

    def __init__(self, mesh: Mesh2D, degree: int, bc: str = "free", *, numbering: str = "host"):
        """numbering: "host" (C++ on the host) or "device" (femd_cuda_lagrange_numbering on the
        GPU; the same map, and the dofs stay on the device as well)."""
        if bc not in ("free", "dirichlet"):
            raise ValueError(f"LagrangeSpace2D: bc is 'free' or 'dirichlet' (every exterior side), got {bc!r}")
        if numbering not in ("host", "device"):
            raise ValueError(f"LagrangeSpace2D: numbering is 'host' or 'device', got {numbering!r}")
        k = int(degree)
        if k < 1:
            raise ValueError("LagrangeSpace2D: degree must be >= 1 (P0 is a DG space)")
        self.mesh, self.degree, self.bc = mesh, k, bc
        self.nloc = (k + 1) * (k + 2) // 2
        self._caches = {}
        self._pattern = None
        self._dofs_dev = None
        dim, raw = C.c_int(), C.c_int()
        if numbering == "device":
            torch = _torch()
            ctx = context()
            _, tris = mesh.device(ctx)
            dofs = torch.empty((mesh.ncells, self.nloc), dtype=torch.int32, device=f"cuda:{ctx.device}")
            ctx.enter()
            st = lib.femd_cuda_lagrange_numbering(ctx.h, mesh.nverts, mesh.ncells, tris.data_ptr(), k,
                                                  int(bc == "dirichlet"), dofs.data_ptr(), C.byref(dim), C.byref(raw))
            ctx.leave()
            check(st)
            self._dofs_dev = dofs
            self.cell_dofs = dofs.cpu().numpy()
        else:
            self.cell_dofs = np.empty((mesh.ncells, self.nloc), dtype=np.int32)
            check(lib.femd_host_lagrange_numbering(mesh.nverts, mesh.ncells, _np_ptr(mesh.tris), k, int(bc == "dirichlet"),
                                                   _np_ptr(self.cell_dofs), C.byref(dim), C.byref(raw)))
        self.dim, self.raw_dim = dim.value, raw.value

    def cache(self, degree: int) -> Cache2D:
        c = self._caches.get(degree)
        if c is None:
            c = self._caches[degree] = Cache2D(self, degree)
        return c

    def cell_dofs_device(self, ctx=None):
        if self._dofs_dev is None:
            torch = _torch()
            ctx = ctx or context()
            self._dofs_dev = torch.from_numpy(self.cell_dofs).to(f"cuda:{ctx.device}")
        return self._dofs_dev

    def pattern(self, ctx=None) -> "SparsityPattern":
        """cell_pattern(V, V), cached on the space (spaces2d.py:272-279)."""
        if self._pattern is None:
            self._pattern = cell_pattern(self, self, ctx)
        return self._pattern


# ---- pattern, matrix, preconditioner ---------------------------------------------------------
class SparsityPattern(_Handle):
    def __init__(self, h, ctx):
        super().__init__(h)
        self.ctx = ctx
        nr, nc, nnz = C.c_int(), C.c_int(), C.c_longlong()
        check(lib.femd_cuda_pattern_info(h, C.byref(nr), C.byref(nc), C.byref(nnz)))
        self.nrows, self.ncols, self.nnz = nr.value, nc.value, nnz.value

    def to_host(self):
        ip = np.empty(self.nrows + 1, dtype=np.int32)
        ix = np.empty(max(self.nnz, 1), dtype=np.int32)
        check(lib.femd_cuda_pattern_to_host(self.h, _np_ptr(ip), _np_ptr(ix)))
        return ip, ix[:self.nnz]

    @property
    def indptr(self):
        return self.to_host()[0]

    @property
    def indices(self):
        return self.to_host()[1]

    def device_arrays(self):
        ip, ix = C.c_void_p(), C.c_void_p()
        check(lib.femd_cuda_pattern_arrays(self.h, C.byref(ip), C.byref(ix)))
        return ip.value, ix.value

    def batch_layout(self):
        """Build the batched engine's compact layout of this pattern now (else the first
        mixed-precision lockstep solve on it does); returns the reordered bandwidth, -1 when the
        pattern keeps the plain layout."""
        bw = C.c_int()
        check(lib.femd_cuda_pattern_batch_layout(self.ctx.h, self.h, C.byref(bw)))
        return bw.value

    @staticmethod
    def from_arrays(nrows, ncols, indptr, indices, ctx=None):
        ctx = ctx or context()
        ip = np.ascontiguousarray(indptr, dtype=np.int32)
        ix = np.ascontiguousarray(indices, dtype=np.int32)
        if ip.size != nrows + 1:
            raise ValueError("CSRMatrix: indptr length != nrows + 1")
        h = C.c_void_p()
        check(lib.femd_cuda_pattern_from_csr_host(ctx.h, int(nrows), int(ncols), _np_ptr(ip),
                                                  _np_ptr(ix) if ix.size else C.c_void_p(0), C.byref(h)))
        return SparsityPattern(h, ctx)


def cell_pattern(test: LagrangeSpace2D, trial: LagrangeSpace2D, ctx=None) -> SparsityPattern:
    """CSR pattern of every test-trial coupling through a common cell (assembly_2d.hpp:36-41),
    built on the GPU (K1)."""
    if test is not trial:
        if test.mesh is not trial.mesh or test.degree != trial.degree or test.bc != trial.bc:
            raise ValueError("cell_pattern: the two spaces are on different meshes")
    ctx = ctx or context()
    dofs = test.cell_dofs_device(ctx)
    h = C.c_void_p()
    ctx.enter()
    check(lib.femd_cuda_pattern_from_cells(ctx.h, test.dim, test.mesh.ncells, test.nloc, _ptr(dofs), C.byref(h)))
    P = SparsityPattern(h, ctx)
    P.ncells, P.nloc = test.mesh.ncells, test.nloc
    return P


def scatter_map_2d(pattern: SparsityPattern):
    """The element -> nnz map of a cell pattern (assembly_2d.hpp:136-164): an int32 device
    tensor of ncells x nloc x nloc positions, -1 where a node is constrained.  Raises
    RuntimeError("assemble_matrix_2d: entry outside the pattern") as the reference does."""
    torch = _torch()
    p = C.c_void_p()
    check(lib.femd_cuda_pattern_map(pattern.h, C.byref(p)))
    pattern.ctx.leave()
    n = pattern.ncells * pattern.nloc * pattern.nloc
    return _wrap_device(p.value, n, torch.int32, pattern.ctx)


class CSRMatrix(_Handle):
    """Values on a pattern, in HBM (CSRMatrix, include/femd/sparse/csr.hpp:178-185)."""

    def __init__(self, pattern: SparsityPattern, symmetric: bool = False):
        h = C.c_void_p()
        check(lib.femd_cuda_matrix_create(pattern.ctx.h, pattern.h, C.byref(h)))
        super().__init__(h)
        self.pattern = pattern
        self.ctx = pattern.ctx
        self.symmetric = symmetric
        self._jacobi = False

    nrows = property(lambda self: self.pattern.nrows)
    ncols = property(lambda self: self.pattern.ncols)
    nnz = property(lambda self: self.pattern.nnz)

    def _arrays(self):
        d, i = C.c_void_p(), C.c_void_p()
        check(lib.femd_cuda_matrix_arrays(self.h, C.byref(d), C.byref(i)))
        return d.value, i.value

    def data_tensor(self):
        """The values as a torch float64 CUDA tensor view (no copy)."""
        torch = _torch()
        d, _ = self._arrays()
        self.ctx.leave()
        return _wrap_device(d, self.nnz, torch.float64, self.ctx)

    def inv_tensor(self):
        torch = _torch()
        _, i = self._arrays()
        self.ctx.leave()
        return _wrap_device(i, self.nrows, torch.float64, self.ctx)

    @property
    def data(self):
        out = np.empty(max(self.nnz, 1))
        check(lib.femd_cuda_matrix_to_host(self.h, _np_ptr(out)))
        return out[:self.nnz]

    def set_data(self, data):
        a = np.ascontiguousarray(data, dtype=np.float64)
        if a.size != self.nnz:
            raise ValueError("CSRMatrix: data length != nnz")
        check(lib.femd_cuda_matrix_set_host(self.h, _np_ptr(a)))
        self._jacobi = False

    @staticmethod
    def from_arrays(nrows, ncols, indptr, indices, data, symmetric=False, ctx=None):
        P = SparsityPattern.from_arrays(nrows, ncols, indptr, indices, ctx)
        K = CSRMatrix(P, symmetric)
        K.set_data(data)
        return K

    def matvec(self, x):
        """y = K x for a device tensor x (CSRMatrix::apply, csr.hpp:203-215)."""
        torch = _torch()
        x = _as_device(x, self.ctx)
        if x.numel() != self.ncols:
            raise ValueError("matvec: length mismatch")
        y = torch.empty(self.nrows, dtype=torch.float64, device=x.device)
        self.ctx.enter()
        check(lib.femd_cuda_spmv(self.ctx.h, self.h, _ptr(x), _ptr(y)))
        self.ctx.leave()
        return y

    def autotune_spmv(self, set_best: bool = True):
        """Time the SpMV's threads-per-row variants on this matrix; returns (best, microseconds)."""
        t, us = C.c_int(), C.c_double()
        check(lib.femd_cuda_spmv_autotune(self.ctx.h, self.h, int(set_best), C.byref(t), C.byref(us)))
        return t.value, us.value

    def set_spmv_tpr(self, tpr: int):
        check(lib.femd_cuda_spmv_set_tpr(self.h, int(tpr)))

    def asymmetry(self):
        out = C.c_double()
        check(lib.femd_cuda_asymmetry(self.ctx.h, self.h, C.byref(out)))
        return out.value

    def combine(self, B: "CSRMatrix", alpha: float, beta: float) -> "CSRMatrix":
        """alpha self + beta B on the shared pattern (csr.hpp:315-326)."""
        C_ = CSRMatrix(self.pattern, self.symmetric and B.symmetric)
        check(lib.femd_cuda_combine(self.ctx.h, float(alpha), self.h, float(beta), B.h, C_.h))
        return C_

    def diagonal(self):
        inv = self.inv_tensor()
        return (1.0 / inv).cpu().numpy()


def _wrap_device(ptr, n, dtype, ctx):
    """A torch tensor viewing n elements of device memory owned by a library handle."""
    torch = _torch()
    if n == 0:
        return torch.empty(0, dtype=dtype, device=f"cuda:{ctx.device}")
    elt = torch.empty(0, dtype=dtype).element_size()

    class _Mem:
        __cuda_array_interface__ = {"shape": (n,), "typestr": {8: "<f8", 4: "<f4"}[elt] if dtype.is_floating_point else "<i4",
                                    "data": (ptr, False), "version": 3, "strides": None, "stream": None}
    return torch.as_tensor(_Mem(), device=f"cuda:{ctx.device}")


def _as_device(x, ctx):
    torch = _torch()
    if isinstance(x, torch.Tensor) and x.is_cuda:
        return x.contiguous().to(torch.float64)
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64)).to(f"cuda:{ctx.device}")


class JacobiPreconditioner:
    """z = D^{-1} r with D = diag(K) (include/femd/sparse/precond.hpp:82-102).  The inverse
    diagonal lives with the matrix; building it raises ValueError on a zero diagonal entry."""

    def __init__(self, K: CSRMatrix):
        if K.nrows != K.ncols:
            raise ValueError("Jacobi: the matrix must be square")
        if not K._jacobi:
            check(lib.femd_cuda_matrix_jacobi(K.ctx.h, K.h))
            K._jacobi = True
        self.K = K
        self.size = K.nrows
        self.name = "jacobi"

    def inverse_diagonal(self):
        out = np.empty(max(self.size, 1))
        check(lib.femd_cuda_matrix_inv_diag_to_host(self.K.h, _np_ptr(out)))
        return out[:self.size]


class _PCBase(_Handle):
    """A preconditioner of libfemd_cuda (femd_precond) built from a square CSRMatrix."""

    def __init__(self, K: CSRMatrix, kind, omega, name):
        if K.nrows != K.ncols:
            raise ValueError(f"{name}: the matrix must be square")
        h = C.c_void_p()
        K.ctx.enter()
        check(lib.femd_cuda_precond_create(K.ctx.h, K.h, int(kind), float(omega), C.byref(h)))
        super().__init__(h)
        self.K, self.ctx, self.size = K, K.ctx, K.nrows
        k, lf, lb, mp = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        check(lib.femd_cuda_precond_info(h, C.byref(k), C.byref(lf), C.byref(lb), C.byref(mp)))
        self.levels = (lf.value, lb.value)
        self._min_pivot = mp.value

    def apply(self, r):
        """z = M^{-1} r for a device or host vector (returns a float64 device tensor)."""
        torch = _torch()
        rv = _as_device(r, self.ctx)
        if rv.numel() != self.size:
            raise ValueError(f"{self.name}: vector length differs from the matrix")
        z = torch.empty_like(rv)
        self.ctx.enter()
        check(lib.femd_cuda_precond_apply(self.ctx.h, self.h, _ptr(rv), _ptr(z)))
        self.ctx.leave()
        return z


class ILU0Preconditioner(_PCBase):
    """Incomplete LU with no fill on the pattern of K, natural ordering (ILU0Preconditioner,
    include/femd/sparse/precond.hpp:151-213): factors and applications bit-identical to the
    reference's.  Raises ValueError on a zero diagonal entry and RuntimeError on a zero pivot."""

    def __init__(self, K: CSRMatrix):
        super().__init__(K, N.PC_ILU0, 1.0, "ILU(0)")
        self.name = "ilu0"

    def min_pivot(self):
        """The smallest pivot met (negative: the factorization is indefinite, not for CG)."""
        return self._min_pivot


class SSORPreconditioner(_PCBase):
    """Symmetric SOR, M = w/(2-w) (D/w + L) (D/w)^{-1} (D/w + U), natural ordering
    (SSORPreconditioner, include/femd/sparse/precond.hpp:105-149)."""

    def __init__(self, K: CSRMatrix, omega: float = 1.0):
        super().__init__(K, N.PC_SSOR, omega, "SSOR")
        self.name = "ssor"
        self.omega = float(omega)


# ---- coefficients and assembly ---------------------------------------------------------------
class Coef:
    """A term coefficient: Coef.const(v), Coef.sinsin(p0, p1, a, b) = p0 + p1 sin(a x) sin(b y),
    Coef.helmholtz_sinsin(c, a, b) = c s + s with s = sin(a x) sin(b y), Coef.points(t) (values
    at the points [e nq + q], a device tensor), Coef.field(t) (a P_k field at the dofs)."""

    def __init__(self, kind, value=0.0, tensor=None, p=(0.0, 0.0, 0.0, 0.0)):
        self.kind, self.value, self.tensor, self.p = kind, float(value), tensor, tuple(float(v) for v in p)

    @staticmethod
    def const(v):
        return Coef(N.COEF_CONST, value=v)

    @staticmethod
    def sinsin(p0, p1, a, b):
        return Coef(N.COEF_SINSIN, p=(p0, p1, a, b))

    @staticmethod
    def helmholtz_sinsin(c, a, b):
        return Coef(N.COEF_SINSIN_HELM, p=(0.0, c, a, b))

    @staticmethod
    def points(t):
        return Coef(N.COEF_POINTS, tensor=t)

    @staticmethod
    def field(t):
        return Coef(N.COEF_FIELD, tensor=t)

    def c_struct(self):
        c = N.femd_coef()
        c.kind = self.kind
        c.value = self.value
        c.points_dev = self.tensor.data_ptr() if self.kind == N.COEF_POINTS else None
        c.field_dev = self.tensor.data_ptr() if self.kind == N.COEF_FIELD else None
        for i in range(4):
            c.p[i] = self.p[i]
        return c


def _coefs(coeffs):
    out = [c if isinstance(c, Coef) else Coef.const(c) for c in coeffs]
    arr = (N.femd_coef * len(out))(*[c.c_struct() for c in out])
    return out, arr


def assemble_matrix_2d(QT: Cache2D, QS: Cache2D, a, b, coeffs, K: CSRMatrix, row_offset=0, col_offset=0, *,
                       exact=False, jacobi=True):
    """K = sum_t integral c_t (D^a_t T_i)(D^b_t S_j); codes 0 value, 1 d/dx, 2 d/dy
    (assembly_2d.hpp:219-305).  Unlike the reference, K is overwritten (not added to): the
    kernel writes every value once.  exact=True reproduces the reference's operation order."""
    if QT is not QS:
        raise ValueError("assemble_matrix_2d: test and trial caches differ (this path assembles square forms)")
    if row_offset or col_offset:
        raise ValueError("assemble_matrix_2d: offsets (block systems) are not on this path")
    if len(a) != len(b):
        raise ValueError("assemble_matrix_2d: a and b differ in length")
    if len(coeffs) != len(a):
        raise ValueError("assembly_2d: one coefficient array per term")
    V = QT.space
    keep, carr = _coefs(coeffs)
    ai = (C.c_int * len(a))(*a)
    bi = (C.c_int * len(b))(*b)
    mesh = V.mesh.c_struct(K.ctx)
    rule = QT.c_struct()
    K.ctx.enter()
    check(lib.femd_cuda_assemble_matrix(K.ctx.h, C.byref(mesh), C.byref(rule), K.pattern.h, len(a), ai, bi, carr,
                                        N.ASM_EXACT if exact else N.ASM_FAST, K.h, int(bool(jacobi))))
    K.ctx.leave()
    K._jacobi = bool(jacobi)
    del keep
    return K


def assemble_vector_2d(Q: Cache2D, a, coeffs, pattern: SparsityPattern | None = None, *, exact=False, out=None):
    """f_i = sum_t integral c_t D^a_t N_i (assembly_2d.hpp:173-211), as a float64 device tensor.
    exact=True forms every element entry in the reference's operation order."""
    torch = _torch()
    V = Q.space
    P = pattern or V.pattern()
    if len(coeffs) != len(a):
        raise ValueError("assembly_2d: one coefficient array per term")
    keep, carr = _coefs(coeffs)
    ai = (C.c_int * len(a))(*a)
    f = out if out is not None else torch.empty(V.dim, dtype=torch.float64, device=f"cuda:{P.ctx.device}")
    mesh = V.mesh.c_struct(P.ctx)
    rule = Q.c_struct()
    P.ctx.enter()
    check(lib.femd_cuda_assemble_vector(P.ctx.h, C.byref(mesh), C.byref(rule), P.h, len(a), ai, carr,
                                        N.ASM_EXACT if exact else N.ASM_FAST, _ptr(f)))
    P.ctx.leave()
    del keep
    return f


# ---- CG --------------------------------------------------------------------------------------
def cg_solve(A: CSRMatrix, M, b, x0, max_iter: int, tol: float, *, mixed: bool = False):
    """Preconditioned CG, M None or a JacobiPreconditioner (femd_bindings.cpp:799-833 ->
    krylov::cg_jacobi).  b, x0: device tensors or host arrays.  Returns (x, converged,
    iterations, residual, breakdown) with x a float64 device tensor.  mixed=True runs the inner
    iteration in FP32 with FP64 reliable updates (femd_cuda_pcg_mixed)."""
    torch = _torch()
    n = A.nrows
    if A.nrows != A.ncols:
        raise ValueError(f"krylov: A is {A.nrows} x {A.ncols}")
    bv = _as_device(b, A.ctx)
    if bv.numel() != n:
        raise ValueError(f"krylov: A is {n} x {n}, b has length {bv.numel()}")
    x = (torch.zeros(n, dtype=torch.float64, device=bv.device) if x0 is None else _as_device(x0, A.ctx).clone())
    if x.numel() != n:
        raise ValueError("cg: x0 and b differ in length")
    if M is not None and not isinstance(M, (JacobiPreconditioner, _PCBase)):
        raise TypeError("cg_solve: M is None, a JacobiPreconditioner, an ILU0Preconditioner or an SSORPreconditioner")
    if M is not None and M.size != n:
        raise ValueError("krylov: preconditioner and right-hand side differ in size")
    if isinstance(M, _PCBase):
        # krylov::cg with a general preconditioner (cg.hpp:245-290)
        if mixed:
            raise ValueError("pcg_mixed: the mixed-precision solve is Jacobi-preconditioned")
        if M.K.pattern is not A.pattern:
            raise ValueError("krylov: the preconditioner was built on another matrix pattern")
        A.ctx.enter()
        res = N.femd_cg_result()
        check(lib.femd_cuda_cg_precond(A.ctx.h, A.h, M.h, _ptr(bv), _ptr(x), int(max_iter), float(tol), C.byref(res)))
        A.ctx.leave()
        cg_solve.last = res
        return x, bool(res.converged), int(res.iterations), float(res.residual), bool(res.breakdown)
    if M is not None and M.K is not A:
        # the preconditioner of another matrix: its inverse diagonal becomes A's
        _, inv = M.K._arrays()
        A.ctx.enter()
        check(lib.femd_cuda_matrix_set_inv_diag(A.ctx.h, A.h, C.c_void_p(inv)))
        A._jacobi = True
    A.ctx.enter()
    res = N.femd_cg_result()
    if mixed:
        if M is None:
            raise ValueError("pcg_mixed: the mixed-precision solve is Jacobi-preconditioned")
        check(lib.femd_cuda_pcg_mixed(A.ctx.h, A.h, _ptr(bv), _ptr(x), int(max_iter), float(tol), C.byref(res)))
    else:
        check(lib.femd_cuda_cg_jacobi(A.ctx.h, A.h, int(M is not None), _ptr(bv), _ptr(x), int(max_iter), float(tol),
                                      C.byref(res)))
    A.ctx.leave()
    cg_solve.last = res
    return x, bool(res.converged), int(res.iterations), float(res.residual), bool(res.breakdown)


def cg_solve_host(indptr, indices, data, inv, b, x0=None, max_iter=None, tol=1e-10, ctx=None):
    """cg_solve on HOST arrays, exactly the data the reference binding holds (CSR arrays of a
    CSRMatrix, the JacobiPreconditioner's inverse diagonal or None, numpy b and x0).  Returns
    (x as numpy, converged, iterations, residual, breakdown)."""
    ctx = ctx or context()
    ip = np.ascontiguousarray(indptr, dtype=np.int32)
    ix = np.ascontiguousarray(indices, dtype=np.int32)
    dv = np.ascontiguousarray(data, dtype=np.float64)
    bv = np.ascontiguousarray(b, dtype=np.float64)
    n = bv.size
    if ip.size != n + 1:
        raise ValueError(f"krylov: A has {ip.size - 1} rows, b has length {n}")
    x0v = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
    if x0v is not None and x0v.size != n:
        raise ValueError("cg: x0 and b differ in length")
    invv = None if inv is None else np.ascontiguousarray(inv, dtype=np.float64)
    x = np.empty(max(n, 1))
    max_iter = max(1000, 10 * n) if max_iter is None else int(max_iter)
    res = N.femd_cg_result()
    check(lib.femd_cuda_cg_solve_host(ctx.h, n, _np_ptr(ip), _np_ptr(ix) if ix.size else None, _np_ptr(dv) if dv.size else None,
                                      None if invv is None else _np_ptr(invv), _np_ptr(bv) if n else None,
                                      None if x0v is None else _np_ptr(x0v), _np_ptr(x), max_iter, float(tol),
                                      C.byref(res)))
    return x[:n], bool(res.converged), int(res.iterations), float(res.residual), bool(res.breakdown)
