"""CPU oracle (TEST INFRASTRUCTURE ONLY): numpy-facing wrappers of femd_oracle.c.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module,
and only as the checker.  The library (femd_b200) never imports it.

Every function mirrors one reference function; the C file gives the reference file:line of
each.  `problem(...)` builds a whole synthetic problem (mesh, numbering, caches, pattern,
scatter map, assembled matrix and load vector) the way the reference's fd.solve(a, L) does
for the forms used by the configurations.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

PI = 3.141592653589793


def build():
    """Compile liboracle.so (gcc only)."""
    src = os.path.join(_HERE, "femd_oracle.c")
    if os.path.exists(_LIB) and os.path.getmtime(_LIB) >= os.path.getmtime(src):
        return _LIB
    cc = "gcc-13" if subprocess.run(["which", "gcc-13"], capture_output=True).returncode == 0 else "gcc"
    subprocess.run([cc, "-std=c11", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-shared", "-o", _LIB, src, "-lm"],
                   check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---- mesh, numbering, quadrature, tabulation ------------------------------------------------
def rectangle_mesh(N, x0=0.0, y0=0.0, x1=1.0, y1=1.0):
    pts = np.empty(((N + 1) * (N + 1), 2))
    tris = np.empty((2 * N * N, 3), dtype=np.int32)
    lib().or_rectangle_mesh(C.c_double(x0), C.c_double(y0), C.c_double(x1), C.c_double(y1), N, N, _p(pts), _p(tris))
    return pts, tris


def lagrange_numbering(nv, tris, k, all_exterior=True):
    tris = _i32(tris)
    ne = tris.shape[0]
    nloc = (k + 1) * (k + 2) // 2
    raw = np.empty((ne, nloc), dtype=np.int32)
    dofs = np.empty((ne, nloc), dtype=np.int32)
    rd = C.c_int(0)
    dim = lib().or_lagrange_numbering(nv, ne, _p(tris), k, int(all_exterior), _p(raw), _p(dofs), C.byref(rd))
    if dim < 0:
        raise MemoryError("oracle numbering")
    return dofs, raw, int(dim), int(rd.value)


def triangle_quadrature(degree):
    xi, eta, w = np.empty(64), np.empty(64), np.empty(64)
    m = lib().or_triangle_quadrature(int(degree), _p(xi), _p(eta), _p(w))
    if m < 0:
        raise ValueError("quadrature degree too high")
    return xi[:m].copy(), eta[:m].copy(), w[:m].copy()


def tabulate(k, xi, eta):
    xi, eta = _f64(xi), _f64(eta)
    nloc = (k + 1) * (k + 2) // 2
    out = np.empty((xi.size, 3, nloc))
    lib().or_tabulate(k, xi.size, _p(xi), _p(eta), _p(out))
    return out


def cache_points(pts, tris, xi, eta, w):
    pts, tris, xi, eta, w = _f64(pts), _i32(tris), _f64(xi), _f64(eta), _f64(w)
    ne, nq = tris.shape[0], xi.size
    x, y, ww = np.empty(ne * nq), np.empty(ne * nq), np.empty(ne * nq)
    Ji = np.empty(ne * nq * 4)
    bad = lib().or_cache_points(ne, _p(pts), _p(tris), nq, _p(xi), _p(eta), _p(w), _p(x), _p(y), _p(ww), _p(Ji))
    if bad:
        raise ValueError(f"cell {bad - 1} is degenerate or clockwise")
    return x, y, ww, Ji


# ---- pattern, scatter map, assembly ---------------------------------------------------------
def from_cells(n, dofs):
    dofs = _i32(dofs)
    ne, nloc = dofs.shape
    indptr = np.empty(n + 1, dtype=np.int32)
    nnz = _pattern_rows(n, ne, dofs, nloc, indptr)
    indices = np.empty(nnz, dtype=np.int32)
    if lib().or_pattern_fill(n, ne, _p(dofs), nloc, _p(dofs), nloc, _p(indptr), _p(indices)):
        raise MemoryError("oracle pattern")
    return indptr, indices


def _pattern_rows(n, ne, dofs, nloc, indptr):
    f = lib().or_pattern_rows
    f.restype = C.c_longlong
    nnz = f(n, ne, _p(dofs), nloc, _p(dofs), nloc, _p(indptr))
    if nnz < 0:
        raise MemoryError("oracle pattern")
    return int(nnz)


def scatter_map(dofs, indptr, indices):
    dofs = _i32(dofs)
    ne, nloc = dofs.shape
    m = np.empty(ne * nloc * nloc, dtype=np.int32)
    if lib().or_scatter_map(ne, nloc, _p(dofs), _p(_i32(indptr)), _p(_i32(indices)), _p(m)):
        raise RuntimeError("assemble_matrix_2d: entry outside the pattern")
    return m


def assemble_matrix(nnz, ref, w, Ji, a, b, coefs, smap):
    ref, w, Ji = _f64(ref), _f64(w), _f64(Ji)
    nq, _, nloc = ref.shape
    ne = w.size // nq
    coefs = [_f64(c) for c in coefs]
    arr = (C.c_void_p * len(coefs))(*[c.ctypes.data for c in coefs])
    data = np.zeros(nnz)
    rc = lib().or_assemble_matrix(ne, nloc, nq, _p(ref), _p(w), _p(Ji), len(coefs), _p(_i32(a)), _p(_i32(b)), arr,
                                  _p(_i32(smap)), _p(data))
    if rc:
        raise MemoryError("oracle assembly")
    return data


def assemble_vector(n, ref, w, Ji, a, coef, dofs):
    ref, w, Ji, coef = _f64(ref), _f64(w), _f64(Ji), _f64(coef)
    nq, _, nloc = ref.shape
    ne = w.size // nq
    f = np.zeros(n)
    if lib().or_assemble_vector(ne, nloc, nq, _p(ref), _p(w), _p(Ji), int(a), _p(coef), _p(_i32(dofs)), _p(f)):
        raise MemoryError("oracle assembly")
    return f


def exterior_facets(pts, tris, bounds=(0.0, 0.0, 1.0, 1.0), markers=(1, 2, 3, 4)):
    """The exterior facets of a rectangle mesh in (cell, local edge) order with the markers of
    their sides {bottom, right, top, left}: (cell, local, marker)."""
    pts, tris = _f64(pts), _i32(tris)
    ne = tris.shape[0]
    cell, local, marker = (np.empty(3 * ne, dtype=np.int32) for _ in range(3))
    mk = np.asarray(markers, dtype=np.int32)
    nf = lib().or_rect_exterior_facets(ne, _p(tris), _p(pts), *[C.c_double(v) for v in bounds], _p(mk), _p(cell),
                                       _p(local), _p(marker))
    if nf < 0:
        raise MemoryError("oracle facets")
    return cell[:nf].copy(), local[:nf].copy(), marker[:nf].copy()


def facet_cache(pts, tris, cell, local, k, degree):
    """The exterior-facet quadrature cache: x, y, w, nx, ny (nf nq), Ji (4 per point) and the
    tabulation per local edge (3, nq, 3, nloc)."""
    pts, tris, cell, local = _f64(pts), _i32(tris), _i32(cell), _i32(local)
    nf = cell.size
    nq = max(1, (degree + 2) // 2)
    nloc = (k + 1) * (k + 2) // 2
    x, y, w, nx, ny = (np.empty(nf * nq) for _ in range(5))
    Ji = np.empty(4 * nf * nq)
    ref = np.empty((3, nq, 3, nloc))
    got = lib().or_facet_cache(nf, _p(cell), _p(local), _p(pts), _p(tris), k, degree, _p(x), _p(y), _p(w), _p(nx), _p(ny),
                               _p(Ji), _p(ref))
    if got != nq:
        raise ValueError("oracle facet cache")
    return dict(x=x, y=y, w=w, nx=nx, ny=ny, Ji=Ji, ref=ref, nq=nq)


def assemble_matrix_v(nnz, ref, var, w, Ji, a, b, coefs, smap, into=None):
    """assemble_matrix with a tabulation per entry variant: ref (nvar, nq, 3, nloc), var[e];
    the element matrices are added onto a copy of `into` (default zeros), in entry order."""
    ref, w, Ji = _f64(ref), _f64(w), _f64(Ji)
    _, nq, _, nloc = ref.shape
    ne = w.size // nq
    coefs = [_f64(c) for c in coefs]
    arr = (C.c_void_p * len(coefs))(*[c.ctypes.data for c in coefs])
    data = np.zeros(nnz) if into is None else _f64(into).copy()
    rc = lib().or_assemble_matrix_v(ne, nloc, nq, _p(ref), _p(_i32(var)), _p(w), _p(Ji), len(coefs), _p(_i32(a)),
                                    _p(_i32(b)), arr, _p(_i32(smap)), _p(data))
    if rc:
        raise MemoryError("oracle assembly")
    return data


def assemble_vector_v(n, ref, var, w, Ji, a, coef, dofs, into=None):
    ref, w, Ji, coef = _f64(ref), _f64(w), _f64(Ji), _f64(coef)
    _, nq, _, nloc = ref.shape
    ne = w.size // nq
    f = np.zeros(n) if into is None else _f64(into).copy()
    if lib().or_assemble_vector_v(ne, nloc, nq, _p(ref), _p(_i32(var)), _p(w), _p(Ji), int(a), _p(coef), _p(_i32(dofs)),
                                  _p(f)):
        raise MemoryError("oracle assembly")
    return f


def eval_field(ref, dofs, c):
    ref, c, dofs = _f64(ref), _f64(c), _i32(dofs)
    nq, _, nloc = ref.shape
    ne = dofs.shape[0]
    out = np.empty(ne * nq)
    lib().or_eval_field(ne, nloc, nq, _p(ref), _p(dofs), _p(c), _p(out))
    return out


# ---- sparse kernels and CG ------------------------------------------------------------------
def spmv(indptr, indices, data, x):
    n = indptr.size - 1
    y = np.empty(n)
    lib().or_spmv(n, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data)), _p(_f64(x)), _p(y))
    return y


def jacobi_inverse(indptr, indices, data):
    n = indptr.size - 1
    inv = np.empty(n)
    bad = lib().or_jacobi_inverse(n, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data)), _p(inv))
    if bad >= 0:
        raise ValueError(f"Jacobi: zero diagonal entry in row {bad}")
    return inv


def asymmetry(indptr, indices, data):
    f = lib().or_asymmetry
    f.restype = C.c_double
    return float(f(indptr.size - 1, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data))))


def combine(alpha, A, beta, B):
    A, B = _f64(A), _f64(B)
    out = np.empty_like(A)
    lib().or_combine(C.c_longlong(A.size), C.c_double(alpha), _p(A), C.c_double(beta), _p(B), _p(out))
    return out


def ddot(x, y):
    f = lib().or_ddot
    f.restype = C.c_double
    x, y = _f64(x), _f64(y)
    return float(f(_p(x), _p(y), C.c_size_t(x.size)))


def cg_jacobi(indptr, indices, data, inv, b, x0=None, max_iter=None, tol=1e-10):
    n = indptr.size - 1
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    max_iter = max(1000, 10 * n) if max_iter is None else int(max_iter)
    res = np.zeros(4)
    if lib().or_cg_jacobi(n, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data)), _p(_f64(inv)), _p(_f64(b)), _p(x),
                          max_iter, C.c_double(tol), _p(res)):
        raise MemoryError("oracle cg")
    return x, dict(converged=bool(res[0]), iterations=int(res[1]), residual=float(res[2]), breakdown=bool(res[3]))


def ilu0(indptr, indices, data):
    """ILU(0) on the matrix's pattern (ILU0Preconditioner, natural ordering): (lu, diag, min_pivot)."""
    n = indptr.size - 1
    lu = np.empty(int(indptr[-1]))
    diag = np.empty(n, dtype=np.int32)
    mp = C.c_double()
    st = lib().or_ilu0(n, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data)), _p(lu), _p(diag), C.byref(mp))
    if st >= 0:
        raise ValueError(f"ILU(0): zero diagonal entry in row {st}")
    if st < -1:
        raise RuntimeError(f"ILU(0): zero pivot in row {-st - 2}")
    return lu, diag, mp.value


def ilu0_apply(indptr, indices, lu, diag, r):
    z = np.empty(indptr.size - 1)
    lib().or_ilu0_apply(indptr.size - 1, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(lu)), _p(_i32(diag)), _p(_f64(r)), _p(z))
    return z


def diag_positions(indptr, indices, data):
    diag = np.empty(indptr.size - 1, dtype=np.int32)
    st = lib().or_diag_positions(indptr.size - 1, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data)), _p(diag))
    if st >= 0:
        raise ValueError(f"SSOR: zero diagonal entry in row {st}")
    return diag


def ssor_apply(indptr, indices, data, diag, r, omega=1.0):
    z = np.empty(indptr.size - 1)
    lib().or_ssor_apply(indptr.size - 1, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data)), _p(_i32(diag)),
                        C.c_double(omega), _p(_f64(r)), _p(z))
    return z


def cg_pc(indptr, indices, data, b, kind, x0=None, max_iter=None, tol=1e-10, omega=1.0):
    """CG preconditioned by ILU(0) (kind "ilu0") or SSOR (kind "ssor"), natural ordering
    (krylov::cg with ILU0Preconditioner / SSORPreconditioner)."""
    n = indptr.size - 1
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    max_iter = max(1000, 10 * n) if max_iter is None else int(max_iter)
    if kind == "ilu0":
        lu, diag, _ = ilu0(indptr, indices, data)
        k = 0
    elif kind == "ssor":
        lu, diag, k = np.zeros(1), diag_positions(indptr, indices, data), 1
    else:
        raise ValueError(f"cg_pc: kind is 'ilu0' or 'ssor', got {kind!r}")
    res = np.zeros(4)
    if lib().or_cg_pc(n, _p(_i32(indptr)), _p(_i32(indices)), _p(_f64(data)), k, _p(_f64(lu)), _p(_i32(diag)),
                      C.c_double(omega), _p(_f64(b)), _p(x), max_iter, C.c_double(tol), _p(res)):
        raise MemoryError("oracle cg")
    return x, dict(converged=bool(res[0]), iterations=int(res[1]), residual=float(res[2]), breakdown=bool(res[3]))


def integrand_eval(code, nreg, consts, inputs, xs=None, ys=None, nx=None, ny=None):
    """Integrand(code, nreg, nconst, ninput).evaluate(...) on real values: code is (ninstr, 4)
    int (op, out, a, b); inputs (ninput, npts).  Raises ValueError on a malformed program."""
    code = _i32(code).reshape(-1)
    consts = _f64(consts).reshape(-1)
    inputs = [_f64(v) for v in inputs]
    npts = max([v.size for v in inputs] + [0 if xs is None else np.asarray(xs).size, 0 if nx is None else np.asarray(nx).size])
    ptrs = (C.c_void_p * max(len(inputs), 1))(*[v.ctypes.data for v in inputs])
    arrs = [None if a is None else _f64(a) for a in (xs, ys, nx, ny)]
    out = np.empty(npts)
    f = lib().or_integrand_eval
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]
    st = f(code.ctypes.data, code.size, int(nreg), consts.ctypes.data if consts.size else None, consts.size, ptrs,
           len(inputs), *[None if a is None else a.ctypes.data for a in arrs], npts, out.ctypes.data)
    if st == -1:
        raise MemoryError("oracle integrand")
    if st:
        raise ValueError(f"Integrand: malformed program (check {st})")
    return out


# ---- quadrature degree of the reference's form compiler (forms.py:2487-2500) -----------------
def qdeg(form, k):
    return max({"gradgrad": 2 * (k - 1), "helmholtz": 2 * k, "varcoef": 3 * k - 1, "rhs_data": 2 * k + 1,
                "rhs_field": 2 * k, "mass": 2 * k}[form], 1)


def sin_rhs(x, y, helmholtz=False):
    s = np.sin(PI * x) * np.sin(PI * y)
    return 2.0 * PI * PI * s + s if helmholtz else 2.0 * PI * PI * s


def kcoef(x, y):
    return 1.0 + 0.5 * np.sin(2.0 * PI * x) * np.sin(2.0 * PI * y)


def problem(form, N, k, c=1.0, f_dofs=None, b_vec=None, free=False, robin=0.0, facet_ref=None):
    """The whole reference pipeline for one synthetic problem, on the CPU.

    form: "poisson_sin" | "helmholtz_sin" | "varcoef_field" | "poisson_vec" | "heat"
    free: no Dirichlet elimination; robin: alpha of alpha u v ds, with g v ds (g = 1 + x y) added
    to the load, over every exterior facet (ds degrees 2k and k + 2); facet_ref: the facet
    tabulation to use for the ds matrix (default: this oracle's).
    Returns a dict with pts, tris, dofs, dim, indptr, indices, map, data, rhs (and data_K for heat).
    """
    pts, tris = rectangle_mesh(N)
    dofs, raw, dim, raw_dim = lagrange_numbering(pts.shape[0], tris, k, not free)
    ga = {"poisson_sin": "gradgrad", "poisson_vec": "gradgrad", "helmholtz_sin": "helmholtz",
          "varcoef_field": "varcoef", "heat": "mass"}[form]
    xi, eta, w = triangle_quadrature(qdeg(ga, k))
    ref = tabulate(k, xi, eta)
    x, y, ww, Ji = cache_points(pts, tris, xi, eta, w)
    indptr, indices = from_cells(dim, dofs)
    smap = scatter_map(dofs, indptr, indices)
    nnz = int(indptr[-1])
    one = np.ones(ww.size)
    out = dict(pts=pts, tris=tris, dofs=dofs, raw=raw, dim=dim, raw_dim=raw_dim, indptr=indptr, indices=indices,
               map=smap, ref=ref, quad=(xi, eta, w))
    if form in ("poisson_sin", "poisson_vec"):
        out["data"] = assemble_matrix(nnz, ref, ww, Ji, [1, 2], [1, 2], [c * one, c * one], smap)
    elif form == "helmholtz_sin":
        out["data"] = assemble_matrix(nnz, ref, ww, Ji, [1, 2, 0], [1, 2, 0], [one, one, one], smap)
    elif form == "varcoef_field":
        kc = kcoef(x, y)
        out["data"] = assemble_matrix(nnz, ref, ww, Ji, [1, 2], [1, 2], [kc, kc], smap)
    elif form == "heat":
        out["data"] = assemble_matrix(nnz, ref, ww, Ji, [0], [0], [one], smap)
        out["data_K"] = assemble_matrix(nnz, ref, ww, Ji, [1, 2], [1, 2], [one, one], smap)
        return out
    if form in ("poisson_sin", "helmholtz_sin"):
        xf, yf, wf = triangle_quadrature(qdeg("rhs_data", k))
        reff = tabulate(k, xf, yf)
        px, py, pw, pJ = cache_points(pts, tris, xf, yf, wf)
        out["rhs"] = assemble_vector(dim, reff, pw, pJ, 0, sin_rhs(px, py, form == "helmholtz_sin"), dofs)
    elif form == "varcoef_field":
        xf, yf, wf = triangle_quadrature(qdeg("rhs_field", k))
        reff = tabulate(k, xf, yf)
        px, py, pw, pJ = cache_points(pts, tris, xf, yf, wf)
        fc = eval_field(reff, dofs, f_dofs)
        out["rhs"] = assemble_vector(dim, reff, pw, pJ, 0, fc, dofs)
    else:
        out["rhs"] = _f64(b_vec)
    if robin:
        fcell, flocal, fmarker = exterior_facets(pts, tris)
        fdofs = dofs[fcell]
        fsmap = scatter_map(fdofs, indptr, indices)
        Fa = facet_cache(pts, tris, fcell, flocal, k, 2 * k)
        ra = Fa["ref"] if facet_ref is None else facet_ref
        out["data"] = assemble_matrix_v(nnz, ra, flocal, Fa["w"], Fa["Ji"], [0], [0], [robin * np.ones(Fa["w"].size)], fsmap,
                                        into=out["data"])
        Fb = facet_cache(pts, tris, fcell, flocal, k, k + 2)
        out["rhs"] = assemble_vector_v(dim, Fb["ref"], flocal, Fb["w"], Fb["Ji"], 0, 1.0 + Fb["x"] * Fb["y"], fdofs,
                                       into=out["rhs"])
        out["facets"] = (fcell, flocal, fmarker)
        out["facet_cache"] = Fa
    return out
