"""Compiled 2D forms on the GPU: coefficient programs, the form assembler, the solver dispatch.

The reference compiles a Python form once (python/femd/forms.py:1822-1938, _Program; :2040-2095,
_Compiled2D) into a C++ FormAssembler2D (include/femd/forms/assembler_2d.hpp): known fields read
at the quadrature points, one Integrand register program per term for its coefficient, and the
cell kernels.  This module is that layer over libfemd_cuda:

    Integrand            integrand.hpp:33-109      the register program, run by the device evaluator
    eval_field           cache_2d.hpp:245-288      a P_k field's values / derivatives at the points
    FormAssembler2D      assembler_2d.hpp:38-266   add_field / add_group / add_term / assemble_*
    Form2D               forms.py:2040-2095        a compiled form: assemble() -> CSRMatrix with
                                                   K.symmetric = K.asymmetry() <= 1e-13, or a vector
    SparseSolver         sparse.py:340-483         A.solver(backend, ...): .solve(b), .info, .backend
    solve                linalg.py:710-755         fd.solve(a, L, backend=..., dirichlet=...) on 2D meshes

Every computation runs in libfemd_cuda's kernels; the objects here only hold device buffers and
call the C ABI.  Nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import math
import warnings

import numpy as np

from . import _native as N
from .core import (Cache2D, Coef, CSRMatrix, ILU0Preconditioner, JacobiPreconditioner, LagrangeSpace2D,
                   SSORPreconditioner, _torch, assemble_matrix_2d, assemble_vector_2d, cg_solve, check, context, lib)
from .krylov import KrylovInfo

# opcodes of the reference's instruction set (integrand.hpp:33-45)
CONST, X, Y, NX, NY, INPUT, ADD, MUL, POW, SIN, COS, EXP, LOG, TANH, SQRT, SINH, COSH, SECH, ABS, SIGN = range(20)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _as_dev(a, device):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(device)


class Integrand:
    """A coefficient program (femd::Integrand): code is (ninstr, 4) int -- op, out register, a, b
    -- with the reference's opcodes; the coefficient is the last instruction's register.
    Malformed programs raise ValueError with the reference's messages when evaluated."""

    def __init__(self, code, nreg, nconst, ninput):
        self.code = np.ascontiguousarray(np.asarray(code, dtype=np.int32).reshape(-1, 4))
        self.nreg, self.nconst, self.ninput = int(nreg), int(nconst), int(ninput)

    @property
    def needs_coordinates(self):
        return bool(np.isin(self.code[:, 0], (X, Y)).any())

    @property
    def needs_normal(self):
        return bool(np.isin(self.code[:, 0], (NX, NY)).any())

    def _struct(self):
        return N.femd_integrand(self.code.ctypes.data, self.code.size, self.nreg, self.nconst, self.ninput)

    def _args(self, inputs, consts, device):
        inputs = [_as_dev(v, device) for v in inputs]
        if len(inputs) != self.ninput:
            raise ValueError("Integrand: wrong number of inputs")
        cv = np.ascontiguousarray(np.asarray(consts, dtype=np.float64).reshape(-1))
        if cv.size != self.nconst:
            raise ValueError("Integrand: wrong number of constants")
        arr = (C.c_void_p * max(len(inputs), 1))(*[v.data_ptr() for v in inputs])
        return inputs, cv, arr

    def evaluate(self, npts, inputs, consts, *, xs=None, ys=None, nx=None, ny=None, ctx=None):
        """The coefficient at npts points (Integrand::evaluate): inputs ninput device arrays,
        consts nconst numbers, coordinates / normals device arrays when the program reads them.
        Returns a float64 device tensor."""
        torch = _torch()
        ctx = ctx or context()
        dev = f"cuda:{ctx.device}"
        inputs, cv, arr = self._args(inputs, consts, dev)
        pts = [None if a is None else _as_dev(a, dev) for a in (xs, ys, nx, ny)]
        out = torch.empty(int(npts), dtype=torch.float64, device=dev)
        prog = self._struct()
        ctx.enter()
        st = lib.femd_cuda_integrand_eval(ctx.h, C.byref(prog), cv.ctypes.data if cv.size else None, arr, int(npts),
                                          *[_ptr(a) for a in pts], _ptr(out))
        ctx.leave()
        check(st)
        return out

    def evaluate_cells(self, Q: Cache2D, inputs, consts, *, ctx=None):
        """The coefficient at the points of a cell rule, [e nq + q] (the reference's cell
        group), x and y formed from the mesh as the cell cache does."""
        torch = _torch()
        ctx = ctx or context()
        dev = f"cuda:{ctx.device}"
        inputs, cv, arr = self._args(inputs, consts, dev)
        mesh = Q.space.mesh.c_struct(ctx)
        rule = Q.c_struct()
        out = torch.empty(Q.space.mesh.ncells * Q.nq, dtype=torch.float64, device=dev)
        prog = self._struct()
        ctx.enter()
        st = lib.femd_cuda_integrand_eval_cells(ctx.h, C.byref(prog), cv.ctypes.data if cv.size else None, arr,
                                                C.byref(mesh), C.byref(rule), _ptr(out))
        ctx.leave()
        check(st)
        return out

    # ---- a few programs of the forms on this path --------------------------------------------
    @staticmethod
    def constant():
        """c0: a coefficient read from the constants."""
        return Integrand([[CONST, 0, 0, 0]], 1, 1, 0)

    @staticmethod
    def varcoef(two_pi=2 * math.pi):
        """c0 + c1 sin(c2 x) sin(c2 y), constants (c0, c1, c2) -- config 3's k(x, y) with
        (1, 0.5, 2 pi)."""
        code = [[CONST, 0, 0, 0], [CONST, 1, 1, 0], [CONST, 2, 2, 0], [X, 3, 0, 0], [Y, 4, 0, 0],
                [MUL, 3, 2, 3], [SIN, 3, 3, 0], [MUL, 4, 2, 4], [SIN, 4, 4, 0], [MUL, 3, 1, 3], [MUL, 3, 3, 4],
                [ADD, 0, 0, 3]]
        return Integrand(code, 5, 3, 0)

    @staticmethod
    def field(scale=False):
        """The field value input 0 (times the constant c0 when scale)."""
        if scale:
            return Integrand([[INPUT, 0, 0, 0], [CONST, 1, 0, 0], [MUL, 0, 1, 0]], 2, 1, 1)
        return Integrand([[INPUT, 0, 0, 0]], 1, 0, 1)


def eval_field(Q: Cache2D, c, codes, *, raw_dofs=None, ctx=None):
    """Cache2D::eval_multi: the P_k field with coefficients c (the space's dofs; or, with
    raw_dofs, the ncells x nloc device map of another numbering) at the points of Q, for the
    derivative codes (0 value, 1 d/dx, 2 d/dy): a device tensor of len(codes) x ncells nq values."""
    torch = _torch()
    ctx = ctx or context()
    V = Q.space
    dofs = raw_dofs if raw_dofs is not None else V.cell_dofs_device(ctx)
    cv = _as_dev(c, f"cuda:{ctx.device}")
    codes = [int(m) for m in codes]
    np_ = V.mesh.ncells * Q.nq
    out = torch.empty(len(codes) * np_, dtype=torch.float64, device=cv.device)
    ca = (C.c_int * len(codes))(*codes)
    mesh = V.mesh.c_struct(ctx)
    rule = Q.c_struct()
    ctx.enter()
    st = lib.femd_cuda_eval_field(ctx.h, C.byref(mesh), C.byref(rule), _ptr(dofs), _ptr(cv), len(codes), ca, _ptr(out))
    ctx.leave()
    check(st)
    return out


class FormAssembler2D:
    """The compiled form (femd::FormAssembler2D, include/femd/forms/assembler_2d.hpp:38-266) on
    the GPU: fields read at the points of a cell rule, groups of terms on a rule, each term a
    coefficient program over field values and constants with a test code a and a trial code b
    (0 value, 1 d/dx, 2 d/dy).  assemble_vector zeroes f and adds each group's vector;
    assemble_matrix writes K (the reference adds into a K the caller zeroed: the same values)."""

    def __init__(self, rank, nvectors, nconsts):
        if rank not in (1, 2):
            raise ValueError("FormAssembler2D: rank is 1 or 2 on this path (rank 0 is not assembled here)")
        if nvectors < 0 or nconsts < 0:
            raise ValueError("FormAssembler2D: negative count")
        self.rank, self.nvec, self.ncon = int(rank), int(nvectors), int(nconsts)
        self.fields = []            # (Q, vec, codes, first)
        self.groups = []            # dict(QT, QS, terms=[(prog, inputs, consts, a, b)])
        self.nval = 0

    def add_field(self, Q: Cache2D, vec, offset, dim, codes):
        """Known field vectors[vec][offset : offset + dim] at the points of Q; returns the index
        of its first value array (code i is first + i)."""
        if vec < 0 or vec >= self.nvec:
            raise ValueError("FormAssembler2D::add_field: vector index out of range")
        if offset < 0 or dim < 0:
            raise ValueError("FormAssembler2D::add_field: negative offset or dim")
        if offset != 0:
            raise ValueError("FormAssembler2D::add_field: block offsets are not on this path")
        if dim != Q.space.dim:
            raise ValueError("FormAssembler2D::add_field: dim != the dimension of the field's space")
        codes = [int(m) for m in codes]
        if not codes:
            raise ValueError("FormAssembler2D::add_field: no derivative codes")
        if any(m < 0 or m > 2 for m in codes):
            raise ValueError("FormAssembler2D::add_field: derivative code out of range")
        first = self.nval
        self.fields.append((Q, int(vec), codes, first))
        self.nval += len(codes)
        return first

    def add_group(self, QT: Cache2D, QS: Cache2D | None = None, toff=0, roff=0):
        if self.rank == 2 and QS is None:
            raise ValueError("FormAssembler2D::add_group: a rank-2 form needs the trial cache")
        if QS is not None and (QS.space.mesh is not QT.space.mesh or QS.nq != QT.nq):
            raise ValueError("FormAssembler2D::add_group: test and trial caches differ (entries, points or kind)")
        if toff < 0 or roff < 0:
            raise ValueError("FormAssembler2D::add_group: negative offset")
        if toff or roff:
            raise ValueError("FormAssembler2D::add_group: block offsets are not on this path")
        self.groups.append(dict(QT=QT, QS=QS, terms=[]))
        return len(self.groups) - 1

    def _value_q(self, i):
        for Q, _, codes, first in self.fields:
            if first <= i < first + len(codes):
                return Q
        return None

    def add_term(self, g, prog: Integrand, inputs, consts, a, b=0, sa=0, sb=0):
        if g < 0 or g >= len(self.groups):
            raise ValueError("FormAssembler2D::add_term: no such group")
        G = self.groups[g]
        if len(inputs) != prog.ninput:
            raise ValueError(f"FormAssembler2D::add_term: the program takes {prog.ninput} inputs")
        if len(consts) != prog.nconst:
            raise ValueError(f"FormAssembler2D::add_term: the program takes {prog.nconst} constants")
        for i in inputs:
            if i < 0 or i >= self.nval:
                raise ValueError("FormAssembler2D::add_term: input out of range")
            Qi = self._value_q(i)
            if Qi is not G["QT"] and not (Qi.space.mesh is G["QT"].space.mesh and Qi.nq == G["QT"].nq and
                                          np.array_equal(Qi.xi, G["QT"].xi)):
                raise ValueError("FormAssembler2D::add_term: an input lives on another point set")
        for k in consts:
            if k < 0 or k >= self.ncon:
                raise ValueError("FormAssembler2D::add_term: constant out of range")
        if prog.needs_normal:
            raise ValueError("FormAssembler2D::add_term: the coefficient reads the normal on a cell group")
        if self.rank >= 1 and not 0 <= a <= 2:
            raise ValueError("FormAssembler2D::add_term: test code out of range")
        if self.rank == 2 and not 0 <= b <= 2:
            raise ValueError("FormAssembler2D::add_term: trial code out of range")
        if sa not in (0, 1) or sb not in (0, 1):
            raise ValueError("FormAssembler2D::add_term: a side is 0 or 1")
        G["terms"].append((prog, [int(i) for i in inputs], [int(k) for k in consts], int(a), int(b)))

    # ---- evaluation ------------------------------------------------------------------------
    def _values(self, vectors, ctx):
        if len(vectors) != self.nvec:
            raise ValueError(f"FormAssembler2D: {self.nvec} coefficient vectors expected")
        vals = [None] * self.nval
        for Q, vec, codes, first in self.fields:
            v = vectors[vec]
            n = v.numel() if hasattr(v, "numel") else np.asarray(v).size
            if n < Q.space.dim:
                raise ValueError(f"FormAssembler2D: coefficient vector {vec} has {n} entries, the form reads "
                                 f"{Q.space.dim}")
            out = eval_field(Q, v, codes, ctx=ctx)
            np_ = Q.space.mesh.ncells * Q.nq
            for i in range(len(codes)):
                vals[first + i] = out[i * np_:(i + 1) * np_]
        return vals

    def _coefs(self, G, vals, consts, ctx):
        """Per term: a Coef for the assembly kernel (a constant program stays a constant)."""
        out = []
        for prog, inputs, cidx, a, b in G["terms"]:
            cv = [consts[k] for k in cidx]
            if prog.ninput == 0 and prog.code.shape[0] == 1 and prog.code[0, 0] == CONST:
                out.append(Coef.const(cv[prog.code[0, 2]]))
                continue
            pts = prog.evaluate_cells(G["QT"], [vals[i] for i in inputs], cv, ctx=ctx)
            out.append(Coef.points(pts))
        return out

    def assemble_vector(self, vectors, consts, n, *, ctx=None):
        if self.rank != 1:
            raise ValueError("FormAssembler2D::assemble_vector: not a rank-1 form")
        torch = _torch()
        ctx = ctx or context()
        consts = [float(c) for c in consts]
        if len(consts) != self.ncon:
            raise ValueError(f"FormAssembler2D: {self.ncon} constants expected")
        vals = self._values(vectors, ctx)
        f = torch.zeros(int(n), dtype=torch.float64, device=f"cuda:{ctx.device}")
        for G in self.groups:
            if not G["terms"]:
                continue
            Q = G["QT"]
            if Q.space.dim > n:
                raise ValueError("FormAssembler2D::assemble_vector: f is too short")
            cs = self._coefs(G, vals, consts, ctx)
            block = assemble_vector_2d(Q, [t[3] for t in G["terms"]], cs)
            f[:Q.space.dim] += block
        return f

    def assemble_matrix(self, vectors, consts, K: CSRMatrix, *, ctx=None, jacobi=True):
        if self.rank != 2:
            raise ValueError("FormAssembler2D::assemble_matrix: not a rank-2 form")
        ctx = ctx or K.ctx
        consts = [float(c) for c in consts]
        if len(consts) != self.ncon:
            raise ValueError(f"FormAssembler2D: {self.ncon} constants expected")
        groups = [G for G in self.groups if G["terms"]]
        if len(groups) > 1:
            raise ValueError("FormAssembler2D::assemble_matrix: one cell group per matrix on this path")
        vals = self._values(vectors, ctx)
        for G in groups:
            cs = self._coefs(G, vals, consts, ctx)
            T = G["terms"]
            assemble_matrix_2d(G["QT"], G["QS"], [t[3] for t in T], [t[4] for t in T], cs, K, jacobi=jacobi)
        return K


class Form2D:
    """A compiled 2D form on a Lagrange space (the reference's _Compiled2D,
    python/femd/forms.py:2040-2095): a FormAssembler2D with its test space and the current field
    vectors and constants.  assemble() returns, for rank 2, a new CSRMatrix on the space's
    pattern with symmetric = asymmetry() <= 1e-13 (forms.py:2093-2094), and for rank 1 a float64
    device vector."""

    def __init__(self, rank, V: LagrangeSpace2D, assembler: FormAssembler2D, vectors=(), consts=()):
        self.rank, self.V, self.A = int(rank), V, assembler
        self.vectors, self.consts = list(vectors), list(consts)
        self.test_space = V
        self.trial_space = V if rank == 2 else None

    @staticmethod
    def build(V: LagrangeSpace2D, terms, degree, rank=None, fields=(), consts=()):
        """A form from terms: (a, coef) for rank 1 or (a, b, coef) for rank 2, each coef a number,
        a (Integrand, input value indices, constant indices) tuple, or an Integrand over no
        inputs whose constants are the form's; fields = [(vector, codes)] read at the points;
        degree the quadrature degree of the cell rule."""
        if rank is None:
            rank = len(terms[0]) - 1
        Q = V.cache(int(degree))
        consts = list(consts)
        A = FormAssembler2D(rank, len(fields), 0)
        vecs = []
        for vec, codes in fields:
            A.add_field(Q, len(vecs), 0, V.dim, codes)
            vecs.append(vec)
        g = A.add_group(Q, Q if rank == 2 else None)
        spec = []
        for t in terms:
            a, b, c = (t[0], 0, t[1]) if rank == 1 else t
            if isinstance(c, (int, float)):
                spec.append((Integrand.constant(), [], [len(consts)], a, b))
                consts.append(float(c))
            elif isinstance(c, Integrand):
                ks = list(range(len(consts), len(consts) + c.nconst))
                spec.append((c, [], ks, a, b))
            else:
                prog, inputs, ks = c
                spec.append((prog, list(inputs), list(ks), a, b))
        A.ncon = len(consts)
        for prog, inputs, ks, a, b in spec:
            A.add_term(g, prog, inputs, ks, a, b)
        return Form2D(rank, V, A, vecs, consts)

    def assemble(self, **overrides):
        consts = list(self.consts)
        vectors = list(self.vectors)
        for k, v in overrides.items():
            if k.startswith("c") and k[1:].isdigit():
                consts[int(k[1:])] = float(v)
            elif k.startswith("f") and k[1:].isdigit():
                vectors[int(k[1:])] = v
            else:
                raise KeyError(f"'{k}' is not a constant (c<i>) or field (f<i>) of this form")
        if self.rank == 1:
            return self.A.assemble_vector(vectors, consts, self.V.dim)
        K = CSRMatrix(self.V.pattern())
        self.A.assemble_matrix(vectors, consts, K)
        K.symmetric = bool(K.asymmetry() <= 1e-13)
        return K


# ---- the solver dispatch ---------------------------------------------------------------------
BACKENDS = ("auto", "cg", "cuda-cg", "cuda-cg-mixed")


class SparseSolver:
    """A solver for a CSRMatrix on the GPU (the reference's SparseSolver, python/femd/sparse.py:
    340-483): solve(b, into=None, lift=None) as the reference's does, .backend, .info (the
    KrylovInfo of the last solve).

    backend "cg": krylov.cg with the reference's default M="ilu0" (ILU(0), natural ordering,
    the reference's factors; "ssor", "jacobi" or None too); "cuda-cg": Jacobi-PCG in FP64 (the fast
    path: the fused SpMV / update kernels); "cuda-cg-mixed": the FP32-inner / FP64-refined PCG;
    "auto" (the reference's default picks its sparse Cholesky for a symmetric matrix with a
    positive diagonal, which this path does not build): Jacobi-PCG for such a matrix, and
    ValueError otherwise.  The matrix, its preconditioner and the solver's workspace (vectors,
    captured CUDA graphs) stay resident between solves."""

    def __init__(self, A: CSRMatrix, backend="auto", **options):
        b = getattr(backend, "name", backend)
        b = "auto" if b is None else str(b).lower()
        if A.nrows != A.ncols:
            raise ValueError(f"solver(): the matrix is {A.nrows} x {A.ncols}, not square")
        if b not in BACKENDS:
            raise ValueError(f"unknown backend {backend!r} on the GPU path: 'auto' (default), 'cg' / 'cuda-cg' "
                             "(Jacobi-PCG) or 'cuda-cg-mixed'")
        self.A, self.info = A, None
        M = options.pop("M", "ilu0" if b == "cg" else "jacobi")
        self.tol = float(options.pop("tol", 1e-10))
        self.maxiter = options.pop("maxiter", None)
        self.x0 = options.pop("x0", None)
        self.warn = bool(options.pop("warn", True))
        if options:
            raise TypeError(f"the {b} backend takes M=, tol=, maxiter=, x0= and warn=, got {sorted(options)}")
        if b == "auto":
            if not (A.nrows > 0 and A.symmetric and bool(np.all(A.diagonal() > 0))):
                raise ValueError("solver('auto'): the GPU path solves symmetric matrices with a positive diagonal "
                                 "(Jacobi-PCG); this one is not (SparseMatrix.symmetric is False or a diagonal entry "
                                 "is <= 0)")
            b = "cuda-cg"
        self.backend = b
        if isinstance(M, str):
            M = preconditioner(A, M)
        if M is not None and not isinstance(M, (JacobiPreconditioner, ILU0Preconditioner, SSORPreconditioner)):
            raise TypeError("solver(): M is 'ilu0', 'ssor', 'jacobi', a preconditioner of this path or None")
        if self.backend in ("cuda-cg", "cuda-cg-mixed") and not (M is None or isinstance(M, JacobiPreconditioner)):
            raise ValueError(f"solver({self.backend!r}): the fused GPU loop is Jacobi-preconditioned; use backend 'cg' for "
                             f"{M.name}")
        if self.backend == "cuda-cg-mixed" and M is None:
            raise ValueError("solver('cuda-cg-mixed'): the mixed-precision solve is Jacobi-preconditioned")
        self._M = M

    @property
    def size(self):
        return self.A.nrows

    def _solve_array(self, b):
        n = self.A.nrows
        maxiter = int(self.maxiter if self.maxiter is not None else max(1000, 10 * n))
        x, conv, its, res, brk = cg_solve(self.A, self._M, b, self.x0, maxiter, self.tol,
                                          mixed=self.backend == "cuda-cg-mixed")
        self.info = KrylovInfo(bool(conv), int(its), float(res), float(res), "cg")
        if self.warn and brk:
            warnings.warn("cg broke down (p^T A p <= 0 or r^T M^{-1} r <= 0): A or the preconditioner is not "
                          "symmetric positive definite", RuntimeWarning, stacklevel=3)
        elif self.warn and not conv:
            warnings.warn(f"cg did not converge in {its} iterations (residual {res:.2e}, tol {self.tol:.1e}); raise "
                          "maxiter or improve the preconditioner", RuntimeWarning, stacklevel=3)
        return x

    def solve(self, b, into=None, lift=None):
        """x with A x = b (a float64 device tensor); into: a device tensor that receives it; lift:
        the lifting of Dirichlet data (a Lift from V.lift): the solution is returned on the raw
        (unconstrained) numbering, u = u_0 + u_g."""
        x = self._solve_array(b)
        if lift is not None:
            return lift.compose(x)
        if into is not None:
            into.copy_(x)
            return into
        return x

    def __repr__(self):
        return f"SparseSolver({self.backend}, n={self.size})"


def preconditioner(A: CSRMatrix, name: str):
    """A.preconditioner(name) (python/femd/sparse.py): "ilu0", "ssor" or "jacobi"."""
    n = str(name).lower()
    if n == "ilu0":
        return ILU0Preconditioner(A)
    if n == "ssor":
        return SSORPreconditioner(A)
    if n == "jacobi":
        return JacobiPreconditioner(A)
    raise ValueError(f"preconditioner {name!r}: 'ilu0', 'ssor' or 'jacobi' on the GPU path")


CSRMatrix.preconditioner = preconditioner


def solver(A: CSRMatrix, backend="auto", **options) -> SparseSolver:
    """A.solver(backend, ...) (python/femd/sparse.py:297-299)."""
    return SparseSolver(A, backend, **options)


CSRMatrix.solver = solver


def solve(a: Form2D, L: Form2D, backend="auto", dirichlet=None, **options):
    """fd.solve(a, L) on a 2D mesh (python/femd/linalg.py:710-755): assemble a and L, solve with
    A.solver(backend); with dirichlet= data the Dirichlet lift u_g = V.lift(g) is taken off the
    load vector (b -= a.action(u_g)) and the solution u_0 + u_g is returned on the raw numbering."""
    if a.rank != 2 or L.rank != 1:
        raise TypeError(f"solve(a, L): a must be bilinear (rank 2) and L linear (rank 1), got ranks {a.rank} and {L.rank}")
    V = a.test_space
    if L.test_space is not V:
        raise ValueError("solve(a, L): a and L must have the same test space")
    A = a.assemble()
    b = L.assemble()
    S = A.solver(backend, **options)
    if dirichlet is None or V.bc != "dirichlet":
        if dirichlet is not None and not (isinstance(dirichlet, (int, float)) and dirichlet == 0):
            raise ValueError("solve(dirichlet=...): the space has no Dirichlet condition built in; create it with "
                             "bc='dirichlet'")
        return S.solve(b)
    from .lift import lift as _lift
    ug = _lift(V, dirichlet)
    b -= ug.action(a)
    return S.solve(b, lift=ug)
