"""The coefficient side of a compiled form on the GPU (f3): the Integrand register program and P_k
fields at the points, against the reference's fixtures and the oracle.

Tolerances.  Programs of sums, products, squares, reciprocals, square roots, absolute values
and signs are exact IEEE operations in both, so their values are compared bit for bit.  A program
with a transcendental instruction (sin, cos, exp, log, tanh, sinh, cosh, sech, a general pow) uses
CUDA's double-precision functions where the reference uses the host C library's; their results
differ by a few ulp, so such programs are compared within 1e-12 relative (+ 1e-14 of the largest
value).  Field values and derivatives at the points: within 1e-13 relative of the oracle's
restatement of Cache2D::eval_multi (+ 1e-15 of the largest).
"""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import INTEGRAND_CASES, golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TRANSCENDENTAL = {8, 9, 10, 11, 12, 13, 15, 16, 17}      # POW, SIN ... COSH, SECH (not SQRT, ABS, SIGN)


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


def _dev(torch, a):
    return None if a is None else torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _close(out, ref, exact):
    if exact:
        return np.array_equal(out, ref)
    return bool(np.all(np.abs(out - ref) <= 1e-12 * np.abs(ref) + 1e-14 * np.abs(ref).max()))


@pytest.mark.parametrize("name", INTEGRAND_CASES)
def test_integrand_matches_reference(fb, name):
    import torch
    from femd_b200.forms import Integrand
    z, _ = golden(name)
    code = np.asarray(z["code"], dtype=np.int32)
    prog = Integrand(code, int(z["nreg"]), len(z["consts"]), len(z["inputs"]))
    kw = {}
    if bool(z["has_xy"]):
        kw.update(xs=_dev(torch, z["xs"]), ys=_dev(torch, z["ys"]))
    if bool(z["has_normal"]):
        kw.update(nx=_dev(torch, z["nx"]), ny=_dev(torch, z["ny"]))
    out = prog.evaluate(z["out"].size, [_dev(torch, v) for v in z["inputs"]], list(z["consts"]), **kw).cpu().numpy()
    exact = not (set(code[:, 0].tolist()) & TRANSCENDENTAL)
    assert _close(out, z["out"], exact)


def test_integrand_every_instruction_against_the_oracle(fb):
    """Random points through a program with every instruction, the oracle's restatement as
    the checker (the same C library the reference uses)."""
    import torch
    from femd_b200.forms import Integrand
    rng = np.random.default_rng(3)
    n = 5000
    xs, ys = rng.uniform(0.1, 1.0, n), rng.uniform(0.1, 1.0, n)
    nx, ny = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    u = rng.uniform(0.2, 2.0, n)
    # r0 = x, r1 = y, r2 = nx, r3 = -ny, r4 = u, r5 = 1.5, then every unary op and binary op
    code = [[1, 0, 0, 0], [2, 1, 0, 0], [3, 2, 1, 0], [4, 3, -1, 0], [5, 4, 0, 0], [0, 5, 0, 0],
            [6, 6, 0, 1], [7, 7, 6, 4], [8, 8, 7, 1], [8, 9, 4, 2], [8, 10, 4, 3], [8, 11, 4, 4]]
    reg = 12
    for op in range(9, 20):
        code.append([op, reg, 7, 0])
        code.append([6, reg + 1, reg, 2])
        reg += 2
    code.append([7, reg, reg - 1, 8])
    prog = Integrand(code, reg + 1, 5, 1)
    consts = [1.5, 2.0, 0.5, -1.0, 2.5]
    got = prog.evaluate(n, [_dev(torch, u)], consts, xs=_dev(torch, xs), ys=_dev(torch, ys), nx=_dev(torch, nx),
                        ny=_dev(torch, ny)).cpu().numpy()
    ref = O.integrand_eval(np.array(code), reg + 1, consts, [u], xs, ys, nx, ny)
    assert _close(got, ref, False)


def test_integrand_errors_are_the_references(fb):
    import torch
    from femd_b200.forms import Integrand
    x = _dev(torch, np.zeros(4))
    cases = [([[6, 0, 0, 5]], 2, 0, 1, "Integrand: register out of range"),
             ([[0, 0, 1, 0]], 1, 1, 0, "Integrand: constant out of range"),
             ([[5, 0, 2, 0]], 1, 0, 1, "Integrand: input out of range"),
             ([[8, 0, 0, 3]], 1, 1, 0, "Integrand: pow operands out of range"),
             ([[42, 0, 0, 0]], 1, 0, 0, "Integrand: unknown instruction 42")]
    for code, nreg, nconst, ninput, msg in cases:
        with pytest.raises(ValueError, match=msg):
            Integrand(code, nreg, nconst, ninput).evaluate(4, [x] * ninput, [1.0] * nconst)
    with pytest.raises(ValueError, match="the program reads x or y"):
        Integrand([[1, 0, 0, 0]], 1, 0, 0).evaluate(4, [], [])


def _mesh_case(fb, N=6, k=2, deg=4, free=False):
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, k, bc="free" if free else "dirichlet")
    Q = V.cache(deg)
    return m, V, Q


def test_integrand_at_cell_points(fb):
    """k(x, y) = 1 + 0.5 sin(2 pi x) sin(2 pi y) as a program, at the points of a cell rule:
    against the oracle's program at the oracle's cell points (Cache2D::build_cells)."""
    from femd_b200.forms import Integrand
    m, V, Q = _mesh_case(fb, 7, 2, 5)
    prog = Integrand.varcoef(2 * math.pi)
    got = prog.evaluate_cells(Q, [], [1.0, 0.5, 2 * math.pi]).cpu().numpy()
    x, y, _, _ = O.cache_points(m.points, m.tris, Q.xi, Q.eta, Q.w)
    ref = O.integrand_eval(prog.code, prog.nreg, [1.0, 0.5, 2 * math.pi], [], x, y)
    assert _close(got, ref, False)
    with pytest.raises(ValueError, match="reads the normal on a cell group"):
        Integrand([[3, 0, 1, 0]], 1, 0, 0).evaluate_cells(Q, [], [])


@pytest.mark.parametrize("k", [1, 2, 3])
def test_field_at_cell_points(fb, k):
    """Values and both derivatives of a P_k field at the points of a cell rule."""
    import torch
    from femd_b200.forms import eval_field
    m, V, Q = _mesh_case(fb, 5, k, 2 * k)
    c = np.random.default_rng(k).standard_normal(V.dim)
    vals = eval_field(Q, torch.as_tensor(c).cuda(), [0, 1, 2]).cpu().numpy()
    np_ = m.ncells * Q.nq
    v0 = O.eval_field(Q.ref, V.cell_dofs, c)
    assert np.all(np.abs(vals[:np_] - v0) <= 1e-13 * np.abs(v0) + 1e-15 * np.abs(v0).max())
    # derivatives: J^{-1} of each cell applied to the reference gradients, in numpy
    _, _, _, Ji = O.cache_points(m.points, m.tris, Q.xi, Q.eta, Q.w)
    Ji = Ji.reshape(m.ncells, Q.nq, 4)
    cd = V.cell_dofs
    loc = np.where(cd >= 0, c[np.maximum(cd, 0)], 0.0)
    Rxi, Reta = Q.ref[:, 1, :], Q.ref[:, 2, :]
    dx = (Ji[..., 0:1] * Rxi[None] + Ji[..., 2:3] * Reta[None]) * loc[:, None, :]
    dy = (Ji[..., 1:2] * Rxi[None] + Ji[..., 3:4] * Reta[None]) * loc[:, None, :]
    for i, ref in ((1, dx.sum(-1).reshape(-1)), (2, dy.sum(-1).reshape(-1))):
        got = vals[i * np_:(i + 1) * np_]
        assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref) + 1e-13 * np.abs(ref).max())


def _varcoef_forms(fb, z, meta):
    """The config-3 forms through the compiled-form path: a = k grad.grad with k a program of x
    and y, L = f v with f a field read at the points."""
    import torch
    from femd_b200.forms import Form2D, Integrand
    N, k = int(meta["N"]), int(meta["k"])
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, k, bc="dirichlet")
    kc = Integrand.varcoef()
    a = Form2D.build(V, [(1, 1, (kc, [], [0, 1, 2])), (2, 2, (kc, [], [0, 1, 2]))], fb.quad_degree("varcoef", k),
                     consts=[1.0, 0.5, 2 * math.pi])
    f = torch.as_tensor(z["input_f"]).cuda()
    L = Form2D.build(V, [(0, (Integrand.field(), [0], []))], fb.quad_degree("rhs_field", k), fields=[(f, [0])])
    return V, a, L


@pytest.mark.parametrize("name", ["p2_varcoef_n6", "p2_varcoef_n16"])
def test_compiled_form_assembles_the_references_matrix_and_vector(fb, name):
    """Form2D.assemble: fields at the points, the coefficient program on the device, the cell
    kernels; the symmetric flag set by asymmetry() <= 1e-13 as forms.py:2093-2094 does."""
    z, meta = golden(name)
    V, a, L = _varcoef_forms(fb, z, meta)
    K = a.assemble()
    assert K.symmetric and int(meta["symmetric"]) == 1
    d, d0 = K.data, z["data"]
    assert np.array_equal(K.pattern.indices, z["indices"])
    assert np.all(np.abs(d - d0) <= 1e-12 * np.abs(d0) + 1e-15 * np.abs(d0).max())
    b = L.assemble().cpu().numpy()
    assert np.all(np.abs(b - z["rhs"]) <= 1e-12 * np.abs(z["rhs"]) + 1e-15 * np.abs(z["rhs"]).max())


def test_compiled_form_flags_an_asymmetric_matrix(fb):
    """A convection-like term (test value x trial d/dx) makes the matrix asymmetric: the flag is
    False, and the 'auto' solver refuses it as the GPU path has no LU."""
    from femd_b200.forms import Form2D
    m = fb.rectangle_mesh(0, 0, 1, 1, 6, 6)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    a = Form2D.build(V, [(1, 1, 1.0), (2, 2, 1.0), (0, 1, 3.0)], 2)
    K = a.assemble()
    assert not K.symmetric and K.asymmetry() > 1e-13
    with pytest.raises(ValueError, match="symmetric"):
        K.solver("auto")


@pytest.mark.parametrize("backend", ["auto", "cg", "cuda-cg", "cuda-cg-mixed"])
def test_sparse_solver_backends(fb, backend):
    """A.solver(backend).solve(b) against the reference's FP64 Cholesky solution; .info carries
    the last solve's KrylovInfo; the matrix and preconditioner stay resident between solves."""
    z, meta = golden("p2_varcoef_n16")
    V, a, L = _varcoef_forms(fb, z, meta)
    K = a.assemble()
    S = K.solver(backend)
    assert S.backend == ("cuda-cg" if backend == "auto" else backend) and S.size == K.nrows
    for _ in range(2):
        x = S.solve(L.assemble()).cpu().numpy()
        assert S.info.converged and S.info.residual <= 1e-9
        assert np.linalg.norm(x - z["x_chol"]) <= 1e-8 * np.linalg.norm(z["x_chol"])
    if backend == "cuda-cg":
        assert abs(S.info.iterations - int(meta["cg_iterations"])) <= 0.02 * int(meta["cg_iterations"]) + 2


def test_fd_solve_dispatch(fb):
    """solve(a, L) (fd.solve on a 2D mesh) through the dispatch: assemble, solver, solve."""
    from femd_b200.forms import solve
    z, meta = golden("p2_varcoef_n16")
    V, a, L = _varcoef_forms(fb, z, meta)
    x = solve(a, L, backend="cuda-cg").cpu().numpy()
    assert np.linalg.norm(x - z["x_chol"]) <= 1e-8 * np.linalg.norm(z["x_chol"])
    x = solve(a, L).cpu().numpy()
    assert np.linalg.norm(x - z["x_chol"]) <= 1e-8 * np.linalg.norm(z["x_chol"])
