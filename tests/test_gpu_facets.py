"""Boundary terms on the GPU (f2): ds terms on exterior facets against the reference's fixtures
(Cache2D on facets and assemble_*_2d on it: a free space with alpha u v ds in the matrix and
g v ds, g = 1 + x y, in the load), and the Dirichlet lift of fd.solve(a, L, dirichlet=g) against
the oracle's free-space restatement and an exactly representable solution.

Tolerances.  The facet list and markers: bit for bit.  Facet points, weights and normals: within
4 ulp (the edge length is CUDA's hypot, within an ulp or two of the host C library's).  The
facet tabulation: 1e-13 (as the cell tabulation).  Matrix and load values: within 1e-12 relative
(+ 1e-15 of the largest), the assembly tolerance of the cell kernels.  Solutions: within 1e-8 of
the reference's FP64 Cholesky solution.
"""
import math

import numpy as np
import pytest

from conftest import DS_CASES, golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


def _close(a, b, rtol=1e-12):
    return bool(np.all(np.abs(a - b) <= rtol * np.abs(b) + 1e-15 * np.abs(b).max()))


@pytest.mark.parametrize("name", DS_CASES)
def test_facet_terms_match_reference(fb, name):
    import torch
    from femd_b200.forms import Integrand
    from femd_b200.lift import FacetCache2D, assemble_facet_matrix, assemble_facet_vector
    z, meta = golden(name)
    N, k, alpha = int(meta["N"]), int(meta["k"]), float(meta["robin"])
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, k, bc="free")
    Fa = FacetCache2D(V, 2 * k)
    assert np.array_equal(Fa.cell, z["facet_cell"]) and np.array_equal(Fa.local, z["facet_local"])
    assert np.array_equal(Fa.marker, z["facet_marker"])
    assert Fa.nq == int(meta["facet_nq"])
    assert np.all(np.abs(Fa.ref.reshape(-1) - z["facet_ref"]) <= 1e-13)
    x, y, w, nx, ny = [t.cpu().numpy() for t in Fa.points()]
    for got, ref in ((x, z["facet_x"]), (y, z["facet_y"]), (w, z["facet_w"]), (nx, z["facet_nx"]), (ny, z["facet_ny"])):
        assert np.all(np.abs(got - ref) <= 4 * np.spacing(np.abs(ref)) + 1e-300)
    # the matrix: cells (grad.grad) then alpha u v ds
    Q = V.cache(fb.quad_degree("gradgrad", k))
    K = fb.CSRMatrix(V.pattern())
    fb.assemble_matrix_2d(Q, Q, [1, 2], [1, 2], [1.0, 1.0], K, jacobi=False)
    assemble_facet_matrix(Fa, [0], [0], [alpha], K)
    assert np.array_equal(K.pattern.indices, z["indices"])
    assert _close(K.data, z["data"])
    # the load: cells (2 pi^2 sin sin) then g v ds with g = 1 + x y as a program at the facet points
    Qf = V.cache(fb.quad_degree("rhs_data", k))
    b = fb.assemble_vector_2d(Qf, [0], [fb.Coef.sinsin(0.0, 2 * math.pi ** 2, math.pi, math.pi)])
    Fb = FacetCache2D(V, k + 2)
    fx, fy = Fb.points()[:2]
    g = Integrand([[0, 0, 0, 0], [1, 1, 0, 0], [2, 2, 0, 0], [7, 1, 1, 2], [6, 0, 0, 1]], 3, 1, 0)
    gv = g.evaluate(Fb.nent * Fb.nq, [], [1.0], xs=fx, ys=fy)
    assemble_facet_vector(Fb, [0], [fb.Coef.points(gv)], b)
    assert _close(b.cpu().numpy(), z["rhs"])
    M = fb.JacobiPreconditioner(K)
    xs, conv, its, res, brk = fb.cg_solve(K, M, b, None, 100000, 1e-10)
    assert conv
    assert np.linalg.norm(xs.cpu().numpy() - z["x_chol"]) <= 1e-8 * np.linalg.norm(z["x_chol"])


def test_facets_by_marker_and_errors(fb):
    from femd_b200.lift import FacetCache2D, assemble_facet_matrix
    m = fb.rectangle_mesh(0, 0, 1, 1, 4, 4)
    V = fb.LagrangeSpace2D(m, 1, bc="free")
    F = FacetCache2D(V, 2, markers=[2, 4])
    assert F.nent == 8 and set(F.marker.tolist()) == {2, 4}
    K = fb.CSRMatrix(V.pattern())
    with pytest.raises(ValueError, match="derivative code out of range"):
        assemble_facet_matrix(F, [3], [0], [1.0], K)
    V2 = fb.LagrangeSpace2D(m, 1, bc="free")
    K2 = fb.CSRMatrix(V2.pattern())
    with pytest.raises(ValueError, match="not on the facet set's pattern"):
        assemble_facet_matrix(F, [0], [0], [1.0], K2)


def _free_reference(N, k, g):
    """The oracle's lifted load: the free-space (raw-numbered) matrix and load of -Lap u = f with
    f = 2 pi^2 sin sin, L - A_free u_g restricted to the Dirichlet space's dofs."""
    Pd = O.problem("poisson_sin", N, k)
    Pf = O.problem("poisson_sin", N, k, free=True)
    dofs, raw, dim, raw_dim = O.lagrange_numbering(Pd["pts"].shape[0], Pd["tris"], k, True)
    raw_of = np.empty(dim, dtype=np.int64)
    sel = dofs.reshape(-1) >= 0
    raw_of[dofs.reshape(-1)[sel]] = raw.reshape(-1)[sel]
    ug = np.zeros(raw_dim)
    xi, eta = _nodes(k)
    p, t = Pd["pts"], Pd["tris"]
    p0, p1, p2 = p[t[:, 0]], p[t[:, 1]], p[t[:, 2]]
    xy = np.empty((raw_dim, 2))
    xy[raw.reshape(-1)] = (p0[:, None] + xi[None, :, None] * (p1 - p0)[:, None] + eta[None, :, None] * (p2 - p0)[:, None]).reshape(-1, 2)
    cons = np.setdiff1d(np.arange(raw_dim), raw_of)
    ug[cons] = g(xy[cons, 0], xy[cons, 1])
    Af = O.spmv(Pf["indptr"], Pf["indices"], Pf["data"], ug)
    return (Pf["rhs"] - Af)[raw_of], ug, raw_of, xy, Pd


def _nodes(k):
    xi = [0.0, 1.0, 0.0]
    eta = [0.0, 0.0, 1.0]
    for e in range(3):
        for j in range(1, k):
            a = [0, 0, 0]
            a[(e + 1) % 3] = k - j
            a[(e + 2) % 3] = j
            xi.append(a[1] / k)
            eta.append(a[2] / k)
    for j in range(1, k):
        for i in range(1, k - j):
            xi.append(i / k)
            eta.append(j / k)
    return np.array(xi), np.array(eta)


@pytest.mark.parametrize("N,k", [(6, 1), (5, 2), (4, 3)])
def test_dirichlet_lift_matches_oracle(fb, N, k):
    """fd.solve(a, L, dirichlet=g): the lifted load b - a(u_g, v) against the oracle's free-space
    restatement, the solution on the raw numbering u = prolongate(x) + u_g against the oracle's
    Cholesky solve of the same lifted system."""
    from femd_b200.forms import Form2D, Integrand, solve
    from femd_b200.lift import lift, raw_coordinates
    g = lambda x, y: 1.0 + x * y + 0.5 * x * x
    b_ref, ug_ref, raw_of, xy, Pd = _free_reference(N, k, g)
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, k, bc="dirichlet")
    assert np.allclose(raw_coordinates(V), xy, rtol=0, atol=1e-15)
    qa = fb.quad_degree("gradgrad", k)
    a = Form2D.build(V, [(1, 1, 1.0), (2, 2, 1.0)], qa)
    sinsin = Integrand([[0, 0, 0, 0], [1, 1, 0, 0], [2, 2, 0, 0], [7, 1, 0, 1], [9, 1, 1, 0], [7, 2, 0, 2], [9, 2, 2, 0],
                        [0, 3, 1, 0], [7, 1, 3, 1], [7, 0, 1, 2]], 4, 2, 0)
    L = Form2D.build(V, [(0, (sinsin, [], [0, 1]))], fb.quad_degree("rhs_data", k), consts=[math.pi, 2 * math.pi ** 2])
    ug = lift(V, g)
    assert np.array_equal(ug.vector.cpu().numpy(), ug_ref)
    b = L.assemble() - ug.action(a)
    assert _close(b.cpu().numpy(), b_ref, 1e-11)
    u = solve(a, L, backend="cuda-cg", dirichlet=g).cpu().numpy()
    # the oracle: Cholesky-free check through the reference's own matrix (the Dirichlet space's)
    import scipy.sparse as sps
    import scipy.sparse.linalg as spla
    A = sps.csr_matrix((Pd["data"], Pd["indices"], Pd["indptr"]))
    x = spla.spsolve(A.tocsc(), b_ref)
    u_ref = ug_ref.copy()
    u_ref[raw_of] = x
    assert np.linalg.norm(u - u_ref) <= 1e-8 * np.linalg.norm(u_ref)


def test_dirichlet_lift_reproduces_a_quadratic_exactly(fb):
    """u = x^2 + y^2 + x y solves -Lap u = -4 and lies in P2: with its boundary values as the
    Dirichlet data the P2 solution is u at every node (to the solver's tolerance)."""
    from femd_b200.forms import Form2D, solve
    from femd_b200.lift import raw_coordinates
    m = fb.rectangle_mesh(0, 0, 1, 1, 12, 12)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    a = Form2D.build(V, [(1, 1, 1.0), (2, 2, 1.0)], 2)
    L = Form2D.build(V, [(0, -4.0)], 2)
    ue = lambda x, y: x * x + y * y + x * y
    u = solve(a, L, backend="cuda-cg", dirichlet=ue, tol=1e-13).cpu().numpy()
    xy = raw_coordinates(V)
    assert np.max(np.abs(u - ue(xy[:, 0], xy[:, 1]))) <= 1e-10
