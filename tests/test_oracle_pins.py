"""Pins the CPU oracle (oracle/femd_oracle.c) against the reference's own outputs.

The golden fixtures were written by FEMd's header-only C++ compiled from the reference tree
(oracle/ref_driver.cpp via tests/golden/make_golden.py).  Integer work (numbering, pattern,
scatter map) must match bit for bit; the tabulation to rounding; the assembly bit for bit
when the oracle is given the reference's own tabulation; the Jacobi-PCG iterates bit for bit
when given the reference's matrix.
"""
import numpy as np
import pytest

from conftest import DS_CASES, GOLDEN_CASES, INTEGRAND_CASES, PC_CASES, golden

CASES = GOLDEN_CASES + PC_CASES
from oracle import oracle as O

FORM_ARGS = {
    "poisson_sin": ("gradgrad", [1, 2], [1, 2]),
    "poisson_vec": ("gradgrad", [1, 2], [1, 2]),
    "helmholtz_sin": ("helmholtz", [1, 2, 0], [1, 2, 0]),
    "varcoef_field": ("varcoef", [1, 2], [1, 2]),
    "heat": ("mass", [0], [0]),
}


def _problem(z, meta):
    form = str(z["form"])
    N, k = int(meta["N"]), int(meta["k"])
    c = 1.0
    if form == "poisson_vec":
        # c is stored implicitly: recover it from the reference's matrix and the unit-c oracle matrix
        P1 = O.problem(form, N, k, c=1.0, b_vec=z["input_b"])
        c = float(np.round(z["data"][0] / P1["data"][0], 12))
    kw = {}
    if "input_f" in z:
        kw["f_dofs"] = z["input_f"]
    if "input_b" in z:
        kw["b_vec"] = z["input_b"]
    return O.problem(form, N, k, c=c, **kw), form, c


@pytest.mark.parametrize("name", CASES)
def test_integer_work_bit_exact(name):
    z, meta = golden(name)
    P, form, _ = _problem(z, meta)
    assert P["dim"] == int(meta["dim"]) and P["raw_dim"] == int(meta["raw_dim"])
    assert np.array_equal(P["pts"].ravel(), z["points"])
    assert np.array_equal(P["tris"].ravel(), z["tris"])
    assert np.array_equal(P["dofs"].ravel(), z["cell_dofs"])
    assert np.array_equal(P["raw"].ravel(), z["cell_raw_dofs"])
    assert np.array_equal(P["indptr"], z["indptr"])
    assert np.array_equal(P["indices"], z["indices"])
    assert np.array_equal(P["map"], z["scatter_map"])


@pytest.mark.parametrize("name", CASES)
def test_quadrature_and_tabulation(name):
    z, meta = golden(name)
    P, _, _ = _problem(z, meta)
    xi, eta, w = P["quad"]
    assert np.array_equal(xi, z["quad_xi_a"]) and np.array_equal(eta, z["quad_eta_a"]) and np.array_equal(w, z["quad_w_a"])
    ref = z["ref_tab_a"].reshape(P["ref"].shape)
    assert np.abs(P["ref"] - ref).max() <= 1e-13


@pytest.mark.parametrize("name", CASES)
def test_assembly(name):
    z, meta = golden(name)
    P, form, c = _problem(z, meta)
    data = z["data"]
    big = np.abs(data).max()
    # own tabulation: equal to rounding
    assert np.all(np.abs(P["data"] - data) <= 1e-12 * np.abs(data) + 1e-15 * big)
    # the reference's tabulation: the same bits (the operation order is restated exactly)
    ga, a, b = FORM_ARGS[form]
    xi, eta, w = P["quad"]
    ref = z["ref_tab_a"].reshape(P["ref"].shape)
    x, y, ww, Ji = O.cache_points(P["pts"], P["tris"], xi, eta, w)
    coef = O.kcoef(x, y) if form == "varcoef_field" else c * np.ones(ww.size)
    exact = O.assemble_matrix(int(P["indptr"][-1]), ref, ww, Ji, a, b, [coef] * len(a), P["map"])
    assert np.array_equal(exact, data)
    if form == "heat":
        dk = O.assemble_matrix(int(P["indptr"][-1]), ref, ww, Ji, [1, 2], [1, 2], [np.ones(ww.size)] * 2, P["map"])
        assert np.array_equal(dk, z["data_K"])
        return
    rhs = z["rhs"]
    assert np.all(np.abs(P["rhs"] - rhs) <= 1e-12 * np.abs(rhs) + 1e-15 * np.abs(rhs).max())
    assert O.asymmetry(P["indptr"], P["indices"], data) == pytest.approx(float(meta["asymmetry"]), abs=1e-17)


@pytest.mark.parametrize("name", [n for n in CASES if "heat" not in n])
def test_jacobi_and_cg_bit_exact(name):
    z, meta = golden(name)
    ip, ix, data, rhs = z["indptr"], z["indices"], z["data"], z["rhs"]
    inv = O.jacobi_inverse(ip, ix, data)
    assert np.array_equal(inv, z["inv_diag"])
    n = ip.size - 1
    xs = 1.0 + 0.5 * np.sin(1.0 + 0.7 * np.arange(n))
    assert np.array_equal(O.spmv(ip, ix, data, xs), z["spmv_y"])
    x, info = O.cg_jacobi(ip, ix, data, inv, rhs, tol=1e-10)
    assert info["iterations"] == int(meta["cg_iterations"])
    assert info["residual"] == float(meta["cg_residual"])
    assert info["converged"] == bool(int(meta["cg_converged"]))
    assert np.array_equal(x, z["x_cg"])
    # the reference's Cholesky solution is the FP64 solution oracle
    xc = z["x_chol"]
    assert np.linalg.norm(x - xc) / np.linalg.norm(xc) < 1e-8


@pytest.mark.parametrize("name", PC_CASES)
def test_ilu0_ssor_and_preconditioned_cg_bit_exact(name):
    """ILU(0) and SSOR (omega 1, natural ordering) applied to the fixed vector, and CG
    preconditioned by each, against ILU0Preconditioner / SSORPreconditioner and krylov::cg."""
    z, meta = golden(name)
    ip, ix, data, rhs = z["indptr"], z["indices"], z["data"], z["rhs"]
    n = ip.size - 1
    xs = 1.0 + 0.5 * np.sin(1.0 + 0.7 * np.arange(n))
    lu, diag, min_pivot = O.ilu0(ip, ix, data)
    assert min_pivot == float(meta["ilu0_min_pivot"])
    assert np.array_equal(O.ilu0_apply(ip, ix, lu, diag, xs), z["ilu0_apply_y"])
    assert np.array_equal(O.ssor_apply(ip, ix, data, O.diag_positions(ip, ix, data), xs), z["ssor_apply_y"])
    xc = z["x_chol"]
    for kind in ("ilu0", "ssor"):
        x, info = O.cg_pc(ip, ix, data, rhs, kind, tol=1e-10)
        assert info["iterations"] == int(meta[kind + "_iterations"])
        assert info["residual"] == float(meta[kind + "_residual"])
        assert info["converged"] == bool(int(meta[kind + "_converged"]))
        assert np.array_equal(x, z["x_" + kind])
        assert np.linalg.norm(x - xc) / np.linalg.norm(xc) < 1e-8
    # the stronger preconditioners take fewer iterations than Jacobi on these systems
    assert int(meta["ilu0_iterations"]) < int(meta["cg_iterations"])


@pytest.mark.parametrize("name", DS_CASES)
def test_facet_ds_assembly_bit_exact(name):
    """A free space (no Dirichlet elimination) with alpha u v ds added to the stiffness matrix and
    g v ds (g = 1 + x y) to the load over every exterior facet: the facet list, the facet
    quadrature cache and the ds assembly against Cache2D(V, degree, {}, true) and
    assemble_matrix_2d / assemble_vector_2d on it."""
    z, meta = golden(name)
    N, k, alpha = int(meta["N"]), int(meta["k"]), float(meta["robin"])
    nloc = (k + 1) * (k + 2) // 2
    nq = int(meta["facet_nq"])
    fref = z["facet_ref"].reshape(3, nq, 3, nloc)
    P = O.problem("poisson_sin", N, k, free=True, robin=alpha, facet_ref=fref)
    fcell, flocal, fmarker = P["facets"]
    assert np.array_equal(fcell, z["facet_cell"]) and np.array_equal(flocal, z["facet_local"])
    assert np.array_equal(fmarker, z["facet_marker"])
    F = P["facet_cache"]
    for key in ("x", "y", "w", "nx", "ny"):
        assert np.array_equal(F[key], z["facet_" + key]), key
    assert np.allclose(F["ref"], fref, rtol=0, atol=1e-13)
    assert np.array_equal(P["dofs"].ravel(), z["cell_dofs"]) and P["dim"] == int(meta["dim"])
    assert np.array_equal(P["indptr"], z["indptr"]) and np.array_equal(P["indices"], z["indices"])
    # the matrix with the reference's cell and facet tabulations: the same bits
    xi, eta, w = P["quad"]
    x, y, ww, Ji = O.cache_points(P["pts"], P["tris"], xi, eta, w)
    nnz = int(P["indptr"][-1])
    cell = O.assemble_matrix(nnz, z["ref_tab_a"].reshape(P["ref"].shape), ww, Ji, [1, 2], [1, 2], [np.ones(ww.size)] * 2,
                             P["map"])
    fsmap = O.scatter_map(P["dofs"][fcell], P["indptr"], P["indices"])
    data = O.assemble_matrix_v(nnz, fref, flocal, F["w"], F["Ji"], [0], [0], [alpha * np.ones(F["w"].size)], fsmap, into=cell)
    assert np.array_equal(data, z["data"])
    # own tabulation: equal to rounding
    big = np.abs(z["data"]).max()
    assert np.all(np.abs(P["data"] - z["data"]) <= 1e-12 * np.abs(z["data"]) + 1e-15 * big)
    rhs = z["rhs"]
    assert np.all(np.abs(P["rhs"] - rhs) <= 1e-12 * np.abs(rhs) + 1e-15 * np.abs(rhs).max())
    # the Robin problem is SPD: CG on the reference's system gives its iterates, and Cholesky's x
    x_cg, info = O.cg_jacobi(z["indptr"], z["indices"], z["data"], O.jacobi_inverse(z["indptr"], z["indices"], z["data"]),
                             rhs, tol=1e-10)
    assert info["iterations"] == int(meta["cg_iterations"]) and np.array_equal(x_cg, z["x_cg"])
    assert np.linalg.norm(x_cg - z["x_chol"]) <= 1e-8 * np.linalg.norm(z["x_chol"])


@pytest.mark.parametrize("name", INTEGRAND_CASES)
def test_integrand_programs_bit_exact(name):
    """The coefficient evaluator (Integrand::evaluate, real values) on the convection term, a
    variable coefficient and a program with every instruction, 1,000 points each."""
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = {}
    if z["has_xy"]:
        kw.update(xs=z["xs"], ys=z["ys"])
    if z["has_normal"]:
        kw.update(nx=z["nx"], ny=z["ny"])
    out = O.integrand_eval(z["code"], int(z["nreg"]), z["consts"], list(z["inputs"]), **kw)
    assert np.array_equal(out, z["out"])


def test_integrand_rejects_malformed_programs():
    with pytest.raises(ValueError):
        O.integrand_eval([[6, 0, 0, 5]], 2, [], [np.zeros(3)])          # register out of range
    with pytest.raises(ValueError):
        O.integrand_eval([[0, 0, 1, 0]], 1, [1.0], [np.zeros(3)])       # constant out of range
    with pytest.raises(ValueError):
        O.integrand_eval([[42, 0, 0, 0]], 1, [], [np.zeros(3)])         # unknown instruction


def test_known_answers_from_reference_docs():
    # examples/example13.ipynb cells 3/7: P2 on rectangle_mesh(0,0,1,1,20,20): 800 triangles, 1521 unknowns
    pts, tris = O.rectangle_mesh(20)
    _, _, dim, _ = O.lagrange_numbering(pts.shape[0], tris, 2, True)
    assert tris.shape[0] == 800 and dim == 1521
    # docs/manual.md:1279: P2 on the unit square, h = 1/150: 89,401 unknowns
    pts, tris = O.rectangle_mesh(150)
    _, _, dim, _ = O.lagrange_numbering(pts.shape[0], tris, 2, True)
    assert dim == 89401


def test_ddot_ordered_chunks():
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(10001), rng.standard_normal(10001)
    # the chunked 8-lane order of util/omp.hpp:135-192, restated in numpy
    def chunk(a, b):
        s = np.zeros(8)
        m = (a.size // 8) * 8
        for kk in range(8):
            acc = 0.0
            for v in (a[kk:m:8] * b[kk:m:8]):
                acc += v
            s[kk] = acc
        for v in a[m:] * b[m:]:
            s[0] += v
        return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]))
    want = 0.0
    for lo in range(0, x.size, 4096):
        want += chunk(x[lo:lo + 4096], y[lo:lo + 4096])
    assert O.ddot(x, y) == want
