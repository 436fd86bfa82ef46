"""K3 / K4 on the GPU against the reference (golden fixtures) and the oracle.

* EXACT mode with the reference's own tabulation: the matrix values are the reference's bits
  for constant coefficients (same operation order, no fused multiply-adds, same element order).
* FAST mode (the default): |a - a_ref| <= 1e-12 |a_ref| + 1e-15 max|a|, the tolerance of the
  north-star parity gate (entries that cancel to ~0 get the absolute floor).
* Vectors: 1e-12 relative with the same floor.
"""
import math

import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden
from gpu_problems import FORMS, build
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL, ATOL_REL = 1e-12, 1e-15


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


def close(a, ref):
    return np.all(np.abs(a - ref) <= RTOL * np.abs(ref) + ATOL_REL * np.abs(ref).max())


def _case(z, meta):
    form = str(z["form"])
    c = 1.0
    if form == "poisson_vec":
        P1 = O.problem(form, int(meta["N"]), int(meta["k"]), c=1.0, b_vec=z["input_b"])
        c = float(np.round(z["data"][0] / P1["data"][0], 12))
    return form, c


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_matrix_fast_within_tolerance(fb, name):
    z, meta = golden(name)
    form, c = _case(z, meta)
    pr = build(fb, form, int(meta["N"]), int(meta["k"]), c=c, f_dofs=z.get("input_f"), b_vec=z.get("input_b"))
    assert close(pr["K"].data, z["data"])
    assert np.array_equal(pr["P"].indices, z["indices"])


@pytest.mark.parametrize("name", [n for n in GOLDEN_CASES if "varcoef" not in n])
def test_matrix_exact_bit_identical(fb, name):
    z, meta = golden(name)
    form, c = _case(z, meta)
    k = int(meta["k"])
    nloc = (k + 1) * (k + 2) // 2
    ref = z["ref_tab_a"].reshape(-1, 3, nloc)
    pr = build(fb, form, int(meta["N"]), k, c=c, f_dofs=z.get("input_f"), b_vec=z.get("input_b"), exact=True,
               ref_tables=ref)
    assert np.array_equal(pr["K"].data, z["data"])
    if form != "heat":
        inv = fb.JacobiPreconditioner(pr["K"]).inverse_diagonal()
        assert np.array_equal(inv, z["inv_diag"])


def test_heat_stiffness_exact(fb):
    z, meta = golden("p2_heat_n4")
    nloc = 6
    ref = z["ref_tab_a"].reshape(-1, 3, nloc)
    m = fb.rectangle_mesh(0, 0, 1, 1, 4, 4)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    Q = V.cache(fb.quad_degree("mass", 2)).with_tables(ref)
    K = fb.CSRMatrix(V.pattern())
    fb.assemble_matrix_2d(Q, Q, [1, 2], [1, 2], [1.0, 1.0], K, exact=True)
    assert np.array_equal(K.data, z["data_K"])


@pytest.mark.parametrize("name", [n for n in GOLDEN_CASES if "heat" not in n and "vec" not in n])
def test_rhs_matches_reference(fb, name):
    z, meta = golden(name)
    form, c = _case(z, meta)
    pr = build(fb, form, int(meta["N"]), int(meta["k"]), c=c, f_dofs=z.get("input_f"))
    assert close(pr["rhs"].cpu().numpy(), z["rhs"])


@pytest.mark.parametrize("form,N,k", [("helmholtz_sin", 40, 2), ("poisson_sin", 25, 3), ("varcoef_field", 33, 2),
                                      ("poisson_sin", 70, 1), ("heat", 31, 2)])
def test_matrix_and_rhs_vs_oracle(fb, form, N, k):
    rng = np.random.default_rng(11)
    dim = (k * N - 1) ** 2
    f = rng.standard_normal(dim)
    P = O.problem(form, N, k, f_dofs=f if form == "varcoef_field" else None)
    pr = build(fb, form, N, k, f_dofs=f)
    assert close(pr["K"].data, P["data"])
    if form != "heat":
        assert close(pr["rhs"].cpu().numpy(), P["rhs"])
        inv = fb.JacobiPreconditioner(pr["K"]).inverse_diagonal()
        assert np.allclose(inv, O.jacobi_inverse(P["indptr"], P["indices"], P["data"]), rtol=1e-12, atol=0)


def test_assembly_deterministic(fb):
    pr = build(fb, "varcoef_field", 120, 2, f_dofs=np.ones((2 * 120 - 1) ** 2))
    d1 = pr["K"].data.copy()
    qa, a, b = FORMS["varcoef_field"]
    from gpu_problems import matrix_coefs
    fb.assemble_matrix_2d(pr["Q"], pr["Q"], a, b, matrix_coefs(fb, "varcoef_field"), pr["K"])
    assert np.array_equal(d1, pr["K"].data)


def test_symmetry_and_combine(fb):
    pr = build(fb, "heat", 20, 2)
    M = pr["K"]
    V, P = pr["V"], pr["P"]
    Qk = V.cache(fb.quad_degree("mass", 2))
    K = fb.CSRMatrix(P)
    fb.assemble_matrix_2d(Qk, Qk, [1, 2], [1, 2], [1.0, 1.0], K)
    assert M.asymmetry() <= 1e-13 and K.asymmetry() <= 1e-13
    ref = O.asymmetry(P.indptr, P.indices, K.data)
    assert K.asymmetry() == ref
    dt = 1e-3
    A = M.combine(K, 1.0, dt)
    assert np.array_equal(A.data, O.combine(1.0, M.data, dt, K.data))
    # example13's problem: 800 triangles, 1521 unknowns (examples/example13.ipynb)
    assert V.mesh.ncells == 800 and V.dim == 1521


def test_asymmetry_detects_nonsymmetric(fb):
    pr = build(fb, "poisson_sin", 6, 2)
    K = pr["K"]
    d = K.data.copy()
    d[5] += 1.0
    K.set_data(d)
    assert K.asymmetry() == pytest.approx(O.asymmetry(pr["P"].indptr, pr["P"].indices, d), rel=0, abs=0)
    assert K.asymmetry() > 1e-3


def test_zero_diagonal_raises(fb):
    pr = build(fb, "poisson_sin", 5, 1)
    K = pr["K"]
    d = K.data.copy()
    ip, ix = pr["P"].to_host()
    row = 3
    pos = ip[row] + np.searchsorted(ix[ip[row]:ip[row + 1]], row)
    d[pos] = 0.0
    K.set_data(d)
    with pytest.raises(ValueError, match="zero diagonal entry in row 3"):
        fb.JacobiPreconditioner(K)
