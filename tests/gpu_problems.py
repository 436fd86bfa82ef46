"""Shared builders for the GPU parity tests: the synthetic problems of the configurations,
assembled through femd_b200 (the product path), and the same forms' term lists."""
import math

import numpy as np

PI = math.pi

# form -> (quadrature form of a, codes a, codes b, coefficient kind)
FORMS = {
    "poisson_sin": ("gradgrad", [1, 2], [1, 2]),
    "poisson_vec": ("gradgrad", [1, 2], [1, 2]),
    "helmholtz_sin": ("helmholtz", [1, 2, 0], [1, 2, 0]),
    "varcoef_field": ("varcoef", [1, 2], [1, 2]),
    "heat": ("mass", [0], [0]),
}


def matrix_coefs(fb, form, c=1.0):
    if form == "varcoef_field":
        k = fb.Coef.sinsin(1.0, 0.5, 2.0 * PI, 2.0 * PI)
        return [k, k]
    n = len(FORMS[form][1])
    return [fb.Coef.const(c)] * n


def build(fb, form, N, k, c=1.0, f_dofs=None, b_vec=None, exact=False, ref_tables=None):
    """mesh, space, pattern, matrix (assembled, with its Jacobi inverse diagonal) and rhs (device)."""
    import torch
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, k, bc="dirichlet")
    qa, a, b = FORMS[form]
    Q = V.cache(fb.quad_degree(qa, k))
    if ref_tables is not None:
        Q = Q.with_tables(ref_tables)
    P = V.pattern()
    K = fb.CSRMatrix(P)
    fb.assemble_matrix_2d(Q, Q, a, b, matrix_coefs(fb, form, c), K, exact=exact)
    rhs = None
    if form in ("poisson_sin", "helmholtz_sin"):
        Qf = V.cache(fb.quad_degree("rhs_data", k))
        coef = fb.Coef.sinsin(0.0, 2.0 * PI * PI, PI, PI) if form == "poisson_sin" else \
            fb.Coef.helmholtz_sinsin(2.0 * PI * PI, PI, PI)
        rhs = fb.assemble_vector_2d(Qf, [0], [coef], P)
    elif form == "varcoef_field":
        Qf = V.cache(fb.quad_degree("rhs_field", k))
        f = torch.as_tensor(np.asarray(f_dofs, dtype=np.float64)).cuda()
        rhs = fb.assemble_vector_2d(Qf, [0], [fb.Coef.field(f)], P)
    elif form == "poisson_vec":
        rhs = torch.as_tensor(np.asarray(b_vec, dtype=np.float64)).cuda()
    return dict(mesh=m, V=V, Q=Q, P=P, K=K, rhs=rhs)
