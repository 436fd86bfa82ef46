"""The synthetic workloads of the benchmark configurations, built through femd_b200.

Every input comes from a seed (numpy's default_rng); no dataset is read.

    poisson_batch(seed, nprob)   many independent Poisson problems: rectangle_mesh(0,0,1,1,N,N),
                                 N uniform in {16, ..., 256}, P_k with k uniform in {1, 2, 3},
                                 a = c grad.grad with c log-uniform in [0.1, 10], the load
                                 vector's dof values N(0, 1)
"""
from __future__ import annotations

import math

import numpy as np

from . import core as fb

PI = math.pi


class SpaceCache:
    """Meshes, spaces, caches and patterns shared by every problem on the same (N, k)."""

    def __init__(self):
        self.spaces = {}

    def get(self, N, k, form="gradgrad"):
        key = (N, k)
        s = self.spaces.get(key)
        if s is None:
            m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
            V = fb.LagrangeSpace2D(m, k, bc="dirichlet")
            s = self.spaces[key] = dict(mesh=m, V=V, P=V.pattern(), Q={})
        q = s["Q"].get(form)
        if q is None:
            q = s["Q"][form] = s["V"].cache(fb.quad_degree(form, k))
        return s, q


def poisson_batch_spec(seed=0, nprob=256, nmin=16, nmax=256):
    rng = np.random.default_rng(seed)
    N = rng.integers(nmin, nmax + 1, nprob)
    k = rng.integers(1, 4, nprob)
    c = np.exp(rng.uniform(np.log(0.1), np.log(10.0), nprob))
    return [dict(N=int(N[i]), k=int(k[i]), c=float(c[i]), seed=int(seed) * 100003 + i) for i in range(nprob)]


def build_poisson(spec, cache: SpaceCache):
    """One problem of the batch: the assembled matrix (with its Jacobi inverse) and the load vector."""
    import torch
    s, Q = cache.get(spec["N"], spec["k"], "gradgrad")
    K = fb.CSRMatrix(s["P"])
    fb.assemble_matrix_2d(Q, Q, [1, 2], [1, 2], [spec["c"], spec["c"]], K)
    b = np.random.default_rng(spec["seed"]).standard_normal(s["V"].dim)
    return K, torch.as_tensor(b).cuda()


def l2_error(V, coeffs, exact, degree=None):
    """sqrt(integral over the mesh of (u_h - exact)^2), u_h = sum_i coeffs_i N_i on the space V
    (constrained nodes 0), by the quadrature rule of the given degree (default 2k + 2) on every
    triangle -- the value of form((w - exact)**2 * dx).assemble() in the reference's examples.
    Host numpy; exact(x, y) takes and returns arrays."""
    coeffs = np.asarray(coeffs.cpu().numpy() if hasattr(coeffs, "cpu") else coeffs, dtype=np.float64)
    Q = V.cache(degree or 2 * V.degree + 2)
    pts, tris = V.mesh.points, V.mesh.tris
    p0, p1, p2 = pts[tris[:, 0]], pts[tris[:, 1]], pts[tris[:, 2]]
    e1, e2 = p1 - p0, p2 - p0
    det = np.abs(e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0])
    xq = p0[:, None, :] + Q.xi[None, :, None] * e1[:, None, :] + Q.eta[None, :, None] * e2[:, None, :]
    cd = V.cell_dofs
    cv = np.where(cd >= 0, coeffs[np.maximum(cd, 0)], 0.0)
    uh = cv @ Q.ref[:, 0, :].T
    err = uh - exact(xq[..., 0], xq[..., 1])
    return float(np.sqrt(np.sum(det[:, None] * Q.w[None, :] * err * err)))


def batch_bytes(sizes, results, mixed=True, compact=False):
    """Algorithmic HBM bytes of one batched PCG solve, from each member's (n, nnz) and its result
    (iterations, reliable_updates).  Per member and iteration: the SpMV's matrix (8 B / nonzero
    in FP32, value + column index -- 6 in the compact layout, value + 16-bit offset; 12 in FP64)
    and vectors (reads of z and the previous direction, stores of the direction and A p; the
    update's loads of r, A p, inv, x or d, p and stores of r, z, x or d: 12 accesses of 4 or 8 B
    per row); per reliable update and at the start an FP64 residual (12 B / nonzero, and b, x,
    inv, r, z: 40 B / row); in mixed mode the FP32 copy of the matrix made at the start (12 B /
    nonzero; 16 with the compact layout's position map)."""
    tot = 0
    per_nnz = 6 if compact else 8
    for (n, nnz), r in zip(sizes, results):
        its, rus = r["iterations"], r.get("reliable_updates", 0)
        if mixed:
            tot += its * (per_nnz * nnz + 48 * n) + (rus + 1) * (12 * nnz + 40 * n) + (16 if compact else 12) * nnz
        else:
            tot += its * (12 * nnz + 96 * n) + 2 * (12 * nnz + 40 * n)
    return tot
