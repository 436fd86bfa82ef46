// assemble.cu -- K3: bilinear-form assembly into CSR values, K4: linear-form assembly into a
// vector, on affine P_k triangles.
//
// Scheme (deterministic, no atomics).  Every matrix position p of row i is owned by one lane of
// the sub-warp that owns row i.  The lane walks the row's (cell, local) list in increasing cell
// order (the pattern's rc lists), finds through the scatter map which element entry (l, j) of
// that cell lands on p, forms that entry and adds it.  Each value is therefore the sum of its
// element contributions in increasing element order, starting from 0 -- the order of the
// reference's row-owner scatter (include/femd/forms/assembly_2d.hpp:265-301) -- and is written
// to HBM exactly once.  The Jacobi inverse diagonal (precond.hpp:82-91) is the epilogue of the
// lane that owns the diagonal position.
//
// Element entries.  Per cell: J = [P1-P0, P2-P0], det J, J^{-1} (lagrange_space_2d.hpp:44-52),
// w_q = rw_q |det J| (cache_2d.hpp:113-114).  Derivative code m of basis l at point q is
// row_m(q,l) = R0 (m = 0), Ji0 Rxi + Ji2 Reta (m = 1), Ji1 Rxi + Ji3 Reta (m = 2)
// (Cache2D::row, cache_2d.hpp:211-226).
//   EXACT: Ke(l,j) = sum_t sum_q [(w_q c_t) row_a(q,l)] row_b(q,j), zero products skipped, in
//          the reference's order with no fused multiply-adds (element_matrix_2d, :102-126).
//   FAST:  constant-coefficient terms are contracted with reference tensors staged in shared
//          memory, S^{rs}(l,j) = sum_q rw_q R_r(q,l) R_s(q,j) (r, s in value, d/dxi, d/deta):
//          Ke(l,j) = |det J| sum_t c_t sum_{rs} A_{a_t r} A_{b_t s} S^{rs}(l,j); point
//          coefficients are contracted point by point.
// Coefficients given as closed forms or as a field are first evaluated at the points into a
// scratch array [e nq + q] (the reference's coefficient arrays, assembler_2d.hpp:393-410).
#include <climits>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace femd {

int build_scatter_map(femd_ctx ctx, femd_pattern p);

static constexpr int MAX_TERMS = 8;
static constexpr int MAX_NLOC = 28;    // P_6
static constexpr int MAX_NQ = 64;

struct TermSpec {
    int nterms;
    int a[MAX_TERMS], b[MAX_TERMS];
    int is_const[MAX_TERMS];
    double cval[MAX_TERMS];
    const double *cpts[MAX_TERMS];
};

struct Geo {
    double J0, J1, J2, J3, det;
};

__device__ __forceinline__ Geo load_geo_exact(const double *__restrict__ pts, const int *__restrict__ tris, int e)
{
    const int v0 = tris[3 * e], v1 = tris[3 * e + 1], v2 = tris[3 * e + 2];
    const double x0 = pts[2 * v0], y0 = pts[2 * v0 + 1];
    Geo g;
    g.J0 = __dsub_rn(pts[2 * v1], x0);
    g.J1 = __dsub_rn(pts[2 * v2], x0);
    g.J2 = __dsub_rn(pts[2 * v1 + 1], y0);
    g.J3 = __dsub_rn(pts[2 * v2 + 1], y0);
    g.det = __dsub_rn(__dmul_rn(g.J0, g.J3), __dmul_rn(g.J1, g.J2));
    return g;
}

// ---- coefficient evaluation at the points -------------------------------------------------
// x = P0.x + J0 xi + J1 eta (lagrange_space_2d.hpp:86-87), no contraction.
__global__ void k_coef_points(const double *__restrict__ pts, const int *__restrict__ tris, int ne, int nq,
                              const double *__restrict__ qxi, const double *__restrict__ qeta, int kind, double p0,
                              double p1, double p2, double p3, const double *__restrict__ field,
                              const int *__restrict__ dofs, int nloc, const double *__restrict__ ref,
                              double *__restrict__ out)
{
    const long long total = (long long)ne * nq;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(t / nq), q = (int)(t % nq);
        double v;
        if (kind == FEMD_COEF_FIELD) {
            // Cache2D::eval_multi, value code (cache_2d.hpp:262-270): s = sum_l R_l loc_l
            const double *R = ref + (size_t)q * 3 * nloc;
            double s = 0.0;
            for (int l = 0; l < nloc; ++l) {
                const int d = dofs[(size_t)e * nloc + l];
                const double c = d >= 0 ? field[d] : 0.0;
                s = __dadd_rn(s, __dmul_rn(R[l], c));
            }
            v = s;
        } else {
            const Geo g = load_geo_exact(pts, tris, e);
            const int v0 = tris[3 * e];
            const double x = __dadd_rn(__dadd_rn(pts[2 * v0], __dmul_rn(g.J0, qxi[q])), __dmul_rn(g.J1, qeta[q]));
            const double y = __dadd_rn(__dadd_rn(pts[2 * v0 + 1], __dmul_rn(g.J2, qxi[q])), __dmul_rn(g.J3, qeta[q]));
            const double s = __dmul_rn(sin(__dmul_rn(p2, x)), sin(__dmul_rn(p3, y)));
            if (kind == FEMD_COEF_SINSIN) v = __dadd_rn(p0, __dmul_rn(p1, s));
            else v = __dadd_rn(__dmul_rn(p1, s), s);   // FEMD_COEF_SINSIN_HELM: p1 s + s
        }
        out[t] = v;
    }
}

// ---- K3 ---------------------------------------------------------------------------------------
// shared memory: ref tabulation [nq][3][nloc], then (FAST) S tensors [9][nloc][nloc]
template <int MODE, int G>
__global__ void __launch_bounds__(256) k_assemble_matrix(
    const double *__restrict__ pts, const int *__restrict__ tris, const int *__restrict__ indptr,
    const int *__restrict__ rc_ptr, const int *__restrict__ rc_code, const int *__restrict__ map,
    const int *__restrict__ diag_pos, int nrows, int nloc, int nq, const double *__restrict__ g_ref,
    const double *__restrict__ g_rw, const double *__restrict__ g_S, TermSpec ts, double *__restrict__ data,
    double *__restrict__ inv, int *__restrict__ status)
{
    extern __shared__ double smem[];
    double *sref = smem;                              // nq * 3 * nloc
    double *srw = sref + nq * 3 * nloc;               // nq
    double *sS = srw + nq;                            // 9 * nloc * nloc (FAST)
    const int nref = nq * 3 * nloc;
    for (int t = threadIdx.x; t < nref; t += blockDim.x) sref[t] = g_ref[t];
    for (int t = threadIdx.x; t < nq; t += blockDim.x) srw[t] = g_rw[t];
    if (MODE == FEMD_ASM_FAST)
        for (int t = threadIdx.x; t < 9 * nloc * nloc; t += blockDim.x) sS[t] = g_S[t];
    __syncthreads();

    const int lane = threadIdx.x % G;
    const int groups_per_block = blockDim.x / G;
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
    for (int i = blockIdx.x * groups_per_block + threadIdx.x / G; i < nrows; i += gridDim.x * groups_per_block) {
        const int rlo = indptr[i], len = indptr[i + 1] - rlo;
        const int clo = rc_ptr[i], chi = rc_ptr[i + 1];
        const int dpos = diag_pos ? diag_pos[i] : -1;
        for (int c0 = 0; c0 < len; c0 += G) {
            const int p = rlo + c0 + lane;
            const bool valid = c0 + lane < len;
            double acc = 0.0;
            for (int c = clo; c < chi; ++c) {
                const int code = rc_code[c];
                const int e = code / nloc, l = code - e * nloc;
                // the map row of (e, l): lane j < nloc holds the position of entry (l, j)
                const int mj = lane < nloc ? map[(size_t)code * nloc + lane] : -2;
                // the three vertices, loaded by lanes 0..2 and shared
                double vx = 0.0, vy = 0.0;
                if (lane < 3) {
                    const int v = tris[3 * e + lane];
                    vx = pts[2 * v];
                    vy = pts[2 * v + 1];
                }
                const int gbase = (threadIdx.x & 31) / G * G;
                const double x0 = __shfl_sync(gmask, vx, gbase + 0), y0 = __shfl_sync(gmask, vy, gbase + 0);
                const double x1 = __shfl_sync(gmask, vx, gbase + 1), y1 = __shfl_sync(gmask, vy, gbase + 1);
                const double x2 = __shfl_sync(gmask, vx, gbase + 2), y2 = __shfl_sync(gmask, vy, gbase + 2);
                int myj = -1;
                for (int j = 0; j < nloc; ++j) {
                    const int pj = __shfl_sync(gmask, mj, gbase + j);
                    if (pj == p) myj = j;
                }
                if (!valid || myj < 0) continue;
                const double J0 = __dsub_rn(x1, x0), J1 = __dsub_rn(x2, x0);
                const double J2 = __dsub_rn(y1, y0), J3 = __dsub_rn(y2, y0);
                const double d = __dsub_rn(__dmul_rn(J0, J3), __dmul_rn(J1, J2));
                const double ad = fabs(d);
                double Ke = 0.0;
                if (MODE == FEMD_ASM_EXACT) {
                    const double Ji0 = __ddiv_rn(J3, d), Ji1 = __ddiv_rn(-J1, d);
                    const double Ji2 = __ddiv_rn(-J2, d), Ji3 = __ddiv_rn(J0, d);
                    for (int t = 0; t < ts.nterms; ++t) {
                        const int ma = ts.a[t], mb = ts.b[t];
                        for (int q = 0; q < nq; ++q) {
                            const double w = __dmul_rn(srw[q], ad);
                            const double ct = ts.is_const[t] ? ts.cval[t] : ts.cpts[t][(size_t)e * nq + q];
                            const double s = __dmul_rn(w, ct);
                            if (s == 0.0) continue;
                            const double *R = sref + q * 3 * nloc;
                            double ra, rb;
                            if (ma == 0) ra = R[l];
                            else {
                                const double aa = ma == 1 ? Ji0 : Ji1, bb = ma == 1 ? Ji2 : Ji3;
                                ra = __dadd_rn(__dmul_rn(aa, R[nloc + l]), __dmul_rn(bb, R[2 * nloc + l]));
                            }
                            const double sa = __dmul_rn(s, ra);
                            if (sa == 0.0) continue;
                            if (mb == 0) rb = R[myj];
                            else {
                                const double aa = mb == 1 ? Ji0 : Ji1, bb = mb == 1 ? Ji2 : Ji3;
                                rb = __dadd_rn(__dmul_rn(aa, R[nloc + myj]), __dmul_rn(bb, R[2 * nloc + myj]));
                            }
                            Ke = __dadd_rn(Ke, __dmul_rn(sa, rb));
                        }
                    }
                    acc = __dadd_rn(acc, Ke);
                } else {
                    const double rd = 1.0 / d;
                    // A[m][r]: code m of the physical row in terms of reference row r (value, xi, eta)
                    const double A[3][3] = {{1.0, 0.0, 0.0}, {0.0, J3 * rd, -J2 * rd}, {0.0, -J1 * rd, J0 * rd}};
                    double G9[9];
#pragma unroll
                    for (int r = 0; r < 9; ++r) G9[r] = 0.0;
                    for (int t = 0; t < ts.nterms; ++t) {
                        const int ma = ts.a[t], mb = ts.b[t];
                        if (ts.is_const[t]) {
                            const double cs = ts.cval[t] * ad;
#pragma unroll
                            for (int r = 0; r < 3; ++r)
#pragma unroll
                                for (int s = 0; s < 3; ++s) G9[3 * r + s] += cs * A[ma][r] * A[mb][s];
                        } else {
                            const double *cp = ts.cpts[t] + (size_t)e * nq;
                            for (int q = 0; q < nq; ++q) {
                                const double *R = sref + q * 3 * nloc;
                                const double ra = A[ma][0] * R[l] + A[ma][1] * R[nloc + l] + A[ma][2] * R[2 * nloc + l];
                                const double rb = A[mb][0] * R[myj] + A[mb][1] * R[nloc + myj] + A[mb][2] * R[2 * nloc + myj];
                                Ke += (srw[q] * ad * cp[q]) * ra * rb;
                            }
                        }
                    }
                    const int lj = l * nloc + myj;
#pragma unroll
                    for (int r = 0; r < 9; ++r)
                        if (G9[r] != 0.0) Ke += G9[r] * sS[r * nloc * nloc + lj];
                    acc += Ke;
                }
            }
            if (valid) {
                data[p] = acc;
                if (inv && p == dpos) {
                    if (acc == 0.0) { atomicOr(status, ST_ZERODIAG); atomicMin(status + 1, i); }
                    inv[i] = 1.0 / acc;
                }
            }
        }
        if (inv && lane == 0 && dpos < 0) { atomicOr(status, ST_ZERODIAG); atomicMin(status + 1, i); }
    }
}

// ---- K4 ---------------------------------------------------------------------------------------
// One thread per row; f_i = sum over the row's cells (increasing order) of fe(l), with
// fe(l) = sum_t sum_q (w_q c_t) row_a(q, l) (assemble_vector_2d, assembly_2d.hpp:188-207).
template <int MODE>
__global__ void __launch_bounds__(256) k_assemble_vector(
    const double *__restrict__ pts, const int *__restrict__ tris, const int *__restrict__ rc_ptr,
    const int *__restrict__ rc_code, int nrows, int nloc, int nq, const double *__restrict__ g_ref,
    const double *__restrict__ g_rw, TermSpec ts, double *__restrict__ f)
{
    extern __shared__ double smem[];
    double *sref = smem;
    double *srw = sref + nq * 3 * nloc;
    for (int t = threadIdx.x; t < nq * 3 * nloc; t += blockDim.x) sref[t] = g_ref[t];
    for (int t = threadIdx.x; t < nq; t += blockDim.x) srw[t] = g_rw[t];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += gridDim.x * blockDim.x) {
        double fi = 0.0;
        for (int c = rc_ptr[i]; c < rc_ptr[i + 1]; ++c) {
            const int code = rc_code[c];
            const int e = code / nloc, l = code - e * nloc;
            const Geo g = load_geo_exact(pts, tris, e);
            const double ad = fabs(g.det);
            double Ji0 = 0.0, Ji1 = 0.0, Ji2 = 0.0, Ji3 = 0.0;
            bool need = false;
            for (int t = 0; t < ts.nterms; ++t) need |= ts.a[t] != 0;
            if (need) {
                Ji0 = __ddiv_rn(g.J3, g.det); Ji1 = __ddiv_rn(-g.J1, g.det);
                Ji2 = __ddiv_rn(-g.J2, g.det); Ji3 = __ddiv_rn(g.J0, g.det);
            }
            double fe = 0.0;
            for (int t = 0; t < ts.nterms; ++t) {
                const int ma = ts.a[t];
                for (int q = 0; q < nq; ++q) {
                    const double w = __dmul_rn(srw[q], ad);
                    const double ct = ts.is_const[t] ? ts.cval[t] : ts.cpts[t][(size_t)e * nq + q];
                    const double s = __dmul_rn(w, ct);
                    if (s == 0.0) continue;
                    const double *R = sref + q * 3 * nloc;
                    double r;
                    if (ma == 0) r = R[l];
                    else {
                        const double aa = ma == 1 ? Ji0 : Ji1, bb = ma == 1 ? Ji2 : Ji3;
                        r = __dadd_rn(__dmul_rn(aa, R[nloc + l]), __dmul_rn(bb, R[2 * nloc + l]));
                    }
                    fe = __dadd_rn(fe, __dmul_rn(s, r));
                }
            }
            fi = __dadd_rn(fi, fe);
        }
        f[i] = fi;
    }
}

// ---- FAST path: K3a per-element factors, K3b row-owner accumulation ---------------------------
// The physical derivative code m of a basis function is sum_r A[m][r] R_r, r = 0 value,
// 1 d/dxi, 2 d/deta: A[0] = (1, 0, 0), A[1] = (0, Ji0, Ji2), A[2] = (0, Ji1, Ji3).  A matrix
// form is then Ke(l, j) = sum_{(r,s)} [ F_rs S^{rs}(l, j) + sum_q H_{q,rs} R_r(q,l) R_s(q,j) ]
// with, per cell,
//   F_rs    = |det J| sum_{t constant} c_t A[a_t][r] A[b_t][s]          (constant coefficients)
//   H_{q,rs} = rw_q |det J| sum_{t varying} c_t(q) A[a_t][r] A[b_t][s]   (coefficients at points)
// and the reference tensors S^{rs}(l, j) = sum_q rw_q R_r(q,l) R_s(q,j) computed on the host.
// K3a forms F and H once per cell (evaluating closed-form and field coefficients there), K3b
// walks each row's cells in increasing order and adds the entries in shared memory.
static constexpr int MAX_PAIRS = 9;
static constexpr int FAST_BLOCK = 128;

struct FastSpec {
    int nterms;
    int a[MAX_TERMS], b[MAX_TERMS];           // b unused for vectors
    int kind[MAX_TERMS];
    double cval[MAX_TERMS], p[MAX_TERMS][4];
    const double *pts[MAX_TERMS];             // FEMD_COEF_POINTS arrays
    const double *field[MAX_TERMS];           // FEMD_COEF_FIELD vectors
    int npair, pr[MAX_PAIRS], ps[MAX_PAIRS];  // active (r, s) pairs (matrix) / active r (vector: ps unused)
    int psym[MAX_PAIRS];                      // pair k stands for (r, s) and (s, r) of a symmetric form
    int has_const, has_var, nf;               // factors per cell: npair (const) + nq npair (varying)
    int vector;
    // the constant terms folded per pair onto the 15 monomials of degree <= 2 in J^-1 (1, Ji0..3,
    // Ji_a Ji_b with a <= b): F_k = |det J| sum_m cm[k][m] mono_m (filled by fast_spec)
    double cm[MAX_PAIRS][15];
};

__device__ __forceinline__ double amat(int m, int r, double Ji0, double Ji1, double Ji2, double Ji3)
{
    if (m == 0) return r == 0 ? 1.0 : 0.0;
    if (r == 0) return 0.0;
    if (m == 1) return r == 1 ? Ji0 : Ji2;
    return r == 1 ? Ji1 : Ji3;
}

// coefficient of a varying term at point q of cell e (x, y the physical point)
__device__ __forceinline__ double coef_at(const FastSpec &fs, int t, int e, int q, int nq, double x, double y,
                                          const int *__restrict__ dofs, int nloc, const double *__restrict__ ref)
{
    switch (fs.kind[t]) {
    case FEMD_COEF_POINTS: return fs.pts[t][(size_t)e * nq + q];
    case FEMD_COEF_SINSIN: return fs.p[t][0] + fs.p[t][1] * (sin(fs.p[t][2] * x) * sin(fs.p[t][3] * y));
    case FEMD_COEF_SINSIN_HELM: {
        const double s = sin(fs.p[t][2] * x) * sin(fs.p[t][3] * y);
        return fs.p[t][1] * s + s;
    }
    case FEMD_COEF_FIELD: {
        const double *R = ref + (size_t)q * 3 * nloc;
        double s = 0.0;
        for (int l = 0; l < nloc; ++l) {
            const int d = dofs[(size_t)e * nloc + l];
            s += R[l] * (d >= 0 ? fs.field[t][d] : 0.0);
        }
        return s;
    }
    default: return fs.cval[t];
    }
}

// K3a: one thread per cell.  tables: rw[nq], xi[nq], eta[nq], ref[nq][3][nloc].
__global__ void __launch_bounds__(256) k_elem_factors(const double *__restrict__ pts, const int *__restrict__ tris, int ne,
                                                      int nq, int nloc, const int *__restrict__ dofs,
                                                      const double *__restrict__ tables, FastSpec fs,
                                                      double *__restrict__ factors)
{
    const double *rw = tables, *qxi = tables + nq, *qeta = tables + 2 * nq, *ref = tables + 3 * nq;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const int v0 = tris[3 * e], v1 = tris[3 * e + 1], v2 = tris[3 * e + 2];
        const double x0 = pts[2 * v0], y0 = pts[2 * v0 + 1];
        const double J0 = pts[2 * v1] - x0, J1 = pts[2 * v2] - x0, J2 = pts[2 * v1 + 1] - y0, J3 = pts[2 * v2 + 1] - y0;
        const double d = J0 * J3 - J1 * J2, ad = fabs(d), rd = 1.0 / d;
        const double Ji0 = J3 * rd, Ji1 = -J1 * rd, Ji2 = -J2 * rd, Ji3 = J0 * rd;
        double *F = factors + (size_t)e * fs.nf;
        int o = 0;
        if (fs.has_const) {
            // the constant terms as a dot product with the monomials of J^-1 (no per-term branches)
            const double mono[15] = {1.0, Ji0, Ji1, Ji2, Ji3, Ji0 * Ji0, Ji0 * Ji1, Ji0 * Ji2, Ji0 * Ji3,
                                     Ji1 * Ji1, Ji1 * Ji2, Ji1 * Ji3, Ji2 * Ji2, Ji2 * Ji3, Ji3 * Ji3};
            for (int k = 0; k < fs.npair; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int m = 0; m < 15; ++m) acc += fs.cm[k][m] * mono[m];
                F[o++] = ad * acc;
            }
        }
        if (fs.has_var) {
            for (int q = 0; q < nq; ++q) {
                const double x = x0 + J0 * qxi[q] + J1 * qeta[q], y = y0 + J2 * qxi[q] + J3 * qeta[q];
                double c[MAX_TERMS];
                for (int t = 0; t < fs.nterms; ++t)
                    c[t] = fs.kind[t] == FEMD_COEF_CONST ? 0.0 : coef_at(fs, t, e, q, nq, x, y, dofs, nloc, ref);
                const double wq = rw[q] * ad;
                for (int k = 0; k < fs.npair; ++k) {
                    double acc = 0.0;
                    for (int t = 0; t < fs.nterms; ++t) {
                        if (fs.kind[t] == FEMD_COEF_CONST) continue;
                        const double ar = amat(fs.a[t], fs.pr[k], Ji0, Ji1, Ji2, Ji3);
                        const double bs = fs.vector ? 1.0 : amat(fs.b[t], fs.ps[k], Ji0, Ji1, Ji2, Ji3);
                        acc += c[t] * ar * bs;
                    }
                    F[o++] = wq * acc;
                }
            }
        }
    }
}

// K3b: one thread per row, the row's values accumulated in shared memory (acc[k][thread]) in
// increasing cell order, then written out by each warp as one contiguous, coalesced range.
// smem: S[npair][nloc][nloc] (const part), R[nq][3][nloc] (varying part), acc[maxlen][FAST_BLOCK],
// rlo[FAST_BLOCK + 4 per warp].
__global__ void __launch_bounds__(FAST_BLOCK) k_assemble_rows(
    const int *__restrict__ indptr, const int *__restrict__ rc_ptr, const int *__restrict__ rc_code,
    const int *__restrict__ map, const int *__restrict__ diag_pos, int nrows, int nloc, int nq,
    const double *__restrict__ factors, const double *__restrict__ g_S, const double *__restrict__ g_R, FastSpec fs,
    int maxlen, double *__restrict__ data, double *__restrict__ inv, int *__restrict__ status)
{
    extern __shared__ double smem[];
    const int nl2 = nloc * nloc;
    double *sS = smem;                                        // npair * nl2 (const)
    double *sR = sS + (fs.has_const ? fs.npair * nl2 : 0);    // nq * 3 * nloc (varying)
    double *acc = sR + (fs.has_var ? nq * 3 * nloc : 0);      // maxlen * FAST_BLOCK
    int *srlo = reinterpret_cast<int *>(acc + (size_t)maxlen * FAST_BLOCK);   // FAST_BLOCK + 1 per block... per warp 33
    if (fs.has_const)
        for (int t = threadIdx.x; t < fs.npair * nl2; t += blockDim.x) sS[t] = g_S[t];
    if (fs.has_var)
        for (int t = threadIdx.x; t < nq * 3 * nloc; t += blockDim.x) sR[t] = g_R[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *wrlo = srlo + w * 33;
    // the loop bound is uniform per warp: rows are handed out 32 at a time
    for (int i0 = (blockIdx.x * FAST_BLOCK + w * 32); i0 < nrows; i0 += gridDim.x * FAST_BLOCK) {
        const int i = i0 + lane;
        const bool valid = i < nrows;
        const int rlo = valid ? indptr[i] : 0;
        const int len = valid ? indptr[i + 1] - rlo : 0;
        double *a = acc + threadIdx.x;                        // a[k * FAST_BLOCK]
        for (int k = 0; k < len; ++k) a[k * FAST_BLOCK] = 0.0;
        if (valid) {
            for (int c = rc_ptr[i]; c < rc_ptr[i + 1]; ++c) {
                const int code = rc_code[c];
                const int e = code / nloc, l = code - e * nloc;
                const double *F = factors + (size_t)e * fs.nf;
                double Fc[MAX_PAIRS];
                if (fs.has_const)
                    for (int k = 0; k < fs.npair; ++k) Fc[k] = F[k];
                const double *H = F + (fs.has_const ? fs.npair : 0);
                const int *mrow = map + (size_t)code * nloc;
                for (int j = 0; j < nloc; ++j) {
                    const int pos = mrow[j];
                    if (pos < 0) continue;
                    double v = 0.0;
                    if (fs.has_const)
                        for (int k = 0; k < fs.npair; ++k) v += Fc[k] * sS[k * nl2 + l * nloc + j];
                    if (fs.has_var)
                        for (int q = 0; q < nq; ++q) {
                            const double *R = sR + q * 3 * nloc;
                            for (int k = 0; k < fs.npair; ++k)
                                v += H[q * fs.npair + k] * R[fs.pr[k] * nloc + l] * R[fs.ps[k] * nloc + j];
                        }
                    a[(pos - rlo) * FAST_BLOCK] += v;
                }
            }
            if (inv) {
                const int dp = diag_pos[i];
                if (dp < 0) { atomicOr(status, ST_ZERODIAG); atomicMin(status + 1, i); }
                else {
                    const double dv = a[(dp - rlo) * FAST_BLOCK];
                    if (dv == 0.0) { atomicOr(status, ST_ZERODIAG); atomicMin(status + 1, i); }
                    inv[i] = 1.0 / dv;
                }
            }
        }
        // coalesced write-out of the warp's 32 rows: positions [first, last)
        wrlo[lane] = valid ? rlo : (i0 < nrows ? indptr[nrows] : 0);
        if (lane == 31) wrlo[32] = valid ? rlo + len : indptr[nrows];
        __syncwarp();
        const int first = wrlo[0], last = wrlo[32];
        for (int p = first + lane; p < last; p += 32) {
            int lo = 0, hi = 31;          // the row t with wrlo[t] <= p < wrlo[t + 1]
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (wrlo[mid] <= p) lo = mid; else hi = mid - 1;
            }
            data[p] = acc[(size_t)(p - wrlo[lo]) * FAST_BLOCK + w * 32 + lo];
        }
        __syncwarp();
    }
}

// ---- K3d: one thread per row over the pair offsets ----------------------------------------------
// As K3b, with the scatter map replaced by the row-local byte offsets (a quarter of the bytes),
// the next pair's code, offsets and factors loaded while the current pair's entries are formed,
// and the row written back from the shared-memory accumulator. P1 / P2 with up to 4 pair
// factors are held to 64 registers, 8 blocks per SM (no spills; 5 % faster at 1024^2 P2 than 7
// blocks at 72 registers).
template <int NLOC, int NPAIR>
__global__ void __launch_bounds__(FAST_BLOCK, (NLOC <= 6 && NPAIR <= 4) ? 8 : 1) k_assemble_rows_off(
    const int *__restrict__ indptr, const int *__restrict__ rc_ptr, const int *__restrict__ rc_code,
    const unsigned char *__restrict__ pair_off, const int *__restrict__ diag_pos, int nrows, int nq,
    const double *__restrict__ factors, const double *__restrict__ g_S, const double *__restrict__ g_R, FastSpec fs,
    int maxlen, double *__restrict__ data, double *__restrict__ inv, int *__restrict__ status)
{
    extern __shared__ double smem[];
    constexpr int NL2 = NLOC * NLOC;
    constexpr int OFFS = (NLOC + 3) / 4 * 4;
    constexpr int NW = OFFS / 4;                             // 32-bit words of offsets per pair
    double *sS = smem;
    double *sR = sS + (fs.has_const ? NPAIR * NL2 : 0);
    double *acc = sR + (fs.has_var ? nq * 3 * NLOC : 0);
    if (fs.has_const)
        for (int t = threadIdx.x; t < NPAIR * NL2; t += blockDim.x) sS[t] = g_S[t];
    if (fs.has_var)
        for (int t = threadIdx.x; t < nq * 3 * NLOC; t += blockDim.x) sR[t] = g_R[t];
    __syncthreads();
    const int cst = fs.has_const ? NPAIR : 0;
    const unsigned *offw = reinterpret_cast<const unsigned *>(pair_off);
    // per warp: the first position of each of its 32 rows (+ the end), and for every position of
    // the warp's range the lane that owns it -- for the coalesced write-out below
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *wrlo = reinterpret_cast<int *>(acc + (size_t)maxlen * FAST_BLOCK) + w * 33;
    unsigned char *owner = reinterpret_cast<unsigned char *>(reinterpret_cast<int *>(acc + (size_t)maxlen * FAST_BLOCK) +
                                                             (FAST_BLOCK / 32) * 33) + (size_t)w * 32 * maxlen;
    for (int i0 = blockIdx.x * FAST_BLOCK + w * 32; i0 < nrows; i0 += gridDim.x * FAST_BLOCK) {
    const int i = i0 + lane;
    const bool valid = i < nrows;
    const int rlo = valid ? indptr[i] : 0, len = valid ? indptr[i + 1] - rlo : 0;
    // entry k of the lane's row at column (lane + k) mod 32 of the warp's 32: the write-out below
    // reads consecutive entries of one row, which then fall in different banks
    double *a = acc + w * 32;
    auto slot = [&](int k) -> double & { return a[(size_t)k * FAST_BLOCK + ((lane + k) & 31)]; };
    for (int k = 0; k < len; ++k) slot(k) = 0.0;
    if (valid) {
        const int c0 = rc_ptr[i], c1 = rc_ptr[i + 1];
        int code = 0;
        unsigned ow[NW];
        double Fc[NPAIR];
        if (c0 < c1) {
            code = __ldcs(&rc_code[c0]);
#pragma unroll
            for (int ww = 0; ww < NW; ++ww) ow[ww] = __ldcs(&offw[(size_t)c0 * NW + ww]);
            const double *F = factors + (size_t)(code / NLOC) * fs.nf;
#pragma unroll
            for (int k = 0; k < NPAIR; ++k) Fc[k] = fs.has_const ? __ldg(&F[k]) : 0.0;
        }
        for (int c = c0; c < c1; ++c) {
            const int cur = code;
            unsigned oq[NW];
            double Fq[NPAIR];
#pragma unroll
            for (int ww = 0; ww < NW; ++ww) oq[ww] = ow[ww];
#pragma unroll
            for (int k = 0; k < NPAIR; ++k) Fq[k] = Fc[k];
            if (c + 1 < c1) {                                 // the next pair's loads
                code = __ldcs(&rc_code[c + 1]);
#pragma unroll
                for (int ww = 0; ww < NW; ++ww) ow[ww] = __ldcs(&offw[(size_t)(c + 1) * NW + ww]);
                const double *F = factors + (size_t)(code / NLOC) * fs.nf;
#pragma unroll
                for (int k = 0; k < NPAIR; ++k) Fc[k] = fs.has_const ? __ldg(&F[k]) : 0.0;
            }
            const int e = cur / NLOC, l = cur - e * NLOC;
            double v[NLOC];
#pragma unroll
            for (int j = 0; j < NLOC; ++j) {
                double s = 0.0;
                if (fs.has_const) {
#pragma unroll
                    for (int k = 0; k < NPAIR; ++k) s += Fq[k] * sS[k * NL2 + l * NLOC + j];
                }
                v[j] = s;
            }
            if (fs.has_var) {
                const double *H = factors + (size_t)e * fs.nf + cst;
                for (int q = 0; q < nq; ++q) {
                    const double *R = sR + q * 3 * NLOC;
#pragma unroll
                    for (int k = 0; k < NPAIR; ++k) {
                        const double h = H[q * NPAIR + k] * R[fs.pr[k] * NLOC + l];
                        const double *Rs = R + fs.ps[k] * NLOC;
#pragma unroll
                        for (int j = 0; j < NLOC; ++j) v[j] += h * Rs[j];
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NLOC; ++j) {
                const unsigned o = (oq[j >> 2] >> (8 * (j & 3))) & 0xffu;
                if (o != 0xffu) slot((int)o) += v[j];
            }
        }
        if (inv) {
            const int dp = diag_pos[i];
            if (dp < 0) { atomicOr(status, ST_ZERODIAG); atomicMin(status + 1, i); }
            else {
                const double dv = slot(dp - rlo);
                if (dv == 0.0) { atomicOr(status, ST_ZERODIAG); atomicMin(status + 1, i); }
                inv[i] = 1.0 / dv;
            }
        }
    }
    // coalesced write-out: the warp's rows are contiguous in HBM, [wrlo[0], wrlo[32]); each
    // position is written by consecutive lanes (full sectors, no partial-sector merges in L2)
    const int end_all = indptr[min(i0 + 32, nrows)];
    wrlo[lane] = valid ? rlo : end_all;
    if (lane == 31) wrlo[32] = end_all;
    __syncwarp();
    const int first = wrlo[0];
    for (int k = 0; k < len; ++k) owner[rlo - first + k] = (unsigned char)lane;
    __syncwarp();
    for (int p = first + lane; p < wrlo[32]; p += 32) {
        const int t = owner[p - first], k = p - wrlo[t];
        data[p] = acc[(size_t)k * FAST_BLOCK + w * 32 + ((t + k) & 31)];
    }
    __syncwarp();
    }
}


// The pair offsets: for rc index c (row i, cell entry code = cell nloc + l), byte j of
// off[c * OFFS + j] = position of (i, dof(cell, j)) minus indptr[i], 255 where constrained.
// OFFS = nloc rounded up to a multiple of 4, so a pair's offsets load as whole 32-bit words.
__global__ void k_pair_offsets(const int *__restrict__ rc_ptr, const int *__restrict__ rc_code,
                               const int *__restrict__ indptr, const int *__restrict__ map, int nrows, int nloc, int offs,
                               unsigned char *__restrict__ off)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += gridDim.x * blockDim.x) {
        const int rlo = indptr[i];
        for (int c = rc_ptr[i]; c < rc_ptr[i + 1]; ++c) {
            const int code = rc_code[c];
            for (int j = 0; j < offs; ++j) {
                const int m = j < nloc ? map[(size_t)code * nloc + j] : -1;
                off[(size_t)c * offs + j] = m < 0 ? (unsigned char)255 : (unsigned char)(m - rlo);
            }
        }
    }
}

static int build_pair_offsets(femd_ctx ctx, femd_pattern p)
{
    if (p->pair_off.p) return FEMD_OK;
    const int offs = (p->nloc + 3) / 4 * 4;
    const size_t npairs = (size_t)p->ncells * p->nloc;
    FEMD_TRY(p->pair_off.alloc(npairs * offs + 4));
    if (p->nrows)
        k_pair_offsets<<<grid_for((size_t)p->nrows, 256, 1u << 20), 256, 0, counted(ctx->stream)>>>(
            p->rc_ptr.p, p->rc_code.p, p->indptr.p, p->map.p, p->nrows, p->nloc, offs, p->pair_off.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    return FEMD_OK;
}

// K4 FAST: one thread per row, f_i = sum over the row's cells (increasing order) of
// sum_k F_k R_{r_k}(l) (constant) + sum_q sum_k H_{q,k} R_{r_k}(q, l) (varying), where the
// constant part uses the tabulation integrated against the weights (Sv^{r}(l) = sum_q rw_q R_r(q,l)).
__global__ void __launch_bounds__(256) k_assemble_vector_fast(const int *__restrict__ rc_ptr, const int *__restrict__ rc_code,
                                                              int nrows, int nloc, int nq, const double *__restrict__ factors,
                                                              const double *__restrict__ g_Sv, const double *__restrict__ g_R,
                                                              FastSpec fs, double *__restrict__ f)
{
    extern __shared__ double smem[];
    double *sSv = smem;                        // 3 * nloc
    double *sR = sSv + 3 * nloc;               // nq * 3 * nloc
    for (int t = threadIdx.x; t < 3 * nloc; t += blockDim.x) sSv[t] = g_Sv[t];
    for (int t = threadIdx.x; t < nq * 3 * nloc; t += blockDim.x) sR[t] = g_R[t];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += gridDim.x * blockDim.x) {
        double fi = 0.0;
        for (int c = rc_ptr[i]; c < rc_ptr[i + 1]; ++c) {
            const int code = rc_code[c];
            const int e = code / nloc, l = code - e * nloc;
            const double *F = factors + (size_t)e * fs.nf;
            double v = 0.0;
            int o = 0;
            if (fs.has_const)
                for (int k = 0; k < fs.npair; ++k) v += F[o++] * sSv[fs.pr[k] * nloc + l];
            if (fs.has_var)
                for (int q = 0; q < nq; ++q)
                    for (int k = 0; k < fs.npair; ++k) v += F[o++] * sR[(q * 3 + fs.pr[k]) * nloc + l];
            fi += v;
        }
        f[i] = fi;
    }
}

// ---- host side -----------------------------------------------------------------------------
struct RuleDev {
    DevBuf<double> ref, rw, S, xi, eta;
};

// Active (r, s) pairs of a form, and the factor count per cell.
static void fast_spec(int nterms, const int *a, const int *b, const femd_coef *coef, int nq, bool vector, FastSpec &fs)
{
    fs = FastSpec{};
    fs.nterms = nterms;
    fs.vector = vector ? 1 : 0;
    bool act[3][3] = {};
    for (int t = 0; t < nterms; ++t) {
        fs.a[t] = a[t];
        fs.b[t] = b ? b[t] : 0;
        fs.kind[t] = coef[t].kind;
        fs.cval[t] = coef[t].value;
        for (int u = 0; u < 4; ++u) fs.p[t][u] = coef[t].p[u];
        fs.pts[t] = coef[t].points_dev;
        fs.field[t] = coef[t].field_dev;
        if (coef[t].kind == FEMD_COEF_CONST) fs.has_const = 1; else fs.has_var = 1;
        for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) {
                const bool ra = a[t] == 0 ? r == 0 : r != 0;
                const bool sb = vector ? s == 0 : (b[t] == 0 ? s == 0 : s != 0);
                if (ra && sb) act[r][s] = true;
            }
    }
    // a symmetric form with constant coefficients (every term (a, b) has its mirror (b, a) with
    // the same coefficient) has F_rs = F_sr on every cell: (r, s) and (s, r) share one factor
    bool symmetric = !vector && !fs.has_var;
    for (int t = 0; t < nterms && symmetric; ++t) {
        if (a[t] == b[t]) continue;
        bool found = false;
        for (int u = 0; u < nterms && !found; ++u)
            found = a[u] == b[t] && b[u] == a[t] && coef[u].kind == coef[t].kind && coef[u].value == coef[t].value;
        symmetric = found;
    }
    for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) {
            if (!act[r][s]) continue;
            if (symmetric && s < r && act[s][r]) continue;     // merged into (s, r)
            fs.pr[fs.npair] = r;
            fs.ps[fs.npair] = s;
            fs.psym[fs.npair] = symmetric && r != s && act[s][r];
            ++fs.npair;
        }
    // cm: amat(m, r) is 0, 1 or one entry of J^-1 (index 0 / 1 / 2 + entry); a product of two is a
    // monomial: 0 = 1, 1-4 = Ji0..Ji3, then Ji_a Ji_b (a <= b) in row order
    auto aidx = [](int m, int r) {
        if (m == 0) return r == 0 ? 1 : 0;
        if (r == 0) return 0;
        if (m == 1) return r == 1 ? 2 : 4;    // Ji0 : Ji2
        return r == 1 ? 3 : 5;                // Ji1 : Ji3
    };
    auto mono = [](int i, int j) {            // i, j in 1..5 (1 = the constant, 2..5 = Ji0..Ji3)
        if (i > j) std::swap(i, j);
        if (i == 1) return j - 1;             // 1 -> 0, Ji_x -> 1 + x
        const int a = i - 2, b = j - 2;       // Ji_a Ji_b, a <= b
        static const int base[4] = {5, 9, 12, 14};
        return base[a] + (b - a);
    };
    for (int k = 0; k < fs.npair; ++k)
        for (int t = 0; t < nterms; ++t) {
            if (coef[t].kind != FEMD_COEF_CONST) continue;
            const int i = aidx(a[t], fs.pr[k]), j = vector ? 1 : aidx(b[t], fs.ps[k]);
            if (i && j) fs.cm[k][mono(i, j)] += coef[t].value;
        }
    fs.nf = (fs.has_const ? fs.npair : 0) + (fs.has_var ? nq * fs.npair : 0);
}

static int check_common(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, femd_pattern p, int nterms,
                        const int *a, const int *b, const femd_coef *coef, int mode)
{
    FEMD_CHECK_ARG(ctx && mesh && rule && p && a && coef, "assembly: NULL argument");
    FEMD_CHECK_ARG(p->kind == KIND_PATTERN, "assembly: not a pattern handle");
    FEMD_CHECK_ARG(p->cell_dofs.p != nullptr, "assembly: the pattern was not built from cells (cell_pattern)");
    FEMD_CHECK_ARG(mode == FEMD_ASM_FAST || mode == FEMD_ASM_EXACT, "assembly: mode is FEMD_ASM_FAST or FEMD_ASM_EXACT");
    FEMD_CHECK_ARG(nterms >= 1 && nterms <= MAX_TERMS, "assembly: 1..8 terms");
    FEMD_CHECK_ARG(mesh->ncells == p->ncells, "assembly: the mesh and the pattern have different cell counts");
    FEMD_CHECK_ARG(mesh->ncells == 0 || (mesh->points_dev && mesh->tris_dev), "assembly: mesh arrays are NULL");
    FEMD_CHECK_ARG(rule->nloc == p->nloc && rule->nloc <= MAX_NLOC, "assembly: the rule's nloc differs from the pattern's");
    FEMD_CHECK_ARG(rule->nq >= 1 && rule->nq <= MAX_NQ, "assembly: 1..64 quadrature points");
    FEMD_CHECK_ARG(rule->ref_host && rule->w_host && rule->xi_host && rule->eta_host, "assembly: rule arrays are NULL");
    for (int t = 0; t < nterms; ++t) {
        FEMD_CHECK_ARG(a[t] >= 0 && a[t] <= 2, "assembly_2d: derivative code " + std::to_string(a[t]) + " is not in 0..2");
        if (b) FEMD_CHECK_ARG(b[t] >= 0 && b[t] <= 2, "assembly_2d: derivative code " + std::to_string(b[t]) + " is not in 0..2");
        const int k = coef[t].kind;
        FEMD_CHECK_ARG(k >= FEMD_COEF_CONST && k <= FEMD_COEF_FIELD, "assembly: unknown coefficient kind");
        if (k == FEMD_COEF_POINTS) FEMD_CHECK_ARG(coef[t].points_dev, "assembly: coefficient points array is NULL");
        if (k == FEMD_COEF_FIELD) FEMD_CHECK_ARG(coef[t].field_dev, "assembly: coefficient field array is NULL");
    }
    return FEMD_OK;
}

// Upload the rule; in FAST mode also the reference tensors S^{rs}.
static int upload_rule(const femd_rule *rule, bool want_S, RuleDev &R, cudaStream_t s)
{
    const int nq = rule->nq, nl = rule->nloc;
    FEMD_TRY(R.ref.alloc((size_t)nq * 3 * nl));
    FEMD_TRY(R.rw.alloc(nq));
    FEMD_TRY(R.xi.alloc(nq));
    FEMD_TRY(R.eta.alloc(nq));
    FEMD_TRY_CUDA(cudaMemcpyAsync(R.ref.p, rule->ref_host, (size_t)nq * 3 * nl * sizeof(double), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(R.rw.p, rule->w_host, nq * sizeof(double), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(R.xi.p, rule->xi_host, nq * sizeof(double), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(R.eta.p, rule->eta_host, nq * sizeof(double), cudaMemcpyHostToDevice, s));
    if (want_S) {
        std::vector<double> S((size_t)9 * nl * nl, 0.0);
        for (int r = 0; r < 3; ++r)
            for (int sidx = 0; sidx < 3; ++sidx)
                for (int l = 0; l < nl; ++l)
                    for (int j = 0; j < nl; ++j) {
                        double acc = 0.0;
                        for (int q = 0; q < nq; ++q) {
                            const double *Rq = rule->ref_host + (size_t)q * 3 * nl;
                            acc += rule->w_host[q] * Rq[r * nl + l] * Rq[sidx * nl + j];
                        }
                        S[((size_t)(3 * r + sidx) * nl + l) * nl + j] = acc;
                    }
        FEMD_TRY(R.S.alloc(S.size()));
        FEMD_TRY_CUDA(cudaMemcpyAsync(R.S.p, S.data(), S.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // S is a stack vector
    }
    return FEMD_OK;
}

// Evaluate closed-form and field coefficients into scratch arrays; fill the TermSpec.
static int prepare_terms(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, femd_pattern p, int nterms,
                         const int *a, const int *b, const femd_coef *coef, const RuleDev &R, DevBuf<double> &scratch,
                         TermSpec &ts)
{
    ts.nterms = nterms;
    const size_t np = (size_t)mesh->ncells * rule->nq;
    int nscratch = 0;
    int owner[MAX_TERMS];
    for (int t = 0; t < nterms; ++t) {
        owner[t] = -1;
        if (coef[t].kind >= FEMD_COEF_SINSIN) {
            for (int u = 0; u < t; ++u)   // the same coefficient as an earlier term: share its array
                if (coef[u].kind == coef[t].kind && coef[u].field_dev == coef[t].field_dev && coef[u].p[0] == coef[t].p[0] &&
                    coef[u].p[1] == coef[t].p[1] && coef[u].p[2] == coef[t].p[2] && coef[u].p[3] == coef[t].p[3]) {
                    owner[t] = owner[u];
                    break;
                }
            if (owner[t] < 0) owner[t] = nscratch++;
        }
    }
    if (nscratch) FEMD_TRY(scratch.alloc(np * nscratch));
    bool done[MAX_TERMS] = {};
    for (int t = 0; t < nterms; ++t) {
        ts.a[t] = a[t];
        ts.b[t] = b ? b[t] : 0;
        ts.is_const[t] = coef[t].kind == FEMD_COEF_CONST;
        ts.cval[t] = coef[t].value;
        ts.cpts[t] = coef[t].kind == FEMD_COEF_POINTS ? coef[t].points_dev : nullptr;
        if (owner[t] >= 0) {
            double *dst = scratch.p + np * owner[t];
            ts.cpts[t] = dst;
            if (!done[owner[t]] && np) {
                done[owner[t]] = true;
                k_coef_points<<<grid_for(np, 256, 1u << 20), 256, 0, counted(ctx->stream)>>>(
                    mesh->points_dev, mesh->tris_dev, mesh->ncells, rule->nq, R.xi.p, R.eta.p, coef[t].kind, coef[t].p[0],
                    coef[t].p[1], coef[t].p[2], coef[t].p[3], coef[t].field_dev, p->cell_dofs.p, rule->nloc, R.ref.p, dst);
                FEMD_TRY_CUDA(cudaGetLastError());
            }
        }
    }
    return FEMD_OK;
}

static constexpr int FAST_MAX_ROW = 96;   // longest row the shared-memory accumulator holds

// FAST assembly of a matrix (K non-null) or a vector (f non-null).  Tables and factors live in
// the pattern's workspace; no allocation once the workspace has its size.
static int fast_assemble(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, femd_pattern p, int nterms,
                         const int *a, const int *b, const femd_coef *coef, femd_matrix K, int want_inv, double *f)
{
    cudaStream_t s = ctx->stream;
    const bool vector = K == nullptr;
    const int nq = rule->nq, nl = rule->nloc, nl2 = nl * nl, n = p->nrows, ne = p->ncells;
    FastSpec fs;
    fast_spec(nterms, a, b, coef, nq, vector, fs);
    // host tables: [rw | xi | eta | ref (nq 3 nl) | S (npair nl^2) or Sv (3 nl)]
    const size_t nref = (size_t)nq * 3 * nl;
    const size_t nS = vector ? (size_t)3 * nl : (size_t)fs.npair * nl2;
    std::vector<double> tab(3 * (size_t)nq + nref + nS, 0.0);
    for (int q = 0; q < nq; ++q) { tab[q] = rule->w_host[q]; tab[nq + q] = rule->xi_host[q]; tab[2 * nq + q] = rule->eta_host[q]; }
    std::copy(rule->ref_host, rule->ref_host + nref, tab.begin() + 3 * nq);
    double *S = tab.data() + 3 * nq + nref;
    if (vector) {
        for (int r = 0; r < 3; ++r)
            for (int l = 0; l < nl; ++l) {
                double acc = 0.0;
                for (int q = 0; q < nq; ++q) acc += rule->w_host[q] * rule->ref_host[((size_t)q * 3 + r) * nl + l];
                S[r * nl + l] = acc;
            }
    } else {
        for (int k = 0; k < fs.npair; ++k)
            for (int l = 0; l < nl; ++l)
                for (int j = 0; j < nl; ++j) {
                    double acc = 0.0;
                    for (int q = 0; q < nq; ++q) {
                        const double *Rq = rule->ref_host + (size_t)q * 3 * nl;
                        acc += rule->w_host[q] * Rq[fs.pr[k] * nl + l] * Rq[fs.ps[k] * nl + j];
                        if (fs.psym[k]) acc += rule->w_host[q] * Rq[fs.ps[k] * nl + l] * Rq[fs.pr[k] * nl + j];
                    }
                    S[(size_t)k * nl2 + l * nl + j] = acc;
                }
    }
    if (p->ws_factors.n < (size_t)ne * fs.nf + 1) FEMD_TRY(p->ws_factors.alloc((size_t)ne * fs.nf + 1));
    // the slot holding these tables, else the least recently used one, refilled (stream-ordered,
    // so kernels still reading the slot's old tables finish first)
    femd_pattern_s::TableSlot *slot = nullptr;
    for (auto &t : p->tables)
        if (t.host == tab) { slot = &t; break; }
    if (!slot) {
        slot = &p->tables[0];
        for (auto &t : p->tables)
            if (t.used < slot->used) slot = &t;
        slot->host.clear();
        if (slot->dev.n < tab.size()) FEMD_TRY(slot->dev.alloc(tab.size()));
        FEMD_TRY_CUDA(cudaMemcpyAsync(slot->dev.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        slot->host = std::move(tab);
    }
    slot->used = ++p->table_clock;
    const double *d_tab = slot->dev.p;
    const double *d_ref = d_tab + 3 * nq, *d_S = d_ref + nref;
    if (ne)
        k_elem_factors<<<grid_for((size_t)ne, 256, 1u << 22), 256, 0, counted(s)>>>(
            mesh->points_dev, mesh->tris_dev, ne, nq, nl, p->cell_dofs.p, d_tab, fs, p->ws_factors.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    if (vector) {
        const size_t shm = (3 * (size_t)nl + nref) * sizeof(double);
        if (n) {
            cudaFuncSetAttribute(k_assemble_vector_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
            k_assemble_vector_fast<<<grid_for((size_t)n, 256, 1u << 22), 256, shm, counted(s)>>>(
                p->rc_ptr.p, p->rc_code.p, n, nl, nq, p->ws_factors.p, d_S, d_ref, fs, f);
        }
        FEMD_TRY_CUDA(cudaGetLastError());
        return FEMD_OK;
    }
    FEMD_TRY(reset_status(ctx));
    double *inv = nullptr;
    if (want_inv) {
        if (!K->inv.p) FEMD_TRY(K->inv.alloc((size_t)n + 1));
        inv = K->inv.p;
    }
    const int maxlen = std::max(p->max_row_len, 1);
    const size_t shm = ((fs.has_const ? (size_t)fs.npair * nl2 : 0) + (fs.has_var ? nref : 0) + (size_t)maxlen * FAST_BLOCK) *
                           sizeof(double) + (FAST_BLOCK / 32) * 33 * sizeof(int);
    if (n) {
        const unsigned grid = grid_for((size_t)n, FAST_BLOCK, 1u << 22);
        bool done = false;
        const size_t sho = ((fs.has_const ? (size_t)fs.npair * nl2 : 0) + (fs.has_var ? nref : 0) +
                            (size_t)maxlen * FAST_BLOCK) * sizeof(double) +
                           (FAST_BLOCK / 32) * 33 * sizeof(int) + (size_t)FAST_BLOCK * maxlen;
#define FEMD_ROWS_OFF(NL, NP)                                                                                          \
        if (!done && nl == NL && fs.npair == NP && maxlen < 255) {                                                     \
            FEMD_TRY(build_pair_offsets(ctx, p));                                                                      \
            cudaFuncSetAttribute(k_assemble_rows_off<NL, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sho); \
            k_assemble_rows_off<NL, NP><<<grid, FAST_BLOCK, sho, counted(s)>>>(                                        \
                p->indptr.p, p->rc_ptr.p, p->rc_code.p, p->pair_off.p, p->diag_pos.p, n, nq, p->ws_factors.p, d_S,     \
                d_ref, fs, maxlen, K->data.p, inv, ctx->status_dev);                                                   \
            done = true;                                                                                               \
        }
        FEMD_ROWS_OFF(3, 1) FEMD_ROWS_OFF(3, 3) FEMD_ROWS_OFF(3, 4) FEMD_ROWS_OFF(3, 5)
        FEMD_ROWS_OFF(6, 1) FEMD_ROWS_OFF(6, 3) FEMD_ROWS_OFF(6, 4) FEMD_ROWS_OFF(6, 5)
        FEMD_ROWS_OFF(10, 1) FEMD_ROWS_OFF(10, 3) FEMD_ROWS_OFF(10, 4) FEMD_ROWS_OFF(10, 5)
#undef FEMD_ROWS_OFF
        if (!done) {
            cudaFuncSetAttribute(k_assemble_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
            k_assemble_rows<<<grid, FAST_BLOCK, shm, counted(s)>>>(p->indptr.p, p->rc_ptr.p, p->rc_code.p, p->map.p,
                                                                   p->diag_pos.p, n, nl, nq, p->ws_factors.p, d_S, d_ref,
                                                                   fs, maxlen, K->data.p, inv, ctx->status_dev);
        }
    }
    FEMD_TRY_CUDA(cudaGetLastError());
    K->f32_valid = false;
    if (want_inv) {
        int flags = 0, bad = 0;
        FEMD_TRY(read_status(ctx, &flags, &bad));
        if (flags & ST_ZERODIAG) {
            set_error("Jacobi: zero diagonal entry in row " + std::to_string(bad));
            return FEMD_EZERODIAG;
        }
        K->inv_valid = true;
    }
    return FEMD_OK;
}

}  // namespace femd

using namespace femd;

extern "C" {

int femd_cuda_assemble_matrix(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, femd_pattern p, int nterms,
                              const int *a, const int *b, const femd_coef *coef, int mode, femd_matrix K, int want_inv)
{
    clear_error();
    FEMD_TRY(check_common(ctx, mesh, rule, p, nterms, a, b, coef, mode));
    FEMD_CHECK_ARG(b != nullptr, "assemble_matrix_2d: b is NULL");
    FEMD_CHECK_ARG(K && K->kind == KIND_MATRIX && K->pattern == p, "assemble_matrix_2d: K is not a matrix on this pattern");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    FEMD_TRY(build_scatter_map(ctx, p));
    if (mode == FEMD_ASM_FAST && p->max_row_len <= FAST_MAX_ROW)
        return fast_assemble(ctx, mesh, rule, p, nterms, a, b, coef, K, want_inv, nullptr);
    RuleDev R;
    FEMD_TRY(upload_rule(rule, mode == FEMD_ASM_FAST, R, s));
    DevBuf<double> scratch;
    TermSpec ts;
    FEMD_TRY(prepare_terms(ctx, mesh, rule, p, nterms, a, b, coef, R, scratch, ts));
    FEMD_TRY(reset_status(ctx));
    const int nl = rule->nloc, nq = rule->nq;
    size_t shm = ((size_t)nq * 3 * nl + nq + (mode == FEMD_ASM_FAST ? 9 * nl * nl : 0)) * sizeof(double);
    const int n = p->nrows;
    if (n > 0) {
        double *inv = nullptr;
        if (want_inv) {
            if (!K->inv.p) FEMD_TRY(K->inv.alloc((size_t)n));
            inv = K->inv.p;
        }
        const bool wide = p->max_row_len > 16 || nl > 16;
        const int G = wide ? 32 : 16;
        const unsigned grid = grid_for((size_t)n, 256 / G, 1u << 22);
#define FEMD_LAUNCH_ASM(M, GG)                                                                                        \
    do {                                                                                                             \
        cudaFuncSetAttribute(k_assemble_matrix<M, GG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);        \
        k_assemble_matrix<M, GG><<<grid, 256, shm, counted(s)>>>(mesh->points_dev, mesh->tris_dev, p->indptr.p, p->rc_ptr.p,    \
                                                        p->rc_code.p, p->map.p, p->diag_pos.p, n, nl, nq, R.ref.p,      \
                                                        R.rw.p, R.S.p, ts, K->data.p, inv, ctx->status_dev);           \
    } while (0)
        if (mode == FEMD_ASM_EXACT) { if (wide) FEMD_LAUNCH_ASM(FEMD_ASM_EXACT, 32); else FEMD_LAUNCH_ASM(FEMD_ASM_EXACT, 16); }
        else { if (wide) FEMD_LAUNCH_ASM(FEMD_ASM_FAST, 32); else FEMD_LAUNCH_ASM(FEMD_ASM_FAST, 16); }
#undef FEMD_LAUNCH_ASM
        FEMD_TRY_CUDA(cudaGetLastError());
    }
    K->f32_valid = false;
    int flags = 0, bad = 0;
    FEMD_TRY(read_status(ctx, &flags, &bad));   // also keeps R and scratch alive until the kernels finish
    if (want_inv && (flags & ST_ZERODIAG)) {
        set_error("Jacobi: zero diagonal entry in row " + std::to_string(bad));
        return FEMD_EZERODIAG;
    }
    if (want_inv) K->inv_valid = true;
    return FEMD_OK;
}

int femd_cuda_assemble_vector(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, femd_pattern p, int nterms,
                              const int *a, const femd_coef *coef, int mode, double *f_dev)
{
    clear_error();
    FEMD_TRY(check_common(ctx, mesh, rule, p, nterms, a, nullptr, coef, mode));
    FEMD_CHECK_ARG(p->nrows == 0 || f_dev, "assemble_vector_2d: f is NULL");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    if (mode == FEMD_ASM_FAST) return fast_assemble(ctx, mesh, rule, p, nterms, a, nullptr, coef, nullptr, 0, f_dev);
    RuleDev R;
    FEMD_TRY(upload_rule(rule, false, R, s));
    DevBuf<double> scratch;
    TermSpec ts;
    FEMD_TRY(prepare_terms(ctx, mesh, rule, p, nterms, a, nullptr, coef, R, scratch, ts));
    const int nl = rule->nloc, nq = rule->nq, n = p->nrows;
    const size_t shm = ((size_t)nq * 3 * nl + nq) * sizeof(double);
    if (n > 0) {
        if (mode == FEMD_ASM_EXACT) {
            cudaFuncSetAttribute(k_assemble_vector<FEMD_ASM_EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
            k_assemble_vector<FEMD_ASM_EXACT><<<grid_for((size_t)n, 256, 1u << 22), 256, shm, counted(s)>>>(
                mesh->points_dev, mesh->tris_dev, p->rc_ptr.p, p->rc_code.p, n, nl, nq, R.ref.p, R.rw.p, ts, f_dev);
        } else {
            cudaFuncSetAttribute(k_assemble_vector<FEMD_ASM_FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
            k_assemble_vector<FEMD_ASM_FAST><<<grid_for((size_t)n, 256, 1u << 22), 256, shm, counted(s)>>>(
                mesh->points_dev, mesh->tris_dev, p->rc_ptr.p, p->rc_code.p, n, nl, nq, R.ref.p, R.rw.p, ts, f_dev);
        }
        FEMD_TRY_CUDA(cudaGetLastError());
    }
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // R and scratch are released on return
    return FEMD_OK;
}

}  // extern "C"
