/*
 * femd_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C, single-threaded restatement of the
 * reference algorithm of FEMd's 2D P_k assembly + Jacobi-PCG path.  Only the tests, the
 * smoke check and bench.py's CPU-baseline leg load it, as the checker.  The library never
 * links, loads or calls it.
 *
 * Every function follows the reference file:line named beside it (paths inside the FEMd
 * tree).  Floating-point work keeps the reference's operation order and is compiled with
 * -ffp-contract=off, so the assembly and CG iterates reproduce the reference's bits when
 * given the same inputs.  The one deliberate difference: the Lagrange basis is tabulated
 * with Silvester's closed-form product formula instead of the reference's Dubiner
 * polynomials times an inverted Vandermonde matrix (simplex_basis.hpp:202-251).  Both give
 * the same polynomials on the same equispaced nodes; the values agree to rounding
 * (~1e-15), which tests/test_oracle_pins.py checks against the reference's own tables.
 *
 * The restatement is pinned against golden vectors produced by the reference itself
 * (oracle/ref_driver.cpp, fixtures in tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------------------
 * Mesh: rectangle_mesh / structured_grid_mesh, "right" diagonal.
 * include/femd/mesh/structured.hpp:338-351 (grid), :260-289 (triangles (a,b,c),(a,c,d)).
 * pts: (N+1)^2 x 2 doubles, tris: 2 N^2 x 3 ints.
 * ------------------------------------------------------------------------------------- */
void or_rectangle_mesh(double x0, double y0, double x1, double y1, int nx, int ny, double *pts, int *tris)
{
    for (int j = 0; j <= ny; ++j)
    {
        double y = j == ny ? y1 : y0 + (y1 - y0) * j / ny;
        for (int i = 0; i <= nx; ++i)
        {
            double x = i == nx ? x1 : x0 + (x1 - x0) * i / nx;
            pts[2 * (j * (nx + 1) + i)] = x;
            pts[2 * (j * (nx + 1) + i) + 1] = y;
        }
    }
    int t = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
        {
            int a = j * (nx + 1) + i, b = a + 1, c = a + nx + 2, d = a + nx + 1;
            tris[3 * t] = a; tris[3 * t + 1] = b; tris[3 * t + 2] = c; ++t;
            tris[3 * t] = a; tris[3 * t + 1] = c; tris[3 * t + 2] = d; ++t;
        }
}

/* ---------------------------------------------------------------------------------------
 * Numbering of a continuous P_k space on triangles with every exterior edge Dirichlet
 * (bc="dirichlet" -> all_exterior).  include/femd/fe/space_2d.hpp:390-412 (global edges in
 * first-encounter order over (cell, local edge), edge i from local vertex (i+1)%3 to
 * (i+2)%3, flip when it runs from the higher vertex), :449-475 (raw dofs), :490-498
 * (fixed nodes of exterior edges), :506-526 (adapted numbering in raw order).  An edge is
 * exterior when no second cell holds it (the neighbour array of a valid mesh).
 * Returns dim; cell_dofs/cell_raw: ne x nloc; *raw_dim_out.  Returns -1 on allocation failure.
 * ------------------------------------------------------------------------------------- */
typedef struct { int64_t key; int val; } or_slot;

static uint64_t or_hash(int64_t k)
{
    uint64_t x = (uint64_t)k;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

int or_lagrange_numbering(int nv, int ne, const int *tris, int k, int all_exterior, int *cell_raw, int *cell_dofs,
                          int *raw_dim_out)
{
    const int nloc = (k + 1) * (k + 2) / 2, de = k - 1, nint = (k - 1) * (k - 2) / 2;
    size_t cap = 1;
    while (cap < (size_t)ne * 4) cap <<= 1;
    or_slot *tab = (or_slot *)malloc(cap * sizeof(or_slot));
    int *cell_edge = (int *)malloc((size_t)ne * 3 * sizeof(int));
    char *flip = (char *)malloc((size_t)ne * 3);
    int *ecount = (int *)calloc((size_t)ne * 3, sizeof(int));
    if (!tab || !cell_edge || !flip || !ecount) { free(tab); free(cell_edge); free(flip); free(ecount); return -1; }
    for (size_t s = 0; s < cap; ++s) tab[s].key = -1;
    int nedges = 0;
    for (int c = 0; c < ne; ++c)
        for (int i = 0; i < 3; ++i)
        {
            int a = tris[3 * c + (i + 1) % 3], b = tris[3 * c + (i + 2) % 3];
            int lo = a < b ? a : b, hi = a < b ? b : a;
            int64_t key = ((int64_t)lo << 32) | (uint32_t)hi;
            size_t s = or_hash(key) & (cap - 1);
            while (tab[s].key != -1 && tab[s].key != key) s = (s + 1) & (cap - 1);
            if (tab[s].key == -1) { tab[s].key = key; tab[s].val = nedges++; }
            cell_edge[3 * c + i] = tab[s].val;
            flip[3 * c + i] = a > b;
            ecount[tab[s].val]++;
        }
    const int voff = nv, raw_dim = voff + nedges * de + ne * nint;
    for (int c = 0; c < ne; ++c)
    {
        int *d = cell_raw + (size_t)c * nloc;
        for (int v = 0; v < 3; ++v) d[v] = tris[3 * c + v];
        for (int i = 0; i < 3; ++i)
        {
            int g = cell_edge[3 * c + i];
            for (int j = 0; j < de; ++j)
            {
                int l = 3 + i * de + j;                               /* simplex_basis.hpp:225 */
                d[l] = voff + g * de + (flip[3 * c + i] ? (de - 1 - j) : j);
            }
        }
        int f0 = 3 + 3 * de;                                          /* simplex_basis.hpp:226 */
        for (int j = 0; j < nint; ++j) d[f0 + j] = voff + nedges * de + c * nint + j;
    }
    char *fixed = (char *)calloc((size_t)raw_dim, 1);
    int *raw2ad = (int *)malloc((size_t)raw_dim * sizeof(int));
    if (!fixed || !raw2ad) { free(tab); free(cell_edge); free(flip); free(ecount); free(fixed); free(raw2ad); return -1; }
    if (all_exterior)
        for (int c = 0; c < ne; ++c)
            for (int i = 0; i < 3; ++i)
            {
                int g = cell_edge[3 * c + i];
                if (ecount[g] != 1) continue;
                fixed[tris[3 * c + (i + 1) % 3]] = 1;
                fixed[tris[3 * c + (i + 2) % 3]] = 1;
                for (int j = 0; j < de; ++j) fixed[voff + g * de + j] = 1;
            }
    int dim = 0;
    for (int r = 0; r < raw_dim; ++r) raw2ad[r] = fixed[r] ? -1 : dim++;
    for (size_t i = 0; i < (size_t)ne * nloc; ++i) cell_dofs[i] = raw2ad[cell_raw[i]];
    *raw_dim_out = raw_dim;
    free(tab); free(cell_edge); free(flip); free(ecount); free(fixed); free(raw2ad);
    return dim;
}

/* ---------------------------------------------------------------------------------------
 * Quadrature.  include/femd/quadrature/triangle.hpp:24-58 and gauss_legendre.hpp:104-207.
 * Writes up to 64 points; returns the count.
 * ------------------------------------------------------------------------------------- */
static void or_gauss_legendre(int n, double *x, double *w)
{
    if (n == 1) { x[0] = 0.0; w[0] = 2.0; return; }
    if (n == 2) { x[0] = -1.0 / sqrt(3.0); x[1] = 1.0 / sqrt(3.0); w[0] = w[1] = 1.0; return; }
    if (n == 3) { x[0] = -sqrt(3.0 / 5.0); x[1] = 0.0; x[2] = sqrt(3.0 / 5.0); w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0; return; }
    if (n == 4)
    {
        double a = sqrt((3.0 + 2.0 * sqrt(6.0 / 5.0)) / 7.0), b = sqrt((3.0 - 2.0 * sqrt(6.0 / 5.0)) / 7.0);
        double wa = (18.0 - sqrt(30.0)) / 36.0, wb = (18.0 + sqrt(30.0)) / 36.0;
        x[0] = -a; x[1] = -b; x[2] = b; x[3] = a; w[0] = wa; w[1] = wb; w[2] = wb; w[3] = wa; return;
    }
    if (n == 5)
    {
        double a = sqrt(5.0 + 2.0 * sqrt(10.0 / 7.0)) / 3.0, b = sqrt(5.0 - 2.0 * sqrt(10.0 / 7.0)) / 3.0;
        double wa = (322.0 - 13.0 * sqrt(70.0)) / 900.0, wb = (322.0 + 13.0 * sqrt(70.0)) / 900.0;
        x[0] = -a; x[1] = -b; x[2] = 0.0; x[3] = b; x[4] = a;
        w[0] = wa; w[1] = wb; w[2] = 128.0 / 225.0; w[3] = wb; w[4] = wa; return;
    }
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < n; ++i)
    {
        double xi = cos(PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it)
        {
            double p0 = 1.0, p1 = xi;
            for (int k = 2; k <= n; ++k) { double p2 = ((2.0 * k - 1.0) * xi * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
            double dp = n * (xi * p1 - p0) / (xi * xi - 1.0);
            double dx = -p1 / dp;
            xi += dx;
            if (fabs(dx) <= 1e-15) break;
        }
        double p0 = 1.0, p1 = xi;
        for (int k = 2; k <= n; ++k) { double p2 = ((2.0 * k - 1.0) * xi * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
        double dp = n * (xi * p1 - p0) / (xi * xi - 1.0);
        x[i] = xi;
        w[i] = 2.0 / ((1.0 - xi * xi) * dp * dp);
    }
}

int or_triangle_quadrature(int degree, double *xi, double *eta, double *w)
{
    int d = degree < 0 ? 0 : degree, m = 0;
#define OR_ADD(a, b, c) do { xi[m] = (a); eta[m] = (b); w[m] = (c); ++m; } while (0)
    if (d <= 1) OR_ADD(1.0 / 3.0, 1.0 / 3.0, 0.5);
    else if (d == 2)
    {
        OR_ADD(1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0);
        OR_ADD(2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0);
        OR_ADD(1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0);
    }
    else if (d <= 5)
    {
        const double s15 = sqrt(15.0);
        OR_ADD(1.0 / 3.0, 1.0 / 3.0, 9.0 / 80.0);
        const double a1 = (6.0 - s15) / 21.0, w1 = (155.0 - s15) / 2400.0;
        const double a2 = (6.0 + s15) / 21.0, w2 = (155.0 + s15) / 2400.0;
        OR_ADD(a1, a1, w1); OR_ADD(1.0 - 2.0 * a1, a1, w1); OR_ADD(a1, 1.0 - 2.0 * a1, w1);
        OR_ADD(a2, a2, w2); OR_ADD(1.0 - 2.0 * a2, a2, w2); OR_ADD(a2, 1.0 - 2.0 * a2, w2);
    }
    else
    {
        const int nu = (d + 2) / 2, nv = (d + 3) / 2;
        if (nu * nv > 64) return -1;
        double gux[32], guw[32], gvx[32], gvw[32];
        or_gauss_legendre(nu, gux, guw);
        or_gauss_legendre(nv, gvx, gvw);
        for (int j = 0; j < nv; ++j)
        {
            const double v = 0.5 * (gvx[j] + 1.0), wv = 0.5 * gvw[j];
            for (int i = 0; i < nu; ++i)
            {
                const double u = 0.5 * (gux[i] + 1.0), wu = 0.5 * guw[i];
                OR_ADD(u * (1.0 - v), v, wu * wv * (1.0 - v));
            }
        }
    }
#undef OR_ADD
    return m;
}

/* ---------------------------------------------------------------------------------------
 * Reference tabulation of the equispaced P_k basis, local order of simplex_basis.hpp:17-18,
 * 254-291 (3 vertices; k-1 nodes per edge e from vertex (e+1)%3 to (e+2)%3; interior
 * lattice j = 1.., i = 1.. with i + j < k).  out[q * 3 nloc + r nloc + l], r = value,
 * d/dxi, d/deta (the layout of Cache2D::ref, cache_2d.hpp:97, 205).  Silvester's formula:
 * phi = prod_m P_{a_m}(lambda_m), P_a(t) = prod_{s<a} (k t - s) / (s + 1).
 * ------------------------------------------------------------------------------------- */
static void or_silvester(int k, int a, double t, double *p, double *dp)
{
    double v = 1.0, d = 0.0;
    for (int s = 0; s < a; ++s)
    {
        const double f = (k * t - s) / (s + 1.0), df = k / (s + 1.0);
        d = d * f + v * df;
        v = v * f;
    }
    *p = v; *dp = d;
}

int or_lagrange_nodes(int k, int *bary)          /* bary: nloc x 3 lattice indices */
{
    int m = 0;
    const int V[3][3] = {{k, 0, 0}, {0, k, 0}, {0, 0, k}};
    for (int v = 0; v < 3; ++v) { bary[3 * m] = V[v][0]; bary[3 * m + 1] = V[v][1]; bary[3 * m + 2] = V[v][2]; ++m; }
    for (int e = 0; e < 3; ++e)
    {
        const int a = (e + 1) % 3, b = (e + 2) % 3;
        for (int j = 1; j < k; ++j)
        {
            int idx[3] = {0, 0, 0};
            idx[a] = k - j; idx[b] = j;
            bary[3 * m] = idx[0]; bary[3 * m + 1] = idx[1]; bary[3 * m + 2] = idx[2]; ++m;
        }
    }
    for (int j = 1; j < k; ++j)
        for (int i = 1; i + j < k; ++i) { bary[3 * m] = k - i - j; bary[3 * m + 1] = i; bary[3 * m + 2] = j; ++m; }
    return m;
}

int or_tabulate(int k, int nq, const double *xi, const double *eta, double *out)
{
    const int nloc = (k + 1) * (k + 2) / 2;
    int bary[3 * 231];
    if (k < 1 || k > 20) return -1;
    or_lagrange_nodes(k, bary);
    for (int q = 0; q < nq; ++q)
    {
        const double lam[3] = {1.0 - xi[q] - eta[q], xi[q], eta[q]};
        double *o = out + (size_t)q * 3 * nloc;
        for (int l = 0; l < nloc; ++l)
        {
            double p[3], dp[3];
            for (int m = 0; m < 3; ++m) or_silvester(k, bary[3 * l + m], lam[m], &p[m], &dp[m]);
            o[l] = p[0] * p[1] * p[2];
            o[nloc + l] = -dp[0] * p[1] * p[2] + p[0] * dp[1] * p[2];
            o[2 * nloc + l] = -dp[0] * p[1] * p[2] + p[0] * p[1] * dp[2];
        }
    }
    return nloc;
}

/* ---------------------------------------------------------------------------------------
 * Geometry per cell and per point.  lagrange_space_2d.hpp:41-52 (J = [P1-P0, P2-P0], det,
 * J^{-1}), :82-89 (x = P0 + J (xi, eta)), cache_2d.hpp:105-119 (w = rw |det|, J^{-1} per
 * point from J).  Per point arrays [e nq + q]; Ji: 4 per point.
 * ------------------------------------------------------------------------------------- */
int or_cache_points(int ne, const double *pts, const int *tris, int nq, const double *rxi, const double *reta,
                    const double *rw, double *x, double *y, double *w, double *Ji)
{
    for (int c = 0; c < ne; ++c)
    {
        const double *P0 = pts + 2 * tris[3 * c], *P1 = pts + 2 * tris[3 * c + 1], *P2 = pts + 2 * tris[3 * c + 2];
        double J[4];
        J[0] = P1[0] - P0[0]; J[1] = P2[0] - P0[0];
        J[2] = P1[1] - P0[1]; J[3] = P2[1] - P0[1];
        const double det = J[0] * J[3] - J[1] * J[2];
        if (!(det > 0.0)) return c + 1;
        for (int q = 0; q < nq; ++q)
        {
            const size_t kq = (size_t)c * nq + q;
            x[kq] = P0[0] + J[0] * rxi[q] + J[1] * reta[q];
            y[kq] = P0[1] + J[2] * rxi[q] + J[3] * reta[q];
            const double d = J[0] * J[3] - J[1] * J[2];
            w[kq] = rw[q] * fabs(d);
            double *Jk = Ji + 4 * kq;
            Jk[0] = J[3] / d; Jk[1] = -J[1] / d;
            Jk[2] = -J[2] / d; Jk[3] = J[0] / d;
        }
    }
    return 0;
}

/* Cache2D::row, cache_2d.hpp:211-226 */
static void or_row(const double *R, const double *Ji, int nloc, int m, double *out)
{
    if (m == 0) { for (int l = 0; l < nloc; ++l) out[l] = R[l]; return; }
    const double a = (m == 1) ? Ji[0] : Ji[1];
    const double b = (m == 1) ? Ji[2] : Ji[3];
    for (int l = 0; l < nloc; ++l) out[l] = a * R[nloc + l] + b * R[2 * nloc + l];
}

/* ---------------------------------------------------------------------------------------
 * SparsityPattern::from_cells, csr.hpp:84-125 (square case, rows = cols = cell dofs).
 * Two calls: or_pattern_rows fills indptr and returns nnz; or_pattern_fill writes indices.
 * ------------------------------------------------------------------------------------- */
static int or_cmp_int(const void *a, const void *b) { int x = *(const int *)a, y = *(const int *)b; return (x > y) - (x < y); }

static int or_row_cols(int i, const int *cnt, const int *cellof, const int *cols, int nc, int *buf)
{
    int m = 0;
    for (int t = cnt[i]; t < cnt[i + 1]; ++t)
    {
        const int c = cellof[t];
        for (int kk = 0; kk < nc; ++kk) { int j = cols[(size_t)c * nc + kk]; if (j >= 0) buf[m++] = j; }
    }
    qsort(buf, (size_t)m, sizeof(int), or_cmp_int);
    int u = 0;
    for (int t = 0; t < m; ++t) if (u == 0 || buf[t] != buf[u - 1]) buf[u++] = buf[t];
    return u;
}

static int or_cells_of_rows(int nrows, int ncells, const int *rows, int nr, int **cnt_out, int **cellof_out)
{
    int *cnt = (int *)calloc((size_t)nrows + 1, sizeof(int));
    if (!cnt) return -1;
    for (int c = 0; c < ncells; ++c)
        for (int kk = 0; kk < nr; ++kk) { int i = rows[(size_t)c * nr + kk]; if (i >= 0) ++cnt[i + 1]; }
    for (int i = 0; i < nrows; ++i) cnt[i + 1] += cnt[i];
    int *cellof = (int *)malloc(((size_t)cnt[nrows] + 1) * sizeof(int));
    int *fill = (int *)malloc(((size_t)nrows + 1) * sizeof(int));
    if (!cellof || !fill) { free(cnt); free(cellof); free(fill); return -1; }
    memcpy(fill, cnt, (size_t)nrows * sizeof(int));
    for (int c = 0; c < ncells; ++c)
        for (int kk = 0; kk < nr; ++kk) { int i = rows[(size_t)c * nr + kk]; if (i >= 0) cellof[fill[i]++] = c; }
    free(fill);
    *cnt_out = cnt; *cellof_out = cellof;
    return 0;
}

long long or_pattern_rows(int nrows, int ncells, const int *rows, int nr, const int *cols, int nc, int *indptr)
{
    int *cnt, *cellof;
    if (or_cells_of_rows(nrows, ncells, rows, nr, &cnt, &cellof)) return -1;
    int maxlen = 0;
    for (int i = 0; i < nrows; ++i) if (cnt[i + 1] - cnt[i] > maxlen) maxlen = cnt[i + 1] - cnt[i];
    int *buf = (int *)malloc(((size_t)maxlen * nc + 1) * sizeof(int));
    if (!buf) { free(cnt); free(cellof); return -1; }
    indptr[0] = 0;
    long long nnz = 0;
    for (int i = 0; i < nrows; ++i) { nnz += or_row_cols(i, cnt, cellof, cols, nc, buf); indptr[i + 1] = (int)nnz; }
    free(buf); free(cnt); free(cellof);
    return nnz;
}

int or_pattern_fill(int nrows, int ncells, const int *rows, int nr, const int *cols, int nc, const int *indptr, int *indices)
{
    int *cnt, *cellof;
    if (or_cells_of_rows(nrows, ncells, rows, nr, &cnt, &cellof)) return -1;
    int maxlen = 0;
    for (int i = 0; i < nrows; ++i) if (cnt[i + 1] - cnt[i] > maxlen) maxlen = cnt[i + 1] - cnt[i];
    int *buf = (int *)malloc(((size_t)maxlen * nc + 1) * sizeof(int));
    if (!buf) { free(cnt); free(cellof); return -1; }
    for (int i = 0; i < nrows; ++i)
    {
        int u = or_row_cols(i, cnt, cellof, cols, nc, buf);
        memcpy(indices + indptr[i], buf, (size_t)u * sizeof(int));
    }
    free(buf); free(cnt); free(cellof);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * scatter_map_2d, assembly_2d.hpp:136-164 (square, offsets 0).  Returns 0, or 1 when an
 * entry lies outside the pattern (the reference throws std::logic_error then).
 * ------------------------------------------------------------------------------------- */
int or_scatter_map(int ne, int nloc, const int *dofs, const int *indptr, const int *indices, int *map)
{
    int outside = 0;
    const size_t bs = (size_t)nloc * nloc;
    for (int e = 0; e < ne; ++e)
    {
        const int *d = dofs + (size_t)e * nloc;
        int *pe = map + (size_t)e * bs;
        for (size_t t = 0; t < bs; ++t) pe[t] = -1;
        for (int i = 0; i < nloc; ++i)
        {
            if (d[i] < 0) continue;
            const int I = d[i], lo0 = indptr[I], hi0 = indptr[I + 1];
            for (int j = 0; j < nloc; ++j)
            {
                if (d[j] < 0) continue;
                int lo = lo0, hi = hi0;                      /* std::lower_bound */
                while (lo < hi) { int mid = lo + (hi - lo) / 2; if (indices[mid] < d[j]) lo = mid + 1; else hi = mid; }
                if (lo == hi0 || indices[lo] != d[j]) { outside = 1; continue; }
                pe[(size_t)i * nloc + j] = lo;
            }
        }
    }
    return outside;
}

/* ---------------------------------------------------------------------------------------
 * assemble_matrix_2d with a scatter map, assembly_2d.hpp:219-305 and the element kernel
 * element_matrix_2d, :102-126: per element Ke = 0; for t, q: s = w c_t; skip s == 0; for i:
 * sa = s RT_a[i]; skip sa == 0; for j: Ke_ij += sa RS_b[j]; then K.data[map] += Ke in
 * element order.  data must hold the values to add to (zeroed by the caller for a fresh K).
 * ref: nq x 3 nloc tabulation; w, Ji: per point (or_cache_points); coef: nterms arrays of
 * ne nq values.
 * ------------------------------------------------------------------------------------- */
int or_assemble_matrix_v(int ne, int nloc, int nq, const double *ref, const int *var, const double *w, const double *Ji,
                         int nterms, const int *a, const int *b, const double *const *coef, const int *map, double *data);

int or_assemble_matrix(int ne, int nloc, int nq, const double *ref, const double *w, const double *Ji, int nterms,
                       const int *a, const int *b, const double *const *coef, const int *map, double *data)
{
    return or_assemble_matrix_v(ne, nloc, nq, ref, NULL, w, Ji, nterms, a, b, coef, map, data);
}

/* the same with a tabulation per entry variant (a facet cache's local edge): entry e reads
 * ref + var[e] nq 3 nloc (var NULL: variant 0 for every entry) */
int or_assemble_matrix_v(int ne, int nloc, int nq, const double *ref, const int *var, const double *w, const double *Ji,
                         int nterms, const int *a, const int *b, const double *const *coef, const int *map, double *data)
{
    double *RT = (double *)malloc((size_t)3 * nq * nloc * sizeof(double));
    double *Ke = (double *)malloc((size_t)nloc * nloc * sizeof(double));
    if (!RT || !Ke) { free(RT); free(Ke); return -1; }
    for (int e = 0; e < ne; ++e)
    {
        for (int m = 0; m < 3; ++m)
            for (int q = 0; q < nq; ++q)
                or_row(ref + ((size_t)(var ? var[e] : 0) * nq + q) * 3 * nloc, Ji + 4 * ((size_t)e * nq + q), nloc, m,
                       RT + ((size_t)m * nq + q) * nloc);
        memset(Ke, 0, (size_t)nloc * nloc * sizeof(double));
        for (int t = 0; t < nterms; ++t)
            for (int q = 0; q < nq; ++q)
            {
                const size_t kq = (size_t)e * nq + q;
                const double s = w[kq] * coef[t][kq];
                if (s == 0.0) continue;
                const double *ra = RT + ((size_t)a[t] * nq + q) * nloc, *rb = RT + ((size_t)b[t] * nq + q) * nloc;
                for (int i = 0; i < nloc; ++i)
                {
                    const double sa = s * ra[i];
                    if (sa == 0.0) continue;
                    for (int j = 0; j < nloc; ++j) Ke[i * nloc + j] += sa * rb[j];
                }
            }
        const int *pe = map + (size_t)e * nloc * nloc;
        for (int t = 0; t < nloc * nloc; ++t) if (pe[t] >= 0) data[pe[t]] += Ke[t];
    }
    free(RT); free(Ke);
    return 0;
}

/* assemble_vector_2d, assembly_2d.hpp:173-211 (one term per call, code a) */
int or_assemble_vector_v(int ne, int nloc, int nq, const double *ref, const int *var, const double *w, const double *Ji, int a,
                         const double *coef, const int *dofs, double *f);

int or_assemble_vector(int ne, int nloc, int nq, const double *ref, const double *w, const double *Ji, int a,
                       const double *coef, const int *dofs, double *f)
{
    return or_assemble_vector_v(ne, nloc, nq, ref, NULL, w, Ji, a, coef, dofs, f);
}

/* the same with a tabulation per entry variant, as or_assemble_matrix_v */
int or_assemble_vector_v(int ne, int nloc, int nq, const double *ref, const int *var, const double *w, const double *Ji, int a,
                         const double *coef, const int *dofs, double *f)
{
    double *r = (double *)malloc((size_t)nloc * sizeof(double)), *fe = (double *)malloc((size_t)nloc * sizeof(double));
    if (!r || !fe) { free(r); free(fe); return -1; }
    for (int e = 0; e < ne; ++e)
    {
        for (int l = 0; l < nloc; ++l) fe[l] = 0.0;
        for (int q = 0; q < nq; ++q)
        {
            const size_t kq = (size_t)e * nq + q;
            const double s = w[kq] * coef[kq];
            if (s == 0.0) continue;
            or_row(ref + ((size_t)(var ? var[e] : 0) * nq + q) * 3 * nloc, Ji + 4 * kq, nloc, a, r);
            for (int l = 0; l < nloc; ++l) fe[l] += s * r[l];
        }
        const int *d = dofs + (size_t)e * nloc;
        for (int l = 0; l < nloc; ++l) if (d[l] >= 0) f[d[l]] += fe[l];
    }
    free(r); free(fe);
    return 0;
}

/* Cache2D::eval_multi, code 0 only (a field's values at the points), cache_2d.hpp:260-270 */
void or_eval_field(int ne, int nloc, int nq, const double *ref, const int *dofs, const double *c, double *out)
{
    double loc[231];
    for (int e = 0; e < ne; ++e)
    {
        const int *d = dofs + (size_t)e * nloc;
        for (int l = 0; l < nloc; ++l) loc[l] = d[l] >= 0 ? c[d[l]] : 0.0;
        for (int q = 0; q < nq; ++q)
        {
            const double *R = ref + (size_t)q * 3 * nloc;
            double s = 0.0;
            for (int l = 0; l < nloc; ++l) s += R[l] * loc[l];
            out[(size_t)e * nq + q] = s;
        }
    }
}

/* ---------------------------------------------------------------------------------------
 * Sparse kernels: CSRMatrix::apply csr.hpp:203-215; JacobiPreconditioner precond.hpp:68-91;
 * asymmetry csr.hpp:632-645 with mirror() :43-59; combine (shared pattern) :315-326.
 * ------------------------------------------------------------------------------------- */
void or_spmv(int n, const int *indptr, const int *indices, const double *v, const double *x, double *y)
{
    for (int i = 0; i < n; ++i)
    {
        double s = 0.0;
        for (int p = indptr[i]; p < indptr[i + 1]; ++p) s += v[p] * x[indices[p]];
        y[i] = s;
    }
}

/* returns -1 on success, else the first row with a zero or missing diagonal */
int or_jacobi_inverse(int n, const int *indptr, const int *indices, const double *v, double *inv)
{
    for (int i = 0; i < n; ++i)
    {
        int lo = indptr[i], hi = indptr[i + 1], e = hi;
        while (lo < hi) { int mid = lo + (hi - lo) / 2; if (indices[mid] < i) lo = mid + 1; else hi = mid; }
        if (lo == e || indices[lo] != i || v[lo] == 0.0) return i;
        inv[i] = 1.0 / v[lo];
    }
    return -1;
}

double or_asymmetry(int n, const int *indptr, const int *indices, const double *v)
{
    double big = 0.0, d = 0.0;
    const int nnz = indptr[n];
    for (int p = 0; p < nnz; ++p) if (fabs(v[p]) > big) big = fabs(v[p]);
    for (int i = 0; i < n; ++i)
        for (int p = indptr[i]; p < indptr[i + 1]; ++p)
        {
            const int j = indices[p];
            int lo = indptr[j], hi = indptr[j + 1], e = hi;
            while (lo < hi) { int mid = lo + (hi - lo) / 2; if (indices[mid] < i) lo = mid + 1; else hi = mid; }
            const double m = (lo != e && indices[lo] == i) ? v[lo] : 0.0;
            const double t = fabs(v[p] - m);
            if (t > d) d = t;
        }
    return big > 0.0 ? d / big : 0.0;
}

void or_combine(long long nnz, double alpha, const double *A, double beta, const double *B, double *C)
{
    for (long long p = 0; p < nnz; ++p) C[p] = alpha * A[p] + beta * B[p];
}

/* ---------------------------------------------------------------------------------------
 * Reductions and Jacobi-PCG.  util/omp.hpp:87 (chunk 4096), :135-192 (dot_chunk: eight
 * interleaved partial sums, combined ((s0+s1)+(s2+s3))+((s4+s5)+(s6+s7)); chunk sums added
 * in order); krylov/cg.hpp:99-171 (fused Jacobi update), :192-208, :222-237 (finish),
 * :296-350 (cg_jacobi).
 * ------------------------------------------------------------------------------------- */
#define OR_CHUNK 4096

static double or_dot_chunk(const double *x, const double *y, size_t lo, size_t hi)
{
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t i = lo;
    for (; i + 8 <= hi; i += 8)
        for (int k = 0; k < 8; ++k) s[k] += x[i + k] * y[i + k];
    for (; i < hi; ++i) s[0] += x[i] * y[i];
    return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

double or_ddot(const double *x, const double *y, size_t n)
{
    if (n <= OR_CHUNK) return or_dot_chunk(x, y, 0, n);
    double s = 0.0;
    for (size_t lo = 0; lo < n; lo += OR_CHUNK) s += or_dot_chunk(x, y, lo, lo + OR_CHUNK < n ? lo + OR_CHUNK : n);
    return s;
}

static void or_update_chunk(double *x, double *r, const double *p, const double *Ap, const double *inv, double alpha,
                            size_t lo, size_t hi, double *rr, double *rz)
{
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0}, q[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t i = lo;
    for (; i + 8 <= hi; i += 8)
        for (int k = 0; k < 8; ++k)
        {
            r[i + k] = r[i + k] - alpha * Ap[i + k];
            x[i + k] = x[i + k] + alpha * p[i + k];
            const double t = r[i + k] * r[i + k];
            s[k] += t;
            q[k] += t * inv[i + k];
        }
    for (; i < hi; ++i)
    {
        r[i] -= alpha * Ap[i];
        x[i] += alpha * p[i];
        const double t = r[i] * r[i];
        s[0] += t;
        q[0] += t * inv[i];
    }
    *rr = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
    *rz = ((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]));
}

static void or_update(double *x, double *r, const double *p, const double *Ap, const double *inv, double alpha, size_t n,
                      double *rr, double *rz)
{
    if (n <= OR_CHUNK) { or_update_chunk(x, r, p, Ap, inv, alpha, 0, n, rr, rz); return; }
    double a = 0.0, b = 0.0;
    for (size_t lo = 0; lo < n; lo += OR_CHUNK)
    {
        double s, q;
        or_update_chunk(x, r, p, Ap, inv, alpha, lo, lo + OR_CHUNK < n ? lo + OR_CHUNK : n, &s, &q);
        a += s; b += q;
    }
    *rr = a; *rz = b;
}

/* result[0] converged, [1] iterations, [2] residual, [3] breakdown.  x: initial guess in,
 * solution out.  Returns 0, or -1 on allocation failure. */
int or_cg_jacobi(int n, const int *indptr, const int *indices, const double *v, const double *inv, const double *b,
                 double *x, int max_iter, double tol, double *result)
{
    const size_t N = (size_t)n;
    int converged = 0, breakdown = 0, it = 0;
    double residual = 0.0;
    const double nb = sqrt(or_ddot(b, b, N));
    if (nb == 0.0)
    {
        for (size_t i = 0; i < N; ++i) x[i] = 0.0;
        result[0] = 1; result[1] = 0; result[2] = 0.0; result[3] = 0;
        return 0;
    }
    double *r = (double *)malloc(N * sizeof(double)), *p = (double *)malloc(N * sizeof(double));
    double *Ap = (double *)malloc(N * sizeof(double));
    if (!r || !p || !Ap) { free(r); free(p); free(Ap); return -1; }
    or_spmv(n, indptr, indices, v, x, Ap);
    for (size_t i = 0; i < N; ++i) r[i] = b[i] - Ap[i];
    double rn = sqrt(or_ddot(r, r, N));
    if (rn <= tol * nb)
    {
        result[0] = 1; result[1] = 0; result[2] = rn / nb; result[3] = 0;
        free(r); free(p); free(Ap);
        return 0;
    }
    for (size_t i = 0; i < N; ++i) p[i] = inv[i] * r[i];
    double rz = or_ddot(r, p, N);
    while (it < max_iter)
    {
        if (!(rz > 0.0)) { breakdown = 1; break; }
        or_spmv(n, indptr, indices, v, p, Ap);
        const double pAp = or_ddot(p, Ap, N);
        if (!(pAp > 0.0)) { breakdown = 1; break; }
        const double alpha = rz / pAp;
        double rr, rz_new;
        or_update(x, r, p, Ap, inv, alpha, N, &rr, &rz_new);
        rn = sqrt(rr);
        ++it;
        if (rn <= tol * nb) break;
        const double beta = rz_new / rz;
        rz = rz_new;
        for (size_t i = 0; i < N; ++i) p[i] = inv[i] * r[i] + beta * p[i];
    }
    or_spmv(n, indptr, indices, v, x, Ap);
    for (size_t i = 0; i < N; ++i) r[i] = b[i] - Ap[i];
    residual = sqrt(or_ddot(r, r, N)) / nb;
    converged = !breakdown && residual <= tol * (1.0 + 1e-6) + 1e-15;
    if (!converged && !breakdown && residual <= 10.0 * tol && it < max_iter) converged = 1;
    result[0] = converged; result[1] = it; result[2] = residual; result[3] = breakdown;
    free(r); free(p); free(Ap);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * ILU(0) and SSOR preconditioned CG (the preconditioners beyond Jacobi, natural ordering).
 * ILU(0): Saad's IKJ variant (Iterative Methods for Sparse Linear Systems, 2nd ed., Alg.
 * 10.4) on the matrix's own pattern in row order, the factorization sparse/precond.hpp:151-183
 * builds (unit lower L below the diagonal, U on and above it, in one array); its solve is the
 * forward then backward substitution of precond.hpp:185-200.  SSOR with relaxation w:
 * M = w/(2-w) (D/w + L) (D/w)^-1 (D/w + U), applied as precond.hpp:116-147 does (forward
 * sweep, diagonal scaling, backward sweep).  The CG loop is the generic preconditioned CG of
 * krylov/cg.hpp:245-293 with the ordered reductions above.  Rows must have sorted columns.
 * ------------------------------------------------------------------------------------- */

/* the diagonal position of every row; -1 on success, else the first row whose diagonal is
 * missing or zero (the reference's diagonal check, precond.hpp:69-79) */
int or_diag_positions(int n, const int *indptr, const int *indices, const double *v, int *diag)
{
    for (int i = 0; i < n; ++i)
    {
        diag[i] = -1;
        for (int p = indptr[i]; p < indptr[i + 1]; ++p)
            if (indices[p] == i) { diag[i] = p; break; }
        if (diag[i] < 0 || v[diag[i]] == 0.0) return i;
    }
    return -1;
}

/* lu: the factors (nnz doubles), diag: diagonal positions.  Returns -1 on success, the row of
 * a missing or zero diagonal, or -(2 + i) for a zero pivot in row i; *min_pivot: the smallest
 * pivot met (negative: the factorization is indefinite). */
int or_ilu0(int n, const int *indptr, const int *indices, const double *v, double *lu, int *diag, double *min_pivot)
{
    const long long nnz = indptr[n];
    for (long long q = 0; q < nnz; ++q) lu[q] = v[q];
    const int bad = or_diag_positions(n, indptr, indices, lu, diag);
    if (bad >= 0) return bad;
    int *where = (int *)malloc((size_t)n * sizeof(int));
    if (!where) return -(2 + n);
    for (int i = 0; i < n; ++i) where[i] = -1;
    double mp = INFINITY;
    for (int i = 0; i < n; ++i)
    {
        for (int p = indptr[i]; p < indptr[i + 1]; ++p) where[indices[p]] = p;
        /* eliminate with every earlier row k this row reaches, in increasing k */
        for (int p = indptr[i]; p < diag[i]; ++p)
        {
            const int k = indices[p];
            lu[p] = lu[p] / lu[diag[k]];
            const double l = lu[p];
            for (int q = diag[k] + 1; q < indptr[k + 1]; ++q)
            {
                const int t = where[indices[q]];
                if (t >= 0) lu[t] = lu[t] - l * lu[q];
            }
        }
        for (int p = indptr[i]; p < indptr[i + 1]; ++p) where[indices[p]] = -1;
        const double d = lu[diag[i]];
        if (d == 0.0) { free(where); return -(2 + i); }
        if (d < mp) mp = d;
    }
    free(where);
    *min_pivot = mp;
    return -1;
}

/* z = (L U)^-1 r */
void or_ilu0_apply(int n, const int *indptr, const int *indices, const double *lu, const int *diag, const double *r, double *z)
{
    for (int i = 0; i < n; ++i)
    {
        double s = r[i];
        for (int p = indptr[i]; p < diag[i]; ++p) s = s - lu[p] * z[indices[p]];
        z[i] = s;
    }
    for (int i = n - 1; i >= 0; --i)
    {
        double s = z[i];
        for (int p = diag[i] + 1; p < indptr[i + 1]; ++p) s = s - lu[p] * z[indices[p]];
        z[i] = s / lu[diag[i]];
    }
}

/* z = M_SSOR(w)^-1 r */
void or_ssor_apply(int n, const int *indptr, const int *indices, const double *v, const int *diag, double w, const double *r,
                   double *z)
{
    for (int i = 0; i < n; ++i)
    {
        double s = r[i];
        for (int p = indptr[i]; p < diag[i]; ++p) s = s - v[p] * z[indices[p]];
        z[i] = s * w / v[diag[i]];
    }
    const double c = (2.0 - w) / w;
    for (int i = 0; i < n; ++i) z[i] = z[i] * (c * v[diag[i]] / w);
    for (int i = n - 1; i >= 0; --i)
    {
        double s = z[i];
        for (int p = diag[i] + 1; p < indptr[i + 1]; ++p) s = s - v[p] * z[indices[p]];
        z[i] = s * w / v[diag[i]];
    }
}

/* x += alpha p, r -= alpha Ap; returns ||r||^2 in ordered chunks of eight lanes */
static double or_update_plain_chunk(double *x, double *r, const double *p, const double *Ap, double alpha, size_t lo, size_t hi)
{
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t i = lo;
    for (; i + 8 <= hi; i += 8)
        for (int k = 0; k < 8; ++k)
        {
            r[i + k] = r[i + k] - alpha * Ap[i + k];
            x[i + k] = x[i + k] + alpha * p[i + k];
            s[k] += r[i + k] * r[i + k];
        }
    for (; i < hi; ++i)
    {
        r[i] -= alpha * Ap[i];
        x[i] += alpha * p[i];
        s[0] += r[i] * r[i];
    }
    return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

static double or_update_plain(double *x, double *r, const double *p, const double *Ap, double alpha, size_t n)
{
    if (n <= OR_CHUNK) return or_update_plain_chunk(x, r, p, Ap, alpha, 0, n);
    double s = 0.0;
    for (size_t lo = 0; lo < n; lo += OR_CHUNK) s += or_update_plain_chunk(x, r, p, Ap, alpha, lo, lo + OR_CHUNK < n ? lo + OR_CHUNK : n);
    return s;
}

/* CG preconditioned by ILU(0) (kind 0: lu, diag from or_ilu0) or SSOR (kind 1: diag, w).
 * result as or_cg_jacobi's.  Returns 0, or -1 on allocation failure. */
int or_cg_pc(int n, const int *indptr, const int *indices, const double *v, int kind, const double *lu, const int *diag,
             double w, const double *b, double *x, int max_iter, double tol, double *result)
{
    const size_t N = (size_t)n;
    int converged = 0, breakdown = 0, it = 0;
    const double nb = sqrt(or_ddot(b, b, N));
    if (nb == 0.0)
    {
        for (size_t i = 0; i < N; ++i) x[i] = 0.0;
        result[0] = 1; result[1] = 0; result[2] = 0.0; result[3] = 0;
        return 0;
    }
    double *r = (double *)malloc(N * sizeof(double)), *z = (double *)malloc(N * sizeof(double));
    double *p = (double *)malloc(N * sizeof(double)), *Ap = (double *)malloc(N * sizeof(double));
    if (!r || !z || !p || !Ap) { free(r); free(z); free(p); free(Ap); return -1; }
#define OR_APPLY(in, out)                                                        \
    do {                                                                         \
        if (kind == 0) or_ilu0_apply(n, indptr, indices, lu, diag, in, out);     \
        else or_ssor_apply(n, indptr, indices, v, diag, w, in, out);             \
    } while (0)
    or_spmv(n, indptr, indices, v, x, Ap);
    for (size_t i = 0; i < N; ++i) r[i] = b[i] - Ap[i];
    double rn = sqrt(or_ddot(r, r, N));
    if (rn <= tol * nb)
    {
        result[0] = 1; result[1] = 0; result[2] = rn / nb; result[3] = 0;
        free(r); free(z); free(p); free(Ap);
        return 0;
    }
    OR_APPLY(r, z);
    for (size_t i = 0; i < N; ++i) p[i] = z[i];
    double rz = or_ddot(r, z, N);
    while (it < max_iter)
    {
        if (!(rz > 0.0)) { breakdown = 1; break; }
        or_spmv(n, indptr, indices, v, p, Ap);
        const double pAp = or_ddot(p, Ap, N);
        if (!(pAp > 0.0)) { breakdown = 1; break; }
        const double alpha = rz / pAp;
        rn = sqrt(or_update_plain(x, r, p, Ap, alpha, N));
        ++it;
        if (rn <= tol * nb) break;
        OR_APPLY(r, z);
        const double rz_new = or_ddot(r, z, N);
        const double beta = rz_new / rz;
        rz = rz_new;
        for (size_t i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
    }
#undef OR_APPLY
    or_spmv(n, indptr, indices, v, x, Ap);
    for (size_t i = 0; i < N; ++i) r[i] = b[i] - Ap[i];
    const double residual = sqrt(or_ddot(r, r, N)) / nb;
    converged = !breakdown && residual <= tol * (1.0 + 1e-6) + 1e-15;
    if (!converged && !breakdown && residual <= 10.0 * tol && it < max_iter) converged = 1;
    result[0] = converged; result[1] = it; result[2] = residual; result[3] = breakdown;
    free(r); free(z); free(p); free(Ap);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * The coefficient evaluator, real values (Integrand, forms/integrand.hpp:33-45 instruction
 * set, :47-66 checks, :300-342 run): a program of 4-integer instructions (op, out, a, b) over
 * registers of one value per point; the result is the last instruction's register.  Each
 * point is independent, so this evaluates point by point with nreg doubles of scratch.
 * ------------------------------------------------------------------------------------- */
enum { OR_CONST, OR_X, OR_Y, OR_NX, OR_NY, OR_INPUT, OR_ADD, OR_MUL, OR_POW, OR_SIN, OR_COS, OR_EXP, OR_LOG, OR_TANH,
       OR_SQRT, OR_SINH, OR_COSH, OR_SECH, OR_ABS, OR_SIGN };

/* 0 when the program is well formed, else a code: 1 bad length, 2 no register, 3 register,
 * 4 constant, 5 input, 6 pow operands, 7 unknown instruction */
int or_integrand_check(const int *code, int ncode, int nreg, int nconst, int ninput)
{
    if (ncode % 4 != 0) return 1;
    if (nreg < 1) return 2;
    for (int k = 0; k < ncode; k += 4)
    {
        const int op = code[k], out = code[k + 1], a = code[k + 2], b = code[k + 3];
        if (out < 0 || out >= nreg) return 3;
        if (op == OR_CONST && (a < 0 || a >= nconst)) return 4;
        if (op == OR_INPUT && (a < 0 || a >= ninput)) return 5;
        if ((op == OR_ADD || op == OR_MUL) && (a < 0 || a >= nreg || b < 0 || b >= nreg)) return 3;
        if (op == OR_POW && (a < 0 || a >= nreg || b < 0 || b >= nconst)) return 6;
        if (op >= OR_SIN && op <= OR_SIGN && (a < 0 || a >= nreg)) return 3;
        if (op < 0 || op > OR_SIGN) return 7;
    }
    return 0;
}

/* sech z = 2 e / (1 + e^2) with e = exp(-|z|), which neither overflows nor loses the tail */
static double or_sech(double z)
{
    const double e = exp(-fabs(z));
    return 2.0 * e / (1.0 + e * e);
}

/* out[q] for npts points; inputs: ninput arrays of npts values (an array of pointers).
 * Returns the check's code (nothing is written unless it is 0), or -1 on allocation failure. */
int or_integrand_eval(const int *code, int ncode, int nreg, const double *consts, int nconst, const double *const *inputs,
                      int ninput, const double *xs, const double *ys, const double *nx, const double *ny, long long npts,
                      double *out)
{
    const int bad = or_integrand_check(code, ncode, nreg, nconst, ninput);
    if (bad) return bad;
    if (ncode == 0) return 1;
    double *r = (double *)calloc((size_t)nreg, sizeof(double));   /* registers start at 0, as the reference's do */
    if (!r) return -1;
    const int result = code[ncode - 4 + 1];
    for (long long q = 0; q < npts; ++q)
    {
        for (int k = 0; k < ncode; k += 4)
        {
            const int op = code[k], o = code[k + 1], a = code[k + 2], b = code[k + 3];
            double v = 0.0;
            switch (op)
            {
            case OR_CONST: v = consts[a]; break;
            case OR_X: v = xs[q]; break;
            case OR_Y: v = ys[q]; break;
            case OR_NX: v = (a < 0 ? -1.0 : 1.0) * nx[q]; break;
            case OR_NY: v = (a < 0 ? -1.0 : 1.0) * ny[q]; break;
            case OR_INPUT: v = inputs[a][q]; break;
            case OR_ADD: v = r[a] + r[b]; break;
            case OR_MUL: v = r[a] * r[b]; break;
            case OR_POW:
            {
                /* squares, reciprocals and square roots are exact operations, not pow */
                const double n = consts[b];
                if (n == 2.0) v = r[a] * r[a];
                else if (n == -1.0) v = 1.0 / r[a];
                else if (n == 0.5) v = sqrt(r[a]);
                else v = pow(r[a], n);
                break;
            }
            case OR_SIN: v = sin(r[a]); break;
            case OR_COS: v = cos(r[a]); break;
            case OR_EXP: v = exp(r[a]); break;
            case OR_LOG: v = log(r[a]); break;
            case OR_TANH: v = tanh(r[a]); break;
            case OR_SQRT: v = sqrt(r[a]); break;
            case OR_SINH: v = sinh(r[a]); break;
            case OR_COSH: v = cosh(r[a]); break;
            case OR_SECH: v = or_sech(r[a]); break;
            case OR_ABS: v = fabs(r[a]); break;
            case OR_SIGN: v = r[a] > 0.0 ? 1.0 : (r[a] < 0.0 ? -1.0 : 0.0); break;
            default: break;
            }
            r[o] = v;
        }
        out[q] = r[result];
    }
    free(r);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * Exterior facets (ds) on a rectangle mesh (the next row f2).  The facet list of
 * fe/space_2d.hpp:430-446 keeps, in (cell, local edge) order, every edge with no neighbour,
 * with the marker of its boundary segment; on rectangle_mesh the segments carry the markers
 * {bottom, right, top, left} of their side (mesh/structured.hpp:26-31, default {1, 2, 3, 4}).
 * The facet cache of fe/cache_2d.hpp:126-184: Gauss-Legendre with max(1, (degree + 2) / 2)
 * points along each edge, reference points (1 - t) a + t b at t = (node + 1) / 2 between the
 * edge's reference vertices, mapped by the cell's affine map; weight gw len / 2; outward normal
 * (dy, -dx) / len for a counter-clockwise cell; J^{-1} of the cell per point; the tabulation
 * per local edge (3 x nq x 3 nloc).
 * ------------------------------------------------------------------------------------- */
static int or_cmp_u64(const void *a, const void *b)
{
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

static uint64_t or_edge_key(int a, int b)
{
    const uint64_t lo = (uint64_t)(a < b ? a : b), hi = (uint64_t)(a < b ? b : a);
    return (lo << 32) | hi;
}

/* cell, local, marker: room for 3 ne entries.  Returns the number of exterior facets, or -1 on
 * allocation failure. */
int or_rect_exterior_facets(int ne, const int *tris, const double *pts, double x0, double y0, double x1, double y1,
                            const int *markers, int *cell, int *local, int *marker)
{
    const size_t nh = (size_t)ne * 3;
    uint64_t *keys = (uint64_t *)malloc(nh * sizeof(uint64_t));
    if (!keys) return -1;
    for (size_t t = 0; t < nh; ++t)
    {
        const size_t c = t / 3;
        const int i = (int)(t % 3);
        keys[t] = or_edge_key(tris[3 * c + (i + 1) % 3], tris[3 * c + (i + 2) % 3]);
    }
    qsort(keys, nh, sizeof(uint64_t), or_cmp_u64);
    int nf = 0;
    for (int c = 0; c < ne; ++c)
        for (int i = 0; i < 3; ++i)
        {
            const int a = tris[3 * c + (i + 1) % 3], b = tris[3 * c + (i + 2) % 3];
            const uint64_t k = or_edge_key(a, b);
            size_t lo = 0, hi = nh;                          /* first key >= k */
            while (lo < hi) { const size_t mid = (lo + hi) / 2; if (keys[mid] < k) lo = mid + 1; else hi = mid; }
            const int count = (int)(lo + 1 < nh && keys[lo + 1] == k) + 1;
            if (count != 1) continue;
            const double ax = pts[2 * a], ay = pts[2 * a + 1], bx = pts[2 * b], by = pts[2 * b + 1];
            int m = 0;
            if (ay == y0 && by == y0) m = markers[0];
            else if (ax == x1 && bx == x1) m = markers[1];
            else if (ay == y1 && by == y1) m = markers[2];
            else if (ax == x0 && bx == x0) m = markers[3];
            cell[nf] = c; local[nf] = i; marker[nf] = m;
            ++nf;
        }
    free(keys);
    return nf;
}

/* x, y, w, nx, ny: nf nq; Ji: 4 nf nq; ref: 3 nq 3 nloc.  Returns nq (at most 64), or a
 * negative status. */
int or_facet_cache(int nf, const int *cell, const int *local, const double *pts, const int *tris, int k, int degree,
                   double *x, double *y, double *w, double *nx, double *ny, double *Ji, double *ref)
{
    const int n = (degree + 2) / 2 > 1 ? (degree + 2) / 2 : 1;
    if (n > 64) return -1;
    double gx[64], gw[64];
    or_gauss_legendre(n, gx, gw);
    static const double vx[3] = {0.0, 1.0, 0.0}, vy[3] = {0.0, 0.0, 1.0};
    double fx[3 * 64], fy[3 * 64];
    const int nloc = (k + 1) * (k + 2) / 2;
    for (int i = 0; i < 3; ++i)
    {
        const int a = (i + 1) % 3, b = (i + 2) % 3;
        for (int q = 0; q < n; ++q)
        {
            const double t = 0.5 * (gx[q] + 1.0);
            fx[i * n + q] = (1.0 - t) * vx[a] + t * vx[b];
            fy[i * n + q] = (1.0 - t) * vy[a] + t * vy[b];
        }
        const int st = or_tabulate(k, n, fx + i * n, fy + i * n, ref + (size_t)i * n * 3 * nloc);
        if (st < 0) return st;
    }
    for (int e = 0; e < nf; ++e)
    {
        const int c = cell[e], i = local[e];
        const int *T = tris + 3 * c;
        const double *P0 = pts + 2 * T[0], *P1 = pts + 2 * T[1], *P2 = pts + 2 * T[2];
        double J[4];
        J[0] = P1[0] - P0[0]; J[1] = P2[0] - P0[0];
        J[2] = P1[1] - P0[1]; J[3] = P2[1] - P0[1];
        const double *A = pts + 2 * T[(i + 1) % 3], *B = pts + 2 * T[(i + 2) % 3];
        const double dx = B[0] - A[0], dy = B[1] - A[1], len = hypot(dx, dy);
        for (int q = 0; q < n; ++q)
        {
            const size_t kq = (size_t)e * n + q;
            const double xi = fx[i * n + q], eta = fy[i * n + q];
            x[kq] = P0[0] + J[0] * xi + J[1] * eta;
            y[kq] = P0[1] + J[2] * xi + J[3] * eta;
            w[kq] = 0.5 * gw[q] * len;
            nx[kq] = dy / len;
            ny[kq] = -dx / len;
            const double d = J[0] * J[3] - J[1] * J[2];
            double *Jk = Ji + 4 * kq;
            Jk[0] = J[3] / d; Jk[1] = -J[1] / d;
            Jk[2] = -J[2] / d; Jk[3] = J[0] / d;
        }
    }
    return n;
}
