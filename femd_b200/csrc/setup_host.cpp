// setup_host.cpp -- host-side setup of a P_k problem on a structured triangle mesh: the mesh,
// the dof numbering, the quadrature rule and the reference tabulation.  These run once per
// mesh and degree (the reference runs them on the host too) and feed the device kernels.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/femd_cuda.h"
#include "compact_host.h"

namespace femd {
void set_error(const std::string &msg);
void clear_error();

// A reverse Cuthill-McKee order of a square pattern (host CSR): order[new] = old.  Per connected
// component: a pseudo-peripheral start (repeated breadth-first sweeps from the lowest-degree node
// of the last level while the depth grows; George and Liu's heuristic), then the Cuthill-McKee
// breadth-first numbering with each node's unnumbered neighbours taken in increasing degree
// (ties by index); the whole sequence reversed.  Deterministic.
void rcm_order(int n, const std::vector<int> &ip, const std::vector<int> &ix, std::vector<int> &order)
{
    std::vector<int> deg(n), mark(n, -1), num(n, 0), queue;
    for (int i = 0; i < n; ++i) deg[i] = ip[i + 1] - ip[i];
    order.clear();
    order.reserve(n);
    queue.reserve(n);
    int stamp = 0;
    // breadth-first levels from s over the nodes not yet numbered; the depth, and the
    // lowest-degree node of the last level
    auto sweep = [&](int s, int &depth, int &far) {
        ++stamp;
        queue.clear();
        queue.push_back(s);
        mark[s] = stamp;
        size_t head = 0, level_start = 0;
        depth = 0;
        while (true) {
            const size_t level_end = queue.size();
            for (; head < level_end; ++head) {
                const int u = queue[head];
                for (int q = ip[u]; q < ip[u + 1]; ++q) {
                    const int v = ix[q];
                    if (!num[v] && mark[v] != stamp) {
                        mark[v] = stamp;
                        queue.push_back(v);
                    }
                }
            }
            if (queue.size() == level_end) {
                far = queue[level_start];
                for (size_t k = level_start; k < level_end; ++k)
                    if (deg[queue[k]] < deg[far] || (deg[queue[k]] == deg[far] && queue[k] < far)) far = queue[k];
                return;
            }
            level_start = level_end;
            ++depth;
        }
    };
    std::vector<int> nb;
    for (int seed = 0; seed < n; ++seed) {
        if (num[seed]) continue;
        int r = seed, depth = 0, far = seed;
        sweep(r, depth, far);
        for (int t = 0; t < 8; ++t) {
            int d2 = 0, f2 = far;
            sweep(far, d2, f2);
            if (d2 <= depth) break;
            r = far;
            depth = d2;
            far = f2;
        }
        // Cuthill-McKee from r
        const size_t first = order.size();
        order.push_back(r);
        num[r] = 1;
        for (size_t h = first; h < order.size(); ++h) {
            const int u = order[h];
            nb.clear();
            for (int q = ip[u]; q < ip[u + 1]; ++q)
                if (!num[ix[q]]) {
                    num[ix[q]] = 1;
                    nb.push_back(ix[q]);
                }
            std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
            order.insert(order.end(), nb.begin(), nb.end());
        }
    }
    std::reverse(order.begin(), order.end());
}


void compact_layout(int n, const std::vector<int> &ip, const std::vector<int> &ix, CompactLayout &L)
{
    L = CompactLayout();
    std::vector<int> order;
    rcm_order(n, ip, ix, order);
    // rows by length, longest first, within windows of CL_SORT rows of the RCM order, so that
    // the 32 rows of a slice have nearly the same length (P2 / P3 rows of a 6-valent mesh have
    // 7 to 37 entries; unsorted, the slices would be padded by 66 % / 121 %, sorted by 1-5 %)
    auto rlen = [&](int i) { return ip[i + 1] - ip[i]; };
    for (int a = 0; a < n; a += CL_SORT)
        std::stable_sort(order.begin() + a, order.begin() + std::min(n, a + CL_SORT),
                         [&](int u, int v) { return rlen(u) > rlen(v); });
    const int nslice = (n + CL_TILE - 1) / CL_TILE;
    L.iperm.assign((size_t)n, 0);
    L.rstart.assign((size_t)n + 1, 0);
    long long nsell = 0;
    for (int t = 0; t < nslice; ++t) {
        const int k0 = t * CL_TILE, k1 = std::min(n, (t + 1) * CL_TILE);
        int w = 0;
        for (int k = k0; k < k1; ++k) w = std::max(w, rlen(order[k]));
        for (int k = k0; k < k1; ++k) L.rstart[k] = (int)std::min<long long>(nsell + (k - k0), INT_MAX);
        nsell += (long long)CL_TILE * w;
    }
    L.nsell = nsell;
    if (nsell > INT_MAX - 64) {
        L.bw = -1;
        return;
    }
    L.rstart[n] = (int)nsell;
    for (int k = 0; k < n; ++k) L.iperm[order[k]] = k;
    const long long nnz = n ? ip[n] : 0;
    L.dst.assign((size_t)std::max<long long>(nnz, 1), 0);
    L.off.assign((size_t)std::max<long long>(nsell, 1), (short)0);
    L.tlo.assign((size_t)nslice, INT_MAX);
    L.thi.assign((size_t)nslice, INT_MIN);
    std::vector<std::pair<int, int>> row;
    int bw = 0;
    for (int k = 0; k < n; ++k) {
        const int i = order[k];
        row.clear();
        for (int q = ip[i]; q < ip[i + 1]; ++q) row.emplace_back(L.iperm[ix[q]], q);
        std::sort(row.begin(), row.end());
        int pos = L.rstart[k];
        int &lo = L.tlo[k / CL_TILE], &hi = L.thi[k / CL_TILE];
        lo = std::min(lo, k);
        hi = std::max(hi, k);
        for (const auto &e : row) {
            const int d = e.first - k;
            bw = std::max(bw, std::abs(d));
            L.off[pos] = (short)std::max(-32768, std::min(32767, d));
            L.dst[e.second] = pos;
            pos += CL_TILE;
            lo = std::min(lo, e.first);
            hi = std::max(hi, e.first);
        }
    }
    L.bw = bw;
    L.ok = bw <= 32767;
}

}  // namespace femd

using femd::set_error;

extern "C" {

// rectangle_mesh, "right" diagonal: vertex (i, j) = j (nx+1) + i; cell (i, j) holds the
// triangles (a, b, c) and (a, c, d), a = (i, j), b = (i+1, j), c = (i+1, j+1), d = (i, j+1)
// (include/femd/mesh/structured.hpp:282-289, 338-351).
int femd_host_rectangle_mesh(double x0, double y0, double x1, double y1, int nx, int ny, double *points, int *tris)
{
    femd::clear_error();
    if (!(x1 > x0 && y1 > y0)) { set_error("rectangle_mesh: need x1 > x0 and y1 > y0"); return FEMD_EINVAL; }
    if (nx < 1 || ny < 1) { set_error("rectangle_mesh: need nx, ny >= 1"); return FEMD_EINVAL; }
    if (!points || !tris) { set_error("rectangle_mesh: NULL output"); return FEMD_EINVAL; }
    const long long W = nx + 1;
    for (int j = 0; j <= ny; ++j) {
        const double y = j == ny ? y1 : y0 + (y1 - y0) * j / ny;
        for (int i = 0; i <= nx; ++i) {
            const long long v = j * W + i;
            points[2 * v] = i == nx ? x1 : x0 + (x1 - x0) * i / nx;
            points[2 * v + 1] = y;
        }
    }
    long long t = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int a = (int)(j * W + i), b = a + 1, c = (int)(a + W + 1), d = (int)(a + W);
            int *T = tris + 6 * t;
            T[0] = a; T[1] = b; T[2] = c;
            T[3] = a; T[4] = c; T[5] = d;
            ++t;
        }
    return FEMD_OK;
}

// Continuous P_k numbering (include/femd/fe/space_2d.hpp:390-526).  Global edges are numbered
// by their first appearance over (cell, local edge i), edge i running from local vertex
// (i+1)%3 to (i+2)%3.  Here the first appearance is found by sorting the (edge key, c 3 + i)
// pairs: within a key the smallest c 3 + i comes first, and the edges are ranked by it.
// An edge met once is exterior; with all_exterior its vertices and nodes are fixed.
}  // extern "C"

// The numbering of femd_host_lagrange_numbering; cell_raw (optional) receives the raw numbering
// (before the elimination of Dirichlet nodes), cell_dofs (optional) the adapted one.
static int lagrange_numbering(int nverts, int ncells, const int *tris, int k, int all_exterior, int *cell_dofs,
                              int *cell_raw, int *dim, int *raw_dim)
{
    femd::clear_error();
    if (k < 1 || k > 20) { set_error("LagrangeSpace2D: degree must be in 1..20"); return FEMD_EINVAL; }
    if (nverts < 3 || ncells < 1 || !tris || (!cell_dofs && !cell_raw)) { set_error("lagrange_numbering: bad arguments"); return FEMD_EINVAL; }
    const int nloc = (k + 1) * (k + 2) / 2, de = k - 1, nint = (k - 1) * (k - 2) / 2;
    const size_t nh = (size_t)ncells * 3;
    struct Half { uint64_t key; int val; };
    std::vector<Half> h(nh);
    for (size_t c = 0; c < (size_t)ncells; ++c)
        for (int i = 0; i < 3; ++i) {
            const int a = tris[3 * c + (i + 1) % 3], b = tris[3 * c + (i + 2) % 3];
            if (a < 0 || a >= nverts || b < 0 || b >= nverts) { set_error("lagrange_numbering: vertex index out of range"); return FEMD_EINVAL; }
            const uint64_t lo = (uint64_t)std::min(a, b), hi = (uint64_t)std::max(a, b);
            h[3 * c + i] = Half{(lo << 32) | hi, (int)(3 * c + i)};
        }
    std::sort(h.begin(), h.end(), [](const Half &x, const Half &y) { return x.key < y.key || (x.key == y.key && x.val < y.val); });
    std::vector<char> first(nh, 0);
    std::vector<int> seg_first(nh), seg_count(nh);
    for (size_t s = 0; s < nh;) {
        size_t e = s;
        while (e < nh && h[e].key == h[s].key) ++e;
        if (e - s > 2) { set_error("lagrange_numbering: an edge is shared by more than two triangles"); return FEMD_EINVAL; }
        first[h[s].val] = 1;
        for (size_t t = s; t < e; ++t) { seg_first[t] = h[s].val; seg_count[t] = (int)(e - s); }
        s = e;
    }
    std::vector<int> rank(nh);
    int nedges = 0;
    for (size_t v = 0; v < nh; ++v) { rank[v] = nedges; nedges += first[v]; }
    std::vector<int> cell_edge(nh);
    std::vector<char> exterior(nh);
    for (size_t t = 0; t < nh; ++t) {
        cell_edge[h[t].val] = rank[seg_first[t]];
        exterior[h[t].val] = seg_count[t] == 1;
    }
    const long long voff = nverts;
    const long long rd = voff + (long long)nedges * de + (long long)ncells * nint;
    if (rd > 0x7fffffffLL) { set_error("lagrange_numbering: more than 2^31 nodes"); return FEMD_EINVAL; }
    std::vector<int> raw((size_t)ncells * nloc);
    for (size_t c = 0; c < (size_t)ncells; ++c) {
        int *d = raw.data() + c * nloc;
        for (int v = 0; v < 3; ++v) d[v] = tris[3 * c + v];
        for (int i = 0; i < 3; ++i) {
            const int g = cell_edge[3 * c + i];
            const bool flip = tris[3 * c + (i + 1) % 3] > tris[3 * c + (i + 2) % 3];
            for (int j = 0; j < de; ++j) d[3 + i * de + j] = (int)(voff + (long long)g * de + (flip ? de - 1 - j : j));
        }
        for (int j = 0; j < nint; ++j) d[3 + 3 * de + j] = (int)(voff + (long long)nedges * de + (long long)c * nint + j);
    }
    std::vector<char> fixed((size_t)rd, 0);
    if (all_exterior)
        for (size_t c = 0; c < (size_t)ncells; ++c)
            for (int i = 0; i < 3; ++i) {
                if (!exterior[3 * c + i]) continue;
                const int g = cell_edge[3 * c + i];
                fixed[tris[3 * c + (i + 1) % 3]] = 1;
                fixed[tris[3 * c + (i + 2) % 3]] = 1;
                for (int j = 0; j < de; ++j) fixed[voff + (long long)g * de + j] = 1;
            }
    std::vector<int> r2a((size_t)rd);
    int n = 0;
    for (long long r = 0; r < rd; ++r) r2a[r] = fixed[r] ? -1 : n++;
    if (cell_dofs)
        for (size_t q = 0; q < raw.size(); ++q) cell_dofs[q] = r2a[raw[q]];
    if (cell_raw) std::copy(raw.begin(), raw.end(), cell_raw);
    if (dim) *dim = n;
    if (raw_dim) *raw_dim = (int)rd;
    return FEMD_OK;
}

extern "C" {

int femd_host_lagrange_numbering(int nverts, int ncells, const int *tris, int k, int all_exterior, int *cell_dofs,
                                 int *dim, int *raw_dim)
{
    if (!cell_dofs || !dim) { femd::clear_error(); set_error("lagrange_numbering: bad arguments"); return FEMD_EINVAL; }
    return lagrange_numbering(nverts, ncells, tris, k, all_exterior, cell_dofs, nullptr, dim, raw_dim);
}

// The raw numbering of the same space (every node, none eliminated), ncells x nloc: vertices
// first, then edge nodes from the smaller vertex to the larger, then cell interiors
// (include/femd/fe/space_2d.hpp:448-470).
int femd_host_lagrange_raw(int nverts, int ncells, const int *tris, int k, int *cell_raw, int *raw_dim)
{
    return lagrange_numbering(nverts, ncells, tris, k, 0, nullptr, cell_raw, nullptr, raw_dim);
}

// Gauss-Legendre on [-1, 1]: closed forms for 1..5 points, Newton on P_n from Chebyshev-spaced
// guesses for more (include/femd/quadrature/gauss_legendre.hpp:104-207).
static void gauss_legendre(int n, double *x, double *w)
{
    switch (n) {
    case 1: x[0] = 0.0; w[0] = 2.0; return;
    case 2: x[0] = -1.0 / std::sqrt(3.0); x[1] = 1.0 / std::sqrt(3.0); w[0] = w[1] = 1.0; return;
    case 3:
        x[0] = -std::sqrt(3.0 / 5.0); x[1] = 0.0; x[2] = std::sqrt(3.0 / 5.0);
        w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
        return;
    case 4: {
        const double a = std::sqrt((3.0 + 2.0 * std::sqrt(6.0 / 5.0)) / 7.0), b = std::sqrt((3.0 - 2.0 * std::sqrt(6.0 / 5.0)) / 7.0);
        const double wa = (18.0 - std::sqrt(30.0)) / 36.0, wb = (18.0 + std::sqrt(30.0)) / 36.0;
        x[0] = -a; x[1] = -b; x[2] = b; x[3] = a;
        w[0] = wa; w[1] = wb; w[2] = wb; w[3] = wa;
        return;
    }
    case 5: {
        const double a = std::sqrt(5.0 + 2.0 * std::sqrt(10.0 / 7.0)) / 3.0, b = std::sqrt(5.0 - 2.0 * std::sqrt(10.0 / 7.0)) / 3.0;
        const double wa = (322.0 - 13.0 * std::sqrt(70.0)) / 900.0, wb = (322.0 + 13.0 * std::sqrt(70.0)) / 900.0;
        x[0] = -a; x[1] = -b; x[2] = 0.0; x[3] = b; x[4] = a;
        w[0] = wa; w[1] = wb; w[2] = 128.0 / 225.0; w[3] = wb; w[4] = wa;
        return;
    }
    default: break;
    }
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < n; ++i) {
        double t = std::cos(PI * (i + 0.75) / (n + 0.5));
        auto legendre = [n](double z, double &pn, double &pn1) {
            double p0 = 1.0, p1 = z;
            for (int m = 2; m <= n; ++m) { const double p2 = ((2.0 * m - 1.0) * z * p1 - (m - 1.0) * p0) / m; p0 = p1; p1 = p2; }
            pn = p1; pn1 = p0;
        };
        for (int it = 0; it < 100; ++it) {
            double pn, pm;
            legendre(t, pn, pm);
            const double dp = n * (t * pn - pm) / (t * t - 1.0);
            const double dx = -pn / dp;
            t += dx;
            if (std::abs(dx) <= 1e-15) break;
        }
        double pn, pm;
        legendre(t, pn, pm);
        const double dp = n * (t * pn - pm) / (t * t - 1.0);
        x[i] = t;
        w[i] = 2.0 / ((1.0 - t * t) * dp * dp);
    }
}

// TriangleQuadrature(degree): 1 point (degree <= 1), 3 points (2), Radon's 7 points (3..5),
// else the collapsed Gauss rule xi = u (1 - v), eta = v, weight wu wv (1 - v)
// (include/femd/quadrature/triangle.hpp:24-58).
int femd_host_triangle_quadrature(int degree, double *xi, double *eta, double *w)
{
    femd::clear_error();
    if (!xi || !eta || !w) { set_error("triangle_quadrature: NULL output"); return -FEMD_EINVAL; }
    const int d = degree < 0 ? 0 : degree;
    int m = 0;
    auto add = [&](double a, double b, double c) { xi[m] = a; eta[m] = b; w[m] = c; ++m; };
    if (d <= 1) add(1.0 / 3.0, 1.0 / 3.0, 0.5);
    else if (d == 2) {
        add(1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0);
        add(2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0);
        add(1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0);
    } else if (d <= 5) {
        const double s15 = std::sqrt(15.0);
        add(1.0 / 3.0, 1.0 / 3.0, 9.0 / 80.0);
        const double a1 = (6.0 - s15) / 21.0, w1 = (155.0 - s15) / 2400.0;
        const double a2 = (6.0 + s15) / 21.0, w2 = (155.0 + s15) / 2400.0;
        add(a1, a1, w1); add(1.0 - 2.0 * a1, a1, w1); add(a1, 1.0 - 2.0 * a1, w1);
        add(a2, a2, w2); add(1.0 - 2.0 * a2, a2, w2); add(a2, 1.0 - 2.0 * a2, w2);
    } else {
        const int nu = (d + 2) / 2, nv = (d + 3) / 2;
        if (nu * nv > 64) { set_error("triangle_quadrature: degree too high (more than 64 points)"); return -FEMD_EINVAL; }
        double gu[32], wu_[32], gv[32], wv_[32];
        gauss_legendre(nu, gu, wu_);
        gauss_legendre(nv, gv, wv_);
        for (int j = 0; j < nv; ++j) {
            const double v = 0.5 * (gv[j] + 1.0), wv = 0.5 * wv_[j];
            for (int i = 0; i < nu; ++i) {
                const double u = 0.5 * (gu[i] + 1.0), wu = 0.5 * wu_[i];
                add(u * (1.0 - v), v, wu * wv * (1.0 - v));
            }
        }
    }
    return m;
}

// The equispaced P_k Lagrange basis on the reference triangle in FEMd's local order
// (include/femd/fe/simplex_basis.hpp:17-18, 254-291): vertices 0, 1, 2; the k-1 nodes of edge e
// from vertex (e+1)%3 to (e+2)%3; interior nodes j = 1.., i = 1.. with i + j < k.  The node with
// lattice indices (a0, a1, a2), a0 + a1 + a2 = k, has the basis function
// prod_m L_{a_m}(lambda_m), L_a(t) = prod_{s<a} (k t - s) / (s + 1), lambda = (1-xi-eta, xi, eta).
int femd_host_tabulate(int k, int nq, const double *xi, const double *eta, double *out)
{
    femd::clear_error();
    if (k < 1 || k > 20 || nq < 0 || (nq > 0 && (!xi || !eta || !out))) { set_error("tabulate: bad arguments"); return -FEMD_EINVAL; }
    const int nloc = (k + 1) * (k + 2) / 2;
    std::vector<int> lat;
    const int V[3][3] = {{k, 0, 0}, {0, k, 0}, {0, 0, k}};
    for (auto &v : V) lat.insert(lat.end(), v, v + 3);
    for (int e = 0; e < 3; ++e)
        for (int j = 1; j < k; ++j) {
            int a[3] = {0, 0, 0};
            a[(e + 1) % 3] = k - j;
            a[(e + 2) % 3] = j;
            lat.insert(lat.end(), a, a + 3);
        }
    for (int j = 1; j < k; ++j)
        for (int i = 1; i + j < k; ++i) { const int a[3] = {k - i - j, i, j}; lat.insert(lat.end(), a, a + 3); }
    auto L = [k](int a, double t, double &v, double &dv) {
        v = 1.0; dv = 0.0;
        for (int s = 0; s < a; ++s) {
            const double f = (k * t - s) / (s + 1.0);
            dv = dv * f + v * (k / (s + 1.0));
            v *= f;
        }
    };
    for (int q = 0; q < nq; ++q) {
        const double lam[3] = {1.0 - xi[q] - eta[q], xi[q], eta[q]};
        double *o = out + (size_t)q * 3 * nloc;
        for (int l = 0; l < nloc; ++l) {
            double v[3], dv[3];
            for (int m = 0; m < 3; ++m) L(lat[3 * l + m], lam[m], v[m], dv[m]);
            o[l] = v[0] * v[1] * v[2];
            o[nloc + l] = -dv[0] * v[1] * v[2] + v[0] * dv[1] * v[2];
            o[2 * nloc + l] = -dv[0] * v[1] * v[2] + v[0] * v[1] * dv[2];
        }
    }
    return nloc;
}

// The reverse Cuthill-McKee order of a square CSR pattern (femd::rcm_order), order[new] = old: the
// order of the lockstep engine's compact layout.
int femd_host_rcm_order(int n, const int *indptr, const int *indices, int *order)
{
    femd::clear_error();
    if (n < 0 || !indptr || !order || (n > 0 && indptr[n] > 0 && !indices)) { set_error("rcm_order: bad arguments"); return FEMD_EINVAL; }
    for (int i = 0; i < n; ++i)
        if (indptr[i + 1] < indptr[i]) { set_error("rcm_order: indptr is not increasing"); return FEMD_EINVAL; }
    const long long nnz = n ? indptr[n] : 0;
    for (long long q = 0; q < nnz; ++q)
        if (indices[q] < 0 || indices[q] >= n) { set_error("rcm_order: column out of range"); return FEMD_EINVAL; }
    std::vector<int> ip(indptr, indptr + n + 1), ix(indices, indices + nnz), out;
    femd::rcm_order(n, ip, ix, out);
    std::copy(out.begin(), out.end(), order);
    return FEMD_OK;
}

// The lockstep engine's compact layout of a square CSR pattern (femd::compact_layout), what
// femd_cuda_pattern_batch_layout builds and uploads.  Called with off == NULL it reports the sizes
// only (*nsell, *bandwidth); with the arrays it fills them.
int femd_host_compact_layout(int n, const int *indptr, const int *indices, long long *nsell, int *bandwidth, int *iperm,
                             int *rstart, int *dst, short *off, int *tile_lo, int *tile_hi)
{
    femd::clear_error();
    if (n < 0 || !indptr || !nsell || !bandwidth || (n > 0 && indptr[n] > 0 && !indices)) {
        set_error("compact_layout: bad arguments");
        return FEMD_EINVAL;
    }
    for (int i = 0; i < n; ++i)
        if (indptr[i + 1] < indptr[i]) { set_error("compact_layout: indptr is not increasing"); return FEMD_EINVAL; }
    const long long nnz = n ? indptr[n] : 0;
    for (long long q = 0; q < nnz; ++q)
        if (indices[q] < 0 || indices[q] >= n) { set_error("compact_layout: column out of range"); return FEMD_EINVAL; }
    std::vector<int> ip(indptr, indptr + n + 1), ix(indices, indices + nnz);
    femd::CompactLayout L;
    femd::compact_layout(n, ip, ix, L);
    *nsell = L.nsell;
    *bandwidth = L.ok ? L.bw : -1;
    if (!off || !L.ok) return FEMD_OK;
    if (!iperm || !rstart || (nnz && !dst) || !tile_lo || !tile_hi) { set_error("compact_layout: NULL array"); return FEMD_EINVAL; }
    std::copy(L.iperm.begin(), L.iperm.end(), iperm);
    std::copy(L.rstart.begin(), L.rstart.end(), rstart);
    std::copy(L.dst.begin(), L.dst.begin() + nnz, dst);
    std::copy(L.off.begin(), L.off.begin() + L.nsell, off);
    std::copy(L.tlo.begin(), L.tlo.end(), tile_lo);
    std::copy(L.thi.begin(), L.thi.end(), tile_hi);
    return FEMD_OK;
}

// The reference coordinates of the nloc local nodes of equispaced P_k (the lattice of
// femd_host_tabulate: the three vertices, k - 1 nodes per edge, then the interior): xi, eta.
int femd_host_lagrange_nodes(int k, double *xi, double *eta)
{
    femd::clear_error();
    if (k < 1 || k > 20 || !xi || !eta) { set_error("lagrange_nodes: bad arguments"); return -FEMD_EINVAL; }
    int l = 0;
    const int V[3][2] = {{0, 0}, {k, 0}, {0, k}};
    for (auto &v : V) { xi[l] = (double)v[0] / k; eta[l] = (double)v[1] / k; ++l; }
    for (int e = 0; e < 3; ++e)
        for (int j = 1; j < k; ++j) {
            int a[3] = {0, 0, 0};
            a[(e + 1) % 3] = k - j;
            a[(e + 2) % 3] = j;
            xi[l] = (double)a[1] / k;
            eta[l] = (double)a[2] / k;
            ++l;
        }
    for (int j = 1; j < k; ++j)
        for (int i = 1; i + j < k; ++i) { xi[l] = (double)i / k; eta[l] = (double)j / k; ++l; }
    return l;
}

// The exterior facets of a rectangle mesh in (cell, local edge) order -- an edge (local edge i
// joins vertices (i + 1) % 3 and (i + 2) % 3) held by one cell only -- with the marker of its side
// of [x0, x1] x [y0, y1]: markers[0..3] for bottom, right, top, left, 0 for none
// (include/femd/fe/space_2d.hpp:430-446 facets, mesh/structured.hpp:26-31 side markers).  cell,
// local, marker: room for 3 ncells entries.  Returns the number of facets, or -FEMD_E*.
int femd_host_exterior_facets(int nverts, int ncells, const int *tris, const double *points, double x0, double y0,
                              double x1, double y1, const int *markers, int *cell, int *local, int *marker)
{
    femd::clear_error();
    if (nverts < 3 || ncells < 1 || !tris || !points || !markers || !cell || !local || !marker) {
        set_error("exterior_facets: bad arguments");
        return -FEMD_EINVAL;
    }
    const size_t nh = (size_t)ncells * 3;
    std::vector<uint64_t> keys(nh);
    for (size_t t = 0; t < nh; ++t) {
        const size_t c = t / 3;
        const int i = (int)(t % 3);
        const int a = tris[3 * c + (i + 1) % 3], b = tris[3 * c + (i + 2) % 3];
        if (a < 0 || a >= nverts || b < 0 || b >= nverts) { set_error("exterior_facets: vertex index out of range"); return -FEMD_EINVAL; }
        keys[t] = ((uint64_t)std::min(a, b) << 32) | (uint64_t)std::max(a, b);
    }
    std::vector<uint64_t> sorted(keys);
    std::sort(sorted.begin(), sorted.end());
    int nf = 0;
    for (size_t t = 0; t < nh; ++t) {
        const auto r = std::equal_range(sorted.begin(), sorted.end(), keys[t]);
        if (r.second - r.first != 1) continue;
        const size_t c = t / 3;
        const int i = (int)(t % 3);
        const int a = tris[3 * c + (i + 1) % 3], b = tris[3 * c + (i + 2) % 3];
        const double ax = points[2 * a], ay = points[2 * a + 1], bx = points[2 * b], by = points[2 * b + 1];
        int m = 0;
        if (ay == y0 && by == y0) m = markers[0];
        else if (ax == x1 && bx == x1) m = markers[1];
        else if (ay == y1 && by == y1) m = markers[2];
        else if (ax == x0 && bx == x0) m = markers[3];
        cell[nf] = (int)c;
        local[nf] = i;
        marker[nf] = m;
        ++nf;
    }
    return nf;
}

// The rule of a facet cache (include/femd/fe/cache_2d.hpp:126-149): Gauss-Legendre with
// max(1, (degree + 2) / 2) points, on local edge i (from reference vertex (i + 1) % 3 to (i + 2) % 3)
// at t = (node + 1) / 2: xi, eta (3 x nq), the Gauss weights gw (nq), and the P_k tabulation per
// local edge ref (3 x nq x 3 x nloc).  Returns nq (at most 64), or -FEMD_E*.
int femd_host_facet_rule(int k, int degree, double *xi, double *eta, double *gw, double *ref)
{
    femd::clear_error();
    if (k < 1 || k > 20 || degree < 0 || !xi || !eta || !gw || !ref) { set_error("facet_rule: bad arguments"); return -FEMD_EINVAL; }
    const int n = std::max(1, (degree + 2) / 2);
    if (n > 64) { set_error("facet_rule: more than 64 points"); return -FEMD_EINVAL; }
    double gx[64];
    gauss_legendre(n, gx, gw);
    const double vx[3] = {0.0, 1.0, 0.0}, vy[3] = {0.0, 0.0, 1.0};
    const int nloc = (k + 1) * (k + 2) / 2;
    for (int i = 0; i < 3; ++i) {
        const int a = (i + 1) % 3, b = (i + 2) % 3;
        for (int q = 0; q < n; ++q) {
            const double t = 0.5 * (gx[q] + 1.0);
            xi[i * n + q] = (1.0 - t) * vx[a] + t * vx[b];
            eta[i * n + q] = (1.0 - t) * vy[a] + t * vy[b];
        }
        const int st = femd_host_tabulate(k, n, xi + i * n, eta + i * n, ref + (size_t)i * n * 3 * nloc);
        if (st < 0) return st;
    }
    return n;
}

}  // extern "C"
