// facets.cu -- ds terms on the exterior facets of a mesh (the boundary integrals of Robin and
// Neumann data), and the two small kernels of the Dirichlet lift.
//
// A facet set is a list of (cell, local edge) in the reference's facet order (exterior facets in
// (cell, local edge) order, include/femd/fe/space_2d.hpp:430-446).  Its rule is the facet cache's
// (include/femd/fe/cache_2d.hpp:126-184): Gauss-Legendre points t_q along local edge i (from the
// cell's vertex (i + 1) % 3 to (i + 2) % 3), mapped by the cell's affine map; weight
// w = 0.5 gw_q len, outward normal (dy, -dx) / len for a counter-clockwise cell, J^{-1} of the
// cell; the basis tabulated per local edge.
//
// Assembly (assembly_2d.hpp:102-126 element kernel, :219-305 matrix, :173-211 vector, on a facet
// cache): every facet's element matrix Ke(i, j) = sum_t sum_q [(w_q c_t) row_a(q, i)] row_b(q, j)
// (zero products skipped, no contraction) is formed by one thread per entry; then every matrix
// position the facets touch is owned by one thread, which adds the position's element entries to
// the stored value in increasing facet order -- the order in which the reference adds them -- so
// there are no atomics and the result is deterministic.  The position lists (for every touched
// position, its element entries in facet order) are built once per facet set on the host from the
// pattern's scatter map and kept with the set; vectors use the rows' lists the same way.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"

namespace femd {
int build_scatter_map(femd_ctx ctx, femd_pattern p);
}

struct femd_facets_s : femd::HandleBase {
    femd_ctx ctx = nullptr;
    femd_pattern pattern = nullptr;
    int nf = 0, nloc = 0;
    femd::DevBuf<int> cell, local;
    // matrix: touched positions, their entry lists (f nloc^2 + i nloc + j) in facet order
    bool mat_ready = false;
    int npos = 0;
    femd::DevBuf<int> mpos, mptr, ment;
    // vector: touched rows, their entry lists (f nloc + l) in facet order
    bool vec_ready = false;
    int nrow = 0;
    femd::DevBuf<int> vrow, vptr, vent;
    femd::DevBuf<double> ke;              // element matrices / vectors of the last assembly
    femd_facets_s() : HandleBase(femd::KIND_FACETS) {}
    ~femd_facets_s() override { femd::ctx_release(ctx); }
};

namespace femd {

static constexpr int FC_MAX_TERMS = 8;

struct FacetTerms {
    int nterms;
    int a[FC_MAX_TERMS], b[FC_MAX_TERMS];
    double cval[FC_MAX_TERMS];
    const double *cpts[FC_MAX_TERMS];     // per-point coefficient [f nq + q], or null for cval
};

// rows of derivative code m at point q of facet f (Cache2D::row, cache_2d.hpp:211-226)
__device__ __forceinline__ double fc_row(const double *R, int nloc, int m, int l, const double *Ji)
{
    if (m == 0) return R[l];
    const double a = m == 1 ? Ji[0] : Ji[1], b = m == 1 ? Ji[2] : Ji[3];
    return __dadd_rn(__dmul_rn(a, R[nloc + l]), __dmul_rn(b, R[2 * nloc + l]));
}

// the cell's J^{-1} (lagrange_space_2d.hpp:44-52, cache_2d.hpp:116-117)
__device__ __forceinline__ void fc_jinv(const double *pts, const int *tris, int c, double *Ji)
{
    const int v0 = tris[3 * c], v1 = tris[3 * c + 1], v2 = tris[3 * c + 2];
    const double x0 = pts[2 * v0], y0 = pts[2 * v0 + 1];
    const double J0 = __dsub_rn(pts[2 * v1], x0), J1 = __dsub_rn(pts[2 * v2], x0);
    const double J2 = __dsub_rn(pts[2 * v1 + 1], y0), J3 = __dsub_rn(pts[2 * v2 + 1], y0);
    const double d = __dsub_rn(__dmul_rn(J0, J3), __dmul_rn(J1, J2));
    Ji[0] = __ddiv_rn(J3, d);
    Ji[1] = __ddiv_rn(-J1, d);
    Ji[2] = __ddiv_rn(-J2, d);
    Ji[3] = __ddiv_rn(J0, d);
}

// per (facet, point): x, y, w, nx, ny (any output may be null)
__global__ void k_facet_points(const double *__restrict__ pts, const int *__restrict__ tris, int nf,
                               const int *__restrict__ fcell, const int *__restrict__ flocal, int nq,
                               const double *__restrict__ fxi, const double *__restrict__ feta, const double *__restrict__ gw,
                               double *x, double *y, double *w, double *nx, double *ny)
{
    const long long total = (long long)nf * nq;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / nq), q = (int)(t % nq);
        const int c = fcell[f], i = flocal[f];
        const int *T = tris + 3 * c;
        const double x0 = pts[2 * T[0]], y0 = pts[2 * T[0] + 1];
        const double J0 = __dsub_rn(pts[2 * T[1]], x0), J1 = __dsub_rn(pts[2 * T[2]], x0);
        const double J2 = __dsub_rn(pts[2 * T[1] + 1], y0), J3 = __dsub_rn(pts[2 * T[2] + 1], y0);
        const int a = T[(i + 1) % 3], b = T[(i + 2) % 3];
        const double dx = __dsub_rn(pts[2 * b], pts[2 * a]), dy = __dsub_rn(pts[2 * b + 1], pts[2 * a + 1]);
        const double len = hypot(dx, dy);
        const double xi = fxi[i * nq + q], eta = feta[i * nq + q];
        if (x) x[t] = __dadd_rn(__dadd_rn(x0, __dmul_rn(J0, xi)), __dmul_rn(J1, eta));
        if (y) y[t] = __dadd_rn(__dadd_rn(y0, __dmul_rn(J2, xi)), __dmul_rn(J3, eta));
        if (w) w[t] = __dmul_rn(__dmul_rn(0.5, gw[q]), len);
        if (nx) nx[t] = __ddiv_rn(dy, len);
        if (ny) ny[t] = __ddiv_rn(-dx, len);
    }
}

// element matrices (vector: nj = 1 and b unused) of the facets: ke[f][i][j]
template <bool MATRIX>
__global__ void k_facet_elements(const double *__restrict__ pts, const int *__restrict__ tris, int nf,
                                 const int *__restrict__ fcell, const int *__restrict__ flocal, int nloc, int nq,
                                 const double *__restrict__ ref, const double *__restrict__ gw, FacetTerms ts,
                                 double *__restrict__ ke)
{
    const int nj = MATRIX ? nloc : 1;
    const long long per = (long long)nloc * nj, total = (long long)nf * per;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / per), ij = (int)(t % per), i = ij / nj, j = ij % nj;
        const int c = fcell[f], le = flocal[f];
        double Ji[4];
        fc_jinv(pts, tris, c, Ji);
        const int *T = tris + 3 * c;
        const int a = T[(le + 1) % 3], b = T[(le + 2) % 3];
        const double dx = __dsub_rn(pts[2 * b], pts[2 * a]), dy = __dsub_rn(pts[2 * b + 1], pts[2 * a + 1]);
        const double len = hypot(dx, dy);
        double acc = 0.0;
        for (int tt = 0; tt < ts.nterms; ++tt)
            for (int q = 0; q < nq; ++q) {
                const double wq = __dmul_rn(__dmul_rn(0.5, gw[q]), len);
                const double cq = ts.cpts[tt] ? ts.cpts[tt][(size_t)f * nq + q] : ts.cval[tt];
                const double s = __dmul_rn(wq, cq);
                if (s == 0.0) continue;
                const double *R = ref + ((size_t)le * nq + q) * 3 * nloc;
                const double sa = __dmul_rn(s, fc_row(R, nloc, ts.a[tt], i, Ji));
                if (MATRIX) {
                    if (sa == 0.0) continue;
                    acc = __dadd_rn(acc, __dmul_rn(sa, fc_row(R, nloc, ts.b[tt], j, Ji)));
                } else {
                    acc = __dadd_rn(acc, sa);
                }
            }
        ke[t] = acc;
    }
}

// data[pos[p]] += the position's entries in facet order
__global__ void k_facet_scatter(int npos, const int *__restrict__ pos, const int *__restrict__ ptr,
                                const int *__restrict__ ent, const double *__restrict__ ke, double *__restrict__ data)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npos; p += gridDim.x * blockDim.x) {
        double acc = data[pos[p]];
        for (int k = ptr[p]; k < ptr[p + 1]; ++k) acc = __dadd_rn(acc, ke[ent[k]]);
        data[pos[p]] = acc;
    }
}

// the positions (matrix: the scatter map; vector: the dofs) of every element entry of the facets
__global__ void k_facet_targets(int nf, const int *__restrict__ fcell, int nloc, int matrix, const int *__restrict__ map,
                                const int *__restrict__ dofs, int *__restrict__ out)
{
    const int nj = matrix ? nloc : 1;
    const long long per = (long long)nloc * nj, total = (long long)nf * per;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / per), ij = (int)(t % per);
        const size_t c = (size_t)fcell[f];
        out[t] = matrix ? map[c * per + ij] : dofs[c * nloc + ij];
    }
}

// u_raw[raw_of[i]] = x[i]: a solution on the constrained dofs written into the raw numbering
__global__ void k_prolongate(int n, const int *__restrict__ raw_of, const double *__restrict__ x, double *__restrict__ u)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) u[raw_of[i]] = x[i];
}

// the lists of a facet set: targets downloaded, grouped by target (stable: facet order kept)
static int build_lists(femd_ctx ctx, femd_facets_s *F, bool matrix)
{
    cudaStream_t s = ctx->stream;
    femd_pattern P = F->pattern;
    const int nl = F->nloc, nj = matrix ? nl : 1;
    const size_t total = (size_t)F->nf * nl * nj;
    if (matrix) FEMD_TRY(build_scatter_map(ctx, P));
    DevBuf<int> tg;
    FEMD_TRY(tg.alloc(std::max<size_t>(total, 1)));
    if (total)
        k_facet_targets<<<grid_for(total, 256, 1u << 20), 256, 0, counted(s)>>>(F->nf, F->cell.p, nl, matrix ? 1 : 0, P->map.p,
                                                                                P->cell_dofs.p, tg.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    std::vector<int> h(total);
    if (total) FEMD_TRY_CUDA(cudaMemcpyAsync(h.data(), tg.p, total * sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    std::vector<int> order;
    order.reserve(total);
    for (size_t t = 0; t < total; ++t)
        if (h[t] >= 0) order.push_back((int)t);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h[a] < h[b]; });
    std::vector<int> pos, ptr(1, 0), ent;
    for (size_t k = 0; k < order.size(); ++k) {
        if (k == 0 || h[order[k]] != h[order[k - 1]]) {
            if (k) ptr.push_back((int)k);
            pos.push_back(h[order[k]]);
        }
        ent.push_back(order[k]);
    }
    ptr.push_back((int)order.size());
    if (pos.empty()) ptr.assign(1, 0);
    DevBuf<int> &dp = matrix ? F->mpos : F->vrow, &dq = matrix ? F->mptr : F->vptr, &de = matrix ? F->ment : F->vent;
    FEMD_TRY(dp.alloc(std::max<size_t>(pos.size(), 1)));
    FEMD_TRY(dq.alloc(ptr.size()));
    FEMD_TRY(de.alloc(std::max<size_t>(ent.size(), 1)));
    if (!pos.empty()) {
        FEMD_TRY_CUDA(cudaMemcpyAsync(dp.p, pos.data(), pos.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        FEMD_TRY_CUDA(cudaMemcpyAsync(de.p, ent.data(), ent.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    FEMD_TRY_CUDA(cudaMemcpyAsync(dq.p, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    if (matrix) { F->npos = (int)pos.size(); F->mat_ready = true; }
    else { F->nrow = (int)pos.size(); F->vec_ready = true; }
    return FEMD_OK;
}

static femd_facets_s *as_facets(void *h)
{
    femd_facets_s *f = static_cast<femd_facets_s *>(h);
    return (f && f->kind == KIND_FACETS) ? f : nullptr;
}

struct RuleDevF {
    DevBuf<double> buf;   // xi (3 nq), eta (3 nq), gw (nq), ref (3 nq 3 nloc)
};

static int check_rule(const femd_facet_rule *r, int nloc)
{
    FEMD_CHECK_ARG(r && r->xi_host && r->eta_host && r->gw_host && r->ref_host, "facet rule: NULL table");
    FEMD_CHECK_ARG(r->nq >= 1 && r->nq <= 64, "facet rule: 1 to 64 points");
    FEMD_CHECK_ARG(r->nloc == nloc && r->k >= 1 && (r->k + 1) * (r->k + 2) / 2 == nloc, "facet rule: degree differs from the space");
    return FEMD_OK;
}

static int upload_rule(const femd_facet_rule *r, RuleDevF &R, cudaStream_t s)
{
    const size_t nq = (size_t)r->nq, nref = 3 * nq * 3 * (size_t)r->nloc;
    std::vector<double> h(7 * nq + nref);
    std::copy(r->xi_host, r->xi_host + 3 * nq, h.begin());
    std::copy(r->eta_host, r->eta_host + 3 * nq, h.begin() + 3 * nq);
    std::copy(r->gw_host, r->gw_host + nq, h.begin() + 6 * nq);
    std::copy(r->ref_host, r->ref_host + nref, h.begin() + 7 * nq);
    FEMD_TRY(R.buf.alloc(h.size()));
    FEMD_TRY_CUDA(cudaMemcpyAsync(R.buf.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // h is a host vector released on return
    return FEMD_OK;
}

static int facet_terms(int nterms, const int *a, const int *b, const femd_coef *coef, bool matrix, FacetTerms &ts)
{
    FEMD_CHECK_ARG(nterms >= 1 && nterms <= FC_MAX_TERMS && a && coef && (!matrix || b), "facet assembly: 1 to 8 terms");
    ts.nterms = nterms;
    for (int t = 0; t < nterms; ++t) {
        FEMD_CHECK_ARG(a[t] >= 0 && a[t] <= 2 && (!matrix || (b[t] >= 0 && b[t] <= 2)), "assembly_2d: derivative code out of range");
        FEMD_CHECK_ARG(coef[t].kind == FEMD_COEF_CONST || (coef[t].kind == FEMD_COEF_POINTS && coef[t].points_dev),
                       "facet assembly: a coefficient is a constant or an array at the facet points");
        ts.a[t] = a[t];
        ts.b[t] = matrix ? b[t] : 0;
        ts.cval[t] = coef[t].value;
        ts.cpts[t] = coef[t].kind == FEMD_COEF_POINTS ? coef[t].points_dev : nullptr;
    }
    return FEMD_OK;
}

static int facet_assemble(femd_ctx ctx, femd_facets_s *F, const femd_mesh2d *mesh, const femd_facet_rule *rule, int nterms,
                          const int *a, const int *b, const femd_coef *coef, double *data, bool matrix)
{
    FEMD_TRY(check_rule(rule, F->nloc));
    FEMD_CHECK_ARG(mesh && mesh->points_dev && mesh->tris_dev && mesh->ncells == F->pattern->ncells, "facet assembly: bad mesh");
    FacetTerms ts{};
    FEMD_TRY(facet_terms(nterms, a, b, coef, matrix, ts));
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    if (matrix && !F->mat_ready) FEMD_TRY(build_lists(ctx, F, true));
    if (!matrix && !F->vec_ready) FEMD_TRY(build_lists(ctx, F, false));
    if (F->nf == 0) return FEMD_OK;
    RuleDevF R;
    FEMD_TRY(upload_rule(rule, R, s));
    const int nl = F->nloc, nq = rule->nq;
    const size_t total = (size_t)F->nf * nl * (matrix ? nl : 1);
    if (F->ke.n < total) FEMD_TRY(F->ke.alloc(total));
    const double *gw = R.buf.p + 6 * nq, *ref = R.buf.p + 7 * nq;
    const unsigned g = grid_for(total, 256, 1u << 20);
    if (matrix)
        k_facet_elements<true><<<g, 256, 0, counted(s)>>>(mesh->points_dev, mesh->tris_dev, F->nf, F->cell.p, F->local.p, nl, nq,
                                                          ref, gw, ts, F->ke.p);
    else
        k_facet_elements<false><<<g, 256, 0, counted(s)>>>(mesh->points_dev, mesh->tris_dev, F->nf, F->cell.p, F->local.p, nl, nq,
                                                           ref, gw, ts, F->ke.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    const int np = matrix ? F->npos : F->nrow;
    if (np)
        k_facet_scatter<<<grid_for((size_t)np, 256, 1u << 20), 256, 0, counted(s)>>>(
            np, matrix ? F->mpos.p : F->vrow.p, matrix ? F->mptr.p : F->vptr.p, matrix ? F->ment.p : F->vent.p, F->ke.p, data);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // the rule buffer is released on return
    return FEMD_OK;
}

}  // namespace femd

using namespace femd;

extern "C" {

int femd_cuda_facets_create(femd_ctx ctx, femd_pattern p, int nf, const int *fcell_host, const int *flocal_host,
                            femd_facets *out)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && p && p->kind == KIND_PATTERN && out && nf >= 0, "facets: bad arguments");
    FEMD_CHECK_ARG(p->cell_dofs.p && p->ncells > 0 && p->nloc > 0, "facets: the pattern has no cell->dof map (a cell pattern)");
    FEMD_CHECK_ARG(nf == 0 || (fcell_host && flocal_host), "facets: NULL facet list");
    for (int f = 0; f < nf; ++f)
        FEMD_CHECK_ARG(fcell_host[f] >= 0 && fcell_host[f] < p->ncells && flocal_host[f] >= 0 && flocal_host[f] < 3,
                       "facets: a facet's cell or local edge is out of range");
    *out = nullptr;
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    auto F = new femd_facets_s();
    F->ctx = ctx;
    ctx_retain(ctx);
    F->pattern = p;
    F->nf = nf;
    F->nloc = p->nloc;
    int st;
    if ((st = F->cell.alloc(std::max(nf, 1))) || (st = F->local.alloc(std::max(nf, 1)))) { delete F; return st; }
    cudaError_t e = cudaSuccess;
    if (nf) e = cudaMemcpyAsync(F->cell.p, fcell_host, nf * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    if (nf && e == cudaSuccess) e = cudaMemcpyAsync(F->local.p, flocal_host, nf * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { delete F; set_error(std::string("facets: ") + cudaGetErrorString(e)); return FEMD_ECUDA; }
    *out = reinterpret_cast<femd_facets>(F);
    return FEMD_OK;
}

int femd_cuda_facet_points(femd_ctx ctx, femd_facets handle, const femd_mesh2d *mesh, const femd_facet_rule *rule,
                           double *x_dev, double *y_dev, double *w_dev, double *nx_dev, double *ny_dev)
{
    clear_error();
    femd_facets_s *F = as_facets(handle);
    FEMD_CHECK_ARG(ctx && F && mesh && mesh->points_dev && mesh->tris_dev, "facet_points: bad arguments");
    FEMD_TRY(check_rule(rule, F->nloc));
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    if (F->nf == 0) return FEMD_OK;
    RuleDevF R;
    FEMD_TRY(upload_rule(rule, R, ctx->stream));
    const int nq = rule->nq;
    const size_t total = (size_t)F->nf * nq;
    k_facet_points<<<grid_for(total, 256, 1u << 20), 256, 0, counted(ctx->stream)>>>(
        mesh->points_dev, mesh->tris_dev, F->nf, F->cell.p, F->local.p, nq, R.buf.p, R.buf.p + 3 * nq, R.buf.p + 6 * nq, x_dev,
        y_dev, w_dev, nx_dev, ny_dev);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return FEMD_OK;
}

int femd_cuda_assemble_facet_matrix(femd_ctx ctx, femd_facets handle, const femd_mesh2d *mesh, const femd_facet_rule *rule,
                                    int nterms, const int *a, const int *b, const femd_coef *coef, femd_matrix K)
{
    clear_error();
    femd_facets_s *F = as_facets(handle);
    FEMD_CHECK_ARG(ctx && F && K && K->kind == KIND_MATRIX, "assemble_facet_matrix: bad arguments");
    FEMD_CHECK_ARG(K->pattern == F->pattern, "assemble_facet_matrix: K is not on the facet set's pattern");
    FEMD_TRY(facet_assemble(ctx, F, mesh, rule, nterms, a, b, coef, K->data.p, true));
    K->f32_valid = false;
    return FEMD_OK;
}

int femd_cuda_assemble_facet_vector(femd_ctx ctx, femd_facets handle, const femd_mesh2d *mesh, const femd_facet_rule *rule,
                                    int nterms, const int *a, const femd_coef *coef, double *f_dev)
{
    clear_error();
    femd_facets_s *F = as_facets(handle);
    FEMD_CHECK_ARG(ctx && F && (F->pattern->nrows == 0 || f_dev), "assemble_facet_vector: bad arguments");
    return facet_assemble(ctx, F, mesh, rule, nterms, a, nullptr, coef, f_dev, false);
}

int femd_cuda_prolongate(femd_ctx ctx, int n, const int *raw_of_dev, const double *x_dev, double *u_raw_dev)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && n >= 0 && (n == 0 || (raw_of_dev && x_dev && u_raw_dev)), "prolongate: bad arguments");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    if (n) k_prolongate<<<grid_for((size_t)n, 256, 1u << 20), 256, 0, counted(ctx->stream)>>>(n, raw_of_dev, x_dev, u_raw_dev);
    FEMD_TRY_CUDA(cudaGetLastError());
    return FEMD_OK;
}

}  // extern "C"
