// pattern.cu -- K1: the CSR sparsity pattern of a cell->dof map (sort + segmented unique per
// row, bit-identical to SparsityPattern::from_cells, include/femd/sparse/csr.hpp:84-125), the
// row -> (cell, local) lists in increasing cell order (the reference's cellof lists,
// csr.hpp:90-98), the diagonal positions, and K2: the element -> nnz scatter map
// (scatter_map_2d, include/femd/forms/assembly_2d.hpp:136-164).
//
// Layout in HBM (all int32):
//   cell_dofs  ncells x nloc           the cell -> dof map (-1: constrained)
//   rc_ptr     nrows + 1               row i holds rc_code[rc_ptr[i] .. rc_ptr[i+1])
//   rc_code    sum of row cell counts  cell * nloc + local index, increasing cell order
//   indptr     nrows + 1, indices nnz  the pattern (sorted, unique columns per row)
//   map        ncells x nloc x nloc    position of (dof(e,i), dof(e,j)) in indices, or -1
#include <algorithm>
#include <climits>
#include <string>

#include "common.cuh"

namespace femd {

static constexpr int ST_BADDOF = 32;

// ---- row -> (cell, local) lists -------------------------------------------------------------
__global__ void k_count_rows(const int *__restrict__ dofs, long long total, int nrows, int *__restrict__ cnt,
                             int *__restrict__ status)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int d = dofs[t];
        if (d >= nrows) atomicOr(status, ST_BADDOF);
        else if (d >= 0) atomicAdd(&cnt[d], 1);
    }
}

__global__ void k_fill_rows(const int *__restrict__ dofs, long long total, int nrows, int nloc,
                            int *__restrict__ fill, int *__restrict__ rc_code)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int d = dofs[t];
        if (d >= 0 && d < nrows) {
            const int pos = atomicAdd(&fill[d], 1);
            rc_code[pos] = (int)t;   // t = cell * nloc + local
        }
    }
}

// Sort each row's list (a handful of entries) by insertion: the fill order above is not
// deterministic, the sorted order is.
__global__ void k_sort_rows(const int *__restrict__ rc_ptr, int *__restrict__ rc_code, int nrows, int *__restrict__ maxcells)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const int lo = rc_ptr[i], hi = rc_ptr[i + 1];
    for (int a = lo + 1; a < hi; ++a) {
        const int v = rc_code[a];
        int b = a - 1;
        while (b >= lo && rc_code[b] > v) { rc_code[b + 1] = rc_code[b]; --b; }
        rc_code[b + 1] = v;
    }
    atomicMax(maxcells, hi - lo);
}

// ---- K1, short rows: one thread per row -----------------------------------------------------
// Each thread keeps its row's sorted unique columns in shared memory and inserts every candidate
// column (the dofs of the row's cells, in increasing cell order) at its place, skipping the ones
// already there. Entry s of thread t sits at s * PT_THREADS + t, so the 32 lanes of a warp hit 32
// different banks whatever entry each one is at. A row with more than PT_CAP columns is put on a
// list for the warp-per-row kernel below (counting pass); the filling pass skips it, since its
// length (from indptr) is then known to be above PT_CAP.
static constexpr int PT_THREADS = 128;
static constexpr int PT_CAP = 40;   // P1..P3 rows of a 6-valent mesh have 7, 19, 37 columns

template <bool FILL>
__global__ void __launch_bounds__(PT_THREADS) k_pattern_rows_t(const int *__restrict__ dofs, int nloc,
                                                               const int *__restrict__ rc_ptr,
                                                               const int *__restrict__ rc_code, int nrows,
                                                               int *__restrict__ rowlen, const int *__restrict__ indptr,
                                                               int *__restrict__ indices, int *__restrict__ list,
                                                               int *__restrict__ nlist, int *__restrict__ status)
{
    __shared__ int sbuf[PT_CAP * PT_THREADS];
    int *buf = sbuf + threadIdx.x;
    // every thread of a block takes the same number of turns, so the warp reduction below has all lanes
    for (int base = blockIdx.x * PT_THREADS; base < nrows; base += gridDim.x * PT_THREADS) {
        const int i = base + threadIdx.x;
        int len = 0;
        if (i < nrows && !(FILL && indptr[i + 1] - indptr[i] > PT_CAP)) {
            const int lo = rc_ptr[i], hi = rc_ptr[i + 1];
            bool over = false;
            for (int a = lo; a < hi && !over; ++a) {
                const int *cd = dofs + (size_t)(rc_code[a] / nloc) * nloc;
                for (int j = 0; j < nloc; ++j) {
                    const int d = cd[j];
                    if (d < 0) continue;
                    int b = len - 1, w = -1;   // b: the last entry <= d
                    while (b >= 0) {
                        w = buf[b * PT_THREADS];
                        if (w <= d) break;
                        --b;
                    }
                    if (b >= 0 && w == d) continue;
                    if (len == PT_CAP) { over = true; break; }
                    for (int c = len; c > b + 1; --c) buf[c * PT_THREADS] = buf[(c - 1) * PT_THREADS];
                    buf[(b + 1) * PT_THREADS] = d;
                    ++len;
                }
            }
            if (over) {
                // only the counting pass gets here: the warp kernel counts and later fills this row
                if (!FILL) list[atomicAdd(nlist, 1)] = i;
                len = 0;
            } else if (FILL) {
                int *out = indices + indptr[i];
                for (int c = 0; c < len; ++c) out[c] = buf[c * PT_THREADS];
            } else {
                rowlen[i] = len;
            }
        }
        if (!FILL) {
            const int m = __reduce_max_sync(0xffffffffu, len);
            if ((threadIdx.x & 31) == 0 && m) atomicMax(status + 2, m);
        }
    }
}

// ---- K1, long rows: one warp per listed row, bitonic sort in shared memory, unique ----------
static constexpr int PAT_WARPS = 4;
static constexpr int PAT_CAP = 1024;   // candidate columns per row (cells of the row x nloc, padded)

template <bool FILL>
__global__ void __launch_bounds__(PAT_WARPS * 32) k_pattern_rows(const int *__restrict__ dofs, int nloc,
                                                                  const int *__restrict__ rc_ptr,
                                                                  const int *__restrict__ rc_code,
                                                                  const int *__restrict__ list,
                                                                  const int *__restrict__ nlist,
                                                                  int *__restrict__ rowlen, const int *__restrict__ indptr,
                                                                  int *__restrict__ indices, int *__restrict__ status)
{
    __shared__ int sbuf[PAT_WARPS][PAT_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *buf = sbuf[w];
    const int nl = *nlist;
    for (int j = blockIdx.x * PAT_WARPS + w; j < nl; j += gridDim.x * PAT_WARPS) {
        const int i = list[j];
        const int lo = rc_ptr[i], ncell = rc_ptr[i + 1] - lo;
        const int m = ncell * nloc;
        int P = 32;
        while (P < m) P <<= 1;
        if (P > PAT_CAP) {
            if (lane == 0) { atomicOr(status, ST_ROW_TOO_LONG); atomicMin(status + 1, i); }
            if (!FILL) { if (lane == 0) rowlen[i] = 0; }
            continue;
        }
        for (int c = lane; c < P; c += 32) {
            int v = INT_MAX;
            if (c < m) {
                const int code = rc_code[lo + c / nloc];
                const int cell = code / nloc;
                const int d = dofs[(size_t)cell * nloc + (c % nloc)];
                v = d >= 0 ? d : INT_MAX;
            }
            buf[c] = v;
        }
        __syncwarp();
        for (int k = 2; k <= P; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int t = lane; t < P; t += 32) {
                    const int u = t ^ j;
                    if (u > t) {
                        const int a = buf[t], b = buf[u];
                        const bool up = (t & k) == 0;
                        if ((a > b) == up) { buf[t] = b; buf[u] = a; }
                    }
                }
                __syncwarp();
            }
        int base = FILL ? indptr[i] : 0;
        int count = 0;
        for (int t0 = 0; t0 < P; t0 += 32) {
            const int t = t0 + lane;
            const int v = buf[t];
            const bool keep = v != INT_MAX && (t == 0 || buf[t - 1] != v);
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (FILL && keep) indices[base + count + __popc(bal & ((1u << lane) - 1u))] = v;
            count += __popc(bal);
        }
        if (!FILL && lane == 0) { rowlen[i] = count; atomicMax(status + 2, count); }
        __syncwarp();
    }
}

__global__ void k_diag_pos(const int *__restrict__ indptr, const int *__restrict__ indices, int nrows, int ncols,
                           int *__restrict__ diag, int *__restrict__ missing)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    int lo = indptr[i], hi = indptr[i + 1];
    const int end = hi;
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (indices[mid] < i) lo = mid + 1; else hi = mid;
    }
    diag[i] = (i < ncols && lo < end && indices[lo] == i) ? lo : -1;
    if (diag[i] < 0 && missing) atomicAdd(missing, 1);
}

// ---- K2: scatter map ------------------------------------------------------------------------
__global__ void k_scatter_map(const int *__restrict__ dofs, long long ne_nloc, int nloc, const int *__restrict__ indptr,
                              const int *__restrict__ indices, int *__restrict__ map, int *__restrict__ status)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ne_nloc; t += (long long)gridDim.x * blockDim.x) {
        const long long e = t / nloc;
        const int *d = dofs + e * nloc;
        int *out = map + t * nloc;
        const int I = dofs[t];
        if (I < 0) {
            for (int j = 0; j < nloc; ++j) out[j] = -1;
            continue;
        }
        const int rlo = indptr[I], rhi = indptr[I + 1];
        for (int j = 0; j < nloc; ++j) {
            const int J = d[j];
            int pos = -1;
            if (J >= 0) {
                int lo = rlo, hi = rhi;
                while (lo < hi) {
                    const int mid = lo + ((hi - lo) >> 1);
                    if (indices[mid] < J) lo = mid + 1; else hi = mid;
                }
                if (lo < rhi && indices[lo] == J) pos = lo;
                else atomicOr(status, ST_OUTSIDE);
            }
            out[j] = pos;
        }
    }
}

int build_scatter_map(femd_ctx ctx, femd_pattern p)
{
    if (p->map.p) return FEMD_OK;
    if (p->cell_dofs.p == nullptr) {
        set_error("scatter map: the pattern was not built from cells");
        return FEMD_EINVAL;
    }
    const long long tot = (long long)p->ncells * p->nloc;
    FEMD_TRY(p->map.alloc((size_t)tot * p->nloc));
    FEMD_TRY(reset_status(ctx));
    if (tot > 0)
        k_scatter_map<<<grid_for((size_t)tot, 256, 1u << 20), 256, 0, counted(ctx->stream)>>>(
            p->cell_dofs.p, tot, p->nloc, p->indptr.p, p->indices.p, p->map.p, ctx->status_dev);
    FEMD_TRY_CUDA(cudaGetLastError());
    int flags = 0;
    FEMD_TRY(read_status(ctx, &flags, nullptr));
    if (flags & ST_OUTSIDE) {
        p->map.release();
        set_error("assemble_matrix_2d: entry outside the pattern");
        return FEMD_EOUTSIDE;
    }
    return FEMD_OK;
}

}  // namespace femd

using namespace femd;

static femd_pattern as_pattern(void *h)
{
    femd_pattern p = static_cast<femd_pattern>(h);
    return (p && p->kind == KIND_PATTERN) ? p : nullptr;
}

extern "C" {

int femd_cuda_pattern_from_cells(femd_ctx ctx, int nrows, int ncells, int nloc, const int *cell_dofs_dev, femd_pattern *out)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && out, "cell_pattern: ctx and out must not be NULL");
    FEMD_CHECK_ARG(nrows >= 0 && ncells >= 0, "cell_pattern: negative size");
    FEMD_CHECK_ARG(nloc >= 1 && nloc <= 64, "cell_pattern: nloc must be in 1..64");
    FEMD_CHECK_ARG(ncells == 0 || cell_dofs_dev, "cell_pattern: cell_dofs is NULL");
    *out = nullptr;
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    femd_pattern p = new femd_pattern_s();
    p->ctx = ctx;
    ctx_retain(ctx);
    p->nrows = p->ncols = nrows;
    p->ncells = ncells;
    p->nloc = nloc;
    auto fail = [&](int st) { delete p; return st; };
    const long long tot = (long long)ncells * nloc;
    int st;
    if ((st = p->cell_dofs.alloc((size_t)tot)) != FEMD_OK) return fail(st);
    if (tot) {
        cudaError_t e = cudaMemcpyAsync(p->cell_dofs.p, cell_dofs_dev, (size_t)tot * sizeof(int), cudaMemcpyDefault, s);
        if (e != cudaSuccess) { set_error(std::string("cell_pattern: copy of cell_dofs: ") + cudaGetErrorString(e)); return fail(FEMD_ECUDA); }
    }
    DevBuf<int> cnt, tmp, fill, rowlen;
    DevBuf<int> maxc;
    if ((st = cnt.alloc((size_t)nrows + 1)) || (st = tmp.alloc(scan_tmp_ints((size_t)nrows + 1))) ||
        (st = p->rc_ptr.alloc((size_t)nrows + 1)) || (st = p->indptr.alloc((size_t)nrows + 1)) ||
        (st = fill.alloc((size_t)nrows + 1)) || (st = rowlen.alloc((size_t)nrows + 1)) || (st = maxc.alloc(3)))
        return fail(st);
    if ((st = reset_status(ctx))) return fail(st);
    cudaMemsetAsync(cnt.p, 0, ((size_t)nrows + 1) * sizeof(int), s);
    // the most cells of a row, the rows without a diagonal, the rows on the long-row list
    cudaMemsetAsync(maxc.p, 0, 3 * sizeof(int), s);
    if (tot) k_count_rows<<<grid_for((size_t)tot, 256, 1u << 20), 256, 0, counted(s)>>>(p->cell_dofs.p, tot, nrows, cnt.p, ctx->status_dev);
    if ((st = exclusive_scan_int(cnt.p, p->rc_ptr.p, (size_t)nrows + 1, tmp.p, s))) return fail(st);
    int flags = 0;
    if ((st = read_status(ctx, &flags, nullptr))) return fail(st);
    if (flags & ST_BADDOF) { set_error("cell_pattern: a cell dof is >= nrows"); return fail(FEMD_EINVAL); }
    int total_rc = 0;
    cudaError_t e = cudaMemcpyAsync(&ctx->status_host[2], p->rc_ptr.p + nrows, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(std::string("cell_pattern: ") + cudaGetErrorString(e)); return fail(FEMD_ECUDA); }
    total_rc = ctx->status_host[2];
    if ((st = p->rc_code.alloc((size_t)total_rc + 1))) return fail(st);
    cudaMemcpyAsync(fill.p, p->rc_ptr.p, ((size_t)nrows + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s);
    if (tot) k_fill_rows<<<grid_for((size_t)tot, 256, 1u << 20), 256, 0, counted(s)>>>(p->cell_dofs.p, tot, nrows, nloc, fill.p, p->rc_code.p);
    if (nrows) k_sort_rows<<<grid_for((size_t)nrows, 256), 256, 0, counted(s)>>>(p->rc_ptr.p, p->rc_code.p, nrows, maxc.p);
    // K1: row lengths, scan, fill. Rows of up to PT_CAP columns take a thread each; the longer
    // ones go on a list (in `fill`, free again by now) that a warp per row takes.
    cudaMemsetAsync(rowlen.p + nrows, 0, sizeof(int), s);
    const unsigned tgrid = grid_for((size_t)nrows, PT_THREADS, 1u << 20);
    const unsigned lgrid = std::min(grid_for((size_t)nrows, PAT_WARPS, 1u << 20), 1184u);
    int *const long_rows = fill.p, *const nlong = maxc.p + 2;
    if (nrows) {
        k_pattern_rows_t<false><<<tgrid, PT_THREADS, 0, counted(s)>>>(p->cell_dofs.p, nloc, p->rc_ptr.p, p->rc_code.p, nrows,
                                                                     rowlen.p, nullptr, nullptr, long_rows, nlong,
                                                                     ctx->status_dev);
        k_pattern_rows<false><<<lgrid, PAT_WARPS * 32, 0, counted(s)>>>(p->cell_dofs.p, nloc, p->rc_ptr.p, p->rc_code.p,
                                                                long_rows, nlong, rowlen.p, nullptr, nullptr,
                                                                ctx->status_dev);
    }
    if ((st = exclusive_scan_int(rowlen.p, p->indptr.p, (size_t)nrows + 1, tmp.p, s))) return fail(st);
    int nnz = 0;
    e = cudaMemcpyAsync(&ctx->status_host[2], p->indptr.p + nrows, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(std::string("cell_pattern: ") + cudaGetErrorString(e)); return fail(FEMD_ECUDA); }
    nnz = ctx->status_host[2];
    int bad = 0;
    if ((st = read_status(ctx, &flags, &bad))) return fail(st);
    p->max_row_len = ctx->status_host[2];
    if (flags & ST_ROW_TOO_LONG) {
        set_error("cell_pattern: row " + std::to_string(bad) + " couples more than " + std::to_string(PAT_CAP) +
                  " cell dofs (too many cells around one node)");
        return fail(FEMD_EINVAL);
    }
    p->nnz = nnz;
    if ((st = p->indices.alloc((size_t)nnz + 1))) return fail(st);
    if (nrows) {
        k_pattern_rows_t<true><<<tgrid, PT_THREADS, 0, counted(s)>>>(p->cell_dofs.p, nloc, p->rc_ptr.p, p->rc_code.p, nrows,
                                                                    nullptr, p->indptr.p, p->indices.p, nullptr, nullptr,
                                                                    ctx->status_dev);
        k_pattern_rows<true><<<lgrid, PAT_WARPS * 32, 0, counted(s)>>>(p->cell_dofs.p, nloc, p->rc_ptr.p, p->rc_code.p,
                                                               long_rows, nlong, nullptr, p->indptr.p, p->indices.p,
                                                               ctx->status_dev);
    }
    if ((st = p->diag_pos.alloc((size_t)nrows + 1))) return fail(st);
    if (nrows)
        k_diag_pos<<<grid_for((size_t)nrows, 256), 256, 0, counted(s)>>>(p->indptr.p, p->indices.p, nrows, nrows, p->diag_pos.p,
                                                                          maxc.p + 1);
    e = cudaGetLastError();
    if (e != cudaSuccess) { set_error(std::string("cell_pattern: ") + cudaGetErrorString(e)); return fail(FEMD_ECUDA); }
    e = cudaMemcpyAsync(&ctx->status_host[2], maxc.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(std::string("cell_pattern: ") + cudaGetErrorString(e)); return fail(FEMD_ECUDA); }
    p->max_row_cells = ctx->status_host[2];
    p->all_diag = ctx->status_host[3] == 0;
    *out = p;
    return FEMD_OK;
}

int femd_cuda_pattern_from_csr_host(femd_ctx ctx, int nrows, int ncols, const int *indptr_host, const int *indices_host,
                                    femd_pattern *out)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && out && indptr_host, "pattern_from_csr: NULL argument");
    FEMD_CHECK_ARG(nrows >= 0 && ncols >= 0, "pattern_from_csr: negative size");
    *out = nullptr;
    const int nnz = indptr_host[nrows];
    FEMD_CHECK_ARG(indptr_host[0] == 0 && nnz >= 0, "CSRMatrix: indptr must start at 0");
    bool all_diag = nrows == ncols;
    for (int i = 0; i < nrows; ++i) {
        FEMD_CHECK_ARG(indptr_host[i + 1] >= indptr_host[i], "CSRMatrix: indptr must be non-decreasing");
        bool has = false;
        for (int q = indptr_host[i]; q < indptr_host[i + 1] && !has; ++q) has = indices_host[q] == i;
        all_diag = all_diag && has;
        for (int q = indptr_host[i] + 1; q < indptr_host[i + 1]; ++q)
            FEMD_CHECK_ARG(indices_host[q] > indices_host[q - 1],
                           "CSRMatrix.from_arrays: column indices must be sorted (call sort_indices())");
        if (indptr_host[i + 1] > indptr_host[i])
            FEMD_CHECK_ARG(indices_host[indptr_host[i]] >= 0 && indices_host[indptr_host[i + 1] - 1] < ncols,
                           "CSRMatrix: column index out of range");
    }
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    femd_pattern p = new femd_pattern_s();
    p->ctx = ctx;
    ctx_retain(ctx);
    p->nrows = nrows;
    p->ncols = ncols;
    p->nnz = nnz;
    p->all_diag = all_diag;
    int st;
    if ((st = p->indptr.alloc((size_t)nrows + 1)) || (st = p->indices.alloc((size_t)nnz + 1)) ||
        (st = p->diag_pos.alloc((size_t)nrows + 1))) { delete p; return st; }
    cudaError_t e = cudaMemcpyAsync(p->indptr.p, indptr_host, ((size_t)nrows + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && nnz)
        e = cudaMemcpyAsync(p->indices.p, indices_host, (size_t)nnz * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && nrows) {
        k_diag_pos<<<grid_for((size_t)nrows, 256), 256, 0, counted(ctx->stream)>>>(p->indptr.p, p->indices.p, nrows, ncols, p->diag_pos.p,
                                                                                      nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { set_error(std::string("pattern_from_csr: ") + cudaGetErrorString(e)); delete p; return FEMD_ECUDA; }
    *out = p;
    return FEMD_OK;
}

int femd_cuda_pattern_info(femd_pattern p, int *nrows, int *ncols, long long *nnz)
{
    clear_error();
    p = as_pattern(p);
    FEMD_CHECK_ARG(p, "pattern_info: not a pattern handle");
    if (nrows) *nrows = p->nrows;
    if (ncols) *ncols = p->ncols;
    if (nnz) *nnz = p->nnz;
    return FEMD_OK;
}

int femd_cuda_pattern_arrays(femd_pattern p, const int **indptr_dev, const int **indices_dev)
{
    clear_error();
    p = as_pattern(p);
    FEMD_CHECK_ARG(p, "pattern_arrays: not a pattern handle");
    if (indptr_dev) *indptr_dev = p->indptr.p;
    if (indices_dev) *indices_dev = p->indices.p;
    return FEMD_OK;
}

int femd_cuda_pattern_to_host(femd_pattern p, int *indptr_host, int *indices_host)
{
    clear_error();
    p = as_pattern(p);
    FEMD_CHECK_ARG(p, "pattern_to_host: not a pattern handle");
    FEMD_TRY_CUDA(cudaSetDevice(p->ctx->device));
    cudaStream_t s = p->ctx->stream;
    if (indptr_host)
        FEMD_TRY_CUDA(cudaMemcpyAsync(indptr_host, p->indptr.p, ((size_t)p->nrows + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (indices_host && p->nnz)
        FEMD_TRY_CUDA(cudaMemcpyAsync(indices_host, p->indices.p, (size_t)p->nnz * sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    return FEMD_OK;
}

int femd_cuda_scatter_map(femd_ctx ctx, femd_pattern p, int *map_dev)
{
    clear_error();
    p = as_pattern(p);
    FEMD_CHECK_ARG(ctx && p, "scatter_map: NULL argument");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    FEMD_TRY(build_scatter_map(ctx, p));
    if (map_dev && p->map.n)
        FEMD_TRY_CUDA(cudaMemcpyAsync(map_dev, p->map.p, p->map.n * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
    return FEMD_OK;
}

int femd_cuda_pattern_map(femd_pattern p, const int **map_dev)
{
    clear_error();
    p = as_pattern(p);
    FEMD_CHECK_ARG(p && map_dev, "pattern_map: NULL argument");
    FEMD_TRY(build_scatter_map(p->ctx, p));
    *map_dev = p->map.p;
    return FEMD_OK;
}

}  // extern "C"
