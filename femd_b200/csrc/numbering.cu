// numbering.cu -- continuous P_k dof numbering on the device, the same map as the host's
// femd_host_lagrange_numbering (include/femd/fe/space_2d.hpp:390-526): global edges numbered by
// their first appearance over (cell, local edge i), edge i running from local vertex (i+1)%3 to
// (i+2)%3; vertex dofs, then k-1 nodes per edge (reversed when the edge runs from the larger
// vertex index to the smaller), then the interior nodes cell by cell; with all_exterior every
// node of an edge met once is eliminated (-1) and the rest are renumbered in raw order.
//
// The host sorts the half-edges by (edge key, c 3 + i).  Here the same order comes from a
// counting sort by the smaller vertex (a bucket per vertex) and a sort of each bucket by (larger
// vertex, c 3 + i) -- buckets are a vertex's edges, a handful -- so no general sort is needed:
//   cnt, bptr     3 ncells half-edges counted per smaller vertex, bucket offsets by a scan
//   hs_hi, hs_val the half-edges grouped by bucket, each bucket sorted (larger vertex, c 3 + i)
//   first         1 at the half-edge that appears first for its edge; its scan ranks the edges
//   cell_edge     per half-edge (c 3 + i): the global edge; exterior: met once
//   keep          per raw node: 1 unless eliminated; its scan renumbers the kept nodes
#include <algorithm>
#include <climits>
#include <string>

#include "common.cuh"

namespace femd {

static constexpr int NB_BADVERT = 1, NB_NONMANIFOLD = 2;
static constexpr int MAX_BUCKET = 512;   // half-edges whose smaller vertex is one vertex

// ends of half-edge t = c 3 + i: local vertices (i+1)%3 and (i+2)%3 of cell c
__device__ __forceinline__ void half_ends(const int *tris, long long t, int &a, int &b)
{
    const long long c = t / 3;
    const int i = (int)(t - 3 * c);
    a = tris[3 * c + (i + 1) % 3];
    b = tris[3 * c + (i + 2) % 3];
}

__global__ void k_half_count(const int *__restrict__ tris, long long nh, int nverts, int *__restrict__ cnt, int *status)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += (long long)gridDim.x * blockDim.x) {
        int a, b;
        half_ends(tris, t, a, b);
        if (a < 0 || a >= nverts || b < 0 || b >= nverts) {
            atomicOr(status, NB_BADVERT);
            continue;
        }
        atomicAdd(&cnt[min(a, b)], 1);
    }
}

__global__ void k_half_fill(const int *__restrict__ tris, long long nh, int nverts, const int *__restrict__ bptr,
                            int *__restrict__ fill, int *__restrict__ hs_hi, int *__restrict__ hs_val)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += (long long)gridDim.x * blockDim.x) {
        int a, b;
        half_ends(tris, t, a, b);
        if (a < 0 || a >= nverts || b < 0 || b >= nverts) continue;
        const int lo = min(a, b);
        const int pos = bptr[lo] + atomicAdd(&fill[lo], 1);
        hs_hi[pos] = max(a, b);
        hs_val[pos] = (int)t;
    }
}

__global__ void k_max_bucket(const int *__restrict__ cnt, int n, int *out)
{
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, cnt[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// per bucket (at most MAX_BUCKET half-edges): insertion sort by (larger vertex, half-edge), then
// first-appearance flags; a key met more than twice marks the mesh non-manifold
__global__ void k_bucket_sort(const int *__restrict__ bptr, int nverts, int *__restrict__ hs_hi, int *__restrict__ hs_val,
                              int *__restrict__ first, int *status)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nverts) return;
    const int p0 = bptr[v], p1 = bptr[v + 1];
    for (int p = p0 + 1; p < p1; ++p) {
        const int h = hs_hi[p], w = hs_val[p];
        int q = p - 1;
        while (q >= p0 && (hs_hi[q] > h || (hs_hi[q] == h && hs_val[q] > w))) {
            hs_hi[q + 1] = hs_hi[q];
            hs_val[q + 1] = hs_val[q];
            --q;
        }
        hs_hi[q + 1] = h;
        hs_val[q + 1] = w;
    }
    for (int p = p0; p < p1;) {
        int e = p + 1;
        while (e < p1 && hs_hi[e] == hs_hi[p]) ++e;
        if (e - p > 2) atomicOr(status, NB_NONMANIFOLD);
        first[hs_val[p]] = 1;
        p = e;
    }
}

// per bucket: every half-edge gets its edge (the rank of its key's first half-edge) and whether
// the edge is exterior (met once)
__global__ void k_bucket_edges(const int *__restrict__ bptr, int nverts, const int *__restrict__ hs_hi,
                               const int *__restrict__ hs_val, const int *__restrict__ rank, int *__restrict__ cell_edge,
                               unsigned char *__restrict__ exterior)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nverts) return;
    const int p0 = bptr[v], p1 = bptr[v + 1];
    for (int p = p0; p < p1;) {
        int e = p + 1;
        while (e < p1 && hs_hi[e] == hs_hi[p]) ++e;
        const int g = rank[hs_val[p]];
        for (int q = p; q < e; ++q) {
            cell_edge[hs_val[q]] = g;
            exterior[hs_val[q]] = e - p == 1;
        }
        p = e;
    }
}

__global__ void k_fill_int(int *__restrict__ a, long long n, int v)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) a[t] = v;
}

// the nodes of exterior edges (vertices and edge nodes) are eliminated
__global__ void k_eliminate(const int *__restrict__ tris, long long nh, const int *__restrict__ cell_edge,
                            const unsigned char *__restrict__ exterior, int de, long long voff, int *__restrict__ keep)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += (long long)gridDim.x * blockDim.x) {
        if (!exterior[t]) continue;
        int a, b;
        half_ends(tris, t, a, b);
        keep[a] = 0;
        keep[b] = 0;
        const long long g = cell_edge[t];
        for (int j = 0; j < de; ++j) keep[voff + g * de + j] = 0;
    }
}

// cell_dofs[c nloc + q]: the raw node of local node q (vertices, edge nodes in edge direction,
// interior nodes), then -1 if eliminated, else its rank among the kept nodes
__global__ void k_cell_dofs(const int *__restrict__ tris, long long ncells, int nloc, int de, int nint, long long voff,
                            long long nedges, const int *__restrict__ cell_edge, const int *__restrict__ keep,
                            const int *__restrict__ r2a, int *__restrict__ cell_dofs)
{
    const long long total = ncells * nloc;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long c = t / nloc;
        const int q = (int)(t - c * nloc);
        long long raw;
        if (q < 3) {
            raw = tris[3 * c + q];
        } else if (q < 3 + 3 * de) {
            const int i = (q - 3) / de, j = (q - 3) - i * de;
            const bool flip = tris[3 * c + (i + 1) % 3] > tris[3 * c + (i + 2) % 3];
            raw = voff + (long long)cell_edge[3 * c + i] * de + (flip ? de - 1 - j : j);
        } else {
            raw = voff + nedges * de + c * nint + (q - 3 - 3 * de);
        }
        cell_dofs[t] = keep[raw] ? r2a[raw] : -1;
    }
}

}  // namespace femd

using namespace femd;

extern "C" {

int femd_cuda_lagrange_numbering(femd_ctx ctx, int nverts, int ncells, const int *tris_dev, int k, int all_exterior,
                                 int *cell_dofs_dev, int *dim, int *raw_dim)
{
    clear_error();
    FEMD_CHECK_ARG(ctx, "lagrange_numbering: NULL context");
    FEMD_CHECK_ARG(k >= 1 && k <= 20, "LagrangeSpace2D: degree must be in 1..20");
    FEMD_CHECK_ARG(nverts >= 3 && ncells >= 1 && tris_dev && cell_dofs_dev && dim, "lagrange_numbering: bad arguments");
    FEMD_CHECK_ARG((long long)ncells * 3 < INT_MAX, "lagrange_numbering: more than 2^31 half-edges");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int nloc = (k + 1) * (k + 2) / 2, de = k - 1, nint = (k - 1) * (k - 2) / 2;
    const long long nh = 3LL * ncells;
    DevBuf<int> cnt, bptr, fill, hs_hi, hs_val, first, rank, cell_edge, tmp, status;
    DevBuf<unsigned char> exterior;
    if (int st = cnt.alloc((size_t)nverts + 1)) return st;
    if (int st = bptr.alloc((size_t)nverts + 1)) return st;
    if (int st = fill.alloc((size_t)nverts)) return st;
    if (int st = hs_hi.alloc((size_t)nh)) return st;
    if (int st = hs_val.alloc((size_t)nh)) return st;
    if (int st = first.alloc((size_t)nh)) return st;
    if (int st = rank.alloc((size_t)nh + 1)) return st;
    if (int st = cell_edge.alloc((size_t)nh)) return st;
    if (int st = exterior.alloc((size_t)nh)) return st;
    if (int st = status.alloc(2)) return st;
    if (int st = tmp.alloc(scan_tmp_ints((size_t)std::max<long long>(nh, nverts) + 1))) return st;
    FEMD_TRY_CUDA(cudaMemsetAsync(cnt.p, 0, ((size_t)nverts + 1) * sizeof(int), s));
    FEMD_TRY_CUDA(cudaMemsetAsync(fill.p, 0, (size_t)nverts * sizeof(int), s));
    FEMD_TRY_CUDA(cudaMemsetAsync(first.p, 0, (size_t)nh * sizeof(int), s));
    FEMD_TRY_CUDA(cudaMemsetAsync(status.p, 0, 2 * sizeof(int), s));
    const unsigned gh = grid_for((size_t)nh, 256, 4096);
    k_half_count<<<gh, 256, 0, counted(s)>>>(tris_dev, nh, nverts, cnt.p, status.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    k_max_bucket<<<grid_for((size_t)nverts, 256, 1024), 256, 0, counted(s)>>>(cnt.p, nverts, status.p + 1);
    FEMD_TRY_CUDA(cudaGetLastError());
    int st_host[2] = {0, 0};
    FEMD_TRY_CUDA(cudaMemcpyAsync(st_host, status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    FEMD_CHECK_ARG(!(st_host[0] & NB_BADVERT), "lagrange_numbering: vertex index out of range");
    FEMD_CHECK_ARG(st_host[1] <= MAX_BUCKET, "lagrange_numbering: a vertex is the smaller end of more than 512 edges "
                                             "(use the host numbering)");
    FEMD_TRY(exclusive_scan_int(cnt.p, bptr.p, (size_t)nverts + 1, tmp.p, s));   // cnt[nverts] = 0: bptr[nverts] = nh
    k_half_fill<<<gh, 256, 0, counted(s)>>>(tris_dev, nh, nverts, bptr.p, fill.p, hs_hi.p, hs_val.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    const unsigned gv = grid_for((size_t)nverts, 128);
    k_bucket_sort<<<gv, 128, 0, counted(s)>>>(bptr.p, nverts, hs_hi.p, hs_val.p, first.p, status.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaMemcpyAsync(st_host, status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    FEMD_CHECK_ARG(!(st_host[0] & NB_NONMANIFOLD), "lagrange_numbering: an edge is shared by more than two triangles");
    FEMD_TRY(exclusive_scan_int(first.p, rank.p, (size_t)nh, tmp.p, s));
    k_bucket_edges<<<gv, 128, 0, counted(s)>>>(bptr.p, nverts, hs_hi.p, hs_val.p, rank.p, cell_edge.p, exterior.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    int tail[2] = {0, 0};
    FEMD_TRY_CUDA(cudaMemcpyAsync(&tail[0], rank.p + nh - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(&tail[1], first.p + nh - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    const long long nedges = (long long)tail[0] + tail[1];
    const long long voff = nverts;
    const long long rd = voff + nedges * de + (long long)ncells * nint;
    FEMD_CHECK_ARG(rd <= 0x7fffffffLL - 1, "lagrange_numbering: more than 2^31 nodes");
    DevBuf<int> keep, r2a, tmp2;
    if (int st = keep.alloc((size_t)rd)) return st;
    if (int st = r2a.alloc((size_t)rd)) return st;
    if (int st = tmp2.alloc(scan_tmp_ints((size_t)rd))) return st;
    k_fill_int<<<grid_for((size_t)rd, 256, 4096), 256, 0, counted(s)>>>(keep.p, rd, 1);
    FEMD_TRY_CUDA(cudaGetLastError());
    if (all_exterior && nh) {
        k_eliminate<<<gh, 256, 0, counted(s)>>>(tris_dev, nh, cell_edge.p, exterior.p, de, voff, keep.p);
        FEMD_TRY_CUDA(cudaGetLastError());
    }
    FEMD_TRY(exclusive_scan_int(keep.p, r2a.p, (size_t)rd, tmp2.p, s));
    k_cell_dofs<<<grid_for((size_t)ncells * nloc, 256, 4096), 256, 0, counted(s)>>>(
        tris_dev, ncells, nloc, de, nint, voff, nedges, cell_edge.p, keep.p, r2a.p, cell_dofs_dev);
    FEMD_TRY_CUDA(cudaGetLastError());
    int last[2] = {0, 0};
    FEMD_TRY_CUDA(cudaMemcpyAsync(&last[0], r2a.p + rd - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(&last[1], keep.p + rd - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    *dim = last[0] + last[1];
    if (raw_dim) *raw_dim = (int)rd;
    return FEMD_OK;
}

}  // extern "C"
