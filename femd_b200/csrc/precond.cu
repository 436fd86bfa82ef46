// precond.cu -- the reference's stronger preconditioners on the GPU: ILU(0) and SSOR on the natural
// ordering (include/femd/sparse/precond.hpp:105-213), for CG (krylov::cg, krylov/cg.hpp:245-290).
//
// Both are sequential sweeps over the rows: ILU(0)'s factorization (IKJ: row i is eliminated with
// the finished rows k < i of its lower part) and the triangular solves of every application.  Row
// i depends only on the rows its lower (forward) or upper (backward) part names, so the rows fall
// into levels -- level(i) = 1 + the largest level among them -- and the rows of one level are
// independent.  The level schedules are built once per pattern on the host.  Each sweep then runs
// as ONE thread block that walks the levels in order with a block barrier between them: a thread
// takes a row and does that row's arithmetic exactly as the reference writes it (the same
// operations in the same order, no contraction), so the factors and every application are
// bit-identical to the reference's; only the order in which independent rows are done differs.
// No block waits on another, so nothing can hang.
//
// The price is parallelism: one SM per sweep, latency-bound by the number of levels (about 4 N
// for P2 on an N x N rectangle).  The reference's natural-order ILU(0) has no more parallelism to
// give; a faster preconditioner would be a different one (another ordering), with other iterates.
#include <algorithm>
#include <climits>
#include <cmath>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

struct femd_precond_s : femd::HandleBase {
    femd_ctx ctx = nullptr;
    femd_pattern pattern = nullptr;
    int pc_kind = 0;                     // FEMD_PC_ILU0 / FEMD_PC_SSOR
    double omega = 1.0, min_pivot = 0.0;
    int n = 0, nlf = 0, nlb = 0;
    femd::DevBuf<double> v;              // ILU(0): the factors L (unit, strict lower) and U; SSOR: the values
    femd::DevBuf<int> diag;              // position of (i, i)
    femd::DevBuf<int> frows, fptr, brows, bptr;   // rows by forward / backward level
    femd_precond_s() : HandleBase(femd::KIND_PRECOND) {}
    ~femd_precond_s() override { femd::ctx_release(ctx); }
};

namespace femd {

static constexpr int PC_BLOCK = 1024;

// ILU(0) factorization, the reference's IKJ loop per row (precond.hpp:172-186): for each k in the
// lower part of row i (increasing), v_ik /= v_kk, then v_ij -= v_ik v_kj over the upper part of
// row k where (i, j) is in the pattern (found by a merge of the two sorted rows).
__global__ void __launch_bounds__(PC_BLOCK) k_ilu0_factor(const int *__restrict__ ip, const int *__restrict__ ix,
                                                         const int *__restrict__ diag, double *__restrict__ v, int nl,
                                                         const int *__restrict__ lptr, const int *__restrict__ rows,
                                                         int *__restrict__ status)
{
    for (int L = 0; L < nl; ++L) {
        for (int t = lptr[L] + (int)threadIdx.x; t < lptr[L + 1]; t += PC_BLOCK) {
            const int i = rows[t];
            const int hi = ip[i + 1], di = diag[i];
            for (int p = ip[i]; p < di; ++p) {
                const int k = ix[p];
                const double lik = __ddiv_rn(v[p], v[diag[k]]);
                v[p] = lik;
                int s = p + 1;                                   // columns of row i after k (sorted)
                for (int q = diag[k] + 1; q < ip[k + 1]; ++q) {
                    const int j = ix[q];
                    while (s < hi && ix[s] < j) ++s;
                    if (s < hi && ix[s] == j) v[s] = __dsub_rn(v[s], __dmul_rn(lik, v[q]));
                }
            }
            if (v[di] == 0.0) atomicMin(status, i);
        }
        __syncthreads();                                         // the level's rows are final
    }
}

// forward sweep: ILU(0) z_i = r_i - sum_{p < d_i} v_p z_col (precond.hpp:193-198); SSOR
// z_i = (r_i - sum ...) w / v_ii (:127-132)
template <bool SSOR>
__global__ void __launch_bounds__(PC_BLOCK) k_pc_forward(const int *__restrict__ ip, const int *__restrict__ ix,
                                                        const int *__restrict__ diag, const double *__restrict__ v, int nl,
                                                        const int *__restrict__ lptr, const int *__restrict__ rows,
                                                        double w, const double *__restrict__ r, double *__restrict__ z,
                                                        const int *__restrict__ skip)
{
    if (skip && *skip) return;
    for (int L = 0; L < nl; ++L) {
        for (int t = lptr[L] + (int)threadIdx.x; t < lptr[L + 1]; t += PC_BLOCK) {
            const int i = rows[t];
            double s = r[i];
            const int di = diag[i];
            for (int p = ip[i]; p < di; ++p) s = __dsub_rn(s, __dmul_rn(v[p], z[ix[p]]));
            z[i] = SSOR ? __ddiv_rn(__dmul_rn(s, w), v[di]) : s;
        }
        __syncthreads();
    }
}

// SSOR's middle step, z_i *= c v_ii / w with c = (2 - w) / w (precond.hpp:134-135)
__global__ void k_ssor_scale(int n, const int *__restrict__ diag, const double *__restrict__ v, double w,
                             double *__restrict__ z, const int *__restrict__ skip)
{
    if (skip && *skip) return;
    const double c = __ddiv_rn(__dsub_rn(2.0, w), w);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        z[i] = __dmul_rn(z[i], __ddiv_rn(__dmul_rn(c, v[diag[i]]), w));
}

// backward sweep: z_i = (z_i - sum_{p > d_i} v_p z_col) / v_ii (ILU(0), :199-204) or * w / v_ii
// (SSOR, :137-142)
template <bool SSOR>
__global__ void __launch_bounds__(PC_BLOCK) k_pc_backward(const int *__restrict__ ip, const int *__restrict__ ix,
                                                         const int *__restrict__ diag, const double *__restrict__ v, int nl,
                                                         const int *__restrict__ lptr, const int *__restrict__ rows,
                                                         double w, double *__restrict__ z, const int *__restrict__ skip)
{
    if (skip && *skip) return;
    for (int L = 0; L < nl; ++L) {
        for (int t = lptr[L] + (int)threadIdx.x; t < lptr[L + 1]; t += PC_BLOCK) {
            const int i = rows[t];
            const int di = diag[i];
            double s = z[i];
            for (int p = di + 1; p < ip[i + 1]; ++p) s = __dsub_rn(s, __dmul_rn(v[p], z[ix[p]]));
            z[i] = SSOR ? __ddiv_rn(__dmul_rn(s, w), v[di]) : __ddiv_rn(s, v[di]);
        }
        __syncthreads();
    }
}

__global__ void k_pc_min_diag(int n, const int *__restrict__ diag, const double *__restrict__ v, double *out)
{
    __shared__ double sh[32];
    double m = INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmin(m, v[diag[i]]);
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = INFINITY;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = fmin(r, sh[k]);
        *out = r;
    }
}

// rows grouped by level: level(i) = 1 + max level over the rows that row i reads (its lower part
// for the forward sweep, its upper part for the backward one, taken from the last row down)
static void level_schedule(int n, const std::vector<int> &ip, const std::vector<int> &ix, const std::vector<int> &dg,
                           bool forward, std::vector<int> &rows, std::vector<int> &ptr)
{
    std::vector<int> lev((size_t)n, 0);
    int nl = 0;
    for (int s = 0; s < n; ++s) {
        const int i = forward ? s : n - 1 - s;
        int l = 0;
        if (forward)
            for (int p = ip[i]; p < dg[i]; ++p) l = std::max(l, lev[ix[p]] + 1);
        else
            for (int p = dg[i] + 1; p < ip[i + 1]; ++p) l = std::max(l, lev[ix[p]] + 1);
        lev[i] = l;
        nl = std::max(nl, l + 1);
    }
    ptr.assign((size_t)nl + 1, 0);
    for (int i = 0; i < n; ++i) ++ptr[lev[i] + 1];
    for (int l = 0; l < nl; ++l) ptr[l + 1] += ptr[l];
    rows.assign((size_t)n, 0);
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < n; ++i) rows[fill[lev[i]]++] = i;
}

static femd_precond_s *as_precond(void *h)
{
    femd_precond_s *p = static_cast<femd_precond_s *>(h);
    return (p && p->kind == KIND_PRECOND) ? p : nullptr;
}

// z = M^{-1} r on the stream, every kernel skipped when *skip is set (a finished CG loop)
int precond_enqueue(femd_precond P, const double *r, double *z, const int *skip, cudaStream_t s)
{
    femd_pattern Q = P->pattern;
    const int *ip = Q->indptr.p, *ix = Q->indices.p;
    if (P->n == 0) return FEMD_OK;
    if (P->pc_kind == FEMD_PC_ILU0) {
        k_pc_forward<false><<<1, PC_BLOCK, 0, counted(s)>>>(ip, ix, P->diag.p, P->v.p, P->nlf, P->fptr.p, P->frows.p, 1.0, r, z,
                                                           skip);
        k_pc_backward<false><<<1, PC_BLOCK, 0, counted(s)>>>(ip, ix, P->diag.p, P->v.p, P->nlb, P->bptr.p, P->brows.p, 1.0, z,
                                                            skip);
    } else {
        k_pc_forward<true><<<1, PC_BLOCK, 0, counted(s)>>>(ip, ix, P->diag.p, P->v.p, P->nlf, P->fptr.p, P->frows.p, P->omega,
                                                          r, z, skip);
        k_ssor_scale<<<grid_for((size_t)P->n, 256, 1u << 16), 256, 0, counted(s)>>>(P->n, P->diag.p, P->v.p, P->omega, z, skip);
        k_pc_backward<true><<<1, PC_BLOCK, 0, counted(s)>>>(ip, ix, P->diag.p, P->v.p, P->nlb, P->bptr.p, P->brows.p,
                                                           P->omega, z, skip);
    }
    FEMD_TRY_CUDA(cudaGetLastError());
    return FEMD_OK;
}

int precond_rows(femd_precond P) { return P->n; }
femd_ctx precond_ctx(femd_precond P) { return P->ctx; }
femd_pattern precond_pattern(femd_precond P) { return P->pattern; }

}  // namespace femd

using namespace femd;

extern "C" {

int femd_cuda_precond_create(femd_ctx ctx, femd_matrix K, int kind, double omega, femd_precond *out)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && K && K->kind == KIND_MATRIX && out, "preconditioner: NULL argument");
    FEMD_CHECK_ARG(kind == FEMD_PC_ILU0 || kind == FEMD_PC_SSOR, "preconditioner: kind is FEMD_PC_ILU0 or FEMD_PC_SSOR");
    const char *what = kind == FEMD_PC_ILU0 ? "ILU(0)" : "SSOR";
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, std::string(what) + ": the matrix must be square");
    FEMD_CHECK_ARG(kind != FEMD_PC_SSOR || (omega > 0.0 && omega < 2.0), "SSOR: omega must lie in (0, 2)");
    *out = nullptr;
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    femd_pattern Q = K->pattern;
    const int n = Q->nrows;
    const long long nnz = Q->nnz;
    // the pattern and the diagonal positions on the host (precond.hpp:68-78: a missing or zero
    // diagonal entry is refused)
    std::vector<int> ip((size_t)n + 1), ix((size_t)std::max<long long>(nnz, 1)), dg((size_t)std::max(n, 1));
    std::vector<double> vals((size_t)std::max<long long>(nnz, 1));
    FEMD_TRY_CUDA(cudaMemcpyAsync(ip.data(), Q->indptr.p, ((size_t)n + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (nnz) {
        FEMD_TRY_CUDA(cudaMemcpyAsync(ix.data(), Q->indices.p, (size_t)nnz * sizeof(int), cudaMemcpyDeviceToHost, s));
        FEMD_TRY_CUDA(cudaMemcpyAsync(vals.data(), K->data.p, (size_t)nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < n; ++i) {
        const int *b = ix.data() + ip[i], *e = ix.data() + ip[i + 1];
        const int *f = std::lower_bound(b, e, i);
        dg[i] = (f != e && *f == i) ? (int)(f - ix.data()) : -1;
        FEMD_CHECK_ARG(dg[i] >= 0 && vals[dg[i]] != 0.0, std::string(what) + ": zero diagonal entry in row " + std::to_string(i));
    }
    auto P = new femd_precond_s();
    std::unique_ptr<femd_precond_s> guard(P);
    P->ctx = ctx;
    ctx_retain(ctx);
    P->pattern = Q;
    P->pc_kind = kind;
    P->omega = omega;
    P->n = n;
    std::vector<int> fr, fp, br, bp;
    level_schedule(n, ip, ix, dg, true, fr, fp);
    level_schedule(n, ip, ix, dg, false, br, bp);
    P->nlf = (int)fp.size() - 1;
    P->nlb = (int)bp.size() - 1;
    int st;
    if ((st = P->v.alloc((size_t)std::max<long long>(nnz, 1))) || (st = P->diag.alloc((size_t)std::max(n, 1))) ||
        (st = P->frows.alloc((size_t)std::max(n, 1))) || (st = P->fptr.alloc(fp.size())) ||
        (st = P->brows.alloc((size_t)std::max(n, 1))) || (st = P->bptr.alloc(bp.size())))
        return st;
    if (nnz) FEMD_TRY_CUDA(cudaMemcpyAsync(P->v.p, K->data.p, (size_t)nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (n) {
        FEMD_TRY_CUDA(cudaMemcpyAsync(P->diag.p, dg.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
        FEMD_TRY_CUDA(cudaMemcpyAsync(P->frows.p, fr.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
        FEMD_TRY_CUDA(cudaMemcpyAsync(P->brows.p, br.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    FEMD_TRY_CUDA(cudaMemcpyAsync(P->fptr.p, fp.data(), fp.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(P->bptr.p, bp.data(), bp.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    if (kind == FEMD_PC_ILU0 && n) {
        FEMD_TRY(reset_status(ctx));
        // status [1] holds the first row with a zero pivot (INT_MAX: none)
        k_ilu0_factor<<<1, PC_BLOCK, 0, counted(s)>>>(Q->indptr.p, Q->indices.p, P->diag.p, P->v.p, P->nlf, P->fptr.p, P->frows.p,
                                                       ctx->status_dev + 1);
        FEMD_TRY_CUDA(cudaGetLastError());
        int flags = 0, bad = 0;
        FEMD_TRY(read_status(ctx, &flags, &bad));
        if (bad != INT_MAX) {
            set_error("ILU(0): zero pivot in row " + std::to_string(bad));
            return FEMD_EPIVOT;
        }
        DevBuf<double> mp;
        FEMD_TRY(mp.alloc(1));
        k_pc_min_diag<<<1, 1024, 0, counted(s)>>>(n, P->diag.p, P->v.p, mp.p);
        FEMD_TRY_CUDA(cudaGetLastError());
        FEMD_TRY_CUDA(cudaMemcpyAsync(&P->min_pivot, mp.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // the host vectors are released on return
    *out = reinterpret_cast<femd_precond>(guard.release());
    return FEMD_OK;
}

int femd_cuda_precond_info(femd_precond handle, int *kind, int *levels_forward, int *levels_backward, double *min_pivot)
{
    clear_error();
    femd_precond_s *P = as_precond(handle);
    FEMD_CHECK_ARG(P, "preconditioner: not a preconditioner handle");
    if (kind) *kind = P->pc_kind;
    if (levels_forward) *levels_forward = P->nlf;
    if (levels_backward) *levels_backward = P->nlb;
    if (min_pivot) *min_pivot = P->pc_kind == FEMD_PC_ILU0 ? P->min_pivot : 0.0;
    return FEMD_OK;
}

int femd_cuda_precond_apply(femd_ctx ctx, femd_precond handle, const double *r_dev, double *z_dev)
{
    clear_error();
    femd_precond_s *P = as_precond(handle);
    FEMD_CHECK_ARG(ctx && P && (P->n == 0 || (r_dev && z_dev)), "preconditioner: bad arguments");
    FEMD_CHECK_ARG(r_dev != z_dev || P->n == 0, "preconditioner: r and z must be separate vectors");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    return precond_enqueue(P, r_dev, z_dev, nullptr, ctx->stream);
}

}  // extern "C"
