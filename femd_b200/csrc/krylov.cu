// krylov.cu -- K5: CSR SpMV (sub-warp per row) fused with p^T A p; K6: the fused Jacobi-PCG
// update (x += a p, r -= a Ap, ||r||^2 and r^T D^-1 r in one pass) and direction update; the
// whole CG loop runs on the device with no host round trip per iteration.
//
// Reference: krylov::cg_jacobi (include/femd/krylov/cg.hpp:296-350), cg_update_chunk_jacobi
// (:99-171), detail_cg::finish (:222-237), CSRMatrix::apply (include/femd/sparse/csr.hpp:203-215).
//
// Reductions.  Every kernel that produces a dot product writes one partial per block; the
// last block to finish (an atomic ticket, no waiting) adds the partials in block order and
// updates the scalar state (alpha, beta, the stopping test).  The grid of each kernel depends
// only on n, so the sums -- and the iterates -- have the same bits on every run.  Kernels of an
// iteration that starts after the stopping test has fired return at once, so whole chunks of
// iterations are queued (captured in a CUDA graph) and the host only polls between chunks.
//
// HBM bytes per FP64 iteration (n rows, nnz entries): SpMV 12 nnz + 4 (n+1) + 8 n (p) + 8 n (Ap);
// update 40 n read + 16 n written; direction 24 n read + 8 n written.
#include <climits>
#include <type_traits>
#include <cmath>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace femd {

static constexpr int RED_BLOCK = 256;

template <class T>
struct CGState {
    double rz, pAp, alpha, beta, rr;       // scalars and dot products in FP64 for both precisions
    double nb, tol_nb, rn, res64;          // FP64 scalars (norms of b and of the true residual)
    double maxr;                           // mixed precision: largest ||r|| since the last reliable update
    double rz_prev;                        // mixed precision: r.z before the last recurrence step
    int it, done, breakdown, max_iter;
    int want_ru, ru_count;
    // mixed precision: the true residual of the last reliable update, the updates in a row that
    // reduced it by less than 2x, and the switch to FP64 after two of them (or a non-finite one)
    double prt;
    int stall, fallback;
    unsigned ticket;
};

// block reduction of NV values per thread into smem[v][0]; deterministic (fixed tree)
template <class T, int NV>
__device__ __forceinline__ void block_reduce(T (&v)[NV], T *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        T x = warp_sum(v[k]);
        if (lane == 0) sh[k * 32 + w] = x;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            T x = lane < nw ? sh[k * 32 + lane] : T(0);
            x = warp_sum(x);
            v[k] = x;
        }
    }
}

// Last-block ticket: returns true in the last block (all threads); partials visible to it.
__device__ __forceinline__ bool last_block(unsigned *ticket)
{
    __shared__ bool amlast;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ticket, 1u);
        amlast = (t == gridDim.x - 1);
    }
    __syncthreads();
    return amlast;
}

// Sum of NV partial arrays (each gridDim.x long, stride ld) in a fixed order by one block.
template <class T, int NV>
__device__ __forceinline__ void reduce_partials(const T *part, int np, int ld, T (&out)[NV], T *sh)
{
    T v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = T(0);
    for (int b = threadIdx.x; b < np; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += ((volatile const T *)part)[k * ld + b];
    block_reduce<T, NV>(v, sh);
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = v[k];
}

// ---- SpMV: y = A x, TPR lanes per row; DOT adds x_i y_i into the block partial ------------
// Each lane takes the entries lo + lane, lo + lane + TPR, ... of its row, U at a time: the U
// index and value loads are issued together, then the U gathers of x, then the U products
// (memory-level parallelism for a latency-bound stream).  The lane's additions stay in entry
// order, so U does not change the result; TPR does (the shuffle tree).
// With FP32 values (the mixed-precision copy, made by f32_rowsum_copy) the row is in row-sum
// form: y_i = s_i x_i + sum_{j != i} a_ij (x_j - x_i), s_i the row's sum, held at the diagonal
// position.  The represented matrix keeps the FP64 matrix's row sums, so rounding the entries to
// FP32 perturbs its quadratic form by O(eps_32) relative instead of O(eps_32 cond(A)), and the
// differences keep the FP32 products of smooth vectors accurate.
template <class V, class T, int TPR, int U, bool DOT>
__global__ void __launch_bounds__(RED_BLOCK) k_spmv(const int *__restrict__ indptr, const int *__restrict__ indices,
                                                    const V *__restrict__ vals, const T *__restrict__ x,
                                                    T *__restrict__ y, int n, double *__restrict__ part,
                                                    CGState<T> *__restrict__ st)
{
    __shared__ double sh[32];
    constexpr bool ROWSUM = std::is_same<V, float>::value;
    if (DOT && (st->done || st->want_ru)) return;
    const int lane = threadIdx.x % TPR;
    constexpr int GPW = 32 / TPR;   // rows per warp per step
    const int gwarp = (blockIdx.x * RED_BLOCK + threadIdx.x) >> 5, nwarp = (gridDim.x * RED_BLOCK) >> 5;
    double dot = 0.0;                                     // x.y accumulated in FP64 (FP32 vectors too)
    // the loop bound is uniform across the warp, so the full-warp shuffles below are safe
    for (int i0 = gwarp * GPW; i0 < n; i0 += nwarp * GPW) {
        const int i = i0 + (threadIdx.x & 31) / TPR;
        T s = T(0);
        if (i < n) {
            const int lo = indptr[i], hi = indptr[i + 1];
            const T xi = ROWSUM ? __ldg(&x[i]) : T(0);
            for (int base = lo + lane; base < hi; base += U * TPR) {
                int c[U];
                V v[U];
                T xv[U];
                // the matrix is streamed once (evict-first loads); x is gathered through the
                // read-only path and stays cached
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int q = base + u * TPR;
                    c[u] = q < hi ? __ldcs(&indices[q]) : 0;
                    v[u] = q < hi ? __ldcs(&vals[q]) : V(0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) xv[u] = base + u * TPR < hi ? __ldg(&x[c[u]]) : T(0);
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (base + u * TPR < hi) s += (T)v[u] * (ROWSUM && c[u] != i ? xv[u] - xi : xv[u]);
            }
        }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, TPR);
        if (lane == 0 && i < n) {
            y[i] = s;
            if (DOT) dot += (double)x[i] * (double)s;
        }
    }
    if (!DOT) return;
    double v[1] = {dot};
    block_reduce<double, 1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    if (!last_block(&st->ticket)) return;
    double tot[1];
    reduce_partials<double, 1>(part, gridDim.x, 0, tot, sh);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        const double pAp = tot[0];
        st->pAp = pAp;
        if (!(pAp > 0.0)) { st->breakdown = 1; st->done = 1; }
        else st->alpha = st->rz / pAp;
    }
}

// ---- fused update: x += a p; r -= a Ap; rr = r.r; rz = r.(inv r) ------------------------------
// JAC: with the Jacobi inverse diagonal; otherwise rz = rr (cg.hpp:330-331).
template <class T, bool JAC>
__global__ void __launch_bounds__(RED_BLOCK) k_cg_update(T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p,
                                                         const T *__restrict__ Ap, const T *__restrict__ inv, int n,
                                                         double *__restrict__ part, CGState<T> *__restrict__ st,
                                                         int mixed)
{
    __shared__ double sh[64];
    if (st->done || st->want_ru) return;                  // want_ru: paused for a reliable update (mixed)
    const T a = (T)st->alpha;
    double rr = 0.0, rz = 0.0;                            // FP64 accumulation (FP32 vectors too)
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) {
        const T ri = r[i] - a * Ap[i];
        r[i] = ri;
        x[i] = x[i] + a * p[i];
        const double t = (double)ri * (double)ri;
        rr += t;
        if (JAC) rz += t * (double)inv[i];
    }
    double v[2] = {rr, rz};
    block_reduce<double, 2>(v, sh);
    if (threadIdx.x == 0) { part[blockIdx.x] = v[0]; part[gridDim.x + blockIdx.x] = v[1]; }
    if (!last_block(&st->ticket)) return;
    double tot[2];
    reduce_partials<double, 2>(part, gridDim.x, gridDim.x, tot, sh);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        const double rrn = tot[0], rzn = JAC ? tot[1] : tot[0];
        st->rr = rrn;
        st->it += 1;
        const double rn = sqrt((double)rrn);
        st->rn = rn;
        if (!mixed) {
            if (rn <= st->tol_nb) { st->done = 1; return; }            // cg.hpp:334
            if (st->it >= st->max_iter) { st->done = 1; return; }      // loop condition
            st->beta = rzn / st->rz;                                   // cg.hpp:335-336
            st->rz = rzn;
            if (!(rzn > 0.0)) { st->breakdown = 1; st->done = 1; }     // cg.hpp:324 at the next loop top
        } else {
            // mixed precision: ask for a reliable update when the recurrence residual has
            // dropped by a decade since the last one, or looks converged
            if (rn <= 0.1 * st->maxr || rn <= st->tol_nb || st->it >= st->max_iter) st->want_ru = 1;
            st->rz_prev = st->rz;
            st->beta = rzn / st->rz;
            st->rz = rzn;
            if (!(rzn > 0.0)) st->want_ru = 1;
        }
    }
}

// ---- direction: p = inv r + beta p (or r + beta p) ------------------------------------------
template <class T, bool JAC>
__global__ void __launch_bounds__(RED_BLOCK) k_cg_direction(T *__restrict__ p, const T *__restrict__ r,
                                                            const T *__restrict__ inv, int n,
                                                            const CGState<T> *__restrict__ st)
{
    if (st->done || st->want_ru) return;
    const T b = (T)st->beta;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK)
        p[i] = (JAC ? inv[i] * r[i] : r[i]) + b * p[i];
}

// ---- start: r = b - Ax; p = inv r; nb, ||r||, rz ------------------------------------------
template <bool JAC>
__global__ void __launch_bounds__(RED_BLOCK) k_cg_start(const double *__restrict__ b, const double *__restrict__ Ax,
                                                        double *__restrict__ r, double *__restrict__ p,
                                                        const double *__restrict__ inv, int n, double *__restrict__ part,
                                                        CGState<double> *__restrict__ st, double tol)
{
    __shared__ double sh[96];
    double bb = 0.0, rr = 0.0, rz = 0.0;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) {
        const double bi = b[i], ri = bi - Ax[i];
        const double zi = JAC ? inv[i] * ri : ri;
        r[i] = ri;
        p[i] = zi;
        bb += bi * bi;
        rr += ri * ri;
        rz += ri * zi;
    }
    double v[3] = {bb, rr, rz};
    block_reduce<double, 3>(v, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = v[0];
        part[gridDim.x + blockIdx.x] = v[1];
        part[2 * gridDim.x + blockIdx.x] = v[2];
    }
    if (!last_block(&st->ticket)) return;
    double tot[3];
    reduce_partials<double, 3>(part, gridDim.x, gridDim.x, tot, sh);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        const double nb = sqrt(tot[0]), rn = sqrt(tot[1]);
        st->nb = nb;
        st->tol_nb = tol * nb;
        st->rn = rn;
        st->maxr = rn;
        st->rz = tot[2];
        st->rr = tot[1];
        st->it = 0;
        st->breakdown = 0;
        st->done = 0;
        if (nb == 0.0) { st->done = 1; return; }                        // cg.hpp:306
        if (rn <= tol * nb) { st->done = 1; return; }                   // cg.hpp:312
        if (!(tot[2] > 0.0)) { st->breakdown = 1; st->done = 1; }       // cg.hpp:324
    }
}

// ---- finish: r = b - Ax, ||r|| (cg.hpp:222-237) ---------------------------------------------
__global__ void __launch_bounds__(RED_BLOCK) k_cg_finish(const double *__restrict__ b, const double *__restrict__ Ax,
                                                         double *__restrict__ r, int n, double *__restrict__ part,
                                                         CGState<double> *__restrict__ st)
{
    __shared__ double sh[32];
    double rr = 0.0;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) {
        const double ri = b[i] - Ax[i];
        r[i] = ri;
        rr += ri * ri;
    }
    double v[1] = {rr};
    block_reduce<double, 1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    if (!last_block(&st->ticket)) return;
    double tot[1];
    reduce_partials<double, 1>(part, gridDim.x, 0, tot, sh);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        st->res64 = sqrt(tot[0]);
    }
}

// ---- CG with a general preconditioner M (cg.hpp:245-290) -------------------------------------
// start: r = b - Ax; nb, ||r||; done when b = 0 or ||r|| <= tol ||b|| (then M and the loop are skipped)
__global__ void __launch_bounds__(RED_BLOCK) k_pc_start(const double *__restrict__ b, const double *__restrict__ Ax,
                                                        double *__restrict__ r, int n, double *__restrict__ part,
                                                        CGState<double> *__restrict__ st, double tol)
{
    __shared__ double sh[64];
    double bb = 0.0, rr = 0.0;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) {
        const double bi = b[i], ri = bi - Ax[i];
        r[i] = ri;
        bb += bi * bi;
        rr += ri * ri;
    }
    double v[2] = {bb, rr};
    block_reduce<double, 2>(v, sh);
    if (threadIdx.x == 0) { part[blockIdx.x] = v[0]; part[gridDim.x + blockIdx.x] = v[1]; }
    if (!last_block(&st->ticket)) return;
    double tot[2];
    reduce_partials<double, 2>(part, gridDim.x, gridDim.x, tot, sh);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        const double nb = sqrt(tot[0]), rn = sqrt(tot[1]);
        st->nb = nb;
        st->tol_nb = tol * nb;
        st->rn = rn;
        st->it = 0;
        st->breakdown = 0;
        st->done = nb == 0.0 || rn <= tol * nb;                           // cg.hpp:259, 265
    }
}

// rz = r.z; FIRST: p = z and the breakdown test of the loop top (cg.hpp:266-271); else
// beta = rz_new / rz (cg.hpp:283-285), and the loop top's test on the new rz
template <bool FIRST>
__global__ void __launch_bounds__(RED_BLOCK) k_pc_rz(const double *__restrict__ r, const double *__restrict__ z,
                                                     double *__restrict__ p, int n, double *__restrict__ part,
                                                     CGState<double> *__restrict__ st)
{
    __shared__ double sh[32];
    if (st->done) return;
    double rz = 0.0;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) {
        rz += r[i] * z[i];
        if (FIRST) p[i] = z[i];
    }
    double v[1] = {rz};
    block_reduce<double, 1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    if (!last_block(&st->ticket)) return;
    double tot[1];
    reduce_partials<double, 1>(part, gridDim.x, 0, tot, sh);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        const double rzn = tot[0];
        if (!FIRST) st->beta = rzn / st->rz;
        st->rz = rzn;
        if (!(rzn > 0.0)) { st->breakdown = 1; st->done = 1; }
    }
}

// x += a p; r -= a Ap; ||r||; the stopping test (cg.hpp:278-281)
__global__ void __launch_bounds__(RED_BLOCK) k_pc_update(double *__restrict__ x, double *__restrict__ r,
                                                         const double *__restrict__ p, const double *__restrict__ Ap, int n,
                                                         double *__restrict__ part, CGState<double> *__restrict__ st)
{
    __shared__ double sh[32];
    if (st->done) return;
    const double a = st->alpha;
    double rr = 0.0;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) {
        const double ri = r[i] - a * Ap[i];
        r[i] = ri;
        x[i] = x[i] + a * p[i];
        rr += ri * ri;
    }
    double v[1] = {rr};
    block_reduce<double, 1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    if (!last_block(&st->ticket)) return;
    double tot[1];
    reduce_partials<double, 1>(part, gridDim.x, 0, tot, sh);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        st->rr = tot[0];
        st->it += 1;
        const double rn = sqrt(tot[0]);
        st->rn = rn;
        if (rn <= st->tol_nb || st->it >= st->max_iter) st->done = 1;
    }
}

// p = z + beta p (cg.hpp:286-288)
__global__ void __launch_bounds__(RED_BLOCK) k_pc_direction(double *__restrict__ p, const double *__restrict__ z, int n,
                                                            const CGState<double> *__restrict__ st)
{
    if (st->done) return;
    const double b = st->beta;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) p[i] = z[i] + b * p[i];
}

// ---- mixed precision kernels -----------------------------------------------------------------
// x64 += d32; d32 = 0 (reliable update of the solution), when st32->want_ru
__global__ void k_mixed_flush(double *__restrict__ x, float *__restrict__ d, int n, const CGState<float> *__restrict__ st)
{
    if (st->done || !st->want_ru) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += (double)d[i];
        d[i] = 0.0f;
    }
}

// y = A64 x when st32->want_ru (the FP64 residual of the reliable update)
template <int TPR>
__global__ void __launch_bounds__(RED_BLOCK) k_mixed_spmv64(const int *__restrict__ indptr, const int *__restrict__ indices,
                                                            const double *__restrict__ vals, const double *__restrict__ x,
                                                            double *__restrict__ y, int n, const CGState<float> *__restrict__ st)
{
    if (st->done || !st->want_ru) return;
    const int lane = threadIdx.x % TPR;
    constexpr int GPW = 32 / TPR;
    const int gwarp = (blockIdx.x * RED_BLOCK + threadIdx.x) >> 5, nwarp = (gridDim.x * RED_BLOCK) >> 5;
    for (int i0 = gwarp * GPW; i0 < n; i0 += nwarp * GPW) {
        const int i = i0 + (threadIdx.x & 31) / TPR;
        double s = 0.0;
        if (i < n)
            for (int q = indptr[i] + lane; q < indptr[i + 1]; q += TPR) s += __ldcs(&vals[q]) * __ldg(&x[__ldcs(&indices[q])]);
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, TPR);
        if (lane == 0 && i < n) y[i] = s;
    }
}

// r64 = b - A x; r32 = r64; ||r64||^2, r32.(inv32 r32); then the convergence test on the FP64
// residual and the restart of the recurrence from it.
__global__ void __launch_bounds__(RED_BLOCK) k_mixed_residual(const double *__restrict__ b, const double *__restrict__ Ax,
                                                              float *__restrict__ r32, const float *__restrict__ inv32, int n,
                                                              double *__restrict__ part64, double *__restrict__ part32,
                                                              CGState<float> *__restrict__ st)
{
    __shared__ double sh64[32];
    __shared__ double sh32[32];
    if (st->done || !st->want_ru) return;
    double rr = 0.0, rz = 0.0;
    for (int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += gridDim.x * RED_BLOCK) {
        const double ri = b[i] - Ax[i];
        const float rf = (float)ri;
        r32[i] = rf;
        rr += ri * ri;
        rz += (double)rf * (double)rf * (double)inv32[i];
    }
    double v[1] = {rr};
    block_reduce<double, 1>(v, sh64);
    double w[1] = {rz};
    __syncthreads();
    block_reduce<double, 1>(w, sh32);
    if (threadIdx.x == 0) { part64[blockIdx.x] = v[0]; part32[blockIdx.x] = w[0]; }
    if (!last_block(&st->ticket)) return;
    double t64[1];
    double t32[1];
    reduce_partials<double, 1>(part64, gridDim.x, 0, t64, sh64);
    __syncthreads();
    reduce_partials<double, 1>(part32, gridDim.x, 0, t32, sh32);
    if (threadIdx.x == 0) {
        st->ticket = 0;
        st->want_ru = 0;
        st->ru_count += 1;
        const double rn = sqrt(t64[0]);
        const double rn_rec = st->rn;                     // the FP32 recurrence's own residual norm
        st->res64 = rn;
        st->rn = rn;
        st->maxr = rn;
        if (rn <= st->tol_nb || st->it >= st->max_iter) { st->done = 1; return; }
        // stagnation of the FP32 recurrence (the FP32 matrix too coarse for the slowest modes):
        // the solve goes on in FP64 from this iterate
        st->stall = (rn > 0.5 * st->prt) ? st->stall + 1 : 0;
        st->prt = rn;
        if (st->stall >= 2 || !(rn < 1e300)) { st->fallback = 1; st->done = 1; return; }
        // continue the recurrence from the true residual: beta from the refreshed r.z; when the
        // recurrence has drifted (true residual over twice its own) restart the direction
        const double rzn = t32[0];
        if (!(rzn > 0.0)) { st->breakdown = 1; st->done = 1; return; }
        st->beta = rn > 2.0 * rn_rec ? 0.0 : rzn / st->rz_prev;
        st->rz = rzn;
    }
}

// x64 += d32 unconditionally (the correction still held when the loop stops)
__global__ void k_mixed_flush_all(double *__restrict__ x, float *__restrict__ d, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += (double)d[i];
        d[i] = 0.0f;
    }
}

// the FP32 recurrence starts from r32 = (float)(b - A x), p32 = inv32 r32, d32 = 0
__global__ void k_mixed_init(const double *__restrict__ b, const double *__restrict__ Ax, float *__restrict__ r32,
                             float *__restrict__ p32, float *__restrict__ d32, const float *__restrict__ inv32, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float rf = (float)(b[i] - Ax[i]);
        r32[i] = rf;
        p32[i] = inv32[i] * rf;
        d32[i] = 0.0f;
    }
}

__global__ void k_to_f32(const double *__restrict__ a, float *__restrict__ b, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

__global__ void k_jacobi_inv(const int *__restrict__ diag_pos, const double *__restrict__ data, double *__restrict__ inv,
                             int n, int *__restrict__ status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d = diag_pos[i];
    const double a = d >= 0 ? data[d] : 0.0;
    if (d < 0 || a == 0.0) { atomicOr(status, ST_ZERODIAG); atomicMin(status + 1, i); }
    inv[i] = 1.0 / a;
}

__global__ void k_asym(const int *__restrict__ indptr, const int *__restrict__ indices, const double *__restrict__ v,
                       int n, unsigned long long *__restrict__ out)
{
    // max |a_ij| and max |a_ij - a_ji| as the bit patterns of non-negative doubles (exact maxima)
    unsigned long long big = 0, dif = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int q = indptr[i]; q < indptr[i + 1]; ++q) {
            const int j = indices[q];
            int lo = indptr[j], hi = indptr[j + 1];
            const int end = hi;
            while (lo < hi) {
                const int mid = lo + ((hi - lo) >> 1);
                if (indices[mid] < i) lo = mid + 1; else hi = mid;
            }
            const double m = (lo < end && indices[lo] == i) ? v[lo] : 0.0;
            const unsigned long long a = __double_as_longlong(fabs(v[q]));
            const unsigned long long d = __double_as_longlong(fabs(v[q] - m));
            big = a > big ? a : big;
            dif = d > dif ? d : dif;
        }
    atomicMax(out, big);
    atomicMax(out + 1, dif);
}

__global__ void k_combine(double alpha, const double *__restrict__ A, double beta, const double *__restrict__ B,
                          double *__restrict__ C, long long nnz)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (long long)gridDim.x * blockDim.x)
        C[q] = alpha * A[q] + beta * B[q];
}

// ---- host side -------------------------------------------------------------------------------
unsigned red_grid(femd_ctx ctx, int n)
{
    // a fixed function of n (deterministic reductions): enough blocks to fill the GPU
    const unsigned cap = (unsigned)ctx->sm_count * 8;
    return grid_for((size_t)n, RED_BLOCK * 4, cap);
}

int pick_tpr(femd_matrix K)
{
    if (K->spmv_tpr) return K->spmv_tpr;
    // 4 loads in flight per lane and the fewest lanes (a power of 2) that cover the mean row in
    // one round: 2 lanes for P1, 4 for P2 and P3 (what the autotuner picks at those sizes)
    const double avg = K->pattern->nrows ? (double)K->pattern->nnz / K->pattern->nrows : 1.0;
    int tpr = 2;
    while (tpr * 4 < avg && tpr < 32) tpr <<= 1;
    return tpr | (4 << 8);
}

// shape = threads per row (low byte) | loads in flight per lane (next byte)
static inline int shape_tpr(int shape) { return shape & 0xff; }
static inline int shape_u(int shape) { return (shape >> 8) ? (shape >> 8) : 1; }

template <class V, class T, bool DOT, int U>
static void launch_spmv_u(int tpr, unsigned grid, cudaStream_t s, const int *ip, const int *ix, const V *v, const T *x, T *y,
                          int n, double *part, CGState<T> *st)
{
    switch (tpr) {
    case 2: k_spmv<V, T, 2, U, DOT><<<grid, RED_BLOCK, 0, counted(s)>>>(ip, ix, v, x, y, n, part, st); break;
    case 4: k_spmv<V, T, 4, U, DOT><<<grid, RED_BLOCK, 0, counted(s)>>>(ip, ix, v, x, y, n, part, st); break;
    case 8: k_spmv<V, T, 8, U, DOT><<<grid, RED_BLOCK, 0, counted(s)>>>(ip, ix, v, x, y, n, part, st); break;
    case 16: k_spmv<V, T, 16, U, DOT><<<grid, RED_BLOCK, 0, counted(s)>>>(ip, ix, v, x, y, n, part, st); break;
    default: k_spmv<V, T, 32, U, DOT><<<grid, RED_BLOCK, 0, counted(s)>>>(ip, ix, v, x, y, n, part, st); break;
    }
}

template <class V, class T, bool DOT>
static void launch_spmv(int shape, unsigned grid, cudaStream_t s, const int *ip, const int *ix, const V *v, const T *x, T *y,
                        int n, double *part, CGState<T> *st)
{
    const int tpr = shape_tpr(shape);
    switch (shape_u(shape)) {
    case 2: launch_spmv_u<V, T, DOT, 2>(tpr, grid, s, ip, ix, v, x, y, n, part, st); break;
    case 4: launch_spmv_u<V, T, DOT, 4>(tpr, grid, s, ip, ix, v, x, y, n, part, st); break;
    default: launch_spmv_u<V, T, DOT, 1>(tpr, grid, s, ip, ix, v, x, y, n, part, st); break;
    }
}

unsigned spmv_grid(femd_ctx ctx, int n, int shape)
{
    const int gpb = RED_BLOCK / shape_tpr(shape);
    const unsigned cap = (unsigned)ctx->sm_count * 16;
    return grid_for((size_t)n, gpb, cap);
}

// The solver workspace of a matrix: vectors, reduction partials, device and pinned host state,
// events, and the CUDA graphs of a chunk of iterations.  The graphs run on the workspace's own
// solution and right-hand-side vectors (wx, wb), so their pointers never change and a graph is
// captured once per matrix; a solve copies b and x0 in and x out.  After the first solve on a
// matrix, a solve makes no allocation, capture or instantiation.
struct SolverWS {
    int n = 0, shape = 0;
    unsigned gs = 0, gr = 0;
    // FP64
    DevBuf<double> r, p, Ap, part, wx, wb;
    DevBuf<CGState<double>> st;
    CGState<double> *st_host = nullptr;
    int *maxit_host = nullptr;
    cudaGraphExec_t x64[2] = {nullptr, nullptr};
    size_t nodes64[2] = {0, 0};
    int ch64 = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr, ev[2] = {nullptr, nullptr};
    // mixed precision
    bool mixed_ready = false;
    DevBuf<double> Ax64, r64, part64;
    DevBuf<float> r32, p32, Ap32, d32;
    DevBuf<double> part32;                       // the FP32 recurrence's block partials (FP64 sums)
    DevBuf<CGState<float>> st32;
    CGState<float> *st32_host = nullptr;
    cudaGraphExec_t xm = nullptr;
    size_t nodesm = 0;
    int chm = 0;
    // CG with a general preconditioner: z, and the graph of a chunk for the preconditioner it was
    // captured with
    DevBuf<double> z;
    cudaGraphExec_t xpc = nullptr;
    size_t nodespc = 0;
    femd_precond pc_for = nullptr;
    int chpc = 0;
    ~SolverWS()
    {
        for (auto &g : x64) if (g) cudaGraphExecDestroy(g);
        if (xm) cudaGraphExecDestroy(xm);
        if (xpc) cudaGraphExecDestroy(xpc);
        for (cudaEvent_t e : {e0, e1, ev[0], ev[1]}) if (e) cudaEventDestroy(e);
        if (st_host) cudaFreeHost(st_host);
        if (maxit_host) cudaFreeHost(maxit_host);
        if (st32_host) cudaFreeHost(st32_host);
    }
};

static void solver_ws_free(void *w) { delete static_cast<SolverWS *>(w); }

static int get_ws(femd_ctx ctx, femd_matrix K, SolverWS **out)
{
    const int n = K->pattern->nrows, shape = pick_tpr(K);
    SolverWS *W = static_cast<SolverWS *>(K->solver_ws);
    if (W && W->n == n && W->shape == shape) { *out = W; return FEMD_OK; }
    if (W) { solver_ws_free(W); K->solver_ws = nullptr; K->solver_ws_free = nullptr; }
    W = new SolverWS();
    std::unique_ptr<SolverWS> guard(W);
    W->n = n;
    W->shape = shape;
    W->gs = spmv_grid(ctx, n, shape);
    W->gr = red_grid(ctx, n);
    for (DevBuf<double> *b : {&W->r, &W->p, &W->Ap, &W->wx, &W->wb}) FEMD_TRY(b->alloc((size_t)n + 1));
    FEMD_TRY(W->part.alloc(3 * (size_t)std::max(W->gs, W->gr) + 3));
    FEMD_TRY(W->st.alloc(1));
    FEMD_TRY_CUDA(cudaMallocHost(&W->st_host, sizeof(CGState<double>)));
    FEMD_TRY_CUDA(cudaMallocHost(&W->maxit_host, sizeof(int)));
    FEMD_TRY_CUDA(cudaEventCreate(&W->e0));
    FEMD_TRY_CUDA(cudaEventCreate(&W->e1));
    FEMD_TRY_CUDA(cudaEventCreateWithFlags(&W->ev[0], cudaEventDisableTiming));
    FEMD_TRY_CUDA(cudaEventCreateWithFlags(&W->ev[1], cudaEventDisableTiming));
    W->ch64 = n > (1 << 18) ? 8 : 32;
    K->solver_ws = guard.release();
    K->solver_ws_free = solver_ws_free;
    *out = W;
    return FEMD_OK;
}

// Capture CH iterations of the FP64 loop on the workspace vectors (once per matrix and variant).
static int capture_cg64(femd_ctx ctx, femd_matrix K, SolverWS &W, bool jac)
{
    if (W.x64[jac]) return FEMD_OK;
    femd_pattern P = K->pattern;
    cudaStream_t s = ctx->stream;
    const int n = W.n;
    cudaGraph_t graph = nullptr;
    FEMD_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < W.ch64; ++k) {
        launch_spmv<double, double, true>(W.shape, W.gs, s, P->indptr.p, P->indices.p, K->data.p, W.p.p, W.Ap.p, n, W.part.p,
                                          W.st.p);
        if (jac) {
            k_cg_update<double, true><<<W.gr, RED_BLOCK, 0, counted(s)>>>(W.wx.p, W.r.p, W.p.p, W.Ap.p, K->inv.p, n, W.part.p,
                                                                          W.st.p, 0);
            k_cg_direction<double, true><<<W.gr, RED_BLOCK, 0, counted(s)>>>(W.p.p, W.r.p, K->inv.p, n, W.st.p);
        } else {
            k_cg_update<double, false><<<W.gr, RED_BLOCK, 0, counted(s)>>>(W.wx.p, W.r.p, W.p.p, W.Ap.p, nullptr, n, W.part.p,
                                                                           W.st.p, 0);
            k_cg_direction<double, false><<<W.gr, RED_BLOCK, 0, counted(s)>>>(W.p.p, W.r.p, nullptr, n, W.st.p);
        }
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) { set_error(std::string("cg: graph capture: ") + cudaGetErrorString(ce)); return FEMD_ECUDA; }
    ce = cudaGraphInstantiate(&W.x64[jac], graph, 0);
    cudaGraphGetNodes(graph, nullptr, &W.nodes64[jac]);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) { W.x64[jac] = nullptr; set_error(std::string("cg: graph instantiate: ") + cudaGetErrorString(ce)); return FEMD_ECUDA; }
    return FEMD_OK;
}

// One FP64 CG solve (cg.hpp:296-350) on the matrix's workspace.
static int cg_run(femd_ctx ctx, femd_matrix K, bool jac, const double *b, double *x, int max_iter, double tol,
                  femd_cg_result *res)
{
    femd_pattern P = K->pattern;
    const int n = P->nrows;
    cudaStream_t s = ctx->stream;
    SolverWS *Wp = nullptr;
    FEMD_TRY(get_ws(ctx, K, &Wp));
    SolverWS &W = *Wp;
    FEMD_TRY(capture_cg64(ctx, K, W, jac));
    const unsigned gs = W.gs, gr = W.gr;
    const int CH = W.ch64;
    *W.maxit_host = max_iter;
    FEMD_TRY_CUDA(cudaEventRecord(W.e0, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.wb.p, b, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.wx.p, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    FEMD_TRY_CUDA(cudaMemsetAsync(W.st.p, 0, sizeof(CGState<double>), s));
    // start (cg.hpp:305-320)
    launch_spmv<double, double, false>(W.shape, gs, s, P->indptr.p, P->indices.p, K->data.p, W.wx.p, W.Ap.p, n, nullptr, nullptr);
    if (jac) k_cg_start<true><<<gr, RED_BLOCK, 0, counted(s)>>>(W.wb.p, W.Ap.p, W.r.p, W.p.p, K->inv.p, n, W.part.p, W.st.p, tol);
    else k_cg_start<false><<<gr, RED_BLOCK, 0, counted(s)>>>(W.wb.p, W.Ap.p, W.r.p, W.p.p, nullptr, n, W.part.p, W.st.p, tol);
    FEMD_TRY_CUDA(cudaGetLastError());
    // max_iter on the device state (after start zeroed the counters)
    FEMD_TRY_CUDA(cudaMemcpyAsync(&W.st.p->max_iter, W.maxit_host, sizeof(int), cudaMemcpyHostToDevice, s));
    // the loop, in chunks of CH iterations (one graph launch each); poll the state between
    // chunks, keeping one chunk queued ahead
    int status = FEMD_OK;
    long long launched = 0;
    const long long max_chunks = (long long)max_iter / CH + 2;
    cudaGraphExec_t exec = W.x64[jac];
    const size_t nodes = W.nodes64[jac];
    cudaError_t ce = launch_graph(exec, nodes, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(W.st_host, W.st.p, sizeof(CGState<double>), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaEventRecord(W.ev[0], s);
    launched = 1;
    while (ce == cudaSuccess) {
        if (launched < max_chunks) {
            ce = launch_graph(exec, nodes, s);
            if (ce != cudaSuccess) break;
        }
        ce = cudaEventSynchronize(W.ev[(launched - 1) & 1]);
        if (ce != cudaSuccess) break;
        if (W.st_host->done) break;
        if (launched >= max_chunks) break;
        ce = cudaMemcpyAsync(W.st_host, W.st.p, sizeof(CGState<double>), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaEventRecord(W.ev[launched & 1], s);
        ++launched;
    }
    if (ce != cudaSuccess) { set_error(std::string("cg: ") + cudaGetErrorString(ce)); status = FEMD_ECUDA; }
    // finish (cg.hpp:222-237)
    if (status == FEMD_OK) {
        launch_spmv<double, double, false>(W.shape, gs, s, P->indptr.p, P->indices.p, K->data.p, W.wx.p, W.Ap.p, n, nullptr,
                                           nullptr);
        k_cg_finish<<<gr, RED_BLOCK, 0, counted(s)>>>(W.wb.p, W.Ap.p, W.r.p, n, W.part.p, W.st.p);
        ce = cudaMemcpyAsync(W.st_host, W.st.p, sizeof(CGState<double>), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(x, W.wx.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (ce == cudaSuccess) ce = cudaEventRecord(W.e1, s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
        if (ce != cudaSuccess) { set_error(std::string("cg: ") + cudaGetErrorString(ce)); status = FEMD_ECUDA; }
    }
    if (status == FEMD_OK) {
        const CGState<double> &S = *W.st_host;
        if (S.nb == 0.0) {
            cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), s);
            cudaStreamSynchronize(s);
            res->converged = 1; res->iterations = 0; res->residual = 0.0; res->breakdown = 0;
        } else {
            res->iterations = S.it;
            res->breakdown = S.breakdown;
            res->residual = S.res64 / S.nb;
            int conv = !S.breakdown && res->residual <= tol * (1.0 + 1e-6) + 1e-15;
            if (!conv && !S.breakdown && res->residual <= 10.0 * tol && S.it < max_iter) conv = 1;
            res->converged = conv;
        }
        res->status = FEMD_OK;
        res->outer = 0;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, W.e0, W.e1);
        res->seconds = ms * 1e-3;
    }
    return status;
}

__global__ void k_f32_rowsum(const int *__restrict__ indptr, const int *__restrict__ diag_pos, const double *__restrict__ a,
                             const int *__restrict__ dst, float *__restrict__ a32, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int lo = indptr[i], hi = indptr[i + 1];
        double sum = 0.0;
        for (int q = lo; q < hi; ++q) {
            const double v = a[q];
            sum += v;
            a32[dst ? dst[q] : q] = (float)v;
        }
        const int d = diag_pos[i];
        a32[dst ? dst[d] : d] = (float)sum;
    }
}

int f32_rowsum_copy(femd_pattern P, const double *a, const int *dst, float *a32, cudaStream_t s)
{
    if (!P->all_diag) {
        set_error("mixed precision: a row of the matrix has no diagonal entry (the matrix is not SPD)");
        return FEMD_EINVAL;
    }
    if (P->nrows)
        k_f32_rowsum<<<grid_for((size_t)P->nrows, 128, 1u << 20), 128, 0, counted(s)>>>(P->indptr.p, P->diag_pos.p, a, dst, a32,
                                                                                       P->nrows);
    FEMD_TRY_CUDA(cudaGetLastError());
    return FEMD_OK;
}

static int ensure_f32(femd_ctx ctx, femd_matrix K)
{
    if (K->f32_valid) return FEMD_OK;
    const long long nnz = K->pattern->nnz;
    const int n = K->pattern->nrows;
    if (!K->data32.p) FEMD_TRY(K->data32.alloc((size_t)nnz + 1));
    if (!K->inv32.p) FEMD_TRY(K->inv32.alloc((size_t)n + 1));
    FEMD_TRY(f32_rowsum_copy(K->pattern, K->data.p, nullptr, K->data32.p, ctx->stream));
    if (n) k_to_f32<<<grid_for((size_t)n, 256, 1u << 20), 256, 0, counted(ctx->stream)>>>(K->inv.p, K->inv32.p, n);
    FEMD_TRY_CUDA(cudaGetLastError());
    K->f32_valid = true;
    return FEMD_OK;
}

// The mixed-precision buffers of the workspace and the graph of a chunk (once per matrix).
static int prepare_mixed(femd_ctx ctx, femd_matrix K, SolverWS &W)
{
    if (W.mixed_ready) return FEMD_OK;
    femd_pattern P = K->pattern;
    cudaStream_t s = ctx->stream;
    const int n = W.n;
    const size_t npart = 3 * (size_t)std::max(W.gs, W.gr) + 3;
    for (DevBuf<double> *b : {&W.Ax64, &W.r64}) FEMD_TRY(b->alloc((size_t)n + 1));
    for (DevBuf<float> *b : {&W.r32, &W.p32, &W.Ap32, &W.d32}) FEMD_TRY(b->alloc((size_t)n + 1));
    FEMD_TRY(W.part64.alloc(npart));
    FEMD_TRY(W.part32.alloc(npart));
    FEMD_TRY(W.st32.alloc(1));
    FEMD_TRY_CUDA(cudaMallocHost(&W.st32_host, sizeof(CGState<float>)));
    // a chunk is CHM iterations of the FP32 recurrence only (SpMV with p.Ap, update, direction);
    // when the update asks for a reliable update the rest of the chunk is skipped (want_ru) and
    // the host runs the FP64 tail (mixed_ru) before the next chunk
    W.chm = 32;
    const unsigned gs = W.gs, gr = W.gr;
    cudaGraph_t graph = nullptr;
    FEMD_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < W.chm; ++k) {
        launch_spmv<float, float, true>(W.shape, gs, s, P->indptr.p, P->indices.p, K->data32.p, W.p32.p, W.Ap32.p, n,
                                        W.part32.p, W.st32.p);
        k_cg_update<float, true><<<gr, RED_BLOCK, 0, counted(s)>>>(W.d32.p, W.r32.p, W.p32.p, W.Ap32.p, K->inv32.p, n, W.part32.p,
                                                                   W.st32.p, 1);
        k_cg_direction<float, true><<<gr, RED_BLOCK, 0, counted(s)>>>(W.p32.p, W.r32.p, K->inv32.p, n, W.st32.p);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) { set_error(std::string("pcg_mixed: graph capture: ") + cudaGetErrorString(ce)); return FEMD_ECUDA; }
    ce = cudaGraphInstantiate(&W.xm, graph, 0);
    cudaGraphGetNodes(graph, nullptr, &W.nodesm);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) { W.xm = nullptr; set_error(std::string("pcg_mixed: ") + cudaGetErrorString(ce)); return FEMD_ECUDA; }
    W.mixed_ready = true;
    return FEMD_OK;
}

// The reliable update, when the FP32 recurrence asked for it: x += d, d = 0; r = b - A64 x in
// FP64, r32 = (float) r, the convergence test on it and the restart of the recurrence; then the
// direction update the paused chunk skipped.
static void mixed_ru(femd_ctx ctx, femd_matrix K, SolverWS &W)
{
    femd_pattern P = K->pattern;
    cudaStream_t s = ctx->stream;
    const int n = W.n;
    const unsigned gs = W.gs, gr = W.gr;
    double *x = W.wx.p;
    const double *b = W.wb.p;
    k_mixed_flush<<<grid_for((size_t)n, 256, 1u << 20), 256, 0, counted(s)>>>(x, W.d32.p, n, W.st32.p);
    switch (shape_tpr(W.shape)) {
    case 2: k_mixed_spmv64<2><<<gs, RED_BLOCK, 0, counted(s)>>>(P->indptr.p, P->indices.p, K->data.p, x, W.Ax64.p, n, W.st32.p); break;
    case 4: k_mixed_spmv64<4><<<gs, RED_BLOCK, 0, counted(s)>>>(P->indptr.p, P->indices.p, K->data.p, x, W.Ax64.p, n, W.st32.p); break;
    case 8: k_mixed_spmv64<8><<<gs, RED_BLOCK, 0, counted(s)>>>(P->indptr.p, P->indices.p, K->data.p, x, W.Ax64.p, n, W.st32.p); break;
    case 16: k_mixed_spmv64<16><<<gs, RED_BLOCK, 0, counted(s)>>>(P->indptr.p, P->indices.p, K->data.p, x, W.Ax64.p, n, W.st32.p); break;
    default: k_mixed_spmv64<32><<<gs, RED_BLOCK, 0, counted(s)>>>(P->indptr.p, P->indices.p, K->data.p, x, W.Ax64.p, n, W.st32.p); break;
    }
    k_mixed_residual<<<gr, RED_BLOCK, 0, counted(s)>>>(b, W.Ax64.p, W.r32.p, K->inv32.p, n, W.part64.p, W.part32.p, W.st32.p);
    k_cg_direction<float, true><<<gr, RED_BLOCK, 0, counted(s)>>>(W.p32.p, W.r32.p, K->inv32.p, n, W.st32.p);
}

// Mixed precision solve: inner FP32 Jacobi-PCG with reliable FP64 updates, on the workspace.
static int mixed_run(femd_ctx ctx, femd_matrix K, const double *b_in, double *x_out, int max_iter, double tol,
                     femd_cg_result *res)
{
    femd_pattern P = K->pattern;
    const int n = P->nrows;
    cudaStream_t s = ctx->stream;
    FEMD_TRY(ensure_f32(ctx, K));
    SolverWS *Wp = nullptr;
    FEMD_TRY(get_ws(ctx, K, &Wp));
    SolverWS &W = *Wp;
    FEMD_TRY(prepare_mixed(ctx, K, W));
    const unsigned gs = W.gs, gr = W.gr;
    double *x = W.wx.p;
    const double *b = W.wb.p;
    CGState<double> *st64 = W.st.p;
    cudaEventRecord(W.e0, s);
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.wb.p, b_in, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.wx.p, x_out, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // FP64 start: r64 = b - A x, nb, ||r64||; the FP32 recurrence starts from (float) r64
    FEMD_TRY_CUDA(cudaMemsetAsync(st64, 0, sizeof(CGState<double>), s));
    launch_spmv<double, double, false>(W.shape, gs, s, P->indptr.p, P->indices.p, K->data.p, x, W.Ax64.p, n, nullptr, nullptr);
    k_cg_start<true><<<gr, RED_BLOCK, 0, counted(s)>>>(b, W.Ax64.p, W.r64.p, W.r64.p, K->inv.p, n, W.part64.p, st64, tol);
    k_mixed_init<<<grid_for((size_t)n, 256, 1u << 20), 256, 0, counted(s)>>>(b, W.Ax64.p, W.r32.p, W.p32.p, W.d32.p, K->inv32.p, n);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.st_host, st64, sizeof(CGState<double>), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    const CGState<double> s64 = *W.st_host;
    if (s64.nb == 0.0) {
        cudaMemsetAsync(x_out, 0, (size_t)n * sizeof(double), s);
        cudaStreamSynchronize(s);
        *res = femd_cg_result{1, 0, 0.0, 0, FEMD_OK, 0, 0.0};
        return FEMD_OK;
    }
    if (s64.done) {   // already converged at x0, or breakdown at the start
        res->converged = !s64.breakdown; res->iterations = 0; res->residual = s64.rn / s64.nb;
        res->breakdown = s64.breakdown; res->status = FEMD_OK; res->outer = 0; res->seconds = 0.0;
        return FEMD_OK;
    }
    // FP32 state seeded from the FP64 start
    CGState<float> &s32 = *W.st32_host;
    s32 = CGState<float>{};
    s32.rz = s64.rz;
    s32.nb = s64.nb;
    s32.tol_nb = s64.tol_nb;
    s32.rn = s64.rn;
    s32.maxr = s64.rn;
    s32.prt = s64.rn;
    s32.max_iter = max_iter;
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.st32.p, W.st32_host, sizeof(CGState<float>), cudaMemcpyHostToDevice, s));
    // every chunk either advances the recurrence or (paused) does nothing; a reliable update
    // is run between chunks when the state asks for one (about once per decade of residual)
    const long long max_polls = 2 * ((long long)max_iter / W.chm + 2) + 64;
    int status = FEMD_OK;
    cudaError_t ce = cudaSuccess;
    for (long long c = 0; c < max_polls; ++c) {
        ce = launch_graph(W.xm, W.nodesm, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(W.st32_host, W.st32.p, sizeof(CGState<float>), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
        if (ce != cudaSuccess) { set_error(std::string("pcg_mixed: ") + cudaGetErrorString(ce)); status = FEMD_ECUDA; break; }
        if (W.st32_host->done) break;
        if (W.st32_host->want_ru) {
            mixed_ru(ctx, K, W);
            ce = cudaMemcpyAsync(W.st32_host, W.st32.p, sizeof(CGState<float>), cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) { set_error(std::string("pcg_mixed: ") + cudaGetErrorString(ce)); status = FEMD_ECUDA; break; }
            if (W.st32_host->done) break;
        }
    }
    // final true residual in FP64 (cg.hpp:222-237)
    if (status == FEMD_OK) {
        const CGState<float> sh = *W.st32_host;
        // flush any correction still held in FP32 (when the loop ended on max_iter)
        k_mixed_flush_all<<<grid_for((size_t)n, 256, 1u << 20), 256, 0, counted(s)>>>(x, W.d32.p, n);
        launch_spmv<double, double, false>(W.shape, gs, s, P->indptr.p, P->indices.p, K->data.p, x, W.Ax64.p, n, nullptr,
                                           nullptr);
        FEMD_TRY_CUDA(cudaMemsetAsync(st64, 0, sizeof(CGState<double>), s));
        k_cg_finish<<<gr, RED_BLOCK, 0, counted(s)>>>(b, W.Ax64.p, W.Ax64.p, n, W.part64.p, st64);
        FEMD_TRY_CUDA(cudaMemcpyAsync(x_out, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        cudaEventRecord(W.e1, s);
        FEMD_TRY_CUDA(cudaMemcpyAsync(W.st_host, st64, sizeof(CGState<double>), cudaMemcpyDeviceToHost, s));
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));
        res->iterations = sh.it;
        res->breakdown = sh.breakdown;
        res->residual = W.st_host->res64 / sh.nb;
        int conv = !sh.breakdown && res->residual <= tol * (1.0 + 1e-6) + 1e-15;
        if (!conv && !sh.breakdown && res->residual <= 10.0 * tol && sh.it < max_iter) conv = 1;
        res->converged = conv;
        res->status = FEMD_OK;
        res->outer = sh.ru_count;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, W.e0, W.e1);
        res->seconds = ms * 1e-3;
        if (sh.fallback && sh.it < max_iter) {
            // the FP32 recurrence stagnated: FP64 Jacobi-PCG from the current iterate (x_out),
            // with the rest of the iteration budget; the result counts both phases
            femd_cg_result r64{};
            FEMD_TRY(cg_run(ctx, K, true, b_in, x_out, max_iter - sh.it, tol, &r64));
            res->iterations = sh.it + r64.iterations;
            res->residual = r64.residual;
            res->breakdown = r64.breakdown;
            res->converged = r64.converged;
            res->seconds += r64.seconds;
        }
    }
    return status;
}

// CG preconditioned by P (cg.hpp:245-290) on the matrix's workspace: the loop in captured chunks
// of CH iterations (SpMV with p.Ap, update, M, r.z, direction), polled between chunks.
static int pc_run(femd_ctx ctx, femd_matrix K, femd_precond P, const double *b, double *x, int max_iter, double tol,
                  femd_cg_result *res)
{
    femd_pattern Q = K->pattern;
    const int n = Q->nrows;
    cudaStream_t s = ctx->stream;
    SolverWS *Wp = nullptr;
    FEMD_TRY(get_ws(ctx, K, &Wp));
    SolverWS &W = *Wp;
    if (!W.z.p) FEMD_TRY(W.z.alloc((size_t)n + 1));
    const unsigned gs = W.gs, gr = W.gr;
    const int *done = &W.st.p->done;
    if (W.pc_for != P) {
        if (W.xpc) cudaGraphExecDestroy(W.xpc);
        W.xpc = nullptr;
        W.pc_for = P;
        W.chpc = n > (1 << 18) ? 2 : 8;
        cudaGraph_t graph = nullptr;
        FEMD_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int st = FEMD_OK;
        for (int k = 0; k < W.chpc && st == FEMD_OK; ++k) {
            launch_spmv<double, double, true>(W.shape, gs, s, Q->indptr.p, Q->indices.p, K->data.p, W.p.p, W.Ap.p, n, W.part.p,
                                              W.st.p);
            k_pc_update<<<gr, RED_BLOCK, 0, counted(s)>>>(W.wx.p, W.r.p, W.p.p, W.Ap.p, n, W.part.p, W.st.p);
            st = precond_enqueue(P, W.r.p, W.z.p, done, s);
            k_pc_rz<false><<<gr, RED_BLOCK, 0, counted(s)>>>(W.r.p, W.z.p, nullptr, n, W.part.p, W.st.p);
            k_pc_direction<<<gr, RED_BLOCK, 0, counted(s)>>>(W.p.p, W.z.p, n, W.st.p);
        }
        cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (st != FEMD_OK) { if (graph) cudaGraphDestroy(graph); W.pc_for = nullptr; return st; }
        if (ce != cudaSuccess) {
            W.pc_for = nullptr;
            set_error(std::string("cg: graph capture: ") + cudaGetErrorString(ce));
            return FEMD_ECUDA;
        }
        ce = cudaGraphInstantiate(&W.xpc, graph, 0);
        cudaGraphGetNodes(graph, nullptr, &W.nodespc);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
            W.xpc = nullptr;
            W.pc_for = nullptr;
            set_error(std::string("cg: graph instantiate: ") + cudaGetErrorString(ce));
            return FEMD_ECUDA;
        }
    }
    *W.maxit_host = max_iter;
    FEMD_TRY_CUDA(cudaEventRecord(W.e0, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.wb.p, b, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.wx.p, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    FEMD_TRY_CUDA(cudaMemsetAsync(W.st.p, 0, sizeof(CGState<double>), s));
    launch_spmv<double, double, false>(W.shape, gs, s, Q->indptr.p, Q->indices.p, K->data.p, W.wx.p, W.Ap.p, n, nullptr, nullptr);
    k_pc_start<<<gr, RED_BLOCK, 0, counted(s)>>>(W.wb.p, W.Ap.p, W.r.p, n, W.part.p, W.st.p, tol);
    FEMD_TRY(precond_enqueue(P, W.r.p, W.z.p, done, s));
    k_pc_rz<true><<<gr, RED_BLOCK, 0, counted(s)>>>(W.r.p, W.z.p, W.p.p, n, W.part.p, W.st.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaMemcpyAsync(&W.st.p->max_iter, W.maxit_host, sizeof(int), cudaMemcpyHostToDevice, s));
    int status = FEMD_OK;
    const long long max_chunks = (long long)max_iter / W.chpc + 2;
    cudaError_t ce = cudaSuccess;
    for (long long c = 0; c < max_chunks && ce == cudaSuccess; ++c) {
        ce = launch_graph(W.xpc, W.nodespc, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(W.st_host, W.st.p, sizeof(CGState<double>), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
        if (ce == cudaSuccess && W.st_host->done) break;
    }
    if (ce != cudaSuccess) { set_error(std::string("cg: ") + cudaGetErrorString(ce)); status = FEMD_ECUDA; }
    if (status == FEMD_OK) {
        // finish (cg.hpp:222-237)
        launch_spmv<double, double, false>(W.shape, gs, s, Q->indptr.p, Q->indices.p, K->data.p, W.wx.p, W.Ap.p, n, nullptr,
                                           nullptr);
        k_cg_finish<<<gr, RED_BLOCK, 0, counted(s)>>>(W.wb.p, W.Ap.p, W.r.p, n, W.part.p, W.st.p);
        ce = cudaMemcpyAsync(W.st_host, W.st.p, sizeof(CGState<double>), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(x, W.wx.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (ce == cudaSuccess) ce = cudaEventRecord(W.e1, s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
        if (ce != cudaSuccess) { set_error(std::string("cg: ") + cudaGetErrorString(ce)); status = FEMD_ECUDA; }
    }
    if (status == FEMD_OK) {
        const CGState<double> &S = *W.st_host;
        if (S.nb == 0.0) {
            cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), s);
            cudaStreamSynchronize(s);
            *res = femd_cg_result{1, 0, 0.0, 0, FEMD_OK, 0, 0.0};
        } else {
            res->iterations = S.it;
            res->breakdown = S.breakdown;
            res->residual = S.res64 / S.nb;
            int conv = !S.breakdown && res->residual <= tol * (1.0 + 1e-6) + 1e-15;
            if (!conv && !S.breakdown && res->residual <= 10.0 * tol && S.it < max_iter) conv = 1;
            res->converged = conv;
            res->status = FEMD_OK;
            res->outer = 0;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, W.e0, W.e1);
        res->seconds = ms * 1e-3;
    }
    return status;
}

}  // namespace femd

using namespace femd;

// the error of a preconditioned solve on a matrix whose inverse diagonal was never written
static const char *const JACOBI_MISSING =
    "Jacobi: the matrix has no inverse diagonal; call JacobiPreconditioner first (femd_cuda_matrix_jacobi, "
    "an assembly with want_inv, or femd_cuda_matrix_set_inv_diag)";

static femd_matrix as_matrix(void *h)
{
    femd_matrix m = static_cast<femd_matrix>(h);
    return (m && m->kind == KIND_MATRIX) ? m : nullptr;
}

extern "C" {

int femd_cuda_matrix_create(femd_ctx ctx, femd_pattern p, femd_matrix *out)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && p && out && p->kind == KIND_PATTERN, "CSRMatrix: NULL or invalid argument");
    *out = nullptr;
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    femd_matrix K = new femd_matrix_s();
    K->ctx = ctx;
    ctx_retain(ctx);
    K->pattern = p;
    int st = K->data.alloc((size_t)p->nnz + 1);
    if (st == FEMD_OK) st = K->inv.alloc((size_t)p->nrows + 1);
    if (st != FEMD_OK) { delete K; return st; }
    cudaMemsetAsync(K->data.p, 0, ((size_t)p->nnz + 1) * sizeof(double), ctx->stream);
    *out = K;
    return FEMD_OK;
}

int femd_cuda_matrix_arrays(femd_matrix K, double **data_dev, double **inv_diag_dev)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(K, "matrix_arrays: not a matrix handle");
    if (data_dev) *data_dev = K->data.p;
    if (inv_diag_dev) *inv_diag_dev = K->inv.p;
    K->f32_valid = false;   // the caller may write through these pointers
    return FEMD_OK;
}

int femd_cuda_matrix_set_host(femd_matrix K, const double *data_host)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(K && data_host, "matrix_set_host: NULL argument");
    FEMD_TRY_CUDA(cudaSetDevice(K->ctx->device));
    if (K->pattern->nnz)
        FEMD_TRY_CUDA(cudaMemcpyAsync(K->data.p, data_host, (size_t)K->pattern->nnz * sizeof(double), cudaMemcpyHostToDevice,
                                      K->ctx->stream));
    FEMD_TRY_CUDA(cudaStreamSynchronize(K->ctx->stream));
    K->f32_valid = false;
    return FEMD_OK;
}

int femd_cuda_matrix_to_host(femd_matrix K, double *data_host)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(K && data_host, "matrix_to_host: NULL argument");
    FEMD_TRY_CUDA(cudaSetDevice(K->ctx->device));
    if (K->pattern->nnz)
        FEMD_TRY_CUDA(cudaMemcpyAsync(data_host, K->data.p, (size_t)K->pattern->nnz * sizeof(double), cudaMemcpyDeviceToHost,
                                      K->ctx->stream));
    FEMD_TRY_CUDA(cudaStreamSynchronize(K->ctx->stream));
    return FEMD_OK;
}

int femd_cuda_matrix_jacobi(femd_ctx ctx, femd_matrix K)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K, "Jacobi: NULL argument");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "Jacobi: the matrix must be square");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    FEMD_TRY(reset_status(ctx));
    const int n = K->pattern->nrows;
    if (n) k_jacobi_inv<<<grid_for((size_t)n, 256), 256, 0, counted(ctx->stream)>>>(K->pattern->diag_pos.p, K->data.p, K->inv.p, n,
                                                                           ctx->status_dev);
    FEMD_TRY_CUDA(cudaGetLastError());
    int flags = 0, bad = 0;
    FEMD_TRY(read_status(ctx, &flags, &bad));
    K->f32_valid = false;
    if (flags & ST_ZERODIAG) {
        set_error("Jacobi: zero diagonal entry in row " + std::to_string(bad));
        return FEMD_EZERODIAG;
    }
    K->inv_valid = true;
    return FEMD_OK;
}

int femd_cuda_matrix_set_inv_diag(femd_ctx ctx, femd_matrix K, const double *inv_dev)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K, "Jacobi: NULL argument");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "Jacobi: the matrix must be square");
    const int n = K->pattern->nrows;
    FEMD_CHECK_ARG(n == 0 || inv_dev, "Jacobi: NULL inverse diagonal");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    if (n && inv_dev != K->inv.p)
        FEMD_TRY_CUDA(cudaMemcpyAsync(K->inv.p, inv_dev, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    K->f32_valid = false;
    K->inv_valid = true;
    return FEMD_OK;
}

int femd_cuda_matrix_inv_diag_to_host(femd_matrix K, double *inv_host)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(K && inv_host, "inv_diag_to_host: NULL argument");
    FEMD_TRY_CUDA(cudaSetDevice(K->ctx->device));
    if (K->pattern->nrows)
        FEMD_TRY_CUDA(cudaMemcpyAsync(inv_host, K->inv.p, (size_t)K->pattern->nrows * sizeof(double), cudaMemcpyDeviceToHost,
                                      K->ctx->stream));
    FEMD_TRY_CUDA(cudaStreamSynchronize(K->ctx->stream));
    return FEMD_OK;
}

int femd_cuda_spmv(femd_ctx ctx, femd_matrix K, const double *x_dev, double *y_dev)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K, "matvec: NULL argument");
    const int n = K->pattern->nrows;
    FEMD_CHECK_ARG(n == 0 || (x_dev && y_dev), "matvec: NULL vector");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    if (n == 0) return FEMD_OK;
    const int tpr = pick_tpr(K);
    launch_spmv<double, double, false>(tpr, spmv_grid(ctx, n, tpr), ctx->stream, K->pattern->indptr.p, K->pattern->indices.p,
                                       K->data.p, x_dev, y_dev, n, nullptr, nullptr);
    FEMD_TRY_CUDA(cudaGetLastError());
    return FEMD_OK;
}

int femd_cuda_spmv_autotune(femd_ctx ctx, femd_matrix K, int set, int *tpr_out, double *us_out)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K, "spmv_autotune: NULL argument");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    const int n = K->pattern->nrows;
    if (n == 0) { if (tpr_out) *tpr_out = pick_tpr(K); if (us_out) *us_out = 0.0; return FEMD_OK; }
    DevBuf<double> x, y;
    FEMD_TRY(x.alloc(K->pattern->ncols + 1));
    FEMD_TRY(y.alloc(n + 1));
    FEMD_TRY_CUDA(cudaMemsetAsync(x.p, 0, (K->pattern->ncols + 1) * sizeof(double), ctx->stream));
    cudaEvent_t e0, e1;
    FEMD_TRY_CUDA(cudaEventCreate(&e0));
    FEMD_TRY_CUDA(cudaEventCreate(&e1));
    // shapes: threads per row 2..32 x loads in flight per lane 1, 2, 4
    std::vector<int> cand;
    for (int t : {2, 4, 8, 16, 32})
        for (int u : {1, 2, 4}) cand.push_back(t | (u << 8));
    int best = pick_tpr(K);
    float best_ms = 1e30f;
    for (int c : cand) {
        const unsigned g = spmv_grid(ctx, n, c);
        for (int w = 0; w < 2; ++w)
            launch_spmv<double, double, false>(c, g, ctx->stream, K->pattern->indptr.p, K->pattern->indices.p, K->data.p,
                                               x.p, y.p, n, nullptr, nullptr);
        cudaEventRecord(e0, ctx->stream);
        const int reps = 5;
        for (int r = 0; r < reps; ++r)
            launch_spmv<double, double, false>(c, g, ctx->stream, K->pattern->indptr.p, K->pattern->indices.p, K->data.p,
                                               x.p, y.p, n, nullptr, nullptr);
        cudaEventRecord(e1, ctx->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) { cudaEventDestroy(e0); cudaEventDestroy(e1); set_error(cudaGetErrorString(e)); return FEMD_ECUDA; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= reps;
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (set) K->spmv_tpr = best;
    if (tpr_out) *tpr_out = best;
    if (us_out) *us_out = best_ms * 1e3;
    return FEMD_OK;
}

int femd_cuda_spmv_set_tpr(femd_matrix K, int tpr)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(K, "spmv_set_tpr: not a matrix handle");
    const int t = shape_tpr(tpr), u = tpr >> 8;
    FEMD_CHECK_ARG(tpr == 0 || ((t == 2 || t == 4 || t == 8 || t == 16 || t == 32) && (u == 0 || u == 1 || u == 2 || u == 4)),
                   "spmv_set_tpr: shape = threads per row (0 heuristic, 2..32) | loads per lane (1, 2, 4) << 8");
    K->spmv_tpr = tpr;
    return FEMD_OK;
}

int femd_cuda_asymmetry(femd_ctx ctx, femd_matrix K, double *out)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K && out, "asymmetry: NULL argument");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    if (K->pattern->nrows != K->pattern->ncols) { *out = 1.0; return FEMD_OK; }
    DevBuf<unsigned long long> m;
    FEMD_TRY(m.alloc(2));
    FEMD_TRY_CUDA(cudaMemsetAsync(m.p, 0, 2 * sizeof(unsigned long long), ctx->stream));
    const int n = K->pattern->nrows;
    if (n) k_asym<<<grid_for((size_t)n, 256, (unsigned)ctx->sm_count * 8), 256, 0, counted(ctx->stream)>>>(
        K->pattern->indptr.p, K->pattern->indices.p, K->data.p, n, m.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    unsigned long long h[2];
    FEMD_TRY_CUDA(cudaMemcpyAsync(h, m.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    FEMD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    double big, dif;
    memcpy(&big, &h[0], 8);
    memcpy(&dif, &h[1], 8);
    *out = big > 0.0 ? dif / big : 0.0;
    return FEMD_OK;
}

int femd_cuda_combine(femd_ctx ctx, double alpha, femd_matrix A, double beta, femd_matrix B, femd_matrix C)
{
    clear_error();
    A = as_matrix(A); B = as_matrix(B); C = as_matrix(C);
    FEMD_CHECK_ARG(ctx && A && B && C, "combine: NULL argument");
    FEMD_CHECK_ARG(A->pattern == B->pattern && A->pattern == C->pattern,
                   "combine: A, B and C must share one pattern (CSRMatrix: shape mismatch in a sum)");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    const long long nnz = A->pattern->nnz;
    if (nnz) k_combine<<<grid_for((size_t)nnz, 256, 1u << 20), 256, 0, counted(ctx->stream)>>>(alpha, A->data.p, beta, B->data.p, C->data.p, nnz);
    FEMD_TRY_CUDA(cudaGetLastError());
    C->f32_valid = false;
    return FEMD_OK;
}

int femd_cuda_cg_jacobi(femd_ctx ctx, femd_matrix K, int use_jacobi, const double *b_dev, double *x_dev, int max_iter,
                        double tol, femd_cg_result *res)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K && res, "cg: NULL argument");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "cg: the matrix must be square");
    const int n = K->pattern->nrows;
    FEMD_CHECK_ARG(n == 0 || (b_dev && x_dev), "cg: NULL vector");
    FEMD_CHECK_ARG(max_iter >= 0, "cg: max_iter must be >= 0");
    FEMD_CHECK_ARG(!use_jacobi || K->inv_valid, JACOBI_MISSING);
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    *res = femd_cg_result{1, 0, 0.0, 0, FEMD_OK, 0, 0.0};
    if (n == 0) return FEMD_OK;
    return cg_run(ctx, K, use_jacobi != 0, b_dev, x_dev, max_iter, tol, res);
}

int femd_cuda_pcg_mixed(femd_ctx ctx, femd_matrix K, const double *b_dev, double *x_dev, int max_iter, double tol,
                        femd_cg_result *res)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K && res, "pcg_mixed: NULL argument");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "pcg_mixed: the matrix must be square");
    const int n = K->pattern->nrows;
    FEMD_CHECK_ARG(n == 0 || (b_dev && x_dev), "pcg_mixed: NULL vector");
    FEMD_CHECK_ARG(K->inv_valid, JACOBI_MISSING);
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    *res = femd_cg_result{1, 0, 0.0, 0, FEMD_OK, 0, 0.0};
    if (n == 0) return FEMD_OK;
    return mixed_run(ctx, K, b_dev, x_dev, max_iter, tol, res);
}

int femd_cuda_kernel_time(femd_ctx ctx, femd_matrix K, int kernel, int reps, double *us_out)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K && us_out && reps >= 1, "kernel_time: bad arguments");
    FEMD_CHECK_ARG(kernel >= 0 && kernel <= 2, "kernel_time: kernel is 0 (SpMV + p.Ap), 1 (fused update) or 2 (direction)");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "kernel_time: the matrix must be square");
    FEMD_CHECK_ARG(K->inv_valid, JACOBI_MISSING);
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    const int n = K->pattern->nrows;
    *us_out = 0.0;
    if (n == 0) return FEMD_OK;
    SolverWS *Wp = nullptr;
    FEMD_TRY(get_ws(ctx, K, &Wp));
    SolverWS &W = *Wp;
    cudaStream_t s = ctx->stream;
    femd_pattern P = K->pattern;
    // a state that never stops the loop: max_iter huge, r = p = D^-1 (so ||r||, r.z and p.Ap stay
    // positive for an SPD matrix), alpha and beta 0 (every launch streams the same bytes and leaves
    // the vectors as they are)
    CGState<double> S{};
    S.rz = 1.0;
    S.max_iter = INT_MAX;
    *W.st_host = S;
    const unsigned gn = grid_for((size_t)n, 256, 1u << 20);
    k_combine<<<gn, 256, 0, counted(s)>>>(1.0, K->inv.p, 0.0, K->inv.p, W.r.p, n);
    k_combine<<<gn, 256, 0, counted(s)>>>(1.0, K->inv.p, 0.0, K->inv.p, W.p.p, n);
    FEMD_TRY_CUDA(cudaMemsetAsync(W.wx.p, 0, (size_t)n * sizeof(double), s));
    auto one = [&]() {
        if (kernel == 0)
            launch_spmv<double, double, true>(W.shape, W.gs, s, P->indptr.p, P->indices.p, K->data.p, W.p.p, W.Ap.p, n, W.part.p,
                                              W.st.p);
        else if (kernel == 1)
            k_cg_update<double, true><<<W.gr, RED_BLOCK, 0, counted(s)>>>(W.wx.p, W.r.p, W.p.p, W.Ap.p, K->inv.p, n, W.part.p,
                                                                          W.st.p, 0);
        else
            k_cg_direction<double, true><<<W.gr, RED_BLOCK, 0, counted(s)>>>(W.p.p, W.r.p, K->inv.p, n, W.st.p);
    };
    for (int w = 0; w < 3; ++w) {
        FEMD_TRY_CUDA(cudaMemcpyAsync(W.st.p, W.st_host, sizeof(CGState<double>), cudaMemcpyHostToDevice, s));
        one();
    }
    FEMD_TRY_CUDA(cudaMemcpyAsync(W.st.p, W.st_host, sizeof(CGState<double>), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaEventRecord(W.e0, s));
    for (int r = 0; r < reps; ++r) one();
    FEMD_TRY_CUDA(cudaEventRecord(W.e1, s));
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaEventSynchronize(W.e1));
    float ms = 0.f;
    FEMD_TRY_CUDA(cudaEventElapsedTime(&ms, W.e0, W.e1));
    *us_out = (double)ms * 1e3 / reps;
    return FEMD_OK;
}

int femd_cuda_cg_precond(femd_ctx ctx, femd_matrix K, femd_precond P, const double *b_dev, double *x_dev, int max_iter,
                         double tol, femd_cg_result *res)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K && P && res, "cg: NULL argument");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "cg: the matrix must be square");
    FEMD_CHECK_ARG(precond_pattern(P) == K->pattern && precond_ctx(P) == ctx,
                   "krylov: the preconditioner was built on another matrix pattern or context");
    const int n = K->pattern->nrows;
    FEMD_CHECK_ARG(n == 0 || (b_dev && x_dev), "cg: NULL vector");
    FEMD_CHECK_ARG(max_iter >= 0, "cg: max_iter must be >= 0");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    *res = femd_cg_result{1, 0, 0.0, 0, FEMD_OK, 0, 0.0};
    if (n == 0) return FEMD_OK;
    return pc_run(ctx, K, P, b_dev, x_dev, max_iter, tol, res);
}

int femd_cuda_cg_solve_host(femd_ctx ctx, int n, const int *indptr_host, const int *indices_host, const double *data_host,
                            const double *inv_host, const double *b_host, const double *x0_host, double *x_host,
                            int max_iter, double tol, femd_cg_result *res)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && indptr_host && res && b_host && x_host, "cg: NULL argument");
    FEMD_CHECK_ARG(n >= 0, "cg: negative size");
    femd_pattern P = nullptr;
    FEMD_TRY(femd_cuda_pattern_from_csr_host(ctx, n, n, indptr_host, indices_host, &P));
    femd_matrix K = nullptr;
    int st = femd_cuda_matrix_create(ctx, P, &K);
    if (st) { femd_cuda_release(P); return st; }
    DevBuf<double> b, x;
    cudaStream_t s = ctx->stream;
    const long long nnz = P->nnz;
    st = b.alloc((size_t)n + 1);
    if (!st) st = x.alloc((size_t)n + 1);
    cudaError_t e = cudaSuccess;
    if (!st) {
        if (nnz) e = cudaMemcpyAsync(K->data.p, data_host, (size_t)nnz * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && inv_host) e = cudaMemcpyAsync(K->inv.p, inv_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s);
        if (inv_host) K->inv_valid = true;
        if (e == cudaSuccess) e = cudaMemcpyAsync(b.p, b_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) {
            if (x0_host) e = cudaMemcpyAsync(x.p, x0_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s);
            else e = cudaMemsetAsync(x.p, 0, (size_t)n * sizeof(double), s);
        }
        if (e != cudaSuccess) { set_error(std::string("cg: ") + cudaGetErrorString(e)); st = FEMD_ECUDA; }
    }
    if (!st) st = femd_cuda_cg_jacobi(ctx, K, inv_host != nullptr, b.p, x.p, max_iter, tol, res);
    if (!st && n) {
        e = cudaMemcpyAsync(x_host, x.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error(std::string("cg: ") + cudaGetErrorString(e)); st = FEMD_ECUDA; }
    }
    femd_cuda_release(K);
    femd_cuda_release(P);
    return st;
}

}  // extern "C"

// ==============================================================================================
// Jacobi-PCG that allocates nothing.
//
// For callers that cannot call cudaMalloc while they solve: a solver embedded in a program whose
// allocator already owns the device memory (a serving engine that reserved the HBM up front, or a
// framework whose memory pool must not be bypassed), or a latency-bound loop where an allocation
// and the device synchronization it may bring are not allowed.  The three work vectors, the
// reduction partials and the scalar state of the solve live in one fixed static device array,
// g_cg_scratch, sized for NOALLOC_MAX_ROWS rows; larger systems are rejected.  The kernels and
// launch shapes are those of femd_cuda_cg_jacobi, so the iterates are the same.
// ==============================================================================================
namespace femd {

static constexpr int NOALLOC_MAX_ROWS = 1 << 20;             // 1,048,576 rows
static constexpr int NOALLOC_PART = 3 * 8192;                // reduction partials (3 per block)
static constexpr size_t NOALLOC_STATE_DOUBLES = (sizeof(CGState<double>) + sizeof(double) - 1) / sizeof(double);
static constexpr size_t NOALLOC_DOUBLES = 3 * (size_t)NOALLOC_MAX_ROWS + NOALLOC_PART + NOALLOC_STATE_DOUBLES;

// about 25 MB per device, held by every GPU that loads the library until the process exits
static __device__ __align__(256) double g_cg_scratch[NOALLOC_DOUBLES];

static constexpr int NOALLOC_MAX_DEVICES = 64;
// per device: the CUDA context the address was looked up in, and the address
static void *g_cg_scratch_ctx[NOALLOC_MAX_DEVICES] = {};
static double *g_cg_scratch_addr[NOALLOC_MAX_DEVICES] = {};
static std::mutex g_cg_scratch_lock;

// The driver's cuCtxGetCurrent, reached through the runtime (the library links no libcuda): the
// key that tells a cached address from one of a context that has since been destroyed and made
// again (after cudaDeviceReset the array lives at a new address in the new context).
typedef int (*CtxGetCurrentFn)(void **);
static CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

// The device address of g_cg_scratch on the current device (host code cannot use the symbol
// itself: on the host it names a stand-in, not device memory).  Looked up once per device and
// CUDA context; the caller has made the device current.
static int noalloc_scratch(int device, double **out)
{
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) {
        set_error("cg_jacobi_noalloc: device index " + std::to_string(device) + " is out of range");
        return FEMD_EINVAL;
    }
    std::lock_guard<std::mutex> g(g_cg_scratch_lock);
    void *cur = nullptr;
    const CtxGetCurrentFn get = ctx_get_current();
    if (!get || get(&cur) != 0 || !cur) {
        set_error("cg_jacobi_noalloc: no current CUDA context on the device");
        return FEMD_ECUDA;
    }
    if (!g_cg_scratch_addr[device] || g_cg_scratch_ctx[device] != cur) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_cg_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("cg_jacobi_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return FEMD_ECUDA;
        }
        g_cg_scratch_addr[device] = static_cast<double *>(p);
        g_cg_scratch_ctx[device] = cur;
    }
    *out = g_cg_scratch_addr[device];
    return FEMD_OK;
}

}  // namespace femd

extern "C" {

int femd_cuda_cg_jacobi_noalloc(femd_ctx ctx, femd_matrix K, int use_jacobi, const double *b_dev, double *x_dev,
                                int max_iter, double tol, femd_cg_result *res)
{
    clear_error();
    K = as_matrix(K);
    FEMD_CHECK_ARG(ctx && K && res, "cg_jacobi_noalloc: NULL argument");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "cg_jacobi_noalloc: the matrix must be square");
    const int n = K->pattern->nrows;
    FEMD_CHECK_ARG(n <= NOALLOC_MAX_ROWS, "cg_jacobi_noalloc: " + std::to_string(n) + " rows exceed the fixed scratch of " +
                                              std::to_string(NOALLOC_MAX_ROWS) + " rows; use femd_cuda_cg_jacobi");
    FEMD_CHECK_ARG(n == 0 || (b_dev && x_dev), "cg_jacobi_noalloc: NULL vector");
    // the solve works on x in place and reads b every chunk: the two must not share memory
    FEMD_CHECK_ARG(n == 0 || b_dev + n <= x_dev || x_dev + n <= b_dev,
                   "cg_jacobi_noalloc: b and x overlap; pass separate vectors");
    FEMD_CHECK_ARG(max_iter >= 0, "cg_jacobi_noalloc: max_iter must be >= 0");
    FEMD_CHECK_ARG(!use_jacobi || K->inv_valid, JACOBI_MISSING);
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    // the solve reads its state back between chunks (a stream synchronization), which a stream
    // capture does not allow
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    FEMD_TRY_CUDA(cudaStreamIsCapturing(ctx->stream, &cap));
    FEMD_CHECK_ARG(cap == cudaStreamCaptureStatusNone,
                   "cg_jacobi_noalloc: the context's stream is being captured; the solve synchronizes between chunks "
                   "and cannot be captured");
    *res = femd_cg_result{1, 0, 0.0, 0, FEMD_OK, 0, 0.0};
    if (n == 0) return FEMD_OK;
    double *base = nullptr;
    FEMD_TRY(noalloc_scratch(ctx->device, &base));
    const femd_pattern P = K->pattern;
    const bool jac = use_jacobi != 0;
    const int tpr = pick_tpr(K);
    const unsigned gs = spmv_grid(ctx, n, tpr), gr = red_grid(ctx, n);
    FEMD_CHECK_ARG(3 * (size_t)std::max(gs, gr) + 3 <= (size_t)NOALLOC_PART,
                   "cg_jacobi_noalloc: the device has more blocks than the fixed reduction scratch holds");
    double *r = base, *p = base + NOALLOC_MAX_ROWS, *Ap = base + 2 * (size_t)NOALLOC_MAX_ROWS;
    double *part = base + 3 * (size_t)NOALLOC_MAX_ROWS;
    CGState<double> *st = reinterpret_cast<CGState<double> *>(part + NOALLOC_PART);
    cudaStream_t s = ctx->stream;
    // the array keeps the previous call's contents: the state (with its reduction ticket) must
    // start at zero; r, p, Ap and the partials are written before they are read
    FEMD_TRY_CUDA(cudaMemsetAsync(st, 0, sizeof(CGState<double>), s));
    launch_spmv<double, double, false>(tpr, gs, s, P->indptr.p, P->indices.p, K->data.p, x_dev, Ap, n, nullptr, nullptr);
    if (jac) k_cg_start<true><<<gr, RED_BLOCK, 0, counted(s)>>>(b_dev, Ap, r, p, K->inv.p, n, part, st, tol);
    else k_cg_start<false><<<gr, RED_BLOCK, 0, counted(s)>>>(b_dev, Ap, r, p, nullptr, n, part, st, tol);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaMemcpyAsync(&st->max_iter, &max_iter, sizeof(int), cudaMemcpyHostToDevice, s));
    CGState<double> S;
    const int CH = 16;
    const long long max_chunks = (long long)max_iter / CH + 2;
    for (long long c = 0; c < max_chunks; ++c) {
        for (int k = 0; k < CH; ++k) {
            launch_spmv<double, double, true>(tpr, gs, s, P->indptr.p, P->indices.p, K->data.p, p, Ap, n, part, st);
            if (jac) {
                k_cg_update<double, true><<<gr, RED_BLOCK, 0, counted(s)>>>(x_dev, r, p, Ap, K->inv.p, n, part, st, 0);
                k_cg_direction<double, true><<<gr, RED_BLOCK, 0, counted(s)>>>(p, r, K->inv.p, n, st);
            } else {
                k_cg_update<double, false><<<gr, RED_BLOCK, 0, counted(s)>>>(x_dev, r, p, Ap, nullptr, n, part, st, 0);
                k_cg_direction<double, false><<<gr, RED_BLOCK, 0, counted(s)>>>(p, r, nullptr, n, st);
            }
        }
        FEMD_TRY_CUDA(cudaGetLastError());
        FEMD_TRY_CUDA(cudaMemcpyAsync(&S, st, sizeof(S), cudaMemcpyDeviceToHost, s));
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));
        if (S.done) break;
    }
    // final true residual (cg.hpp:222-237)
    launch_spmv<double, double, false>(tpr, gs, s, P->indptr.p, P->indices.p, K->data.p, x_dev, Ap, n, nullptr, nullptr);
    k_cg_finish<<<gr, RED_BLOCK, 0, counted(s)>>>(b_dev, Ap, r, n, part, st);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaMemcpyAsync(&S, st, sizeof(S), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    if (S.nb == 0.0) {
        FEMD_TRY_CUDA(cudaMemsetAsync(x_dev, 0, (size_t)n * sizeof(double), s));
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));
        return FEMD_OK;
    }
    res->iterations = S.it;
    res->breakdown = S.breakdown;
    res->residual = S.res64 / S.nb;
    int conv = !S.breakdown && res->residual <= tol * (1.0 + 1e-6) + 1e-15;
    if (!conv && !S.breakdown && res->residual <= 10.0 * tol && S.it < max_iter) conv = 1;
    res->converged = conv;
    return FEMD_OK;
}

}  // extern "C"
