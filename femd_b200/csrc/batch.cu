// batch.cu -- K7: many independent Jacobi-PCG solves in one persistent, cooperative launch.
//
// Every problem p gets a team of T_p thread blocks (T_p from its size alone).  Blocks take
// (problem, member) slots from a queue, largest teams first; a member owns a contiguous range of
// the problem's rows.  The members of a team meet at software barriers (a counter per problem,
// waited on with a bounded spin: a wait that runs out sets FEMD_ETIMEOUT and every block
// returns).  Dot products are summed per block, then across the team's members in member order,
// so a problem's iterates depend on the problem alone -- the same bits alone or in any mix.
//
// The launch is cooperative (all blocks resident), so a team whose members are still busy
// elsewhere only delays; at most one team is incomplete at any time (slots are taken in order),
// so every team completes.
//
// Modes: FP64 Jacobi-PCG (cg.hpp:296-350 semantics) or mixed precision (FP32 matrix copy,
// vectors and reductions; FP64 residual b - A x and solution update at reliable updates).
#include <algorithm>
#include <cmath>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"

namespace femd {

static constexpr int BB = 256;                 // threads per block
static constexpr long long SPIN_LIMIT = 1ll << 25;   // default bound: x ~64 ns sleeps, a few seconds at most

struct BProb {
    int n, tpr, team, max_iter;
    double tol;
    const int *indptr, *indices;
    const float *A32, *inv32;
    const double *A64, *inv64;
    const double *b;
    double *x;
    float *r32, *p32, *Ap32, *d32;
    double *r64, *p64, *Ap64;
    double *part;          // 8 kinds x team
    unsigned *bar;
    int *res_i;            // [0] iterations [1] converged [2] breakdown [3] status [4] reliable updates
    double *res_d;         // [0] residual
};

struct BQueue {
    unsigned next;
    int flag;              // FEMD_ETIMEOUT / FEMD_EABORT seen by any block
    long long spin_limit;  // the bound of every barrier wait (spins)
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// team barrier: returns false when the batch has to stop (timeout or abort)
__device__ bool team_barrier(const BProb &P, unsigned &phase, BQueue *q, volatile const int *abort_flag)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (P.team > 1) {
            __threadfence();
            atomicAdd(P.bar, 1u);
            const unsigned target = (phase + 1) * (unsigned)P.team;
            long long spins = 0;
            while (ld_acquire(P.bar) < target) {
                if (((spins & 1023) == 0) && *(volatile int *)&q->flag) { ok = 0; break; }
                if (++spins > q->spin_limit) { atomicCAS(&q->flag, 0, FEMD_ETIMEOUT); ok = 0; break; }
                __nanosleep(64);
            }
            __threadfence();
        }
        // the host's abort flag (mapped host memory, a PCIe read): every 64th barrier
        if (abort_flag && (phase & 63) == 0 && *abort_flag) atomicCAS(&q->flag, 0, FEMD_EABORT);
        if (*(volatile int *)&q->flag) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    ++phase;
    return s_ok != 0;
}

template <class T>
__device__ __forceinline__ T block_sum(T v, T *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T s = T(0);
    for (int k = 0; k < BB / 32; ++k) s += sh[k];
    return s;
}

// team reduction of NV values of kind base..base+NV-1: each member writes its block sum, the team
// meets, and warp 0 of every member sums the T partials in one fixed order (lane-strided, then a
// shuffle tree), so the result depends on T and the partials only
template <int NV>
__device__ bool team_reduce(const BProb &P, int m, int base, double (&v)[NV], unsigned &phase, BQueue *q,
                            volatile const int *abort_flag)
{
    __shared__ double sh[BB / 32];
    __shared__ double tot[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        v[k] = block_sum<double>(v[k], sh);
        if (threadIdx.x == 0) P.part[(base + k) * P.team + m] = v[k];
    }
    if (!team_barrier(P, phase, q, abort_flag)) return false;
    if (P.team == 1) return true;
    if (threadIdx.x < 32) {
        const volatile double *part = P.part;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = 0.0;
            for (int u = threadIdx.x; u < P.team; u += 32) s += part[(base + k) * P.team + u];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (threadIdx.x == 0) tot[k] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = tot[k];
    return true;
}

// y = A x on rows [r0, r1) with TPR lanes per row; returns this thread's share of x.y.  x and y are
// written during the launch (by this team's members), so they take plain coherent loads: no
// __restrict__, which would let the compiler use the non-coherent read-only path
template <class V, class X, int TPR>
__device__ __forceinline__ double spmv_rows(const int *__restrict__ ip, const int *__restrict__ ix, const V *__restrict__ A,
                                            const X *x, X *y, int r0, int r1)
{
    const int lane = threadIdx.x % TPR;
    constexpr int GPW = 32 / TPR;
    const int w = threadIdx.x >> 5;
    double dot = 0.0;
    for (int i0 = r0 + w * GPW; i0 < r1; i0 += (BB / 32) * GPW) {
        const int i = i0 + (threadIdx.x & 31) / TPR;
        X s = X(0);
        if (i < r1) {
            const int lo = ip[i], hi = ip[i + 1];
            for (int q = lo + lane; q < hi; q += 2 * TPR) {
                const int c0 = ix[q];
                const V a0 = A[q];
                const bool two = q + TPR < hi;
                const int c1 = two ? ix[q + TPR] : c0;
                const V a1 = two ? A[q + TPR] : V(0);
                s += (X)a0 * x[c0];
                if (two) s += (X)a1 * x[c1];
            }
        }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, TPR);
        if (lane == 0 && i < r1) {
            y[i] = s;
            dot += (double)x[i] * (double)s;
        }
    }
    return dot;
}

template <class V, class X>
__device__ double spmv_dispatch(int tpr, const int *ip, const int *ix, const V *A, const X *x, X *y, int r0, int r1)
{
    switch (tpr) {
    case 2: return spmv_rows<V, X, 2>(ip, ix, A, x, y, r0, r1);
    case 4: return spmv_rows<V, X, 4>(ip, ix, A, x, y, r0, r1);
    case 8: return spmv_rows<V, X, 8>(ip, ix, A, x, y, r0, r1);
    case 16: return spmv_rows<V, X, 16>(ip, ix, A, x, y, r0, r1);
    default: return spmv_rows<V, X, 32>(ip, ix, A, x, y, r0, r1);
    }
}

// residual r64 = b - A64 x on [r0, r1): returns the shares of ||r||^2, and (mixed) of r32.(inv r32)
// after writing r32 = (float) r (mixed) or r64 (FP64 mode, into P.r64)
template <int TPR>
__device__ __forceinline__ void residual_rows(const BProb &P, int r0, int r1, bool mixed, double &rr, double &rz)
{
    const int lane = threadIdx.x % TPR;
    constexpr int GPW = 32 / TPR;
    const int w = threadIdx.x >> 5;
    for (int i0 = r0 + w * GPW; i0 < r1; i0 += (BB / 32) * GPW) {
        const int i = i0 + (threadIdx.x & 31) / TPR;
        double s = 0.0;
        if (i < r1)
            for (int q = P.indptr[i] + lane; q < P.indptr[i + 1]; q += TPR) s += P.A64[q] * P.x[P.indices[q]];
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, TPR);
        if (lane == 0 && i < r1) {
            const double ri = P.b[i] - s;
            rr += ri * ri;
            if (mixed) {
                const float rf = (float)ri;
                P.r32[i] = rf;
                rz += (double)(rf * rf * P.inv32[i]);
            } else {
                P.r64[i] = ri;
                rz += ri * ri * P.inv64[i];
            }
        }
    }
}

__device__ void residual_dispatch(const BProb &P, int r0, int r1, bool mixed, double &rr, double &rz)
{
    switch (P.tpr) {
    case 2: residual_rows<2>(P, r0, r1, mixed, rr, rz); break;
    case 4: residual_rows<4>(P, r0, r1, mixed, rr, rz); break;
    case 8: residual_rows<8>(P, r0, r1, mixed, rr, rz); break;
    case 16: residual_rows<16>(P, r0, r1, mixed, rr, rz); break;
    default: residual_rows<32>(P, r0, r1, mixed, rr, rz); break;
    }
}

// one problem, as member m of its team; returns false when the batch has to stop
template <bool MIXED>
__device__ bool solve_member(const BProb &P, int m, BQueue *q, volatile const int *abort_flag)
{
    const int n = P.n, T = P.team;
    const int r0 = (int)((long long)n * m / T), r1 = (int)((long long)n * (m + 1) / T);
    unsigned phase = 0;
    // start: x = x0 (given), r = b - A x, nb, rz, p = inv r; d = 0 (mixed)
    {
        double v[3] = {0.0, 0.0, 0.0};                     // ||r||^2, r.z, ||b||^2
        residual_dispatch(P, r0, r1, MIXED, v[0], v[1]);
        __syncthreads();                                   // r is written by row-group leaders, read strided
        for (int i = r0 + threadIdx.x; i < r1; i += BB) {
            v[2] += P.b[i] * P.b[i];
            if (MIXED) { P.p32[i] = P.inv32[i] * P.r32[i]; P.d32[i] = 0.0f; }
            else P.p64[i] = P.inv64[i] * P.r64[i];
        }
        if (!team_reduce<3>(P, m, 0, v, phase, q, abort_flag)) return false;
        const double nb = sqrt(v[2]), rn0 = sqrt(v[0]);
        if (nb == 0.0) {
            for (int i = r0 + threadIdx.x; i < r1; i += BB) P.x[i] = 0.0;
            if (m == 0 && threadIdx.x == 0) { P.res_i[0] = 0; P.res_i[1] = 1; P.res_i[2] = 0; P.res_d[0] = 0.0; }
            return true;
        }
        if (rn0 <= P.tol * nb) {
            if (m == 0 && threadIdx.x == 0) { P.res_i[0] = 0; P.res_i[1] = 1; P.res_i[2] = 0; P.res_d[0] = rn0 / nb; }
            return true;
        }
        double rz = v[1], maxr = rn0, rz_prev = rz;
        int it = 0, breakdown = 0, rus = 0;
        bool done = false;
        double res_final = rn0 / nb;
        if (!(rz > 0.0)) { breakdown = 1; done = true; }
        while (!done && it < P.max_iter) {
            // Ap = A p, p.Ap
            double pap[1];
            pap[0] = MIXED ? spmv_dispatch<float, float>(P.tpr, P.indptr, P.indices, P.A32, P.p32, P.Ap32, r0, r1)
                           : spmv_dispatch<double, double>(P.tpr, P.indptr, P.indices, P.A64, P.p64, P.Ap64, r0, r1);
            if (!team_reduce<1>(P, m, 3, pap, phase, q, abort_flag)) return false;
            if (!(pap[0] > 0.0)) { breakdown = 1; break; }
            const double alpha = rz / pap[0];
            // x (or d) += alpha p, r -= alpha Ap; ||r||^2, r.z
            double u[2] = {0.0, 0.0};
            for (int i = r0 + threadIdx.x; i < r1; i += BB) {
                if (MIXED) {
                    const float af = (float)alpha;
                    const float ri = P.r32[i] - af * P.Ap32[i];
                    P.r32[i] = ri;
                    P.d32[i] += af * P.p32[i];
                    u[0] += (double)(ri * ri);
                    u[1] += (double)(ri * ri * P.inv32[i]);
                } else {
                    const double ri = P.r64[i] - alpha * P.Ap64[i];
                    P.r64[i] = ri;
                    P.x[i] += alpha * P.p64[i];
                    u[0] += ri * ri;
                    u[1] += ri * ri * P.inv64[i];
                }
            }
            if (!team_reduce<2>(P, m, 4, u, phase, q, abort_flag)) return false;
            ++it;
            const double rn = sqrt(u[0]);
            double beta;
            if (!MIXED) {
                res_final = rn / nb;
                if (rn <= P.tol * nb) { done = true; break; }
                beta = u[1] / rz;
                rz = u[1];
                if (!(rz > 0.0)) { breakdown = 1; break; }
            } else {
                const bool ru = rn <= 0.1 * maxr || rn <= P.tol * nb || it >= P.max_iter || !(u[1] > 0.0);
                if (ru) {
                    // reliable update: x += d, d = 0; r = b - A64 x (FP64), r32 = (float) r
                    for (int i = r0 + threadIdx.x; i < r1; i += BB) { P.x[i] += (double)P.d32[i]; P.d32[i] = 0.0f; }
                    if (!team_barrier(P, phase, q, abort_flag)) return false;
                    double w2[2] = {0.0, 0.0};
                    residual_dispatch(P, r0, r1, true, w2[0], w2[1]);
                    if (!team_reduce<2>(P, m, 6, w2, phase, q, abort_flag)) return false;
                    ++rus;
                    const double rt = sqrt(w2[0]);
                    res_final = rt / nb;
                    maxr = rt;
                    if (rt <= P.tol * nb || it >= P.max_iter) { done = true; break; }
                    if (!(w2[1] > 0.0)) { breakdown = 1; break; }
                    beta = w2[1] / rz;
                    rz = w2[1];
                } else {
                    rz_prev = rz;
                    beta = u[1] / rz;
                    rz = u[1];
                }
            }
            (void)rz_prev;
            // p = inv r + beta p
            for (int i = r0 + threadIdx.x; i < r1; i += BB) {
                if (MIXED) P.p32[i] = P.inv32[i] * P.r32[i] + (float)beta * P.p32[i];
                else P.p64[i] = P.inv64[i] * P.r64[i] + beta * P.p64[i];
            }
            if (!team_barrier(P, phase, q, abort_flag)) return false;
        }
        // the true residual for the FP64 path (cg.hpp:222-237): r = b - A x
        if (!MIXED) {
            if (!team_barrier(P, phase, q, abort_flag)) return false;
            double w3[2] = {0.0, 0.0};
            residual_dispatch(P, r0, r1, false, w3[0], w3[1]);
            if (!team_reduce<2>(P, m, 6, w3, phase, q, abort_flag)) return false;
            res_final = sqrt(w3[0]) / nb;
        } else if (breakdown) {
            for (int i = r0 + threadIdx.x; i < r1; i += BB) { P.x[i] += (double)P.d32[i]; P.d32[i] = 0.0f; }
        }
        if (m == 0 && threadIdx.x == 0) {
            const double tol = P.tol;
            int conv = !breakdown && res_final <= tol * (1.0 + 1e-6) + 1e-15;
            if (!conv && !breakdown && res_final <= 10.0 * tol && it < P.max_iter) conv = 1;
            P.res_i[0] = it; P.res_i[1] = conv; P.res_i[2] = breakdown; P.res_i[4] = rus;
            P.res_d[0] = res_final;
        }
    }
    return true;
}

template <bool MIXED>
__global__ void __launch_bounds__(BB) k_batch_pcg(const BProb *__restrict__ probs, const int *__restrict__ slot_prob,
                                                  const int *__restrict__ slot_member, int nslots, BQueue *q,
                                                  volatile const int *abort_flag)
{
    __shared__ int s_slot, s_stop;
    for (;;) {
        if (threadIdx.x == 0) {
            s_slot = (int)atomicAdd(&q->next, 1u);
            s_stop = *(volatile int *)&q->flag;
        }
        __syncthreads();
        const int slot = s_slot, stop = s_stop;
        __syncthreads();
        if (slot >= nslots || stop) return;
        const BProb P = probs[slot_prob[slot]];
        if (!solve_member<MIXED>(P, slot_member[slot], q, abort_flag)) {
            if (threadIdx.x == 0) P.res_i[3] = *(volatile int *)&q->flag ? *(volatile int *)&q->flag : FEMD_ETIMEOUT;
            return;
        }
    }
}

// f32 copies of a matrix's values and inverse diagonal
__global__ void k_batch_f32(const double *__restrict__ a, float *__restrict__ b, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

}  // namespace femd

using namespace femd;

struct femd_batch_s : femd::HandleBase {
    femd_ctx ctx = nullptr;
    int nprob = 0;
    std::vector<femd_matrix> mats;
    std::vector<int> team, tpr;
    std::vector<int> order;                    // problems, largest teams first
    DevBuf<BProb> d_probs;
    DevBuf<int> d_slot_prob, d_slot_member, d_res_i;
    DevBuf<double> d_res_d, d_part;
    DevBuf<unsigned> d_bar;
    DevBuf<BQueue> d_queue;
    DevBuf<float> f32;                          // all problems' FP32 values, inv, r, p, Ap, d
    DevBuf<double> f64;                         // all problems' FP64 r, p, Ap
    std::vector<BProb> probs;
    int nslots = 0, grid = 0, team_target = 0;
    int ghost = -1;                             // test hook: this problem waits for a member that never comes
    long long spin_limit = SPIN_LIMIT;
    int *abort_host = nullptr;                  // mapped pinned flag
    int *abort_dev = nullptr;
    femd_batch_s() : HandleBase(femd::KIND_BATCH) {}
    ~femd_batch_s() override { if (abort_host) cudaFreeHost(abort_host); }
};

static femd_batch_s *as_batch(void *h)
{
    femd_batch_s *b = static_cast<femd_batch_s *>(h);
    return (b && b->kind == KIND_BATCH) ? b : nullptr;
}

extern "C" {

int femd_cuda_batch_create(femd_ctx ctx, int nprob, const femd_matrix *mats, int nnz_per_block, femd_batch *out)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && out && nprob >= 1 && mats, "batch_create: bad arguments");
    *out = nullptr;
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    auto B = new femd_batch_s();
    std::unique_ptr<femd_batch_s> guard(B);
    B->ctx = ctx;
    B->nprob = nprob;
    B->mats.assign(mats, mats + nprob);
    // resident blocks (cooperative launch)
    int bps = 0;
    FEMD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_batch_pcg<true>, BB, 0));
    int bps64 = 0;
    FEMD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps64, k_batch_pcg<false>, BB, 0));
    bps = std::min(bps, bps64);
    FEMD_CHECK_ARG(bps >= 1, "batch_create: the batch kernel does not fit on an SM");
    B->grid = bps * ctx->sm_count;
    B->team_target = nnz_per_block > 0 ? nnz_per_block : 65536;
    size_t nf32 = 0, nf64 = 0;
    B->team.resize(nprob);
    B->tpr.resize(nprob);
    for (int p = 0; p < nprob; ++p) {
        femd_matrix K = mats[p];
        FEMD_CHECK_ARG(K && K->kind == KIND_MATRIX, "batch_create: not a matrix handle");
        FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "batch_create: the matrices must be square");
        const long long nnz = K->pattern->nnz;
        const int n = K->pattern->nrows;
        int T = (int)std::min<long long>((nnz + B->team_target - 1) / B->team_target, (long long)B->grid / 2);
        T = std::max(1, std::min(T, std::max(1, n / 64)));
        B->team[p] = T;
        const int shape = K->spmv_tpr ? K->spmv_tpr : 0;
        const double avg = n ? (double)nnz / n : 1.0;
        B->tpr[p] = shape ? (shape & 0xff) : (avg <= 6 ? 4 : avg <= 14 ? 8 : avg <= 28 ? 16 : 32);
        nf32 += (size_t)nnz + 6 * (size_t)n + 16;
        nf64 += 3 * (size_t)n + 4;
    }
    B->order.resize(nprob);
    std::iota(B->order.begin(), B->order.end(), 0);
    std::stable_sort(B->order.begin(), B->order.end(), [&](int a, int b) {
        if (B->team[a] != B->team[b]) return B->team[a] > B->team[b];
        return B->mats[a]->pattern->nnz > B->mats[b]->pattern->nnz;
    });
    std::vector<int> sp, sm;
    for (int p : B->order)
        for (int m = 0; m < B->team[p]; ++m) { sp.push_back(p); sm.push_back(m); }
    B->nslots = (int)sp.size();
    const size_t totteam = sp.size();
    int st;
    if ((st = B->f32.alloc(nf32)) || (st = B->f64.alloc(nf64)) || (st = B->d_probs.alloc(nprob)) ||
        (st = B->d_slot_prob.alloc(totteam)) || (st = B->d_slot_member.alloc(totteam)) ||
        (st = B->d_res_i.alloc(8 * (size_t)nprob)) || (st = B->d_res_d.alloc(2 * (size_t)nprob)) ||
        (st = B->d_part.alloc(8 * totteam + 8)) || (st = B->d_bar.alloc(nprob)) || (st = B->d_queue.alloc(1)))
        return st;
    FEMD_TRY_CUDA(cudaHostAlloc(&B->abort_host, sizeof(int), cudaHostAllocMapped));
    *B->abort_host = 0;
    FEMD_TRY_CUDA(cudaHostGetDevicePointer(&B->abort_dev, B->abort_host, 0));
    // carve the per-problem vectors
    B->probs.resize(nprob);
    size_t o32 = 0, o64 = 0, opart = 0;
    std::vector<size_t> part_off(nprob);
    for (int p : B->order) { part_off[p] = opart; opart += 8 * (size_t)B->team[p]; }
    for (int p = 0; p < nprob; ++p) {
        femd_matrix K = mats[p];
        const int n = K->pattern->nrows;
        const long long nnz = K->pattern->nnz;
        BProb &P = B->probs[p];
        P = BProb{};
        P.n = n;
        P.tpr = B->tpr[p];
        P.team = B->team[p];
        P.indptr = K->pattern->indptr.p;
        P.indices = K->pattern->indices.p;
        P.A64 = K->data.p;
        P.inv64 = K->inv.p;
        float *f = B->f32.p + o32;
        P.A32 = f; f += nnz;
        P.inv32 = f; f += n;
        P.r32 = f; f += n;
        P.p32 = f; f += n;
        P.Ap32 = f; f += n;
        P.d32 = f; f += n;
        o32 += (size_t)nnz + 6 * (size_t)n + 8;
        o32 = (o32 + 7) & ~(size_t)7;
        double *d = B->f64.p + o64;
        P.r64 = d; d += n;
        P.p64 = d; d += n;
        P.Ap64 = d;
        o64 += 3 * (size_t)n + 4;
        P.part = B->d_part.p + part_off[p];
        P.bar = B->d_bar.p + p;
        P.res_i = B->d_res_i.p + 8 * (size_t)p;
        P.res_d = B->d_res_d.p + 2 * (size_t)p;
    }
    FEMD_TRY_CUDA(cudaMemcpyAsync(B->d_slot_prob.p, sp.data(), sp.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    FEMD_TRY_CUDA(cudaMemcpyAsync(B->d_slot_member.p, sm.data(), sm.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    FEMD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = reinterpret_cast<femd_batch>(guard.release());
    return FEMD_OK;
}

int femd_cuda_batch_solve(femd_ctx ctx, femd_batch handle, const double *const *b_dev, double *const *x_dev, int max_iter,
                          double tol, int mixed, femd_cg_result *results)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(ctx && B && b_dev && x_dev && results, "batch_solve: NULL argument");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    // refresh the FP32 copies (the matrices may have been re-assembled)
    for (int p = 0; p < B->nprob; ++p) {
        femd_matrix K = B->mats[p];
        BProb &P = B->probs[p];
        FEMD_CHECK_ARG(b_dev[p] && x_dev[p], "batch_solve: NULL vector");
        P.b = b_dev[p];
        P.x = x_dev[p];
        P.tol = tol;
        P.max_iter = max_iter > 0 ? max_iter : std::max(1000, 10 * P.n);
        if (mixed) {
            const long long nnz = K->pattern->nnz;
            k_batch_f32<<<grid_for((size_t)nnz + 1, 256, 1u << 16), 256, 0, counted(s)>>>(K->data.p, const_cast<float *>(P.A32), nnz);
            k_batch_f32<<<grid_for((size_t)P.n + 1, 256, 1u << 16), 256, 0, counted(s)>>>(K->inv.p, const_cast<float *>(P.inv32), P.n);
        }
    }
    FEMD_TRY_CUDA(cudaGetLastError());
    std::vector<BProb> desc = B->probs;
    if (B->ghost >= 0 && B->ghost < B->nprob) desc[B->ghost].team += 1;   // test hook (femd_cuda_batch_debug)
    FEMD_TRY_CUDA(cudaMemcpyAsync(B->d_probs.p, desc.data(), desc.size() * sizeof(BProb), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemsetAsync(B->d_bar.p, 0, B->nprob * sizeof(unsigned), s));
    BQueue q0{0u, 0, B->spin_limit};
    FEMD_TRY_CUDA(cudaMemcpyAsync(B->d_queue.p, &q0, sizeof(BQueue), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemsetAsync(B->d_res_i.p, 0, 8 * (size_t)B->nprob * sizeof(int), s));
    *B->abort_host = 0;
    const BProb *probs = B->d_probs.p;
    const int *sp = B->d_slot_prob.p, *sm = B->d_slot_member.p;
    int nslots = B->nslots;
    BQueue *q = B->d_queue.p;
    const int *ab = B->abort_dev;
    void *args[] = {(void *)&probs, (void *)&sp, (void *)&sm, (void *)&nslots, (void *)&q, (void *)&ab};
    cudaEvent_t e0, e1;
    FEMD_TRY_CUDA(cudaEventCreate(&e0));
    FEMD_TRY_CUDA(cudaEventCreate(&e1));
    cudaEventRecord(e0, s);
    cudaError_t e = mixed ? cudaLaunchCooperativeKernel((const void *)k_batch_pcg<true>, B->grid, BB, args, 0, s)
                          : cudaLaunchCooperativeKernel((const void *)k_batch_pcg<false>, B->grid, BB, args, 0, s);
    if (e == cudaSuccess) add_launches(1);
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) { set_error(std::string("batch_solve: ") + cudaGetErrorString(e)); return FEMD_ECUDA; }
    std::vector<int> ri(8 * (size_t)B->nprob);
    std::vector<double> rd(2 * (size_t)B->nprob);
    BQueue qh;
    FEMD_TRY_CUDA(cudaMemcpyAsync(ri.data(), B->d_res_i.p, ri.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(rd.data(), B->d_res_d.p, rd.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(&qh, B->d_queue.p, sizeof(BQueue), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    for (int p = 0; p < B->nprob; ++p) {
        femd_cg_result &r = results[p];
        r.iterations = ri[8 * p];
        r.converged = ri[8 * p + 1];
        r.breakdown = ri[8 * p + 2];
        r.status = qh.flag ? qh.flag : ri[8 * p + 3];
        r.outer = ri[8 * p + 4];
        r.residual = rd[2 * p];
        r.seconds = ms * 1e-3;
    }
    if (qh.flag == FEMD_ETIMEOUT) { set_error("batch_solve: a team barrier wait ran out"); return FEMD_ETIMEOUT; }
    if (qh.flag == FEMD_EABORT) { set_error("batch_solve: aborted by the host"); return FEMD_EABORT; }
    return FEMD_OK;
}

int femd_cuda_batch_abort(femd_batch handle)
{
    femd_batch_s *B = as_batch(handle);
    if (!B || !B->abort_host) return FEMD_EINVAL;
    *(volatile int *)B->abort_host = 1;
    return FEMD_OK;
}

int femd_cuda_batch_debug(femd_batch handle, int ghost_problem, long long spin_limit)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_debug: not a batch handle");
    FEMD_CHECK_ARG(ghost_problem < B->nprob, "batch_debug: problem index out of range");
    B->ghost = ghost_problem;
    B->spin_limit = spin_limit > 0 ? spin_limit : SPIN_LIMIT;
    return FEMD_OK;
}

int femd_cuda_batch_info(femd_batch handle, int *nprob, int *grid, int *nslots, int *team_out)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_info: not a batch handle");
    if (nprob) *nprob = B->nprob;
    if (grid) *grid = B->grid;
    if (nslots) *nslots = B->nslots;
    if (team_out) for (int p = 0; p < B->nprob; ++p) team_out[p] = B->team[p];
    return FEMD_OK;
}

}  // extern "C"
