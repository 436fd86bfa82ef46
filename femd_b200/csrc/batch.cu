// batch.cu -- K7: many independent Jacobi-PCG solves in one persistent, cooperative launch.
//
// A batch is a set of member systems (CSR matrices with their Jacobi inverse diagonals).  Every
// member gets a team of T thread blocks (T from its size and the batch's launch shape only).
// Blocks take (member, team rank) slots from a queue, largest teams first; a rank owns a
// contiguous range of the member's rows.  The ranks of a team meet at software barriers (a
// counter per member, waited on with a bounded spin: a wait that runs out sets FEMD_ETIMEOUT and
// every block returns).  Dot products are summed per block, then across the team in one fixed
// order, so a member's iterates depend on the member and the launch shape alone -- the same bits
// alone or in any mix.
//
// The launch is cooperative (all blocks resident), so a team whose ranks are still busy
// elsewhere only delays; at most one team is incomplete at any time (slots are taken in order and
// no team is larger than half the grid), so every team completes.
//
// Solves are resumable: a launch advances every armed member by at most `iters` iterations and
// saves its scalars (BState) for the next launch.  One launch with iters = max_iter solves a
// fixed batch; short launches with members joining and leaving between them are the continuous
// batching of the request loop.
//
// SpMV: CSR-stream over precomputed chunks of whole rows (at most BB x NPT nonzeros): bulk
// asynchronous copies (TMA) bring chunk c+1's column indices and values into shared memory while
// chunk c is computed; the block gathers, stores the products in shared memory (two buffers, one
// barrier per chunk), and one thread per row sums its products in order.
//
// One iteration is two team reductions.  The search direction is never written before the SpMV
// that needs it: the SpMV forms p_j = z_j + beta p_j (one fused multiply-add, the same one the
// row's owner stores) from the previous direction, held in a second buffer.
//
// Modes: FP64 Jacobi-PCG (cg.hpp:296-350 semantics, final true residual included) or mixed
// precision: FP32 matrix copy (made by k_batch_f32 before the member's first launch -- the bulk
// copies only read what earlier launches wrote),
// FP32 vectors and SpMV accumulation; FP64 residual b - A x on the FP64 matrix and FP64 solution
// update at reliable updates.
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "compact_host.h"

namespace femd {

static constexpr long long SPIN_LIMIT = 1ll << 25;   // default bound of a barrier wait (spins of ~0.5 us)

enum : int { BS_STARTED = 1, BS_DONE = 2, BS_BREAKDOWN = 4, BS_CONVERGED = 8, BS_FALLBACK = 16 };

// a member's solver scalars, kept in device memory between launches
struct BState {
    double rz, beta, maxr, nb, res;
    double prt;            // mixed: the true residual of the last reliable update
    int it, rus, flags, status;
    int stall;             // mixed: reliable updates in a row that reduced it by less than 2x
    int pad;
};

struct BProb {
    int n, team, max_iter, nch, nnz;
    int tpr;               // lockstep engine: lanes per row of its row-group SpMV
    const int *wrow;       // lockstep engine: first rows of its SpMV windows (null: row groups)
    double tol;
    const int *indptr, *indices;
    const int *crow, *cq;  // chunk c = rows [crow[c], crow[c+1]) = nonzeros [cq[c], cq[c+1])
    const double *A64, *inv64;
    float *A32, *inv32;
    const double *b;
    double *x;
    float *r32, *z32, *pa32, *pb32, *Ap32, *d32;
    double *r64, *z64, *pa64, *pb64, *Ap64;
    double *part;          // 8 kinds x team
    double *cpart;         // per-chunk sums of the SpMV passes: 6 kinds x nch (start 0-2, direction 3, residual 4-5)
    unsigned long long *claim;   // chunk claims of the SpMV passes
    unsigned *bar;
    BState *st;
    // lockstep engine, compact layout (mixed precision; null otherwise): the member's FP32 matrix
    // and its vectors are in the pattern's reverse Cuthill-McKee order; iperm maps an original row
    // to its reordered one, cptr / coff are the reordered rows' pointers and 16-bit column offsets
    // ctab: per reordered row its first position and the bits of the FP32 low part of its split
    // diagonal (k_ls_split_rows), one table per member; row n holds the end
    const int *iperm;
    const int2 *ctab;
    const short *coff;
};

struct BQueue {
    unsigned next;
    int flag;              // FEMD_ETIMEOUT / FEMD_EABORT seen by any block
    long long spin_limit;  // the bound of every barrier wait (spins)
    int nslots;
    int iters;             // iterations per member in this launch
    // cycle counters of the launch (thread 0 of every block): in the kernel, waiting at team
    // barriers, and waiting at the SpMV chunk barriers
    unsigned long long block_cycles, team_wait_cycles, chunk_sync_cycles;
    // the first wait that gave up: 1 a team barrier, 2 a staging barrier; the barrier phase (team)
    // or the chunk (staging) it was at, and the member's id in the launch (its slot's member)
    int fail_where, fail_at, fail_team, fail_rank;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ float pdir(const float *z, const float *p, float beta, int j) { return __fmaf_rn(beta, p[j], z[j]); }

__device__ __forceinline__ double pdir(const double *z, const double *p, double beta, int j) { return __fma_rn(beta, p[j], z[j]); }

// team barrier: false when the batch has to stop (timeout or abort).  lead_sync: the block has
// not synchronised since its last global writes.
__device__ bool team_barrier(const BProb &P, unsigned &phase, BQueue *q, volatile const int *abort_flag, bool lead_sync)
{
    __shared__ int s_ok;
    const bool check = (phase & 15) == 0;
    if (P.team == 1 && !check) {
        if (lead_sync) __syncthreads();
        ++phase;
        return true;
    }
    if (lead_sync) __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (P.team > 1) {
            __threadfence();
            atomicAdd(P.bar, 1u);
            const unsigned target = (phase + 1) * (unsigned)P.team;
            const long long lim = q->spin_limit;
            long long spins = 0;
            const long long t0 = clock64();
            while (ld_acquire(P.bar) < target) {
                if (((++spins) & 255) == 0) {
                    if (*(volatile int *)&q->flag) { ok = 0; break; }
                    if (spins > lim) {
                        if (atomicCAS(&q->flag, 0, FEMD_ETIMEOUT) == 0) {
                            q->fail_where = 1;
                            q->fail_at = (int)phase;
                            q->fail_team = P.team;
                            q->fail_rank = (int)ld_acquire(P.bar);
                        }
                        ok = 0;
                        break;
                    }
                }
                __nanosleep(32);
            }
            atomicAdd(&q->team_wait_cycles, (unsigned long long)(clock64() - t0));
            __threadfence();
        }
        if (check) {
            // the host's abort flag (mapped host memory, a PCIe read): every 64th barrier
            if (abort_flag && (phase & 63) == 0 && *abort_flag) atomicCAS(&q->flag, 0, FEMD_EABORT);
            if (*(volatile int *)&q->flag) ok = 0;
        }
        s_ok = ok;
    }
    __syncthreads();
    ++phase;
    return s_ok != 0;
}

// the block's reduction scratch, one row per kind: consecutive reductions of the same kind are
// always separated by a reduction of another kind (and its __syncthreads)
struct RedSmem {
    double warp[8][16];
    double tot[8];
};
__device__ __forceinline__ RedSmem &red_smem()
{
    __shared__ RedSmem s;
    return s;
}

// team reduction of NV values of kinds base..base+NV-1: block sums, each rank writes its own,
// the team meets, and warp 0 of every rank sums the T partials in one fixed order (lane-strided,
// then a shuffle tree), so the result depends on T and the partials only
template <int NV, int BB>
__device__ bool team_reduce(const BProb &P, int m, int base, double (&v)[NV], unsigned &phase, BQueue *q,
                            volatile const int *abort_flag)
{
    static_assert(BB / 32 <= 16, "at most 16 warps per block");
    RedSmem &S = red_smem();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) S.warp[base + k][threadIdx.x >> 5] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < BB / 32; ++w) s += S.warp[base + k][w];
        v[k] = s;
    }
    if (P.team > 1 && threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) P.part[(base + k) * P.team + m] = v[k];
    }
    if (!team_barrier(P, phase, q, abort_flag, false)) return false;
    if (P.team == 1) return true;
    if (threadIdx.x < 32) {
        const volatile double *part = P.part;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = 0.0;
            for (int u = threadIdx.x; u < P.team; u += 32) s += part[(base + k) * P.team + u];
            s = warp_sum(s);
            if (threadIdx.x == 0) S.tot[base + k] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = S.tot[base + k];
    return true;
}

// ---- chunk staging: bulk asynchronous copies (TMA, into this block's own shared memory) ------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *m, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t *m, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for a phase of a staging barrier (a copy that never lands ends the batch)
__device__ __forceinline__ bool mbar_wait(uint64_t *m, unsigned parity)
{
    for (int k = 0; k < (1 << 22); ++k)
        if (mbar_try_wait(m, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *m)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// a block's SpMV shared memory: two staging buffers of column indices and values (filled by bulk
// copies, 16-byte aligned), two product buffers, and the staging barriers
template <int CAP>
struct ChunkSmem {
    static constexpr int IXN = CAP + 4;
    int ix[2][IXN];
    double val[2][IXN];        // FP64 values, or FP32 values in the first half
    double prod[2][CAP];       // FP64 products, or FP32 products in the first half
    uint64_t mbar[2];
    int fail;
    int cid[2];                // the chunk staged in each buffer (-1: none)
    double wsum[2][16][3];     // a chunk's warp partial sums, per buffer
    double ctot[16][3];        // warp partials of the chunk-ordered team sums
};

// the part of chunk c that bulk copies bring in: nonzeros [qa, qb) with qa = qs rounded down to
// 4 (16 bytes of indices) and qb = qe rounded up but not past nnz rounded down; the rest of the
// chunk (at most 3 nonzeros at the matrix's end) is read directly
__device__ __forceinline__ int staged_end(int qa, int qe, int nnz4)
{
    int qb = (qe + 3) & ~3;
    if (qb > nnz4) qb = nnz4;
    return qb < qa ? qa : qb;
}

template <class V, int CAP>
__device__ __forceinline__ void stage_issue(const BProb &P, const V *A, int c, int s, ChunkSmem<CAP> &S)
{
    const int qs = P.cq[c], qe = P.cq[c + 1];
    const int qa = qs & ~3, qb = staged_end(qa, qe, P.nnz & ~3);
    const unsigned n = (unsigned)(qb - qa);
    fence_proxy_async_smem();                                 // the buffer's last readers were generic
    mbar_arrive_tx(&S.mbar[s], n * (unsigned)(sizeof(int) + sizeof(V)));
    if (n) {
        bulk_g2s(S.ix[s], P.indices + qa, n * (unsigned)sizeof(int), &S.mbar[s]);
        bulk_g2s(S.val[s], A + qa, n * (unsigned)sizeof(V), &S.mbar[s]);
    }
}

// CSR-stream SpMV over the member's chunks, claimed dynamically by the ranks of its team from
// the member's counter (claims base .. base + nch - 1 are the chunks of this pass; every rank
// makes exactly one claim past them, so the next pass starts at base + nch + team).  Chunk
// claims run two ahead: bulk copies bring a claimed chunk's column indices and values into
// shared memory while the one before it is computed.  Products a_q * g(col_q) go to shared
// memory and out(row, sum, pre(row), acc) gets each row's products summed in order by one
// thread and adds the row's share of NK sums to acc; the block sums acc per chunk in warp
// order and writes it to cpart[k * nch + chunk].  So a sum over the chunks in chunk order (team
// sum below) depends on the member and the launch shape alone, whichever rank took which chunk.
// Vectors that the team writes during the launch take plain coherent loads (inside g).
// false: a staging copy did not land (the batch is stopped; the outstanding copy was waited for).
template <class V, class F, int BB, int NPT, int NK, class Gather, class Pre, class RowOut>
__device__ __forceinline__ bool chunk_spmv(const BProb &P, const V *A, unsigned long long base, double *cpart, int kbase,
                                           ChunkSmem<BB * NPT> &S, unsigned &par, BQueue *q, Gather g, Pre pre, RowOut out)
{
    const int nch = P.nch;
    const int nnz4 = P.nnz & ~3;
    auto claim = [&]() -> int {
        const unsigned long long v = atomicAdd(P.claim, 1ull) - base;
        return v < (unsigned long long)nch ? (int)v : -1;
    };
    auto flush = [&](int c, int buf) {                    // thread 0: a chunk's sums, warps in order
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < BB / 32; ++w) t += S.wsum[buf][w][k];
            cpart[(size_t)(kbase + k) * nch + c] = t;
        }
    };
    __syncthreads();                                      // earlier readers of cid and the buffers are done
    if (threadIdx.x == 0) {
        fence_proxy_async_global();                       // values written by the team before: bulk-copy readable
        const int a0 = claim();
        S.cid[0] = a0;
        S.cid[1] = -1;
        if (a0 >= 0) {
            stage_issue<V>(P, A, a0, 0, S);
            const int a1 = claim();
            S.cid[1] = a1;
            if (a1 >= 0) stage_issue<V>(P, A, a1, 1, S);
        }
    }
    __syncthreads();
    int j = 0, cprev = -1;
    for (;; ++j) {
        const int b = j & 1;
        const int c = S.cid[b];
        if (c < 0) break;
        const int rs = P.crow[c], re = P.crow[c + 1];
        const int qs = P.cq[c], qe = P.cq[c + 1];
        const int qa = qs & ~3, qb = staged_end(qa, qe, nnz4);
        const int row0 = rs + (int)threadIdx.x;
        int lo0 = 0, hi0 = 0;
        decltype(pre(0)) pv{};
        if (row0 < re) {
            lo0 = P.indptr[row0];
            hi0 = P.indptr[row0 + 1];
            pv = pre(row0);                               // the row's own values, loaded early
        }
        const bool ok = mbar_wait(&S.mbar[b], (par >> b) & 1u);
        par ^= 1u << b;
        if (ok) {
            const int *ixs = S.ix[b];
            const V *vs = reinterpret_cast<const V *>(S.val[b]);
            F *buf = reinterpret_cast<F *>(S.prod[b]);
            int col[NPT];
            V a[NPT];
#pragma unroll
            for (int t = 0; t < NPT; ++t) {
                const int qq = qs + t * BB + (int)threadIdx.x;
                col[t] = -1;
                a[t] = V(0);
                if (qq < qb) { col[t] = ixs[qq - qa]; a[t] = vs[qq - qa]; }
                else if (qq < qe) { col[t] = P.indices[qq]; a[t] = A[qq]; }
            }
            F gv[NPT];
#pragma unroll
            for (int t = 0; t < NPT; ++t) gv[t] = col[t] >= 0 ? g(col[t]) : F(0);
#pragma unroll
            for (int t = 0; t < NPT; ++t)
                if (col[t] >= 0) buf[t * BB + threadIdx.x] = (F)a[t] * gv[t];
        } else {
            S.fail = 1;
        }
        const long long ts = clock64();
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(&q->chunk_sync_cycles, (unsigned long long)(clock64() - ts));
        if (S.fail) {
            // stop the batch; wait (bounded) for the copy still in flight before the block leaves
            if (threadIdx.x == 0) {
                if (atomicCAS(&q->flag, 0, FEMD_ETIMEOUT) == 0) {
                    q->fail_where = 2;
                    q->fail_at = c;
                    q->fail_team = P.team;
                    q->fail_rank = (int)par;
                }
                // a copy that still has not landed may write this block's shared memory after it
                // exits: recorded apart (3), and the host reports the context as suspect
                if (S.cid[b ^ 1] >= 0 && !mbar_wait(&S.mbar[b ^ 1], (par >> (b ^ 1)) & 1u)) atomicExch(&q->fail_where, 3);
            }
            return false;
        }
        if (threadIdx.x == 0) {
            if (cprev >= 0) flush(cprev, b ^ 1);          // its warps' sums were written before the barrier
            // buffer b is free (every thread read it before the barrier): the chunk after next goes
            // there, unless the claim for the next one was already past the end
            int nx = -1;
            if (S.cid[b ^ 1] >= 0) {
                nx = claim();
                if (nx >= 0) stage_issue<V>(P, A, nx, b, S);
            }
            S.cid[b] = nx;
        }
        double acc[NK];
#pragma unroll
        for (int k = 0; k < NK; ++k) acc[k] = 0.0;
        const F *buf = reinterpret_cast<const F *>(S.prod[b]);
        for (int row = row0; row < re; row += BB) {
            int lo = lo0, hi = hi0;
            if (row != row0) {
                lo = P.indptr[row];
                hi = P.indptr[row + 1];
                pv = pre(row);
            }
            F sum = F(0);
            for (int qq = lo; qq < hi; ++qq) sum += buf[qq - qs];
            out(row, sum, pv, acc);
        }
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            const double t = warp_sum(acc[k]);
            if ((threadIdx.x & 31) == 0) S.wsum[b][threadIdx.x >> 5][k] = t;
        }
        cprev = c;
    }
    __syncthreads();
    if (threadIdx.x == 0 && cprev >= 0) flush(cprev, (j - 1) & 1);
    return true;
}

// Regions of the per-chunk sums, one per kind of pass.  A rank that has read a pass's sums goes on
// to the next pass at once, while slower ranks may still be reading: consecutive passes write
// different regions, and a region is written again only after a team barrier that every rank
// reaches after its reads.
static constexpr int KB_START = 0, KB_DIR = 3, KB_RES = 4, KB_KINDS = 6;

// the team's totals of NK chunk sums of region kbase: meet, then every rank sums cpart over the
// chunks in chunk order (thread-strided, then warps in order) -- the same bits on every rank
template <int NK, int BB, int CAP>
__device__ bool team_sum_chunks(const BProb &P, const double *cpart, int kbase, double (&v)[NK], ChunkSmem<CAP> &S,
                                unsigned &phase, BQueue *q, volatile const int *abort_flag)
{
    if (!team_barrier(P, phase, q, abort_flag, true)) return false;
    const int nch = P.nch;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        double t = 0.0;
        for (int i = threadIdx.x; i < nch; i += BB) t += __ldcg(cpart + (size_t)(kbase + k) * nch + i);
        t = warp_sum(t);
        if ((threadIdx.x & 31) == 0) S.ctot[threadIdx.x >> 5][k] = t;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < BB / 32; ++w) t += S.ctot[w][k];
        v[k] = t;
    }
    return true;
}

template <class F>
struct ResPre {
    double b;
    F inv;
};

// the FP64 residual r = b - A64 x over the member's chunks: stores r and z = inv r (FP32 copies
// in mixed mode; the inverse diagonal rounded from the FP64 one, the same value as the FP32
// copy); chunk sums of ||r||^2 (FP64), r.z and, when START, ||b||^2, and then also zeroes the
// previous direction (and the mixed correction d) of every row
template <int BB, int NPT, bool MIXED, bool START>
__device__ __forceinline__ bool residual_chunks(const BProb &P, unsigned long long base, ChunkSmem<BB * NPT> &S, unsigned &par,
                                                BQueue *q)
{
    using F = typename std::conditional<MIXED, float, double>::type;
    constexpr int NK = START ? 3 : 2;
    const double *x = P.x;
    F *pb = MIXED ? (F *)P.pb32 : (F *)P.pb64;
    return chunk_spmv<double, double, BB, NPT, NK>(
        P, P.A64, base, P.cpart, START ? KB_START : KB_RES, S, par, q, [&](int j) { return x[j]; },
        [&](int i) { return ResPre<F>{P.b[i], (F)P.inv64[i]}; },
        [&](int i, double s, const ResPre<F> &pv, double (&acc)[NK]) {
            const double ri = pv.b - s;
            acc[0] += ri * ri;
            if (MIXED) {
                const float rf = (float)ri, zf = (float)pv.inv * rf;
                P.r32[i] = rf;
                P.z32[i] = zf;
                acc[1] += (double)rf * (double)zf;
            } else {
                const double zi = (double)pv.inv * ri;
                P.r64[i] = ri;
                P.z64[i] = zi;
                acc[1] += ri * zi;
            }
            if (START) {
                acc[NK - 1] += pv.b * pv.b;
                pb[i] = F(0);
                if (MIXED) P.d32[i] = 0.0f;
            }
        });
}

// r -= alpha Ap, acc += alpha p (x in FP64 mode, the correction d in mixed mode), z = inv r on
// [r0, r1); two rows per thread per pass with all loads issued first
template <class F, int BB>
__device__ __forceinline__ void update_rows(F *r, F *z, const F *Ap, const F *inv, F *acc, const F *p, F alpha, int r0, int r1,
                                            double &rr, double &rz)
{
    for (int i = r0 + (int)threadIdx.x; i < r1; i += 2 * BB) {
        const int j = i + BB;
        const bool two = j < r1;
        F ri = r[i], api = Ap[i], ivi = inv[i], ai = acc[i], pi = p[i];
        F rj = F(0), apj = F(0), ivj = F(0), aj = F(0), pj = F(0);
        if (two) { rj = r[j]; apj = Ap[j]; ivj = inv[j]; aj = acc[j]; pj = p[j]; }
        ri -= alpha * api;
        const F zi = ivi * ri;
        r[i] = ri;
        z[i] = zi;
        acc[i] = ai + alpha * pi;
        rr += (double)ri * (double)ri;
        rz += (double)ri * (double)zi;
        if (two) {
            rj -= alpha * apj;
            const F zj = ivj * rj;
            r[j] = rj;
            z[j] = zj;
            acc[j] = aj + alpha * pj;
            rr += (double)rj * (double)rj;
            rz += (double)rj * (double)zj;
        }
    }
}

// rank m of the member's team: advance the solve by at most q->iters iterations; false when the
// batch has to stop.  The SpMV passes take chunks dynamically (chunk_spmv); the elementwise update
// and the FP32 copy at the start work on the rank's own rows (the rows of chunks
// [nch m / T, nch (m+1) / T)) and reduce per rank in rank order.
template <bool MIXED, int BB, int NPT>
__device__ bool solve_member(const BProb &P, int m, BQueue *q, volatile const int *abort_flag, ChunkSmem<BB * NPT> &SM,
                             unsigned &par)
{
    using F = typename std::conditional<MIXED, float, double>::type;
    const int T = P.team;
    const int c0 = (int)((long long)P.nch * m / T), c1 = (int)((long long)P.nch * (m + 1) / T);
    const int r0 = P.crow[c0], r1 = P.crow[c1];
    F *r = MIXED ? (F *)P.r32 : (F *)P.r64;
    F *z = MIXED ? (F *)P.z32 : (F *)P.z64;
    F *pa = MIXED ? (F *)P.pa32 : (F *)P.pa64;
    F *pb = MIXED ? (F *)P.pb32 : (F *)P.pb64;
    F *Ap = MIXED ? (F *)P.Ap32 : (F *)P.Ap64;
    const F *inv = MIXED ? (const F *)P.inv32 : (const F *)P.inv64;
    const F *A = MIXED ? (const F *)P.A32 : (const F *)P.A64;
    F *acc = MIXED ? (F *)P.d32 : (F *)P.x;
    unsigned phase = 0;
    unsigned long long base = 0;                          // claim base of the next SpMV pass
    const unsigned long long pass = (unsigned long long)P.nch + (unsigned long long)T;
    const bool lead = m == 0 && threadIdx.x == 0;
    BState S = *P.st;

    if (!(S.flags & BS_STARTED)) {
        // start: r = b - A x0, z = inv r, pold = 0 (the FP32 copies of A and inv were made by
        // k_batch_f32 before the launch: bulk copies read only what earlier launches wrote)
        if (!residual_chunks<BB, NPT, MIXED, true>(P, base, SM, par, q)) return false;
        base += pass;
        double v[3];                                      // ||r||^2, r.z, ||b||^2
        if (!team_sum_chunks<3, BB>(P, P.cpart, KB_START, v, SM, phase, q, abort_flag)) return false;
        const double nb = sqrt(v[2]), rn0 = sqrt(v[0]);
        S.flags = BS_STARTED;
        S.it = 0;
        S.rus = 0;
        S.beta = 0.0;
        S.rz = v[1];
        S.maxr = rn0;
        S.prt = rn0;
        S.stall = 0;
        S.nb = nb;
        S.res = nb == 0.0 ? 0.0 : rn0 / nb;
        if (nb == 0.0) {
            for (int i = r0 + (int)threadIdx.x; i < r1; i += BB) P.x[i] = 0.0;
            S.flags |= BS_DONE | BS_CONVERGED;
        } else if (rn0 <= P.tol * nb) {
            S.flags |= BS_DONE | BS_CONVERGED;
        } else if (!(S.rz > 0.0)) {
            S.flags |= BS_BREAKDOWN;
        }
        if (S.flags & BS_DONE) {
            if (lead) *P.st = S;
            return true;
        }
    }
    double rz = S.rz, beta = S.beta, maxr = S.maxr, res = S.res, prt = S.prt;
    const double nb = S.nb;
    int it = S.it, rus = S.rus, stall = S.stall;
    bool brk = (S.flags & BS_BREAKDOWN) != 0, done = false, fallback = false;
    const long long it_lim = (long long)it + q->iters;
    const int it_end = it_lim < (long long)P.max_iter ? (int)it_lim : P.max_iter;
    F *pold = (it & 1) ? pa : pb, *pnew = (it & 1) ? pb : pa;
    while (!brk && !done && it < it_end) {
        const F fb = (F)beta;
        const bool ok = chunk_spmv<F, F, BB, NPT, 1>(
            P, A, base, P.cpart, KB_DIR, SM, par, q, [&](int j) { return pdir(z, pold, fb, j); },
            [&](int i) { return pdir(z, pold, fb, i); },
            [&](int i, F s, F pi, double (&a)[1]) {
                pnew[i] = pi;
                Ap[i] = s;
                a[0] += (double)pi * (double)s;
            });
        if (!ok) return false;
        base += pass;
        double pap[1];
        if (!team_sum_chunks<1, BB>(P, P.cpart, KB_DIR, pap, SM, phase, q, abort_flag)) return false;
        if (!(pap[0] > 0.0)) { brk = true; break; }
        const double alpha = rz / pap[0];
        double u[2] = {0.0, 0.0};                         // ||r||^2, r.z
        update_rows<F, BB>(r, z, Ap, inv, acc, pnew, (F)alpha, r0, r1, u[0], u[1]);
        if (!team_reduce<2, BB>(P, m, 4, u, phase, q, abort_flag)) return false;
        ++it;
        const double rn = sqrt(u[0]);
        if (!MIXED) {
            res = rn / nb;
            if (rn <= P.tol * nb) { done = true; break; }
            beta = u[1] / rz;
            rz = u[1];
            if (!(rz > 0.0)) { brk = true; break; }
        } else {
            const bool ru = rn <= 0.1 * maxr || rn <= P.tol * nb || it >= P.max_iter || !(u[1] > 0.0);
            if (ru) {
                // reliable update: x += d, d = 0; r = b - A64 x in FP64, r32 = (float) r
                for (int i = r0 + (int)threadIdx.x; i < r1; i += BB) {
                    P.x[i] += (double)P.d32[i];
                    P.d32[i] = 0.0f;
                }
                if (!team_barrier(P, phase, q, abort_flag, true)) return false;
                if (!residual_chunks<BB, NPT, true, false>(P, base, SM, par, q)) return false;
                base += pass;
                double w[2];
                if (!team_sum_chunks<2, BB>(P, P.cpart, KB_RES, w, SM, phase, q, abort_flag)) return false;
                ++rus;
                const double rt = sqrt(w[0]);
                res = rt / nb;
                maxr = rt;
                if (rt <= P.tol * nb || it >= P.max_iter) { done = true; break; }
                // stagnation of the FP32 recurrence (the FP32 matrix too coarse for the slowest
                // modes): the host goes on in FP64 from this iterate
                stall = rt > 0.5 * prt ? stall + 1 : 0;
                prt = rt;
                if (stall >= 2 || !(rt < 1e300)) { fallback = true; break; }
                if (!(w[1] > 0.0)) { brk = true; break; }
                // drifted recurrence (true residual over twice its own): restart the direction
                beta = rt > 2.0 * rn ? 0.0 : w[1] / rz;
                rz = w[1];
            } else {
                beta = u[1] / rz;
                rz = u[1];
            }
        }
        F *t = pold;
        pold = pnew;
        pnew = t;
    }
    const bool finished = brk || done || fallback || it >= P.max_iter;
    if (finished) {
        if (!MIXED) {
            // the true residual (cg.hpp:222-237): every rank's x is final at the last reduction
            if (!residual_chunks<BB, NPT, false, false>(P, base, SM, par, q)) return false;
            base += pass;
            double w[2];
            if (!team_sum_chunks<2, BB>(P, P.cpart, KB_RES, w, SM, phase, q, abort_flag)) return false;
            res = sqrt(w[0]) / nb;
        } else if (brk) {
            for (int i = r0 + (int)threadIdx.x; i < r1; i += BB) {
                P.x[i] += (double)P.d32[i];
                P.d32[i] = 0.0f;
            }
        }
    }
    if (lead) {
        S.rz = rz;
        S.beta = beta;
        S.maxr = maxr;
        S.res = res;
        S.it = it;
        S.rus = rus;
        S.prt = prt;
        S.stall = stall;
        if (brk) S.flags |= BS_BREAKDOWN;
        if (fallback) {
            S.flags |= BS_DONE | BS_FALLBACK;
        } else if (finished) {
            const double tol = P.tol;
            int conv = !brk && res <= tol * (1.0 + 1e-6) + 1e-15;
            if (!conv && !brk && res <= 10.0 * tol && it < P.max_iter) conv = 1;
            S.flags |= BS_DONE | (conv ? BS_CONVERGED : 0);
        }
        *P.st = S;
    }
    return true;
}

template <bool MIXED, int BB, int NPT>
__global__ void __launch_bounds__(BB, 1024 / BB) k_batch_pcg(const BProb *__restrict__ probs, const int *__restrict__ slot_prob,
                                                             const int *__restrict__ slot_member, BQueue *q,
                                                             volatile const int *abort_flag)
{
    __shared__ __align__(16) ChunkSmem<BB * NPT> SM;
    __shared__ int s_slot, s_stop;
    const int nslots = q->nslots;
    if (threadIdx.x == 0) {
        mbar_init(&SM.mbar[0], 1);
        mbar_init(&SM.mbar[1], 1);
        SM.fail = 0;
        fence_mbar_init();
    }
    __syncthreads();
    const long long t_start = clock64();
    unsigned par = 0;                                     // next phase parity of each staging barrier
    for (;;) {
        if (threadIdx.x == 0) {
            s_slot = (int)atomicAdd(&q->next, 1u);
            s_stop = *(volatile int *)&q->flag;
        }
        __syncthreads();
        const int slot = s_slot, stop = s_stop;
        __syncthreads();
        if (slot >= nslots || stop) {
            if (threadIdx.x == 0) atomicAdd(&q->block_cycles, (unsigned long long)(clock64() - t_start));
            return;
        }
        const BProb &P = probs[slot_prob[slot]];
        if (!solve_member<MIXED, BB, NPT>(P, slot_member[slot], q, abort_flag, SM, par)) {
            if (threadIdx.x == 0) {
                const int f = *(volatile int *)&q->flag;
                P.st->status = f ? f : FEMD_ETIMEOUT;
            }
            return;
        }
    }
}

// the FP32 copies of a member's values and inverse diagonal (mixed mode), before its first launch
__global__ void k_batch_f32(const double *__restrict__ a, float *__restrict__ a32, long long nnz, const double *__restrict__ inv,
                            float *__restrict__ inv32, int n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += stride) a32[i] = (float)a[i];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) inv32[i] = (float)inv[i];
}

// the same for the compact layout: value q of the original CSR goes to position dst[q] of the
// reordered one, the inverse diagonal of original row i to reordered row iperm[i]
__global__ void k_ls_f32_perm(const double *__restrict__ a, const int *__restrict__ dst, float *__restrict__ a32,
                              long long nnz, const double *__restrict__ inv, const int *__restrict__ iperm,
                              float *__restrict__ inv32, int n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += stride) a32[dst[q]] = (float)a[q];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) inv32[iperm[i]] = (float)inv[i];
}

// The compact layout's row table of a member and its split diagonal.  With the off-diagonals
// rounded to FP32, d = a_ii + sum_{j != i} (a_ij - fl(a_ij)) (FP64) keeps the FP64 row sum; it is
// stored as hi = fl(d) at the diagonal position and lo = fl(d - hi) beside the row's first
// position.  The represented matrix is then a graph Laplacian of the rounded off-diagonals plus
// the row sums to about eps_32^2, whose quadratic form is within O(eps_32) of the FP64 one instead
// of O(eps_32 cond(A)): the FP32 recurrence needs fewer iterations on large systems.  A pattern
// without every diagonal position keeps the plain copy (lo = 0).  One thread per original row i
// (after k_ls_f32_perm wrote the entries); thread n writes the end.
__global__ void k_ls_split_rows(const int *__restrict__ indptr, const int *__restrict__ diag_pos, const double *__restrict__ a,
                                const int *__restrict__ dst, const int *__restrict__ iperm, const int *__restrict__ cptr,
                                int split, float *__restrict__ a32, int2 *__restrict__ ctab, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        if (i == n) {
            ctab[n] = make_int2(cptr[n], 0);
            continue;
        }
        const int r = iperm[i];
        float lo = 0.0f;
        if (split) {
            const int q0 = indptr[i], q1 = indptr[i + 1], dp = diag_pos[i];
            double d = a[dp];
            for (int q = q0; q < q1; ++q)
                if (q != dp) d += a[q] - (double)(float)a[q];
            const float h = (float)d;
            a32[dst[dp]] = h;
            lo = (float)(d - (double)h);
        }
        ctab[r] = make_int2(cptr[r], __float_as_int(lo));
    }
}

// chunk tables of one matrix: chunk k starts at the first row whose first nonzero is at or after
// k * cp (cp = chunk capacity - longest row), so no chunk holds more than the capacity
__global__ void k_chunk_table(const int *__restrict__ indptr, int n, int nnz, int cp, int nch, int *crow, int *cq)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nch) return;
    if (k == nch) { crow[k] = n; cq[k] = nnz; return; }
    const long long key = (long long)k * cp;
    int lo = 0, hi = n;                                    // first i in [0, n] with indptr[i] >= key
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (indptr[mid] < key) lo = mid + 1; else hi = mid;
    }
    crow[k] = lo;
    cq[k] = indptr[lo];
}

__device__ __forceinline__ int warp_max(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void k_max_row(const int *__restrict__ indptr, int n, int *out)
{
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, indptr[i + 1] - indptr[i]);
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

using BatchKernel = void (*)(const BProb *, const int *, const int *, BQueue *, volatile const int *);

template <bool MIXED>
static BatchKernel batch_kernel_m(int block, int npt)
{
#define FEMD_BK(B_, N_) if (block == B_ && npt == N_) return k_batch_pcg<MIXED, B_, N_>;
    FEMD_BK(128, 2) FEMD_BK(128, 4) FEMD_BK(128, 8)
    FEMD_BK(256, 2) FEMD_BK(256, 4)
    FEMD_BK(512, 2)
#undef FEMD_BK
    return nullptr;
}
static BatchKernel batch_kernel(bool mixed, int block, int npt)
{
    return mixed ? batch_kernel_m<true>(block, npt) : batch_kernel_m<false>(block, npt);
}


// ==== the lockstep engine ====================================================================
// Every iteration is a few whole-grid kernels over all the members still running: an SpMV
// (direction formed on the fly, p.Ap) and the update; in mixed precision also a flush and an
// FP64 residual over the members that asked for a reliable update in this iteration.  An entry
// of the block table is a fixed range of one member's rows (warp row groups, TPR lanes per row,
// 4 loads in flight per lane, no block barriers in the row loop).  A member's sums are entry
// partials summed in entry order by the member's last block (a ticket per member and kernel), so
// a member's iterates depend on the member alone, whatever else is in the batch.

struct LState {
    double rz, alpha, beta, nb, maxr, rz_prev, rn_rec, prt, res;
    int it, done, want_ru, breakdown, conv, rus, stall, fallback, zero, started;
    unsigned t1, t2, t3;   // last-block tickets of the SpMV, the update and the residual
    int pad;
};

struct LBlock {
    int m, r0, r1, b0, b1;  // member, its rows [r0, r1), the member's entries [b0, b1)
    int w0, w1;             // its SpMV windows [w0, w1) (window mode)
};

static constexpr int LS_BB = 256;

// y = A g on rows [r0, r1) with TPR lanes per row; out(row, sum) by the row's first lane
template <int TPR, class V, class F, class Gather, class Pre, class Out>
__device__ __forceinline__ void ls_rows(const BProb &P, const V *A, int r0, int r1, Gather g, Pre pre, Out out)
{
    constexpr int U = 4, GPW = 32 / TPR, STEP = (LS_BB / 32) * GPW;
    const int lane = threadIdx.x % TPR;
    const int sub = (int)(threadIdx.x & 31) / TPR;
    int i0 = r0 + (int)(threadIdx.x >> 5) * GPW;
    int i = i0 + sub;
    int lo = 0, hi = 0;
    if (i < r1) {
        lo = P.indptr[i];
        hi = P.indptr[i + 1];
    }
    for (; i0 < r1; i0 += STEP) {
        // the next pass's row pointers and this row's own values are loaded ahead of the gathers
        const int inext = i + STEP;
        int lo_n = 0, hi_n = 0;
        if (inext < r1) {
            lo_n = P.indptr[inext];
            hi_n = P.indptr[inext + 1];
        }
        decltype(pre(0)) pv{};
        if (i < r1) pv = pre(i);
        F s = F(0);
        for (int base = lo + lane; base < hi; base += U * TPR) {
            int c[U];
            V v[U];
            F xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int q = base + u * TPR;
                c[u] = q < hi ? __ldcs(&P.indices[q]) : 0;
                v[u] = q < hi ? __ldcs(&A[q]) : V(0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = base + u * TPR < hi ? g(c[u]) : F(0);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (base + u * TPR < hi) s += (F)v[u] * xv[u];
        }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, TPR);
        if (lane == 0 && i < r1) out(i, s, pv);
        i = inext;
        lo = lo_n;
        hi = hi_n;
    }
}

// y = A p on reordered rows [r0, r1) of the compact layout (r0 a multiple of 32), the direction
// p staged in shared memory over the entry's column window [c0, ...). One warp per slice of 32
// rows, one lane per row: entry j of the lane's row is at its first position + 32 j, so each
// load of the warp reads 32 consecutive offsets (64 B) and values (128 B), and no lane idles at
// a row's end (the slice's rows have nearly the same length; the padding entries, offset 0 and
// value 0, add nothing). The slice's width comes from the next slice's first position. Each lane
// sums its row in increasing column order. The diagonal is split (k_ls_split_rows): its FP32
// high part is the row's diagonal entry, its low part comes with the row's table entry and is
// added last, so the FP32 matrix keeps the FP64 matrix's row sums.
//
// The warp is latency-bound (a chain of dependent loads per slice), so: SELL_U entries per round,
// the next slice's table entries loaded one slice ahead, and the first slice's table entries and
// first round loaded by sell_prime before the block's window is staged (they do not need it).
static constexpr int SELL_U = 12;
struct SellCursor {
    int base, width, base1, end1;   // this slice's first position and width; the next slice's bounds
    float dl, dl1;                  // this lane's row's low diagonal part, this slice's and the next's
    short o[SELL_U];
    float v[SELL_U];                // the current round of this slice
};

__device__ __forceinline__ void sell_header(const BProb &P, int s0, int r1, int &base, int &end, float &dl)
{
    base = end = 0;
    dl = 0.0f;
    if (s0 < r1) {
        const int i = s0 + (int)(threadIdx.x & 31);
        base = P.ctab[s0].x;
        end = P.ctab[min(s0 + 32, P.n)].x;
        if (i < r1) dl = __int_as_float(P.ctab[i].y);
    }
}

__device__ __forceinline__ void sell_round(const BProb &P, const float *__restrict__ A, int base, int width, int j,
                                           short (&o)[SELL_U], float (&v)[SELL_U])
{
    const int q0 = base + (int)(threadIdx.x & 31);
#pragma unroll
    for (int u = 0; u < SELL_U; ++u) {
        const bool in = j + u < width;
        const int q = q0 + (j + u) * 32;
        o[u] = in ? __ldcs(&P.coff[q]) : (short)0;
        v[u] = in ? __ldcs(&A[q]) : 0.0f;
    }
}

__device__ __forceinline__ void sell_prime(const BProb &P, const float *__restrict__ A, int r0, int r1, SellCursor &c)
{
    const int s0 = r0 + (int)(threadIdx.x >> 5) * 32;
    int end;
    sell_header(P, s0, r1, c.base, end, c.dl);
    c.width = (end - c.base) >> 5;
    sell_header(P, s0 + LS_BB, r1, c.base1, c.end1, c.dl1);
    sell_round(P, A, c.base, c.width, 0, c.o, c.v);
}

__device__ __forceinline__ void ls_rows_sell(const BProb &P, const float *__restrict__ A, const float *win, int c0, int r0,
                                             int r1, float *__restrict__ Ap, double &dot, SellCursor &c)
{
    const int lane = threadIdx.x & 31;
    for (int s0 = r0 + (int)(threadIdx.x >> 5) * 32; s0 < r1; s0 += LS_BB) {
        const int i = s0 + lane;
        const bool ok = i < r1;                                  // lanes past the member's last row: padding
        const float *wrow = win + (ok ? i - c0 : 0);
        float s = 0.0f;
        for (int j = 0;; j += SELL_U) {
#pragma unroll
            for (int u = 0; u < SELL_U; ++u) s += c.v[u] * wrow[c.o[u]];
            if (j + SELL_U >= c.width) break;
            sell_round(P, A, c.base, c.width, j + SELL_U, c.o, c.v);
        }
        if (ok) {
            s = __fmaf_rn(c.dl, wrow[0], s);                     // the split diagonal's low part
            Ap[i] = s;
            dot += (double)wrow[0] * (double)s;
        }
        // the next slice: its bounds were loaded a slice ago; load its first round and the
        // bounds of the slice after it
        c.base = c.base1;
        c.width = (c.end1 - c.base1) >> 5;
        c.dl = c.dl1;
        sell_header(P, s0 + 2 * LS_BB, r1, c.base1, c.end1, c.dl1);
        if (s0 + LS_BB < r1) sell_round(P, A, c.base, c.width, 0, c.o, c.v);
    }
}

// SpMV windows: whole rows with at most LS_W nonzeros each (a window's rows start within LS_W -
// maxlen nonzeros of each other).  A window's column indices and values are read by coalesced
// loads, LS_NPT per thread, all issued before the gathers; the products go to shared memory
// (two buffers, one barrier per window) and each row is summed in order by one thread.
static constexpr int LS_NPT = 4, LS_W = LS_BB * LS_NPT;

template <class V, class F, class Gather, class Pre, class Out>
__device__ __forceinline__ void ls_windows(const BProb &P, const V *A, int w0, int w1, Gather g, Pre pre, Out out)
{
    __shared__ F prod[2][LS_W];
    const int tid = (int)threadIdx.x;
    for (int w = w0; w < w1; ++w) {
        F *pb = prod[(w - w0) & 1];
        const int rs = P.wrow[w], re = P.wrow[w + 1];
        const int qs = P.indptr[rs], qe = P.indptr[re];
        int col[LS_NPT];
        V a[LS_NPT];
#pragma unroll
        for (int t = 0; t < LS_NPT; ++t) {
            const int q = qs + t * LS_BB + tid;
            col[t] = q < qe ? __ldcs(&P.indices[q]) : -1;
            a[t] = q < qe ? __ldcs(&A[q]) : V(0);
        }
        const int row0 = rs + tid;
        int lo = 0, hi = 0;
        if (row0 < re) {
            lo = P.indptr[row0];
            hi = P.indptr[row0 + 1];
        }
        F gv[LS_NPT];
#pragma unroll
        for (int t = 0; t < LS_NPT; ++t) gv[t] = col[t] >= 0 ? g(col[t]) : F(0);
#pragma unroll
        for (int t = 0; t < LS_NPT; ++t)
            if (col[t] >= 0) pb[t * LS_BB + tid] = (F)a[t] * gv[t];
        __syncthreads();
        for (int row = row0; row < re; row += LS_BB) {
            if (row != row0) {
                lo = P.indptr[row];
                hi = P.indptr[row + 1];
            }
            F s = F(0);
            for (int q = lo; q < hi; ++q) s += pb[q - qs];
            out(row, s, pre(row));
        }
    }
}

// y = A g over an entry: by windows when the member has a window table, else by row groups
template <class V, class F, class Gather, class Pre, class Out>
__device__ __forceinline__ void ls_spmv_entry(const BProb &P, const V *A, const LBlock &L, Gather g, Pre pre, Out out)
{
    if (P.wrow) {
        ls_windows<V, F>(P, A, L.w0, L.w1, g, pre, out);
        return;
    }
    switch (P.tpr) {
    case 2: ls_rows<2, V, F>(P, A, L.r0, L.r1, g, pre, out); break;
    case 4: ls_rows<4, V, F>(P, A, L.r0, L.r1, g, pre, out); break;
    case 8: ls_rows<8, V, F>(P, A, L.r0, L.r1, g, pre, out); break;
    case 16: ls_rows<16, V, F>(P, A, L.r0, L.r1, g, pre, out); break;
    default: ls_rows<32, V, F>(P, A, L.r0, L.r1, g, pre, out); break;
    }
}

// The member's totals of NV sums.  The block's sums go to part[k * NE + e]; in the member's last
// block the function returns true (in every thread) with tot = the member's entry partials
// summed in entry order, and resets the ticket.
template <int NV>
__device__ __forceinline__ bool ls_member_sum(const double (&v)[NV], double *part, int NE, int e, const LBlock &L,
                                              unsigned *ticket, double (&tot)[NV])
{
    __shared__ double sh[NV][LS_BB / 32];
    __shared__ int last;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const double t = warp_sum(v[k]);
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < LS_BB / 32; ++w) t += sh[k][w];
            part[(size_t)k * NE + e] = t;
        }
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned)(L.b1 - L.b0 - 1);
    }
    __syncthreads();
    const bool is_last = last;
    if (!is_last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int b = L.b0 + (int)threadIdx.x; b < L.b1; b += LS_BB) t += __ldcg(part + (size_t)k * NE + b);
        t = warp_sum(t);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = t;
        __syncthreads();
        double u = 0.0;
#pragma unroll
        for (int w = 0; w < LS_BB / 32; ++w) u += sh[k][w];
        tot[k] = u;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0;
    return true;
}

__device__ __forceinline__ void ls_finish(LState &S, int *active)
{
    S.done = 1;
    atomicSub(active, 1);
}

// SpMV with the direction formed on the fly: p = z + beta pold (pold = 0 at the start); p.Ap.
// Block 0 also empties the reliable-update list of the iteration.  Mixed precision: at most 64
// registers, 4 blocks per SM. The sliced rows' 12 entries per round need them: at 5 blocks (51
// registers) the rounds spilled and ran 33 % slower than at 4 (64 config-4 problems x 120
// iterations). FP64: at most 51 registers, 5 blocks per SM.
template <bool MIXED>
__global__ void __launch_bounds__(LS_BB, MIXED ? 4 : 5) k_ls_spmv(const BProb *__restrict__ probs, const LBlock *__restrict__ blks, int NE,
                                                   LState *st, double *part, int *active, int *ru_count)
{
    using F = typename std::conditional<MIXED, float, double>::type;
    extern __shared__ float ls_win[];
    if (MIXED && blockIdx.x == 0 && threadIdx.x == 0) *ru_count = 0;
    const int e = blockIdx.x;
    const LBlock L = blks[e];
    const BProb P = probs[L.m];
    LState &S = st[L.m];
    if (S.done) return;
    const F *z = MIXED ? (const F *)P.z32 : (const F *)P.z64;
    F *pa = MIXED ? (F *)P.pa32 : (F *)P.pa64;
    F *pb = MIXED ? (F *)P.pb32 : (F *)P.pb64;
    F *Ap = MIXED ? (F *)P.Ap32 : (F *)P.Ap64;
    const F *A = MIXED ? (const F *)P.A32 : (const F *)P.A64;
    const int it = S.it;
    const F beta = (F)S.beta;
    const F *pold = (it & 1) ? pa : pb;
    F *pnew = (it & 1) ? pb : pa;
    double dot = 0.0;
    if (MIXED && P.coff) {
        // compact layout: p over the entry's column window [w0, w1) into shared memory (the
        // owner's values to pnew), then the rows read it there
        const int c0 = L.w0, c1 = L.w1;
        // WU columns per thread and round, their loads issued before any store (the stores to
        // pnew could alias z and pold for the compiler, which would serialise the round trips)
        constexpr int WU = 4;
        const float *zf = (const float *)z, *pf = (const float *)pold;
        float *pn = (float *)pnew;
        const float bf = (float)beta;
        SellCursor cur;
        sell_prime(P, (const float *)A, L.r0, L.r1, cur);
        for (int w0 = c0 + (int)threadIdx.x; w0 < c1; w0 += WU * LS_BB) {
            float zv[WU], pv[WU];
#pragma unroll
            for (int u = 0; u < WU; ++u) {
                const int w = w0 + u * LS_BB;
                zv[u] = w < c1 ? zf[w] : 0.0f;
                pv[u] = w < c1 ? pf[w] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < WU; ++u) {
                const int w = w0 + u * LS_BB;
                if (w < c1) {
                    const float pw = __fmaf_rn(bf, pv[u], zv[u]);
                    ls_win[w - c0] = pw;
                    if (w >= L.r0 && w < L.r1) pn[w] = pw;
                }
            }
        }
        __syncthreads();
        ls_rows_sell(P, (const float *)A, ls_win, c0, L.r0, L.r1, (float *)Ap, dot, cur);
    } else {
        ls_spmv_entry<F, F>(
            P, A, L, [&](int j) { return pdir(z, pold, beta, j); }, [&](int i) { return pdir(z, pold, beta, i); },
            [&](int i, F s, F pi) {
                pnew[i] = pi;
                Ap[i] = s;
                dot += (double)pi * (double)s;
            });
    }
    const double v[1] = {dot};
    double tot[1];
    if (ls_member_sum<1>(v, part, NE, e, L, &S.t1, tot) && threadIdx.x == 0) {
        if (!(tot[0] > 0.0)) {
            S.breakdown = 1;
            ls_finish(S, active);
        } else {
            S.alpha = S.rz / tot[0];
        }
    }
}

// r -= alpha Ap, (x or d) += alpha p, z = inv r; ||r||^2 and r.z; then the member's stopping
// test.  In mixed precision a member that wants a reliable update puts its entries on the list.
template <bool MIXED>
__global__ void __launch_bounds__(LS_BB) k_ls_update(const BProb *__restrict__ probs, const LBlock *__restrict__ blks, int NE,
                                                     LState *st, double *part, int *active, int *ru_list, int *ru_count)
{
    using F = typename std::conditional<MIXED, float, double>::type;
    __shared__ int s_ru;
    const int e = blockIdx.x;
    const LBlock L = blks[e];
    const BProb P = probs[L.m];
    LState &S = st[L.m];
    if (S.done) return;
    F *r = MIXED ? (F *)P.r32 : (F *)P.r64;
    F *z = MIXED ? (F *)P.z32 : (F *)P.z64;
    const int it = S.it;
    const F *p = (it & 1) ? (MIXED ? (const F *)P.pb32 : (const F *)P.pb64) : (MIXED ? (const F *)P.pa32 : (const F *)P.pa64);
    const F *Ap = MIXED ? (const F *)P.Ap32 : (const F *)P.Ap64;
    const F *inv = MIXED ? (const F *)P.inv32 : (const F *)P.inv64;
    F *acc = MIXED ? (F *)P.d32 : (F *)P.x;
    const F alpha = (F)S.alpha;
    double v[2] = {0.0, 0.0};
    // UU rows per thread and round (rows i, i + LS_BB, ...: the order of the sums is that of a
    // row at a time), every load of the round issued before its stores
    constexpr int UU = 4;
    for (int i0 = L.r0 + (int)threadIdx.x; i0 < L.r1; i0 += UU * LS_BB) {
        F rv[UU], av[UU], iv[UU], cv[UU], pv[UU];
#pragma unroll
        for (int u = 0; u < UU; ++u) {
            const int i = i0 + u * LS_BB;
            const bool ok = i < L.r1;
            rv[u] = ok ? r[i] : F(0);
            av[u] = ok ? Ap[i] : F(0);
            iv[u] = ok ? inv[i] : F(0);
            cv[u] = ok ? acc[i] : F(0);
            pv[u] = ok ? p[i] : F(0);
        }
#pragma unroll
        for (int u = 0; u < UU; ++u) {
            const int i = i0 + u * LS_BB;
            if (i < L.r1) {
                const F ri = rv[u] - alpha * av[u];
                const F zi = iv[u] * ri;
                r[i] = ri;
                z[i] = zi;
                acc[i] = cv[u] + alpha * pv[u];
                v[0] += (double)ri * (double)ri;
                v[1] += (double)ri * (double)zi;
            }
        }
    }
    double tot[2];
    if (!ls_member_sum<2>(v, part, NE, e, L, &S.t2, tot)) return;
    if (threadIdx.x == 0) {
        s_ru = 0;
        const int it1 = it + 1;
        S.it = it1;
        const double rn = sqrt(tot[0]), rzn = tot[1];
        if (!MIXED) {
            S.res = rn / S.nb;
            if (rn <= P.tol * S.nb || it1 >= P.max_iter) {
                ls_finish(S, active);
            } else {
                S.beta = rzn / S.rz;
                S.rz = rzn;
                if (!(rzn > 0.0)) { S.breakdown = 1; ls_finish(S, active); }
            }
        } else if (rn <= 0.1 * S.maxr || rn <= P.tol * S.nb || it1 >= P.max_iter || !(rzn > 0.0)) {
            S.want_ru = 1;
            S.rz_prev = S.rz;
            S.rn_rec = rn;
            s_ru = atomicAdd(ru_count, L.b1 - L.b0) + 1;
        } else {
            S.beta = rzn / S.rz;
            S.rz = rzn;
        }
    }
    __syncthreads();
    if (MIXED && s_ru)
        for (int k = (int)threadIdx.x; k < L.b1 - L.b0; k += LS_BB) ru_list[s_ru - 1 + k] = L.b0 + k;
}

// the reliable update's first half, x += d and d = 0: on the listed entries (ALL false) or on
// every entry of a member that broke down (ALL true)
template <bool ALL>
__global__ void __launch_bounds__(LS_BB) k_ls_flush(const BProb *__restrict__ probs, const LBlock *__restrict__ blks, int NE,
                                                    const LState *__restrict__ st, const int *ru_list, const int *ru_count)
{
    const int cnt = ALL ? NE : *ru_count;
    for (int w = blockIdx.x; w < cnt; w += gridDim.x) {
        const LBlock L = blks[ALL ? w : ru_list[w]];
        const BProb P = probs[L.m];
        if (ALL && !st[L.m].breakdown) continue;
        for (int i = L.r0 + (int)threadIdx.x; i < L.r1; i += LS_BB) {
            const int ii = P.iperm ? P.iperm[i] : i;
            P.x[i] += (double)P.d32[ii];
            P.d32[ii] = 0.0f;
        }
    }
}

// The FP64 residual r = b - A64 x (stored as FP32 in mixed precision), z = inv r, and the
// member's decisions.  MODE 0: the start (also ||b||, pold = 0, d = 0), every entry; MODE 1: a
// reliable update (mixed), the listed entries; MODE 2: the final true residual, every entry.
template <bool MIXED, int MODE>
__global__ void __launch_bounds__(LS_BB, 5) k_ls_resid(const BProb *__restrict__ probs, const LBlock *__restrict__ blks, int NE,
                                                    LState *st, double *part, int *active, const int *ru_list,
                                                    const int *ru_count)
{
    using F = typename std::conditional<MIXED, float, double>::type;
    const int cnt = MODE == 1 ? *ru_count : NE;
    for (int w = blockIdx.x; w < cnt; w += gridDim.x) {
        const int e = MODE == 1 ? ru_list[w] : w;
        const LBlock L = blks[e];
        const BProb P = probs[L.m];
        LState &S = st[L.m];
        if (MODE == 0 && S.started) continue;
        if (MODE == 2 && S.zero) continue;
        F *pb = MIXED ? (F *)P.pb32 : (F *)P.pb64;
        const double *x = P.x;
        double v[3] = {0.0, 0.0, 0.0};
        ls_spmv_entry<double, double>(
            P, P.A64, L, [&](int j) { return x[j]; },
            [&](int i) { return make_double2(P.b[i], MODE == 2 ? 0.0 : P.inv64[i]); },
            [&](int i, double s, double2 own) {
                const double bi = own.x, ri = bi - s;
                const int ii = MIXED && P.iperm ? P.iperm[i] : i;   // the row in the member's vector order
                v[0] += ri * ri;
                if (MODE != 2) {
                    if (MIXED) {
                        const float rf = (float)ri, zf = (float)own.y * rf;
                        P.r32[ii] = rf;
                        P.z32[ii] = zf;
                        v[1] += (double)rf * (double)zf;
                    } else {
                        const double zi = own.y * ri;
                        P.r64[i] = ri;
                        P.z64[i] = zi;
                        v[1] += ri * zi;
                    }
                }
                if (MODE == 0) {
                    v[2] += bi * bi;
                    pb[ii] = F(0);
                    if (MIXED) P.d32[ii] = 0.0f;
                }
            });
        double tot[3];
        if (!ls_member_sum<3>(v, part, NE, e, L, &S.t3, tot) || threadIdx.x != 0) continue;
        const double rn = sqrt(tot[0]);
        if (MODE == 0) {
            const double nb = sqrt(tot[2]);
            S.started = 1;
            S.nb = nb;
            S.rz = tot[1];
            S.maxr = rn;
            S.prt = rn;
            S.beta = 0.0;
            S.res = nb == 0.0 ? 0.0 : rn / nb;
            if (nb == 0.0) {
                S.zero = 1;
                S.conv = 1;
                ls_finish(S, active);
            } else if (rn <= P.tol * nb) {
                S.conv = 1;
                ls_finish(S, active);
            } else if (!(S.rz > 0.0)) {
                S.breakdown = 1;
                ls_finish(S, active);
            }
        } else if (MODE == 1) {
            S.want_ru = 0;
            S.rus += 1;
            S.res = rn / S.nb;
            S.maxr = rn;
            if (rn <= P.tol * S.nb || S.it >= P.max_iter) {
                ls_finish(S, active);
                continue;
            }
            // stagnation of the FP32 recurrence: the host goes on in FP64 from this iterate
            S.stall = rn > 0.5 * S.prt ? S.stall + 1 : 0;
            S.prt = rn;
            if (S.stall >= 2 || !(rn < 1e300)) {
                S.fallback = 1;
                ls_finish(S, active);
                continue;
            }
            if (!(tot[1] > 0.0)) {
                S.breakdown = 1;
                ls_finish(S, active);
                continue;
            }
            // drifted recurrence (true residual over twice its own): restart the direction
            S.beta = rn > 2.0 * S.rn_rec ? 0.0 : tot[1] / S.rz_prev;
            S.rz = tot[1];
        } else {
            S.res = rn / S.nb;
        }
    }
}

// x = 0 for the members with b = 0
__global__ void __launch_bounds__(LS_BB) k_ls_zero(const BProb *__restrict__ probs, const LBlock *__restrict__ blks,
                                                   const LState *__restrict__ st)
{
    const LBlock L = blks[blockIdx.x];
    if (!st[L.m].zero) return;
    for (int i = L.r0 + (int)threadIdx.x; i < L.r1; i += LS_BB) probs[L.m].x[i] = 0.0;
}

}  // namespace femd

using namespace femd;

namespace {

struct Member {
    femd_matrix K = nullptr;
    bool armed = false;
    int n = 0, team = 1, nch = 0, maxlen = 0;
    long long nnz = 0;
    DevBuf<int> tables;                         // crow (nch+1), cq (nch+1)
    DevBuf<double> cpart;                       // per-chunk sums of the SpMV passes (6 x nch)
    float *f32 = nullptr;                       // A32, inv32, r, z, p, p', Ap, d
    long long a32_cap = 0;                      // room for A32 in f32: nnz, or the sliced layout's size
    double *f64 = nullptr;                      // r, z, p, p', Ap
    const double *b = nullptr;
    double *x = nullptr;
    double tol = 0.0;
    int max_iter = 0;
    bool need_f32 = false;                      // armed: the FP32 copies are made before its first mixed launch
    bool f32_compact = false;                   // the FP32 copy is in the compact (reordered) layout
    bool force_fp64 = false;                    // its FP32 recurrence stagnated: FP64 for the rest of the solve
    int prior_its = 0, prior_rus = 0;           // iterations and reliable updates before the switch
    DevBuf<int> ls_tab;                         // lockstep SpMV windows: first rows (nw + 1), scratch
    std::vector<int> ls_wrow;                   // the same on the host (empty: not built)
};

}  // namespace

struct LsLive;
static void live_free(LsLive *L);

struct femd_batch_s : femd::HandleBase {
    femd_ctx ctx = nullptr;
    std::vector<std::unique_ptr<Member>> mem;   // index = member id (null: free)
    // launch shape: threads per block, nonzeros per team rank, nonzeros per thread per chunk
    int block = 256, nnz_per_block = 65536, npt = 4;
    int grid = 0;
    int cap = 0;                                // member capacity of the device arrays
    size_t slot_cap = 0;                        // slot capacity of the device arrays
    DevBuf<BProb> d_probs;
    DevBuf<BState> d_state;
    DevBuf<unsigned> d_bar;
    DevBuf<unsigned long long> d_claim;
    DevBuf<int> d_slots;                        // slot_prob then slot_member (2 x slot_cap)
    DevBuf<double> d_part;
    DevBuf<BQueue> d_queue;
    DevBuf<int> d_scratch;
    size_t part_cap = 0;
    // pinned staging of a launch: descriptors, slots and queue in, states out
    void *pinned = nullptr;
    BProb *h_desc = nullptr;
    BState *h_state = nullptr;
    int *h_slots = nullptr;
    BQueue *h_q0 = nullptr, *h_qout = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int graph_state[2] = {0, 0};                // 0 none, 1 captured, -1 capture refused (direct launches)
    int ghost = -1;                             // test hook: this member waits for a rank that never comes
    long long spin_limit = SPIN_LIMIT;
    int *abort_host = nullptr;                  // mapped pinned flag
    // the lockstep engine: nonzeros per table entry, iterations enqueued between state reads
    int ls_nnz = 16384, ls_chunk = 8;
    bool ls_windows = false;                    // SpMV by windows (else by row groups)
    bool ls_compact = true;                     // mixed precision: the compact layout where it applies
    long long ls_stats[4] = {0, 0, 0, 0};       // last lockstep solve: compact members, plain members, widest window, entries
    struct LiveDel {
        void operator()(LsLive *L) const { live_free(L); }
    };
    std::unique_ptr<LsLive, LiveDel> live;      // the continuous lockstep engine's state (members in flight)
    int *abort_dev = nullptr;
    femd_batch_s() : HandleBase(femd::KIND_BATCH) {}
    void drop_graphs()
    {
        for (int k = 0; k < 2; ++k) {
            if (exec[k]) cudaGraphExecDestroy(exec[k]);
            exec[k] = nullptr;
            graph_state[k] = 0;
        }
    }
    void free_vectors(Member &M)
    {
        if (M.f32) cudaFreeAsync(M.f32, ctx->stream);
        if (M.f64) cudaFreeAsync(M.f64, ctx->stream);
        M.f32 = nullptr;
        M.f64 = nullptr;
    }
    ~femd_batch_s() override
    {
        drop_graphs();
        for (auto &M : mem)
            if (M) free_vectors(*M);
        if (ctx) cudaStreamSynchronize(ctx->stream);
        if (abort_host) cudaFreeHost(abort_host);
        if (pinned) cudaFreeHost(pinned);
        if (h_slots) cudaFreeHost(h_slots);
        femd::ctx_release(ctx);
    }
};

static femd_batch_s *as_batch(void *h)
{
    femd_batch_s *b = static_cast<femd_batch_s *>(h);
    return (b && b->kind == KIND_BATCH) ? b : nullptr;
}

static int chunk_cap(const femd_batch_s *B) { return B->block * B->npt; }

// a member's team size and chunk tables for the current launch shape
static int member_layout(femd_batch_s *B, Member &M)
{
    cudaStream_t s = B->ctx->stream;
    const int C = chunk_cap(B);
    FEMD_CHECK_ARG(M.maxlen <= C / 2, "batch: a row is longer than half the SpMV chunk (block x nonzeros per thread)");
    const int cp = C - M.maxlen;
    const int nch = (int)std::max<long long>(1, (M.nnz + cp - 1) / cp);
    if (M.tables.n < 2 * (size_t)(nch + 1)) {
        int st = M.tables.alloc(2 * (size_t)(nch + 1));
        if (st) return st;
    }
    if (M.cpart.n < KB_KINDS * (size_t)nch) {
        int st = M.cpart.alloc(KB_KINDS * (size_t)nch);
        if (st) return st;
    }
    M.nch = nch;
    k_chunk_table<<<grid_for((size_t)nch + 1, 256), 256, 0, counted(s)>>>(M.K->pattern->indptr.p, M.n, (int)M.nnz, cp, nch,
                                                                          M.tables.p, M.tables.p + nch + 1);
    FEMD_TRY_CUDA(cudaGetLastError());
    int T = (int)std::min<long long>((M.nnz + B->nnz_per_block - 1) / B->nnz_per_block, (long long)B->grid / 2);
    M.team = std::max(1, std::min(T, std::min(nch, std::max(1, M.n / 64))));
    return FEMD_OK;
}

static int grow_arrays(femd_batch_s *B, int cap)
{
    if (cap <= B->cap) return FEMD_OK;
    cap = std::max(cap, 2 * B->cap);
    int st;
    if ((st = B->d_probs.alloc(cap)) || (st = B->d_bar.alloc(cap)) || (st = B->d_claim.alloc(cap))) return st;
    {
        // members may be part-way through a resumable solve: keep their states
        DevBuf<BState> ns;
        if ((st = ns.alloc(cap))) return st;
        cudaStream_t s = B->ctx->stream;
        cudaError_t e = cudaMemsetAsync(ns.p, 0, (size_t)cap * sizeof(BState), s);
        if (e == cudaSuccess && B->d_state.p)
            e = cudaMemcpyAsync(ns.p, B->d_state.p, B->d_state.n * sizeof(BState), cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error(std::string("batch: ") + cudaGetErrorString(e)); return FEMD_ECUDA; }
        std::swap(B->d_state.p, ns.p);
        std::swap(B->d_state.n, ns.n);
    }
    if (B->pinned) cudaFreeHost(B->pinned);
    B->pinned = nullptr;
    B->cap = 0;
    const size_t pin = (size_t)cap * (sizeof(BProb) + sizeof(BState)) + 2 * sizeof(BQueue) + 64;
    FEMD_TRY_CUDA(cudaHostAlloc(&B->pinned, pin, cudaHostAllocDefault));
    char *c = static_cast<char *>(B->pinned);
    B->h_desc = reinterpret_cast<BProb *>(c); c += (size_t)cap * sizeof(BProb);
    B->h_state = reinterpret_cast<BState *>(c); c += (size_t)cap * sizeof(BState);
    B->h_q0 = reinterpret_cast<BQueue *>(c); c += sizeof(BQueue);
    B->h_qout = reinterpret_cast<BQueue *>(c);
    std::memset(B->h_desc, 0, (size_t)cap * sizeof(BProb));
    B->cap = cap;
    B->drop_graphs();
    return FEMD_OK;
}

static int grow_slots(femd_batch_s *B, size_t need)
{
    if (need <= B->slot_cap) return FEMD_OK;
    need = std::max(need, 2 * B->slot_cap);
    int st;
    if ((st = B->d_slots.alloc(2 * need)) || (st = B->d_part.alloc(8 * need + 8))) return st;
    if (B->h_slots) cudaFreeHost(B->h_slots);
    B->h_slots = nullptr;
    FEMD_TRY_CUDA(cudaHostAlloc(&B->h_slots, 2 * need * sizeof(int), cudaHostAllocDefault));
    B->slot_cap = need;
    B->drop_graphs();
    return FEMD_OK;
}

static int batch_shape(femd_batch_s *B)
{
    int bps = 0, bps64 = 0;
    FEMD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, batch_kernel(true, B->block, B->npt), B->block, 0));
    FEMD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps64, batch_kernel(false, B->block, B->npt), B->block, 0));
    bps = std::min(bps, bps64);
    FEMD_CHECK_ARG(bps >= 1, "batch: the batch kernel does not fit on an SM");
    B->grid = bps * B->ctx->sm_count;
    size_t slots = 0;
    for (auto &up : B->mem)
        if (up) {
            int st = member_layout(B, *up);
            if (st) return st;
            slots += (size_t)up->team;
        }
    FEMD_TRY_CUDA(cudaStreamSynchronize(B->ctx->stream));
    B->drop_graphs();
    return grow_slots(B, std::max<size_t>(slots, 1));
}

static int add_member(femd_batch_s *B, femd_matrix K, int *id_out)
{
    FEMD_CHECK_ARG(K && K->kind == KIND_MATRIX, "batch: not a matrix handle");
    FEMD_CHECK_ARG(K->ctx == B->ctx, "batch: the matrix belongs to another context");
    FEMD_CHECK_ARG(K->pattern->nrows == K->pattern->ncols, "batch: the matrices must be square");
    FEMD_CHECK_ARG(K->pattern->nrows >= 1, "batch: empty matrix");
    FEMD_CHECK_ARG(K->pattern->nnz < INT_MAX, "batch: more than 2^31 nonzeros");
    FEMD_CHECK_ARG(K->inv_valid, "batch: the matrix has no inverse diagonal; call JacobiPreconditioner first "
                                 "(femd_cuda_matrix_jacobi, an assembly with want_inv, or femd_cuda_matrix_set_inv_diag)");
    int id = -1;
    for (size_t i = 0; i < B->mem.size(); ++i)
        if (!B->mem[i]) { id = (int)i; break; }
    if (id < 0) { id = (int)B->mem.size(); B->mem.emplace_back(); }
    int st;
    if ((st = grow_arrays(B, (int)B->mem.size()))) return st;
    B->mem[id].reset(new Member());
    Member &M = *B->mem[id];
    M.K = K;
    M.n = K->pattern->nrows;
    M.nnz = K->pattern->nnz;
    cudaStream_t s = B->ctx->stream;
    FEMD_TRY_CUDA(cudaMemsetAsync(B->d_scratch.p, 0, sizeof(int), s));
    k_max_row<<<grid_for((size_t)M.n, 256, 1024), 256, 0, counted(s)>>>(K->pattern->indptr.p, M.n, B->d_scratch.p);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaMemcpyAsync(&M.maxlen, B->d_scratch.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    if ((st = member_layout(B, M))) { B->mem[id].reset(); return st; }
    size_t slots = 0;
    for (auto &X : B->mem)
        if (X) slots += (size_t)X->team;
    if ((st = grow_slots(B, slots))) { B->mem[id].reset(); return st; }
    *id_out = id;
    return FEMD_OK;
}

static int build_compact(femd_ctx ctx, femd_pattern P);

// the member's vectors of one precision (stream-ordered allocation on the first use). With
// `sliced` (a mixed lockstep solve that may use the compact layout) the pattern's compact layout
// is built first and A32 gets room for its padded slices; a smaller arena is replaced (its FP32
// copy is made again).
static int member_vectors(femd_batch_s *B, Member &M, bool mixed, bool sliced = false)
{
    cudaStream_t s = B->ctx->stream;
    const size_t n = (size_t)M.n, nnz = (size_t)M.nnz;
    size_t cap = nnz;
    if (mixed && sliced) {
        femd_pattern P = M.K->pattern;
        int st;
        if ((st = build_compact(B->ctx, P))) return st;
        if (P->cl_state == 1) cap = std::max(cap, (size_t)P->cl_nsell);
    }
    if (mixed && M.f32 && (size_t)M.a32_cap < cap) {
        cudaFreeAsync(M.f32, s);
        M.f32 = nullptr;
        M.need_f32 = true;
    }
    if (mixed && !M.f32) {
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&M.f32), (cap + 9 * n + 40) * sizeof(float), s);
        if (e != cudaSuccess) { M.f32 = nullptr; cudaGetLastError(); set_error("batch: out of device memory"); return FEMD_ENOMEM; }
        M.a32_cap = (long long)cap;
        if (reinterpret_cast<uintptr_t>(M.f32) & 15) {
            // the FP32 values are read by 16-byte bulk copies
            cudaFreeAsync(M.f32, s);
            M.f32 = nullptr;
            set_error("batch: FP32 arena not 16-byte aligned");
            return FEMD_ECUDA;
        }
    }
    if (!mixed && !M.f64) {
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&M.f64), (5 * n + 8) * sizeof(double), s);
        if (e != cudaSuccess) { M.f64 = nullptr; cudaGetLastError(); set_error("batch: out of device memory"); return FEMD_ENOMEM; }
    }
    return FEMD_OK;
}

static BProb describe(femd_batch_s *B, int id, bool mixed)
{
    Member &M = *B->mem[id];
    BProb P{};
    P.n = M.n;
    P.team = M.team;
    P.max_iter = M.max_iter;
    P.nch = M.nch;
    P.nnz = (int)M.nnz;
    P.tol = M.tol;
    P.indptr = M.K->pattern->indptr.p;
    P.indices = M.K->pattern->indices.p;
    P.crow = M.tables.p;
    P.cq = M.tables.p + M.nch + 1;
    P.A64 = M.K->data.p;
    P.inv64 = M.K->inv.p;
    const size_t n = (size_t)M.n, nnz = (size_t)M.nnz;
    if (mixed) {
        float *f = M.f32;
        P.A32 = f;
        f = M.f32 + (((size_t)M.a32_cap + 7) & ~(size_t)7);
        P.inv32 = f; f += n;
        P.r32 = f; f += n;
        P.z32 = f; f += n;
        P.pa32 = f; f += n;
        P.pb32 = f; f += n;
        P.Ap32 = f; f += n;
        P.d32 = f; f += n;
        // the compact layout's row table (n + 1 int2), 8-byte aligned; set by ls_member_setup
        P.ctab = nullptr;
    } else {
        double *d = M.f64;
        P.r64 = d; d += n;
        P.z64 = d; d += n;
        P.pa64 = d; d += n;
        P.pb64 = d; d += n;
        P.Ap64 = d;
    }
    P.b = M.b;
    P.x = M.x;
    P.bar = B->d_bar.p + id;
    P.claim = B->d_claim.p + id;
    P.cpart = M.cpart.p;
    P.st = B->d_state.p + id;
    return P;
}

static cudaError_t launch_batch(femd_batch_s *B, bool mixed, cudaStream_t s)
{
    const BProb *probs = B->d_probs.p;
    const int *sp = B->d_slots.p, *sm = B->d_slots.p + B->slot_cap;
    BQueue *q = B->d_queue.p;
    volatile const int *ab = B->abort_dev;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)B->grid);
    cfg.blockDim = dim3((unsigned)B->block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, batch_kernel(mixed, B->block, B->npt), probs, sp, sm, q, ab);
}

// one launch's device work: descriptors, slots and queue in, the launch, states out
static cudaError_t enqueue_step(femd_batch_s *B, bool mixed, cudaStream_t s)
{
    cudaError_t e;
    const size_t cap = (size_t)B->cap;
    if ((e = cudaMemcpyAsync(B->d_probs.p, B->h_desc, cap * sizeof(BProb), cudaMemcpyHostToDevice, s))) return e;
    if ((e = cudaMemcpyAsync(B->d_slots.p, B->h_slots, 2 * B->slot_cap * sizeof(int), cudaMemcpyHostToDevice, s))) return e;
    if ((e = cudaMemsetAsync(B->d_bar.p, 0, cap * sizeof(unsigned), s))) return e;
    if ((e = cudaMemsetAsync(B->d_claim.p, 0, cap * sizeof(unsigned long long), s))) return e;
    if ((e = cudaMemcpyAsync(B->d_queue.p, B->h_q0, sizeof(BQueue), cudaMemcpyHostToDevice, s))) return e;
    if ((e = launch_batch(B, mixed, s))) return e;
    if ((e = cudaMemcpyAsync(B->h_state, B->d_state.p, cap * sizeof(BState), cudaMemcpyDeviceToHost, s))) return e;
    return cudaMemcpyAsync(B->h_qout, B->d_queue.p, sizeof(BQueue), cudaMemcpyDeviceToHost, s);
}

static void fill_result(const BState &S, femd_cg_result &r, double seconds)
{
    r.iterations = S.it;
    r.converged = (S.flags & BS_CONVERGED) ? 1 : 0;
    r.breakdown = (S.flags & BS_BREAKDOWN) ? 1 : 0;
    r.status = S.status;
    r.outer = S.rus;
    r.residual = S.res;
    r.seconds = seconds;
}

// one launch over the armed members: each advances by at most iters iterations.  Members that
// finish are disarmed and listed (ids, results) when the lists are given.
// one launch over the members `order` (armed), all in one precision: each advances by at most
// iters iterations; the states are in h_state afterwards, the launch time in *ms
static int launch_set(femd_ctx ctx, femd_batch_s *B, std::vector<int> order, int iters, bool mx, float *ms)
{
    cudaStream_t s = ctx->stream;
    int st;
    *ms = 0.f;
    for (int id : order)
        if ((st = member_vectors(B, *B->mem[id], mx))) return st;
    if (mx) {
        for (int id : order) {
            Member &M = *B->mem[id];
            if (!M.need_f32 && !M.f32_compact) continue;
            const BProb P = describe(B, id, true);
            k_batch_f32<<<grid_for((size_t)M.nnz, 256, 4 * (unsigned)B->ctx->sm_count), 256, 0, counted(s)>>>(
                M.K->data.p, P.A32, M.nnz, M.K->inv.p, P.inv32, M.n);
            FEMD_TRY_CUDA(cudaGetLastError());
            M.need_f32 = false;
            M.f32_compact = false;
        }
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        if (B->mem[a]->team != B->mem[b]->team) return B->mem[a]->team > B->mem[b]->team;
        return B->mem[a]->nnz > B->mem[b]->nnz;
    });
    // descriptors, slots and team scratch
    size_t ns = 0, opart = 0;
    for (int id : order) ns += (size_t)B->mem[id]->team + (id == B->ghost ? 1 : 0);
    if ((st = grow_slots(B, ns + 1))) return st;
    int *sp = B->h_slots, *sm = B->h_slots + B->slot_cap;
    ns = 0;
    for (int id : order) {
        BProb P = describe(B, id, mx);
        P.part = B->d_part.p + opart;
        opart += 8 * (size_t)(P.team + 1);
        for (int m = 0; m < P.team; ++m) { sp[ns] = id; sm[ns] = m; ++ns; }
        if (id == B->ghost) P.team += 1;                // test hook (femd_cuda_batch_debug)
        B->h_desc[id] = P;
    }
    if (opart > B->d_part.n) {
        if ((st = B->d_part.alloc(opart + 8))) return st;
        // the part pointers were set from the old buffer: redo them
        opart = 0;
        for (int id : order) {
            B->h_desc[id].part = B->d_part.p + opart;
            opart += 8 * (size_t)(B->mem[id]->team + 1);
        }
        B->drop_graphs();
    }
    *B->h_q0 = BQueue{0u, 0, B->spin_limit, (int)ns, std::max(1, iters), 0ull, 0ull, 0ull, 0, 0, 0, 0};
    *(volatile int *)B->abort_host = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    FEMD_TRY_CUDA(cudaEventCreate(&e0));
    FEMD_TRY_CUDA(cudaEventCreate(&e1));
    cudaError_t e = cudaSuccess;
    const int k = mx ? 1 : 0;
    if (B->graph_state[k] == 0) {
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t e2 = enqueue_step(B, mx, s);
            e = cudaStreamEndCapture(s, &g);
            if (e == cudaSuccess) e = e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&B->exec[k], g, 0);
        if (g) cudaGraphDestroy(g);
        if (e == cudaSuccess) {
            B->graph_state[k] = 1;
        } else {
            cudaGetLastError();
            B->exec[k] = nullptr;
            B->graph_state[k] = -1;                     // this runtime does not capture the launch: launch directly
            e = cudaSuccess;
        }
    }
    cudaEventRecord(e0, s);
    if (B->graph_state[k] == 1) {
        e = launch_graph(B->exec[k], 1, s);
    } else {
        e = enqueue_step(B, mx, s);
        if (e == cudaSuccess) add_launches(1);
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) { set_error(std::string("batch: ") + cudaGetErrorString(e)); return FEMD_ECUDA; }
    if (B->h_qout->fail_where == 3) {
        set_error("batch: a staging copy had not landed when its block gave up and exited; the CUDA context may be "
                  "unusable");
        return FEMD_ECUDA;
    }
    return FEMD_OK;
}

// a member's result: its iterations and reliable updates include those of a mixed-precision
// phase that fell back to FP64
static void fill_member(const femd_batch_s *B, int id, femd_cg_result &r, double seconds)
{
    const BState &S = B->h_state[id];
    const Member &M = *B->mem[id];
    fill_result(S, r, seconds);
    r.iterations += M.prior_its;
    r.outer += M.prior_rus;
}

// one step: every armed member advances by at most iters iterations.  In a mixed step the members
// whose FP32 recurrence stagnated before (or stagnates in this launch) go on in an FP64 launch in
// the same call, from their current iterate.  Members that finish are disarmed and listed.
static int batch_step(femd_ctx ctx, femd_batch_s *B, int iters, bool mx, int *nfinished, int *fin_ids, femd_cg_result *fin_res,
                      double *seconds)
{
    std::vector<int> set32, set64;
    for (int id = 0; id < (int)B->mem.size(); ++id) {
        if (!B->mem[id] || !B->mem[id]->armed) continue;
        (mx && !B->mem[id]->force_fp64 ? set32 : set64).push_back(id);
    }
    if (nfinished) *nfinished = 0;
    if (seconds) *seconds = 0.0;
    int nf = 0, st = FEMD_OK;
    double sec = 0.0;
    int flag = 0;
    auto collect = [&](const std::vector<int> &set, bool mode) {
        for (int id : set) {
            const BState &S = B->h_state[id];
            Member &M = *B->mem[id];
            if (!(S.flags & BS_DONE) && !flag && !S.status) continue;
            if (mode && (S.flags & BS_FALLBACK) && !flag && !S.status) {
                // the FP32 recurrence stagnated: go on in FP64 from the iterate x
                M.force_fp64 = true;
                M.prior_its += S.it;
                M.prior_rus += S.rus;
                M.max_iter = std::max(1, M.max_iter - S.it);
                cudaMemsetAsync(B->d_state.p + id, 0, sizeof(BState), ctx->stream);
                set64.push_back(id);
                continue;
            }
            M.armed = false;
            if (fin_ids) fin_ids[nf] = id;
            if (fin_res) {
                fill_member(B, id, fin_res[nf], sec);
                if (flag) fin_res[nf].status = flag;
            }
            ++nf;
        }
    };
    if (!set32.empty()) {
        float ms = 0.f;
        if ((st = launch_set(ctx, B, set32, iters, true, &ms))) return st;
        sec += ms * 1e-3;
        flag = B->h_qout->flag;
        collect(set32, true);
    }
    if (!set64.empty() && !flag) {
        float ms = 0.f;
        if ((st = launch_set(ctx, B, set64, iters, false, &ms))) return st;
        sec += ms * 1e-3;
        flag = B->h_qout->flag;
        collect(set64, false);
    }
    if (nfinished) *nfinished = nf;
    if (seconds) *seconds = sec;
    if (flag == FEMD_ETIMEOUT) { set_error("batch: a team barrier wait ran out"); return FEMD_ETIMEOUT; }
    if (flag == FEMD_EABORT) { set_error("batch: aborted by the host"); return FEMD_EABORT; }
    return FEMD_OK;
}

static int arm_member(femd_batch_s *B, int id, const double *b, double *x, int max_iter, double tol)
{
    FEMD_CHECK_ARG(id >= 0 && id < (int)B->mem.size() && B->mem[id], "batch: no such member");
    FEMD_CHECK_ARG(b && x, "batch: NULL vector");
    FEMD_CHECK_ARG(tol >= 0.0, "batch: tol < 0");
    Member &M = *B->mem[id];
    M.b = b;
    M.x = x;
    M.tol = tol;
    M.max_iter = max_iter > 0 ? max_iter : std::max(1000, 10 * M.n);
    M.armed = true;
    M.need_f32 = true;
    M.force_fp64 = false;
    M.prior_its = 0;
    M.prior_rus = 0;
    FEMD_TRY_CUDA(cudaMemsetAsync(B->d_state.p + id, 0, sizeof(BState), B->ctx->stream));
    return FEMD_OK;
}

// ---- the lockstep engine: host side ----------------------------------------------------------

// lanes per row of a member's SpMV: the fewest (a power of two, at least 2) whose 4 loads in
// flight each cover the mean row
static int ls_tpr(const Member &M)
{
    const double avg = (double)M.nnz / (double)M.n;
    int tpr = 2;
    while (tpr * 4 < avg && tpr < 32) tpr <<= 1;
    return tpr;
}

// rows of one table entry of a member: about nnz_per_entry nonzeros
static int ls_rows_per_entry(const femd_batch_s *B, const Member &M)
{
    const long long r = (long long)B->ls_nnz * M.n / std::max(1LL, M.nnz);
    return (int)std::max(32LL, std::min((long long)M.n, r));
}

// a member's SpMV windows for the lockstep engine (built once): window c holds the rows that start
// at nonzeros [c cp, (c + 1) cp), cp = LS_W - the longest row, so at most LS_W - 1 nonzeros.  A
// member whose longest row is over LS_W / 2 keeps none (row groups).
static int ls_windows_of(femd_batch_s *B, Member &M)
{
    if (!M.ls_wrow.empty() || M.maxlen > LS_W / 2) return FEMD_OK;
    cudaStream_t s = B->ctx->stream;
    const int cp = LS_W - M.maxlen;
    const int nw = (int)std::max<long long>(1, (M.nnz + cp - 1) / cp);
    int st;
    if ((st = M.ls_tab.alloc(2 * (size_t)(nw + 1)))) return st;
    k_chunk_table<<<grid_for((size_t)nw + 1, 256), 256, 0, counted(s)>>>(M.K->pattern->indptr.p, M.n, (int)M.nnz, cp, nw,
                                                                         M.ls_tab.p, M.ls_tab.p + nw + 1);
    FEMD_TRY_CUDA(cudaGetLastError());
    std::vector<int> h((size_t)nw + 1);
    FEMD_TRY_CUDA(cudaMemcpyAsync(h.data(), M.ls_tab.p, (nw + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    M.ls_wrow.swap(h);
    return FEMD_OK;
}

// ---- the compact layout (lockstep engine, mixed precision) -------------------------------------

// (the host part -- order, slices, offsets -- is femd::compact_layout, setup_host.cpp)
static constexpr int CL_WIN_MAX = 12288;    // largest column window of an entry (FP32: 48 KB of shared memory)

// Build the pattern's compact layout once (cl_state 1), or mark it unsuitable (-1).
static int build_compact(femd_ctx ctx, femd_pattern P)
{
    if (P->cl_state != 0) return FEMD_OK;
    cudaStream_t s = ctx->stream;
    const int n = P->nrows;
    const long long nnz = P->nnz;
    std::vector<int> ip((size_t)n + 1), ix((size_t)std::max<long long>(nnz, 1));
    FEMD_TRY_CUDA(cudaMemcpyAsync(ip.data(), P->indptr.p, ((size_t)n + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (nnz) FEMD_TRY_CUDA(cudaMemcpyAsync(ix.data(), P->indices.p, (size_t)nnz * sizeof(int), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    CompactLayout L;
    compact_layout(n, ip, ix, L);
    P->cl_bw = L.bw;
    if (!L.ok) {
        P->cl_state = -1;
        return FEMD_OK;
    }
    const long long nsell = L.nsell;
    int st;
    if ((st = P->cl_iperm.alloc((size_t)n)) || (st = P->cl_indptr.alloc((size_t)n + 1)) ||
        (st = P->cl_dst.alloc((size_t)std::max<long long>(nnz, 1))) || (st = P->cl_off.alloc((size_t)std::max<long long>(nsell, 1))))
        return st;
    FEMD_TRY_CUDA(cudaMemcpyAsync(P->cl_iperm.p, L.iperm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(P->cl_indptr.p, L.rstart.data(), ((size_t)n + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    if (nnz) FEMD_TRY_CUDA(cudaMemcpyAsync(P->cl_dst.p, L.dst.data(), (size_t)nnz * sizeof(int), cudaMemcpyHostToDevice, s));
    if (nsell) FEMD_TRY_CUDA(cudaMemcpyAsync(P->cl_off.p, L.off.data(), (size_t)nsell * sizeof(short), cudaMemcpyHostToDevice, s));
    P->cl_nsell = nsell;
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // the host vectors are released on return
    P->cl_tile_lo.swap(L.tlo);
    P->cl_tile_hi.swap(L.thi);
    P->cl_state = 1;
    return FEMD_OK;
}

namespace {
struct PinnedBuf {
    void *p = nullptr;
    ~PinnedBuf()
    {
        if (p) cudaFreeHost(p);
    }
};
}  // namespace

// One lockstep solve of the members `ids` (armed, one precision).  The final states go to out.
// One member's part of a lockstep launch: its descriptor (FP32 compact, FP32 plain or FP64 layout)
// and its table entries (r0, r1, w0, w1); maxwin grows to its widest shared-memory window.
// the compact layout's row table of a member: in its FP32 arena after d32, 8-byte aligned
static const int2 *ls_ctab(const Member &M, const BProb &desc)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(desc.d32 + M.n);
    return reinterpret_cast<const int2 *>((a + 7) & ~(uintptr_t)7);
}

static int ls_member_setup(femd_ctx ctx, femd_batch_s *B, int id, bool mx, BProb &desc, std::vector<std::array<int, 4>> &E,
                           bool &compact, int &maxwin)
{
    int st;
    Member &M = *B->mem[id];
    desc = describe(B, id, mx);
    desc.tpr = ls_tpr(M);
    desc.wrow = nullptr;
    desc.iperm = nullptr;
    desc.ctab = nullptr;
    desc.coff = nullptr;
    if (B->ls_windows && (st = ls_windows_of(B, M))) return st;
    E.clear();
    compact = false;
    if (mx && B->ls_compact && !B->ls_windows) {
        femd_pattern P = M.K->pattern;
        if ((st = build_compact(ctx, P))) return st;
        if (P->cl_state == 1) {
            // rows per entry: a multiple of the tile near nnz_per_entry nonzeros, halved while
            // some entry's column window is wider than the shared-memory window
            int R = std::max(CL_TILE, ls_rows_per_entry(B, M) / CL_TILE * CL_TILE);
            while (!compact) {
                E.clear();
                int wmax = 0;
                for (int r = 0; r < M.n; r += R) {
                    const int r1 = std::min(M.n, r + R);
                    int lo = INT_MAX, hi = INT_MIN;
                    for (int t = r / CL_TILE; t <= (r1 - 1) / CL_TILE; ++t) {
                        lo = std::min(lo, P->cl_tile_lo[t]);
                        hi = std::max(hi, P->cl_tile_hi[t]);
                    }
                    E.push_back({r, r1, lo, hi + 1});
                    wmax = std::max(wmax, hi + 1 - lo);
                }
                if (wmax <= CL_WIN_MAX) {
                    compact = true;
                    maxwin = std::max(maxwin, wmax);
                } else if (R > CL_TILE) {
                    R = std::max(CL_TILE, R / 2 / CL_TILE * CL_TILE);
                } else {
                    break;
                }
            }
            if (!compact) E.clear();
        }
    }
    if (compact) {
        femd_pattern P = M.K->pattern;
        desc.iperm = P->cl_iperm.p;
        desc.ctab = ls_ctab(M, desc);
        desc.coff = P->cl_off.p;
    } else if (B->ls_windows && !M.ls_wrow.empty()) {
        desc.wrow = M.ls_tab.p;
        const int nw = (int)M.ls_wrow.size() - 1;
        const int G = std::max(1, B->ls_nnz / LS_W);
        for (int w = 0; w < nw; w += G) {
            const int w1 = std::min(nw, w + G);
            E.push_back({M.ls_wrow[w], M.ls_wrow[w1], w, w1});
        }
    } else {
        const int R = ls_rows_per_entry(B, M);
        for (int r = 0; r < M.n; r += R) E.push_back({r, std::min(M.n, r + R), 0, 0});
    }
    if (mx && (M.need_f32 || M.f32_compact != compact)) {
        cudaStream_t s = ctx->stream;
        const unsigned g = grid_for((size_t)M.nnz, 256, 4 * (unsigned)ctx->sm_count);
        if (compact) {
            const femd_pattern P = M.K->pattern;
            // the padding entries of the slices stay 0
            FEMD_TRY_CUDA(cudaMemsetAsync(desc.A32, 0, (size_t)P->cl_nsell * sizeof(float), s));
            k_ls_f32_perm<<<g, 256, 0, counted(s)>>>(M.K->data.p, P->cl_dst.p, desc.A32, M.nnz, M.K->inv.p, P->cl_iperm.p,
                                                     desc.inv32, M.n);
            k_ls_split_rows<<<grid_for((size_t)M.n + 1, 128, 1u << 20), 128, 0, counted(s)>>>(
                P->indptr.p, P->diag_pos.p, M.K->data.p, P->cl_dst.p, P->cl_iperm.p, P->cl_indptr.p, P->all_diag ? 1 : 0,
                desc.A32, const_cast<int2 *>(desc.ctab), M.n);
        } else
            k_batch_f32<<<g, 256, 0, counted(s)>>>(M.K->data.p, desc.A32, M.nnz, M.K->inv.p, desc.inv32, M.n);
        FEMD_TRY_CUDA(cudaGetLastError());
        M.need_f32 = false;
        M.f32_compact = compact;
    }
    return FEMD_OK;
}

static int ls_run(femd_ctx ctx, femd_batch_s *B, const std::vector<int> &ids, bool mx, std::vector<LState> &out, double *seconds)
{
    cudaStream_t s = ctx->stream;
    int st;
    const int nm = (int)ids.size();
    *seconds = 0.0;
    out.assign(nm, LState{});
    if (nm == 0) return FEMD_OK;
    for (int id : ids)
        if ((st = member_vectors(B, *B->mem[id], mx, B->ls_compact && !B->ls_windows))) return st;
    std::vector<BProb> desc(nm);
    std::vector<std::vector<std::array<int, 4>>> ents(nm);   // per member: r0, r1, w0, w1 of its entries
    std::vector<int> nent(nm);
    int NEfull = 0, max_it = 1;
    int maxwin = 0;                                     // the widest column window of a compact entry
    for (int k = 0; k < nm; ++k) {
        Member &M = *B->mem[ids[k]];
        auto &E = ents[k];
        bool compact = false;
        if ((st = ls_member_setup(ctx, B, ids[k], mx, desc[k], E, compact, maxwin))) return st;
        nent[k] = (int)E.size();
        FEMD_CHECK_ARG((long long)NEfull + nent[k] < INT_MAX / 4, "batch: too many table entries");
        NEfull += nent[k];
        max_it = std::max(max_it, M.max_iter);
    }
    {
        long long nc = 0;
        for (int k = 0; k < nm; ++k) nc += desc[k].coff != nullptr;
        B->ls_stats[0] = nc;
        B->ls_stats[1] = nm - nc;
        B->ls_stats[2] = maxwin;
        B->ls_stats[3] = NEfull;
    }
    DevBuf<BProb> d_desc;
    DevBuf<LState> d_state;
    DevBuf<LBlock> d_tab;
    DevBuf<double> d_part;
    DevBuf<int> d_int;                                  // active, ru_count, ru_list (NEfull)
    if ((st = d_desc.alloc(nm)) || (st = d_state.alloc(nm)) || (st = d_tab.alloc(NEfull)) || (st = d_part.alloc(3 * (size_t)NEfull)) ||
        (st = d_int.alloc(2 + (size_t)NEfull)))
        return st;
    // pinned staging: two tables, two state copies, the descriptors
    PinnedBuf pin;
    const size_t tab_b = (size_t)NEfull * sizeof(LBlock), st_b = (size_t)nm * sizeof(LState);
    FEMD_TRY_CUDA(cudaHostAlloc(&pin.p, 2 * tab_b + 2 * st_b + nm * sizeof(BProb) + 64, cudaHostAllocDefault));
    LBlock *h_tab[2] = {static_cast<LBlock *>(pin.p), static_cast<LBlock *>(pin.p) + NEfull};
    LState *h_st[2] = {reinterpret_cast<LState *>(h_tab[1] + NEfull), nullptr};
    h_st[1] = h_st[0] + nm;
    BProb *h_desc = reinterpret_cast<BProb *>(h_st[1] + nm);
    std::copy(desc.begin(), desc.end(), h_desc);
    // the table of the live members (all of them when live is null)
    auto build = [&](LBlock *T, const LState *live) {
        int e = 0;
        for (int k = 0; k < nm; ++k) {
            if (live && live[k].done) continue;
            const int b0 = e;
            for (const auto &x : ents[k]) T[e++] = LBlock{k, x[0], x[1], b0, b0 + nent[k], x[2], x[3]};
        }
        return e;
    };
    const int G1 = std::max(1, 8 * ctx->sm_count);     // grid of the reliable-update kernels
    int *active = d_int.p, *ru_count = d_int.p + 1, *ru_list = d_int.p + 2;
    int NE = build(h_tab[0], nullptr);
    int tb = 0;                                         // the host table buffer last uploaded
    cudaEvent_t ev[2] = {nullptr, nullptr}, t0 = nullptr, t1 = nullptr;
    struct EvGuard {
        cudaEvent_t *e;
        int n;
        ~EvGuard()
        {
            for (int i = 0; i < n; ++i)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    };
    cudaEvent_t evs[4] = {nullptr, nullptr, nullptr, nullptr};
    EvGuard guard{evs, 4};
    for (int i = 0; i < 4; ++i) FEMD_TRY_CUDA(cudaEventCreateWithFlags(&evs[i], i < 2 ? cudaEventDisableTiming : cudaEventDefault));
    ev[0] = evs[0];
    ev[1] = evs[1];
    t0 = evs[2];
    t1 = evs[3];
    *(volatile int *)B->abort_host = 0;
    FEMD_TRY_CUDA(cudaEventRecord(t0, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(d_desc.p, h_desc, nm * sizeof(BProb), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(d_tab.p, h_tab[0], NE * sizeof(LBlock), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaMemsetAsync(d_state.p, 0, st_b, s));
    FEMD_TRY_CUDA(cudaMemsetAsync(d_int.p, 0, 2 * sizeof(int), s));
    FEMD_TRY_CUDA(cudaMemcpyAsync(active, &nm, sizeof(int), cudaMemcpyHostToDevice, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));           // &nm is a host stack value
    if (mx)
        k_ls_resid<true, 0><<<NE, LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active, ru_list, ru_count);
    else
        k_ls_resid<false, 0><<<NE, LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active, ru_list, ru_count);
    FEMD_TRY_CUDA(cudaGetLastError());
    const size_t win_b = (size_t)maxwin * sizeof(float);   // the SpMV's shared-memory window
    if (mx) FEMD_TRY_CUDA(cudaFuncSetAttribute(k_ls_spmv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)(CL_WIN_MAX * sizeof(float))));
    const int C = std::max(1, B->ls_chunk);
    const long long max_chunks = (long long)max_it / C + 4;
    int aborted = 0;
    for (long long j = 0; j <= max_chunks; ++j) {
        for (int c = 0; c < C; ++c) {
            if (mx) {
                k_ls_spmv<true><<<NE, LS_BB, win_b, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active, ru_count);
                k_ls_update<true><<<NE, LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active, ru_list, ru_count);
                k_ls_flush<false><<<std::min(G1, NE), LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, ru_list, ru_count);
                k_ls_resid<true, 1><<<std::min(G1, NE), LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active,
                                                                                 ru_list, ru_count);
            } else {
                k_ls_spmv<false><<<NE, LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active, ru_count);
                k_ls_update<false><<<NE, LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active, ru_list,
                                                                   ru_count);
            }
        }
        FEMD_TRY_CUDA(cudaGetLastError());
        FEMD_TRY_CUDA(cudaMemcpyAsync(h_st[j & 1], d_state.p, st_b, cudaMemcpyDeviceToHost, s));
        FEMD_TRY_CUDA(cudaEventRecord(ev[j & 1], s));
        if (j == 0) continue;
        // the states after the previous chunk (one chunk stays queued behind them)
        FEMD_TRY_CUDA(cudaEventSynchronize(ev[(j - 1) & 1]));
        const LState *S = h_st[(j - 1) & 1];
        int live = 0, live_e = 0;
        for (int k = 0; k < nm; ++k)
            if (!S[k].done) { ++live; live_e += nent[k]; }
        if (live == 0) break;
        if (*(volatile int *)B->abort_host) { aborted = 1; break; }
        if (live_e <= (NE * 7) / 10) {
            // compact the table to the live members (their entries keep their order)
            tb ^= 1;
            NE = build(h_tab[tb], S);
            FEMD_TRY_CUDA(cudaMemcpyAsync(d_tab.p, h_tab[tb], NE * sizeof(LBlock), cudaMemcpyHostToDevice, s));
        }
    }
    // the end: the final true residual (FP64) or the flush of the members that broke down (mixed),
    // over the whole table; x = 0 for b = 0
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));           // no upload from a table buffer is pending
    tb ^= 1;
    NE = build(h_tab[tb], nullptr);
    FEMD_TRY_CUDA(cudaMemcpyAsync(d_tab.p, h_tab[tb], NE * sizeof(LBlock), cudaMemcpyHostToDevice, s));
    if (!aborted) {
        if (mx)
            k_ls_flush<true><<<std::min(G1, NE), LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, ru_list, ru_count);
        else
            k_ls_resid<false, 2><<<NE, LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, NE, d_state.p, d_part.p, active, ru_list,
                                                                ru_count);
        k_ls_zero<<<NE, LS_BB, 0, counted(s)>>>(d_desc.p, d_tab.p, d_state.p);
        FEMD_TRY_CUDA(cudaGetLastError());
    }
    FEMD_TRY_CUDA(cudaMemcpyAsync(h_st[0], d_state.p, st_b, cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaEventRecord(t1, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    *seconds = ms * 1e-3;
    std::copy(h_st[0], h_st[0] + nm, out.begin());
    if (aborted) { set_error("batch: aborted by the host"); return FEMD_EABORT; }
    return FEMD_OK;
}

// a member's result from its lockstep state (the acceptance of the persistent engine)
static void ls_result(const Member &M, const LState &S, femd_cg_result &r, double seconds)
{
    r.iterations = S.it + M.prior_its;
    r.outer = S.rus + M.prior_rus;
    r.residual = S.res;
    r.breakdown = S.breakdown;
    r.status = 0;
    r.seconds = seconds;
    int conv = S.conv;
    if (!conv && !S.breakdown && S.done) {
        conv = S.res <= M.tol * (1.0 + 1e-6) + 1e-15;
        if (!conv && S.res <= 10.0 * M.tol && S.it < M.max_iter) conv = 1;
    }
    r.converged = conv;
}

// every member of the batch solved by the lockstep engine; in mixed precision the members whose
// FP32 recurrence stagnated go on in an FP64 lockstep solve from their iterate
static int ls_solve(femd_ctx ctx, femd_batch_s *B, const std::vector<int> &ids, bool mx, femd_cg_result *results)
{
    std::vector<LState> S;
    double sec = 0.0;
    int st = ls_run(ctx, B, ids, mx, S, &sec);
    if (st && st != FEMD_EABORT) return st;
    std::vector<int> fb_ids, fb_pos;
    for (size_t p = 0; p < ids.size(); ++p) {
        Member &M = *B->mem[ids[p]];
        if (st == FEMD_OK && mx && S[p].fallback) {
            M.prior_its = S[p].it;
            M.prior_rus = S[p].rus;
            M.max_iter = std::max(1, M.max_iter - S[p].it);
            fb_ids.push_back(ids[p]);
            fb_pos.push_back((int)p);
            continue;
        }
        ls_result(M, S[p], results[p], sec);
        if (st) results[p].status = st;
    }
    if (fb_ids.empty()) return st;
    std::vector<LState> S2;
    double sec2 = 0.0;
    const int st2 = ls_run(ctx, B, fb_ids, false, S2, &sec2);
    if (st2 && st2 != FEMD_EABORT) return st2;
    for (size_t q = 0; q < fb_ids.size(); ++q) {
        ls_result(*B->mem[fb_ids[q]], S2[q], results[fb_pos[q]], sec + sec2);
        if (st2) results[fb_pos[q]].status = st2;
    }
    for (size_t p = 0; p < ids.size(); ++p) results[p].seconds = sec + sec2;
    return st2;
}

// ---- the lockstep engine, continuous ---------------------------------------------------------
// The same kernels, resumable: every call admits the members armed since the last one (their
// start kernels run first), runs a number of chunks of iterations over every member in flight, and
// finishes and returns the members that are done; the others stay on the device for the next call.
// Mixed-precision members run in one table and FP64 members (a mixed member whose FP32 recurrence
// stagnated comes back as one at the next call) in another; each iteration launches the kernels of
// both.  A member's iterates do not depend on when it joined or on the other members.
struct LsLive {
    std::vector<int> ids;                                  // members in flight, in admission order
    std::vector<char> in, f64, started;                    // per member id
    std::vector<std::vector<std::array<int, 4>>> ents;     // per member id: its entries
    int maxwin = 0;
    int cap = 0;
    size_t tab_cap = 0;
    DevBuf<BProb> d_desc;
    DevBuf<LState> d_state;
    DevBuf<LBlock> d_tab;
    DevBuf<double> d_part;
    DevBuf<int> d_int;                                     // active (unused), ru_count, ru_list (tab_cap)
    void *pin = nullptr;                                   // pinned: descriptor staging, states (2 x cap), tables (2 x tab_cap)
    size_t pin_b = 0;
    // the CUDA graph of a chunk and the table shape it was captured for
    cudaGraphExec_t gx = nullptr;
    size_t g_nodes = 0;
    int g_ne32 = -1, g_ne64 = -1, g_chunk = 0;
    const LBlock *g_tab = nullptr;
    const BProb *g_desc = nullptr;
    const LState *g_state = nullptr;
    size_t g_win = 0;
    bool g_refused = false;
    ~LsLive()
    {
        if (gx) cudaGraphExecDestroy(gx);
        if (pin) cudaFreeHost(pin);
    }
};

static void live_free(LsLive *L) { delete L; }

static int live_grow(femd_batch_s *B, LsLive &L, size_t ntab)
{
    cudaStream_t s = B->ctx->stream;
    const int cap = B->cap;
    if (L.cap < cap) {
        DevBuf<BProb> nd;
        DevBuf<LState> ns;
        int st;
        if ((st = nd.alloc(cap)) || (st = ns.alloc(cap))) return st;
        FEMD_TRY_CUDA(cudaMemsetAsync(ns.p, 0, (size_t)cap * sizeof(LState), s));
        if (L.cap) {
            FEMD_TRY_CUDA(cudaMemcpyAsync(nd.p, L.d_desc.p, (size_t)L.cap * sizeof(BProb), cudaMemcpyDeviceToDevice, s));
            FEMD_TRY_CUDA(cudaMemcpyAsync(ns.p, L.d_state.p, (size_t)L.cap * sizeof(LState), cudaMemcpyDeviceToDevice, s));
        }
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));
        std::swap(L.d_desc.p, nd.p);
        std::swap(L.d_desc.n, nd.n);
        std::swap(L.d_state.p, ns.p);
        std::swap(L.d_state.n, ns.n);
        L.in.resize(cap, 0);
        L.f64.resize(cap, 0);
        L.started.resize(cap, 0);
        L.ents.resize(cap);
        L.cap = cap;
    }
    if (ntab > L.tab_cap) {
        const size_t nc = std::max(ntab, 2 * L.tab_cap);
        int st;
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));
        if ((st = L.d_tab.alloc(nc)) || (st = L.d_part.alloc(3 * nc + 3)) || (st = L.d_int.alloc(nc + 2))) return st;
        L.tab_cap = nc;
    }
    const size_t need = 2 * (size_t)cap * sizeof(LState) + sizeof(BProb) + 2 * L.tab_cap * sizeof(LBlock) + 64;
    if (need > L.pin_b) {
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));
        if (L.pin) cudaFreeHost(L.pin);
        L.pin = nullptr;
        L.pin_b = 0;
        FEMD_TRY_CUDA(cudaHostAlloc(&L.pin, 2 * need, cudaHostAllocDefault));
        L.pin_b = 2 * need;
    }
    return FEMD_OK;
}

// the table of the members `sel` (each member's entries together, its b0 / b1 within the table)
static int live_table(const LsLive &L, const std::vector<int> &sel, LBlock *T)
{
    int e = 0;
    for (int id : sel) {
        const int b0 = e, b1 = b0 + (int)L.ents[id].size();
        for (const auto &x : L.ents[id]) T[e++] = LBlock{id, x[0], x[1], b0, b1, x[2], x[3]};
    }
    return e;
}

static int ls_advance(femd_ctx ctx, femd_batch_s *B, bool mx, int chunks, int *nfin, int *fin_ids, femd_cg_result *fin_res)
{
    cudaStream_t s = ctx->stream;
    if (!B->live) B->live.reset(new LsLive());
    LsLive &L = *B->live;
    int st;
    *nfin = 0;
    // members armed since the last call join (a stagnated mixed member comes back in FP64)
    std::vector<int> fresh;
    size_t ntab = 0;
    if ((st = live_grow(B, L, 1))) return st;
    for (int id = 0; id < (int)B->mem.size(); ++id)
        if (B->mem[id] && B->mem[id]->armed && !L.in[id]) fresh.push_back(id);
    for (int id : L.ids) ntab += L.ents[id].size();
    for (int id : fresh) {
        Member &M = *B->mem[id];
        const bool m32 = mx && !M.force_fp64;
        if ((st = member_vectors(B, M, m32, B->ls_compact && !B->ls_windows))) return st;
        BProb d{};
        bool compact = false;
        if ((st = ls_member_setup(ctx, B, id, m32, d, L.ents[id], compact, L.maxwin))) return st;
        BProb *h = reinterpret_cast<BProb *>(L.pin);
        *h = d;
        FEMD_TRY_CUDA(cudaMemcpyAsync(L.d_desc.p + id, h, sizeof(BProb), cudaMemcpyHostToDevice, s));
        FEMD_TRY_CUDA(cudaMemsetAsync(L.d_state.p + id, 0, sizeof(LState), s));
        FEMD_TRY_CUDA(cudaStreamSynchronize(s));           // the staging slot is reused
        L.in[id] = 1;
        L.f64[id] = !m32;
        L.started[id] = 0;
        L.ids.push_back(id);
        ntab += L.ents[id].size();
    }
    if (L.ids.empty()) return FEMD_OK;
    FEMD_CHECK_ARG(ntab < (size_t)INT_MAX / 4, "batch: too many table entries");
    if ((st = live_grow(B, L, ntab + 1))) return st;
    LState *hs = reinterpret_cast<LState *>(static_cast<char *>(L.pin) + sizeof(BProb) + 64);
    LBlock *ht = reinterpret_cast<LBlock *>(hs + 2 * (size_t)L.cap);
    int *active = L.d_int.p, *ru_count = L.d_int.p + 1, *ru_list = L.d_int.p + 2;
    const int G1 = std::max(1, 8 * ctx->sm_count);
    const size_t win_b = (size_t)L.maxwin * sizeof(float);
    FEMD_TRY_CUDA(cudaFuncSetAttribute(k_ls_spmv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(CL_WIN_MAX * sizeof(float))));
    FEMD_TRY_CUDA(cudaMemsetAsync(L.d_int.p, 0, 2 * sizeof(int), s));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    FEMD_TRY_CUDA(cudaEventCreate(&t0));
    FEMD_TRY_CUDA(cudaEventCreate(&t1));
    struct EvG {
        cudaEvent_t a, b;
        ~EvG() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
    } evg{t0, t1};
    FEMD_TRY_CUDA(cudaEventRecord(t0, s));
    {
        // the layout of the members in flight (femd_cuda_batch_lockstep_stats)
        long long nc = 0;
        size_t ne = 0;
        for (int id : L.ids) {
            nc += B->mem[id]->f32_compact && !L.f64[id];
            ne += L.ents[id].size();
        }
        B->ls_stats[0] = nc;
        B->ls_stats[1] = (long long)L.ids.size() - nc;
        B->ls_stats[2] = L.maxwin;
        B->ls_stats[3] = (long long)ne;
    }
    // the start of the new members (r = b - A x, ||b||, z, the first direction's state)
    {
        std::vector<int> n32, n64;
        for (int id : L.ids)
            if (!L.started[id]) (L.f64[id] ? n64 : n32).push_back(id);
        const int NE32 = live_table(L, n32, ht), NE64 = live_table(L, n64, ht + NE32);
        if (NE32 + NE64) {
            FEMD_TRY_CUDA(cudaMemcpyAsync(L.d_tab.p, ht, (size_t)(NE32 + NE64) * sizeof(LBlock), cudaMemcpyHostToDevice, s));
            if (NE32)
                k_ls_resid<true, 0><<<NE32, LS_BB, 0, counted(s)>>>(L.d_desc.p, L.d_tab.p, NE32, L.d_state.p, L.d_part.p, active,
                                                                     ru_list, ru_count);
            if (NE64)
                k_ls_resid<false, 0><<<NE64, LS_BB, 0, counted(s)>>>(L.d_desc.p, L.d_tab.p + NE32, NE64, L.d_state.p, L.d_part.p,
                                                                      active, ru_list, ru_count);
            FEMD_TRY_CUDA(cudaGetLastError());
            FEMD_TRY_CUDA(cudaStreamSynchronize(s));       // the host table is rewritten below
        }
        for (int id : L.ids) L.started[id] = 1;
    }
    // chunks of iterations over the members in flight; the states are read after each chunk
    const int C = std::max(1, B->ls_chunk);
    // host buffers: the states after the previous chunk and after this one, two tables (an upload
    // may still be pending from one while the other is rewritten)
    LState *hsb[2] = {hs, hs + L.cap};
    LBlock *htb[2] = {reinterpret_cast<LBlock *>(hs + 2 * (size_t)L.cap), nullptr};
    htb[1] = htb[0] + L.tab_cap;
    auto enqueue_chunk = [&](int NE32, int NE64) {
        const LBlock *T32 = L.d_tab.p, *T64 = L.d_tab.p + NE32;
        for (int c = 0; c < C; ++c) {
            if (NE32) {
                k_ls_spmv<true><<<NE32, LS_BB, win_b, counted(s)>>>(L.d_desc.p, T32, NE32, L.d_state.p, L.d_part.p, active,
                                                                   ru_count);
                k_ls_update<true><<<NE32, LS_BB, 0, counted(s)>>>(L.d_desc.p, T32, NE32, L.d_state.p, L.d_part.p, active, ru_list,
                                                                 ru_count);
                k_ls_flush<false><<<std::min(G1, NE32), LS_BB, 0, counted(s)>>>(L.d_desc.p, T32, NE32, L.d_state.p, ru_list,
                                                                                ru_count);
                k_ls_resid<true, 1><<<std::min(G1, NE32), LS_BB, 0, counted(s)>>>(L.d_desc.p, T32, NE32, L.d_state.p, L.d_part.p,
                                                                                  active, ru_list, ru_count);
            }
            if (NE64) {
                k_ls_spmv<false><<<NE64, LS_BB, 0, counted(s)>>>(L.d_desc.p, T64, NE64, L.d_state.p, L.d_part.p, active, ru_count);
                k_ls_update<false><<<NE64, LS_BB, 0, counted(s)>>>(L.d_desc.p, T64, NE64, L.d_state.p, L.d_part.p, active, ru_list,
                                                                  ru_count);
            }
        }
    };
    // a chunk runs as one CUDA graph, captured again only when the table changes (the kernels read
    // the table from device memory, so a table of the same shape reuses the graph)
    auto launch_chunk = [&](int NE32, int NE64) -> cudaError_t {
        const bool same = L.gx && L.g_ne32 == NE32 && L.g_ne64 == NE64 && L.g_tab == L.d_tab.p && L.g_desc == L.d_desc.p &&
                          L.g_state == L.d_state.p && L.g_win == win_b && L.g_chunk == C;
        if (!same && !L.g_refused) {
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                enqueue_chunk(NE32, NE64);
                e = cudaStreamEndCapture(s, &g);
            }
            if (e == cudaSuccess && L.gx) {
                cudaGraphExecUpdateResultInfo info;
                if (cudaGraphExecUpdate(L.gx, g, &info) != cudaSuccess) {
                    cudaGetLastError();
                    cudaGraphExecDestroy(L.gx);
                    L.gx = nullptr;
                }
            }
            if (e == cudaSuccess && !L.gx) e = cudaGraphInstantiate(&L.gx, g, 0);
            if (e == cudaSuccess) cudaGraphGetNodes(g, nullptr, &L.g_nodes);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                // this runtime did not capture the chunk: direct launches from now on
                cudaGetLastError();
                if (L.gx) cudaGraphExecDestroy(L.gx);
                L.gx = nullptr;
                L.g_refused = true;
            } else {
                L.g_ne32 = NE32;
                L.g_ne64 = NE64;
                L.g_tab = L.d_tab.p;
                L.g_desc = L.d_desc.p;
                L.g_state = L.d_state.p;
                L.g_win = win_b;
                L.g_chunk = C;
            }
        }
        if (L.gx && !L.g_refused) return launch_graph(L.gx, L.g_nodes, s);
        enqueue_chunk(NE32, NE64);
        return cudaGetLastError();
    };
    // the table of the live members (their entries in admission order)
    auto build = [&](const LState *S, LBlock *T, int &NE32, int &NE64) {
        std::vector<int> l32, l64;
        for (int id : L.ids)
            if (!S[id].done) (L.f64[id] ? l64 : l32).push_back(id);
        NE32 = live_table(L, l32, T);
        NE64 = live_table(L, l64, T + NE32);
        return NE32 + NE64;
    };
    cudaEvent_t ev[2] = {nullptr, nullptr};
    FEMD_TRY_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    FEMD_TRY_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    struct EvG2 {
        cudaEvent_t *e;
        ~EvG2() { for (int k = 0; k < 2; ++k) if (e[k]) cudaEventDestroy(e[k]); }
    } evg2{ev};
    FEMD_TRY_CUDA(cudaMemcpyAsync(hsb[0], L.d_state.p, (size_t)L.cap * sizeof(LState), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    int tb = 0, NE32 = 0, NE64 = 0;
    int NE = build(hsb[0], htb[tb], NE32, NE64);
    if (NE) FEMD_TRY_CUDA(cudaMemcpyAsync(L.d_tab.p, htb[tb], (size_t)NE * sizeof(LBlock), cudaMemcpyHostToDevice, s));
    const int nchunks = std::max(1, chunks);
    for (int j = 0; j < nchunks && NE; ++j) {
        FEMD_TRY_CUDA(launch_chunk(NE32, NE64));
        FEMD_TRY_CUDA(cudaMemcpyAsync(hsb[j & 1], L.d_state.p, (size_t)L.cap * sizeof(LState), cudaMemcpyDeviceToHost, s));
        FEMD_TRY_CUDA(cudaEventRecord(ev[j & 1], s));
        if (j == 0) continue;
        // the states after the previous chunk (this one stays queued behind them)
        FEMD_TRY_CUDA(cudaEventSynchronize(ev[(j - 1) & 1]));
        const LState *S = hsb[(j - 1) & 1];
        int live_e = 0, live = 0;
        for (int id : L.ids)
            if (!S[id].done) { ++live; live_e += (int)L.ents[id].size(); }
        if (live == 0 || *(volatile int *)B->abort_host) break;
        if (live_e <= (NE * 7) / 10) {
            // compact the table to the live members (uploaded behind the queued chunk)
            tb ^= 1;
            NE = build(S, htb[tb], NE32, NE64);
            FEMD_TRY_CUDA(cudaMemcpyAsync(L.d_tab.p, htb[tb], (size_t)NE * sizeof(LBlock), cudaMemcpyHostToDevice, s));
        }
    }
    FEMD_TRY_CUDA(cudaMemcpyAsync(hs, L.d_state.p, (size_t)L.cap * sizeof(LState), cudaMemcpyDeviceToHost, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));                // hs: the states after the last chunk
    ht = htb[tb ^ 1];                                       // free for the finishing table below
    // the members that are done: the end of their solve (the final true residual in FP64, the
    // flush of a mixed member that broke down, x = 0 for b = 0), then their results
    std::vector<int> d32, d64, back, keep;
    for (int id : L.ids) {
        const LState &S = hs[id];
        if (!S.done) { keep.push_back(id); continue; }
        Member &M = *B->mem[id];
        if (!L.f64[id] && S.fallback) {
            // the FP32 recurrence stagnated: FP64 from this iterate at the next call
            M.force_fp64 = true;
            M.prior_its += S.it;
            M.prior_rus += S.rus;
            M.max_iter = std::max(1, M.max_iter - S.it);
            back.push_back(id);
            continue;
        }
        (L.f64[id] ? d64 : d32).push_back(id);
    }
    const int FE32 = live_table(L, d32, ht), FE64 = live_table(L, d64, ht + FE32);
    if (FE32 + FE64) {
        FEMD_TRY_CUDA(cudaMemcpyAsync(L.d_tab.p, ht, (size_t)(FE32 + FE64) * sizeof(LBlock), cudaMemcpyHostToDevice, s));
        if (FE32)
            k_ls_flush<true><<<std::min(G1, FE32), LS_BB, 0, counted(s)>>>(L.d_desc.p, L.d_tab.p, FE32, L.d_state.p, ru_list,
                                                                           ru_count);
        if (FE64)
            k_ls_resid<false, 2><<<FE64, LS_BB, 0, counted(s)>>>(L.d_desc.p, L.d_tab.p + FE32, FE64, L.d_state.p, L.d_part.p,
                                                                  active, ru_list, ru_count);
        k_ls_zero<<<FE32 + FE64, LS_BB, 0, counted(s)>>>(L.d_desc.p, L.d_tab.p, L.d_state.p);
        FEMD_TRY_CUDA(cudaGetLastError());
        FEMD_TRY_CUDA(cudaMemcpyAsync(hs, L.d_state.p, (size_t)L.cap * sizeof(LState), cudaMemcpyDeviceToHost, s));
    }
    FEMD_TRY_CUDA(cudaEventRecord(t1, s));
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    int nf = 0;
    for (const auto *set : {&d32, &d64})
        for (int id : *set) {
            Member &M = *B->mem[id];
            if (fin_res) ls_result(M, hs[id], fin_res[nf], ms * 1e-3);
            if (fin_ids) fin_ids[nf] = id;
            ++nf;
            M.armed = false;
            L.in[id] = 0;
        }
    for (int id : back) L.in[id] = 0;                       // re-admitted (FP64) at the next call
    L.ids = keep;
    *nfin = nf;
    if (*(volatile int *)B->abort_host) { set_error("batch: aborted by the host"); return FEMD_EABORT; }
    return FEMD_OK;
}

extern "C" {

int femd_cuda_batch_create(femd_ctx ctx, int nprob, const femd_matrix *mats, int nnz_per_block, femd_batch *out)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && out && nprob >= 0 && (mats || nprob == 0), "batch_create: bad arguments");
    *out = nullptr;
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    auto B = new femd_batch_s();
    std::unique_ptr<femd_batch_s> guard(B);
    B->ctx = ctx;
    ctx_retain(ctx);
    B->nnz_per_block = nnz_per_block > 0 ? nnz_per_block : 65536;
    int st;
    if ((st = B->d_queue.alloc(1)) || (st = B->d_scratch.alloc(4))) return st;
    FEMD_TRY_CUDA(cudaHostAlloc(&B->abort_host, sizeof(int), cudaHostAllocMapped));
    *B->abort_host = 0;
    FEMD_TRY_CUDA(cudaHostGetDevicePointer(&B->abort_dev, B->abort_host, 0));
    if ((st = grow_arrays(B, std::max(nprob, 4)))) return st;
    if ((st = batch_shape(B))) return st;
    for (int p = 0; p < nprob; ++p) {
        int id = -1;
        if ((st = add_member(B, mats[p], &id))) return st;
    }
    *out = reinterpret_cast<femd_batch>(guard.release());
    return FEMD_OK;
}

int femd_cuda_batch_add(femd_batch handle, femd_matrix K, int *id_out)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B && id_out, "batch_add: bad arguments");
    FEMD_TRY_CUDA(cudaSetDevice(B->ctx->device));
    return add_member(B, K, id_out);
}

int femd_cuda_batch_remove(femd_batch handle, int id)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B && id >= 0 && id < (int)B->mem.size() && B->mem[id], "batch_remove: no such member");
    if (B->live && id < (int)B->live->in.size() && B->live->in[id]) {
        // a member in flight in the continuous lockstep engine leaves it (its solve is dropped)
        FEMD_TRY_CUDA(cudaStreamSynchronize(B->ctx->stream));
        auto &ids = B->live->ids;
        ids.erase(std::remove(ids.begin(), ids.end(), id), ids.end());
        B->live->in[id] = 0;
    }
    B->free_vectors(*B->mem[id]);
    B->mem[id].reset();
    return FEMD_OK;
}

int femd_cuda_batch_arm(femd_batch handle, int id, const double *b_dev, double *x_dev, int max_iter, double tol)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_arm: not a batch handle");
    return arm_member(B, id, b_dev, x_dev, max_iter, tol);
}

int femd_cuda_batch_step(femd_ctx ctx, femd_batch handle, int iters, int mixed, int *nfinished, int *finished_ids,
                         femd_cg_result *finished)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(ctx && B && ctx == B->ctx, "batch_step: bad arguments");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    return batch_step(ctx, B, iters, mixed != 0, nfinished, finished_ids, finished, nullptr);
}

int femd_cuda_batch_step_lockstep(femd_ctx ctx, femd_batch handle, int mixed, int *nfinished, int *finished_ids,
                                  femd_cg_result *finished)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(ctx && B && ctx == B->ctx, "batch_step_lockstep: bad arguments");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    if (nfinished) *nfinished = 0;
    std::vector<int> ids;
    for (int id = 0; id < (int)B->mem.size(); ++id)
        if (B->mem[id] && B->mem[id]->armed) ids.push_back(id);
    if (ids.empty()) return FEMD_OK;
    std::vector<femd_cg_result> res(ids.size());
    const int st = ls_solve(ctx, B, ids, mixed != 0, res.data());
    if (st && st != FEMD_EABORT && st != FEMD_ETIMEOUT) return st;
    for (size_t p = 0; p < ids.size(); ++p) {
        B->mem[ids[p]]->armed = false;
        if (finished_ids) finished_ids[p] = ids[p];
        if (finished) finished[p] = res[p];
    }
    if (nfinished) *nfinished = (int)ids.size();
    return st;
}

int femd_cuda_batch_advance_lockstep(femd_ctx ctx, femd_batch handle, int mixed, int chunks, int *nfinished,
                                     int *finished_ids, femd_cg_result *finished)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(ctx && B && ctx == B->ctx && chunks >= 1, "batch_advance_lockstep: bad arguments");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    *(volatile int *)B->abort_host = 0;
    int nf = 0;
    const int st = ls_advance(ctx, B, mixed != 0, chunks, &nf, finished_ids, finished);
    if (nfinished) *nfinished = nf;
    return st;
}

int femd_cuda_batch_configure(femd_batch handle, int block, int nnz_per_block, int nnz_per_thread)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_configure: not a batch handle");
    FEMD_CHECK_ARG(block == 128 || block == 256 || block == 512, "batch_configure: block is 128, 256 or 512");
    FEMD_CHECK_ARG(nnz_per_block >= 256, "batch_configure: nnz_per_block < 256");
    FEMD_CHECK_ARG(nnz_per_thread == 2 || nnz_per_thread == 4 || nnz_per_thread == 8,
                   "batch_configure: nnz_per_thread is 2, 4 or 8");
    FEMD_CHECK_ARG(block * nnz_per_thread <= 1024, "batch_configure: block x nnz_per_thread > 1024 is not built");
    for (const auto &M : B->mem)
        FEMD_CHECK_ARG(!M || !M->armed, "batch_configure: a solve is in progress");
    FEMD_TRY_CUDA(cudaSetDevice(B->ctx->device));
    const int ob = B->block, on = B->nnz_per_block, ot = B->npt;
    B->block = block;
    B->nnz_per_block = nnz_per_block;
    B->npt = nnz_per_thread;
    int st = batch_shape(B);
    if (st) {
        B->block = ob;
        B->nnz_per_block = on;
        B->npt = ot;
        batch_shape(B);
    }
    return st;
}

int femd_cuda_batch_params(femd_batch handle, int *block, int *nnz_per_block, int *nnz_per_thread, int *graph)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_params: not a batch handle");
    if (block) *block = B->block;
    if (nnz_per_block) *nnz_per_block = B->nnz_per_block;
    if (nnz_per_thread) *nnz_per_thread = B->npt;
    if (graph) *graph = std::max(B->graph_state[0], B->graph_state[1]);
    return FEMD_OK;
}

int femd_cuda_batch_solve(femd_ctx ctx, femd_batch handle, const double *const *b_dev, double *const *x_dev, int max_iter,
                          double tol, int mixed, femd_cg_result *results)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(ctx && B && b_dev && x_dev && results && ctx == B->ctx, "batch_solve: bad arguments");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    std::vector<int> ids;
    for (int id = 0; id < (int)B->mem.size(); ++id)
        if (B->mem[id]) ids.push_back(id);
    int st;
    for (size_t p = 0; p < ids.size(); ++p)
        if ((st = arm_member(B, ids[p], b_dev[p], x_dev[p], max_iter, tol))) return st;
    std::vector<int> fin(ids.size());
    std::vector<femd_cg_result> fr(ids.size());
    int nf = 0;
    double sec = 0.0;
    st = batch_step(ctx, B, INT_MAX, mixed != 0, &nf, fin.data(), fr.data(), &sec);
    for (size_t p = 0; p < ids.size(); ++p) {
        fill_member(B, ids[p], results[p], sec);
        if (B->h_qout->flag) results[p].status = B->h_qout->flag;
        B->mem[ids[p]]->armed = false;
    }
    return st;
}

int femd_cuda_batch_solve_lockstep(femd_ctx ctx, femd_batch handle, const double *const *b_dev, double *const *x_dev,
                                   int max_iter, double tol, int mixed, femd_cg_result *results)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(ctx && B && b_dev && x_dev && results && ctx == B->ctx, "batch_solve_lockstep: bad arguments");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    std::vector<int> ids;
    for (int id = 0; id < (int)B->mem.size(); ++id)
        if (B->mem[id]) ids.push_back(id);
    int st;
    for (size_t p = 0; p < ids.size(); ++p)
        if ((st = arm_member(B, ids[p], b_dev[p], x_dev[p], max_iter, tol))) return st;
    st = ls_solve(ctx, B, ids, mixed != 0, results);
    for (int id : ids) B->mem[id]->armed = false;
    return st;
}

int femd_cuda_batch_lockstep_configure(femd_batch handle, int nnz_per_entry, int chunk, int windows, int compact)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_lockstep_configure: bad handle");
    FEMD_CHECK_ARG(nnz_per_entry >= 0 && chunk >= 0 && windows >= -1 && windows <= 1 && compact >= -1 && compact <= 1,
                   "batch_lockstep_configure: bad argument");
    if (nnz_per_entry) B->ls_nnz = nnz_per_entry;
    if (chunk) B->ls_chunk = chunk;
    if (windows >= 0) B->ls_windows = windows != 0;
    if (compact >= 0) B->ls_compact = compact != 0;
    return FEMD_OK;
}

int femd_cuda_batch_tune(femd_ctx ctx, femd_batch handle, const double *const *b_dev, double *const *x_dev, int max_iter,
                         double tol, int mixed, int *best_out, double *seconds_out)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(ctx && B && b_dev && x_dev, "batch_tune: NULL argument");
    std::vector<int> ids;
    for (int id = 0; id < (int)B->mem.size(); ++id)
        if (B->mem[id]) ids.push_back(id);
    std::vector<femd_cg_result> res(ids.size() + 1);
    auto run = [&](int blk, int npb, int npt, double *sec) -> int {
        if (blk * npt > 1024) { *sec = 1e300; return FEMD_OK; }   // not built
        int st = femd_cuda_batch_configure(handle, blk, npb, npt);
        if (st) return st;
        double best = 1e300;
        for (int rep = 0; rep < 2; ++rep) {
            for (size_t p = 0; p < ids.size(); ++p)
                FEMD_TRY_CUDA(cudaMemsetAsync(x_dev[p], 0, (size_t)B->mem[ids[p]]->n * sizeof(double), ctx->stream));
            st = femd_cuda_batch_solve(ctx, handle, b_dev, x_dev, max_iter, tol, mixed, res.data());
            if (st) return st;
            best = std::min(best, res[0].seconds);
        }
        *sec = best;
        return FEMD_OK;
    };
    // coordinate descent over nonzeros per rank, threads per block and nonzeros per thread
    static const int NPB[] = {8192, 16384, 32768, 65536, 131072};
    static const int BLK[] = {128, 256, 512};
    static const int NPT[] = {2, 4, 8};
    int cb = 256, cn = 65536, ct = 4;
    double tbest = 1e300;
    int st;
    if ((st = run(cb, cn, ct, &tbest))) return st;
    for (int pass = 0; pass < 2; ++pass) {
        for (int v : NPB) {
            if (v == cn) continue;
            double t;
            if ((st = run(cb, v, ct, &t))) return st;
            if (t < tbest) { tbest = t; cn = v; }
        }
        if (pass == 1) break;
        for (int v : BLK) {
            if (v == cb) continue;
            double t;
            if ((st = run(v, cn, ct, &t))) return st;
            if (t < tbest) { tbest = t; cb = v; }
        }
        for (int v : NPT) {
            if (v == ct) continue;
            double t;
            if ((st = run(cb, cn, v, &t))) return st;
            if (t < tbest) { tbest = t; ct = v; }
        }
    }
    if ((st = femd_cuda_batch_configure(handle, cb, cn, ct))) return st;
    if (best_out) { best_out[0] = cb; best_out[1] = cn; best_out[2] = ct; }
    if (seconds_out) *seconds_out = tbest;
    return FEMD_OK;
}

int femd_cuda_pattern_batch_layout(femd_ctx ctx, femd_pattern p, int *bandwidth)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && p && p->kind == KIND_PATTERN, "pattern_batch_layout: NULL argument or not a pattern");
    FEMD_CHECK_ARG(p->nrows == p->ncols, "pattern_batch_layout: the pattern must be square");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    FEMD_TRY(build_compact(ctx, p));
    if (bandwidth) *bandwidth = p->cl_state == 1 ? p->cl_bw : -1;
    return FEMD_OK;
}

int femd_cuda_batch_lockstep_stats(femd_batch handle, long long *out)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B && out, "batch_lockstep_stats: bad arguments");
    for (int k = 0; k < 4; ++k) out[k] = B->ls_stats[k];
    return FEMD_OK;
}

int femd_cuda_batch_abort(femd_batch handle)
{
    femd_batch_s *B = as_batch(handle);
    if (!B || !B->abort_host) return FEMD_EINVAL;
    *(volatile int *)B->abort_host = 1;
    return FEMD_OK;
}

int femd_cuda_batch_profile(femd_batch handle, long long *cycles_out)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B && cycles_out && B->h_qout, "batch_profile: bad arguments");
    cycles_out[0] = (long long)B->h_qout->block_cycles;
    cycles_out[1] = (long long)B->h_qout->team_wait_cycles;
    cycles_out[2] = (long long)B->h_qout->chunk_sync_cycles;
    cycles_out[3] = B->h_qout->fail_where;
    cycles_out[4] = B->h_qout->fail_at;
    cycles_out[5] = B->h_qout->fail_team;
    cycles_out[6] = B->h_qout->fail_rank;
    return FEMD_OK;
}

int femd_cuda_batch_debug(femd_batch handle, int ghost_member, long long spin_limit)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_debug: not a batch handle");
    FEMD_CHECK_ARG(ghost_member < (int)B->mem.size(), "batch_debug: member index out of range");
    B->ghost = ghost_member;
    B->spin_limit = spin_limit > 0 ? spin_limit : SPIN_LIMIT;
    return FEMD_OK;
}

int femd_cuda_batch_info(femd_batch handle, int *nprob, int *grid, int *nslots, int *team_out)
{
    clear_error();
    femd_batch_s *B = as_batch(handle);
    FEMD_CHECK_ARG(B, "batch_info: not a batch handle");
    int np = 0, ns = 0;
    for (const auto &M : B->mem)
        if (M) {
            if (team_out) team_out[np] = M->team;
            ++np;
            ns += M->team;
        }
    if (nprob) *nprob = np;
    if (grid) *grid = B->grid;
    if (nslots) *nslots = ns;
    return FEMD_OK;
}

}  // extern "C"
