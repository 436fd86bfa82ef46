// common.cuh -- shared definitions of libfemd_cuda: handles, error handling, scans,
// warp reductions.  Internal header (not installed).
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/femd_cuda.h"

namespace femd {

// ---- errors -------------------------------------------------------------------------------
void set_error(const std::string &msg);
void clear_error();

#define FEMD_TRY_CUDA(expr)                                                                      \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            ::femd::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));               \
            return e_ == cudaErrorMemoryAllocation ? FEMD_ENOMEM : FEMD_ECUDA;                   \
        }                                                                                        \
    } while (0)

#define FEMD_CHECK_ARG(cond, msg)                                                                \
    do {                                                                                         \
        if (!(cond)) { ::femd::set_error(msg); return FEMD_EINVAL; }                             \
    } while (0)

#define FEMD_TRY(expr)                                                                           \
    do {                                                                                         \
        int s_ = (expr);                                                                         \
        if (s_ != FEMD_OK) return s_;                                                            \
    } while (0)

// ---- handles ------------------------------------------------------------------------------
enum HandleKind : uint32_t { KIND_PATTERN = 0x50415454u, KIND_MATRIX = 0x4d415452u, KIND_SOLVER = 0x534f4c56u,
                             KIND_BATCH = 0x42415443u, KIND_FACETS = 0x46414354u,
                             KIND_PRECOND = 0x50524543u };

struct HandleBase {
    uint32_t kind;
    explicit HandleBase(uint32_t k) : kind(k) {}
    virtual ~HandleBase() {}
};

// Device memory of the library: a stream-ordered pool per device (core.cu). dev_alloc returns
// memory that any stream may use as soon as it returns; dev_free first waits for the device, as
// cudaFree does, then hands the block back to the pool, which keeps a bounded amount of freed
// memory for the next allocation instead of unmapping it.
cudaError_t dev_alloc(void **p, size_t bytes);
void dev_free(void *p);

// A device buffer owned by a handle.
template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    int alloc(size_t count)
    {
        release();
        if (count == 0) return FEMD_OK;
        void *q = nullptr;
        cudaError_t e = dev_alloc(&q, count * sizeof(T));
        if (e != cudaSuccess) {
            set_error(std::string("device allocation of ") + std::to_string(count * sizeof(T)) + " bytes: " +
                      cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? FEMD_ENOMEM : FEMD_ECUDA;
        }
        p = static_cast<T *>(q);
        n = count;
        return FEMD_OK;
    }
    void release()
    {
        if (p) dev_free(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

struct Workspace;

}  // namespace femd

struct femd_ctx_s {
    // handles that keep the context (patterns, matrices, batches) hold a reference each;
    // femd_cuda_ctx_destroy drops the creator's, and the last one frees the stream
    std::atomic<int> refs{1};
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    // a small device status block: [0] error flags, [1] first bad row, [2..] spare
    int *status_dev = nullptr;
    int *status_host = nullptr;   // pinned
};

namespace femd {
void ctx_retain(femd_ctx ctx);
void ctx_release(femd_ctx ctx);
// the preconditioners of precond.cu: z = M^{-1} r enqueued on s (skipped when *skip is set)
int precond_enqueue(femd_precond P, const double *r, double *z, const int *skip, cudaStream_t s);
int precond_rows(femd_precond P);
// The FP32 copy of a matrix in row-sum form (the mixed-precision inner iteration): position q of
// the original CSR goes to a32[dst ? dst[q] : q] as (float) a[q], except each row's diagonal
// position, which takes (float) of the row's FP64 sum.  Needs every diagonal position.
int f32_rowsum_copy(femd_pattern P, const double *a, const int *dst, float *a32, cudaStream_t s);
femd_ctx precond_ctx(femd_precond P);
femd_pattern precond_pattern(femd_precond P);
}  // namespace femd

struct femd_pattern_s : femd::HandleBase {
    femd_ctx ctx = nullptr;
    int nrows = 0, ncols = 0, ncells = 0, nloc = 0;
    long long nnz = 0;
    femd::DevBuf<int> indptr, indices;
    femd::DevBuf<int> cell_dofs;       // ncells x nloc (copy)
    femd::DevBuf<int> rc_ptr, rc_code; // row -> (cell nloc + local), increasing cell order
    femd::DevBuf<int> map;             // scatter map, ne nloc^2 (built on demand)
    femd::DevBuf<int> diag_pos;        // position of (i, i), -1 when absent
    bool all_diag = false;             // every row i holds the position (i, i)
    int max_row_cells = 0, max_row_len = 0;
    // assembly workspace, grown on demand and reused across calls (no allocation per call
    // once it has its size): per-element factors, the rule's tables
    femd::DevBuf<double> ws_factors;
    // the rule's tables (weights, points, reference values, the pair tensors) of the last few
    // forms, each with the host copy it was uploaded from: a repeated assembly of the same form
    // uploads nothing (a pageable upload can wait for the stream)
    struct TableSlot {
        femd::DevBuf<double> dev;
        std::vector<double> host;
        unsigned long long used = 0;
    };
    static constexpr int TABLE_SLOTS = 4;
    TableSlot tables[TABLE_SLOTS];
    unsigned long long table_clock = 0;
    // for every (row, cell) pair of the rc lists, the offsets within the row of the cell's nloc
    // columns (uint8, 255 = constrained): the scatter map in the rows' own order, a quarter of
    // its size (built on the first FAST assembly when every row is shorter than 255)
    femd::DevBuf<unsigned char> pair_off;
    // the batched engine's compact layout of the pattern, built on first use: a reverse
    // Cuthill-McKee order with the rows of every 256 sorted by length (iperm: original row ->
    // reordered row); the entries in slices of 32 reordered rows, column-major within a slice
    // and padded to its longest row (cl_indptr: each reordered row's first position, entry j at
    // + 32 j; row n: the total); every entry's column as a 16-bit offset from its (reordered)
    // row (padding: 0), and for every original entry its position; per slice the smallest and
    // largest column.  cl_state: 0 not built, 1 built, -1 unsuitable (a column offset over 32767)
    int cl_state = 0, cl_bw = 0;
    long long cl_nsell = 0;            // entries of the sliced layout, padding included
    femd::DevBuf<int> cl_iperm, cl_indptr, cl_dst;
    femd::DevBuf<short> cl_off;
    std::vector<int> cl_tile_lo, cl_tile_hi;
    femd_pattern_s() : HandleBase(femd::KIND_PATTERN) {}
    ~femd_pattern_s() override { femd::ctx_release(ctx); }
};

struct femd_matrix_s : femd::HandleBase {
    femd_ctx ctx = nullptr;
    femd_pattern pattern = nullptr;
    femd::DevBuf<double> data, inv;
    femd::DevBuf<float> data32, inv32;   // FP32 copies (mixed precision), built on demand
    bool f32_valid = false;
    // the inverse diagonal has been written (assembly with want_inv, femd_cuda_matrix_jacobi,
    // femd_cuda_matrix_set_inv_diag, or the host upload of femd_cuda_cg_solve_host); until then
    // every preconditioned solve refuses the matrix instead of reading uninitialised memory
    bool inv_valid = false;
    int spmv_tpr = 0;                    // autotuned threads per row (0: not tuned)
    // the solver workspace of this matrix (vectors, pinned state, captured CUDA graphs), kept
    // between solves so that a solve allocates nothing once it has run once
    void *solver_ws = nullptr;
    void (*solver_ws_free)(void *) = nullptr;
    femd_matrix_s() : HandleBase(femd::KIND_MATRIX) {}
    ~femd_matrix_s() override
    {
        if (solver_ws_free) solver_ws_free(solver_ws);
        femd::ctx_release(ctx);
    }
};

namespace femd {

// ---- small device helpers -----------------------------------------------------------------
template <class T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// exclusive scan of n ints in place on the stream; n+1 entries are written when total is
// requested (out[n] = total).  Uses tmp (device) of scan_tmp_size(n) ints.
size_t scan_tmp_ints(size_t n);
int exclusive_scan_int(const int *in, int *out, size_t n, int *tmp, cudaStream_t s);

// Kernel launches issued by this library in this process (graph launches count their nodes).
void add_launches(long long n);
// The launch-configuration stream argument of every kernel launch goes through counted(): it
// counts the launch (unless the stream is being captured into a graph) and returns the stream.
inline cudaStream_t counted(cudaStream_t s)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    if (cs == cudaStreamCaptureStatusNone) add_launches(1);
    return s;
}
// Launch an instantiated graph and count its kernel nodes.
inline cudaError_t launch_graph(cudaGraphExec_t exec, size_t nodes, cudaStream_t s)
{
    const cudaError_t e = cudaGraphLaunch(exec, s);
    if (e == cudaSuccess) add_launches((long long)nodes);
    return e;
}

inline unsigned grid_for(size_t work, unsigned block, unsigned cap = 1u << 30)
{
    size_t g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// status flags written by kernels into ctx->status_dev[0]
enum StatusFlag : int { ST_OUTSIDE = 1, ST_ZERODIAG = 2, ST_ROW_TOO_LONG = 4, ST_TIMEOUT = 8, ST_ABORT = 16 };

int read_status(femd_ctx ctx, int *flags, int *bad_row);
int reset_status(femd_ctx ctx);

}  // namespace femd
