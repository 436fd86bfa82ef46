// core.cu -- contexts, handles, error text, device status words and the integer scan used by
// the pattern builder.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"

namespace femd {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void set_error(const std::string &msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
void add_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ---- device memory: one stream-ordered pool per device -----------------------------------
// A plain cudaMalloc of a few MB or more takes about 0.4 ms on a B200 and cudaFree 0.3 ms (it
// unmaps the memory and waits for the device), which made the allocations of a pattern build cost
// ten times its kernels. The pool maps memory once and keeps up to POOL_KEEP bytes of freed blocks
// for reuse. Allocations are ordered on the pool's own stream and waited for before they are
// returned, so the caller may use them on any stream; a free first waits for the device, as cudaFree
// does, so no kernel still reading the block sees it handed out again.
static constexpr uint64_t POOL_KEEP = 2ull << 30;
static constexpr int POOL_DEVICES = 64;
struct DevicePool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t s = nullptr;
};
static std::mutex g_pool_mu;
static DevicePool g_pools[POOL_DEVICES];

static cudaError_t device_pool(int dev, DevicePool **out)
{
    if (dev < 0 || dev >= POOL_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    DevicePool &P = g_pools[dev];
    if (!P.pool) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = POOL_KEEP;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        cudaStream_t s = nullptr;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        P.pool = pool;
        P.s = s;
    }
    *out = &P;
    return cudaSuccess;
}

cudaError_t dev_alloc(void **p, size_t bytes)
{
    *p = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    DevicePool *P = nullptr;
    if (e == cudaSuccess) e = device_pool(dev, &P);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync(p, bytes, P->pool, P->s);
    if (e == cudaErrorMemoryAllocation) {
        // give the pool's idle blocks back to the device and try once more
        cudaGetLastError();
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(P->pool, 0);
        e = cudaMallocFromPoolAsync(p, bytes, P->pool, P->s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(P->s);
    if (e != cudaSuccess) {
        if (*p) cudaFreeAsync(*p, P->s);
        *p = nullptr;
        cudaGetLastError();
    }
    return e;
}

void dev_free(void *p)
{
    if (!p) return;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    const int dev = attr.device;
    DevicePool *P = nullptr;
    if (device_pool(dev, &P) != cudaSuccess) return;
    if (dev != cur) cudaSetDevice(dev);
    cudaDeviceSynchronize();
    cudaFreeAsync(p, P->s);
    if (dev != cur) cudaSetDevice(cur);
}

// ---- exclusive scan of int32 (three phases: tile scans, scan of tile sums, add) ------------
static constexpr int SCAN_THREADS = 512;
static constexpr int SCAN_ITEMS = 8;
static constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const int *__restrict__ in, int *__restrict__ out,
                                                            size_t n, int *__restrict__ tile_sums)
{
    __shared__ int warp_tot[SCAN_THREADS / 32];
    const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int run = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const size_t g = base + i;
        const int x = g < n ? in[g] : 0;
        v[i] = run;
        run += x;
    }
    // inclusive warp scan of the per-thread totals
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int w = lane < SCAN_THREADS / 32 ? warp_tot[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < SCAN_THREADS / 32) warp_tot[lane] = wi - w;   // exclusive warp offsets
        if (lane == SCAN_THREADS / 32 - 1 && tile_sums) tile_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    const int off = warp_tot[wid] + inc - run;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const size_t g = base + i;
        if (g < n) out[g] = v[i] + off;
    }
}

__global__ void k_scan_add(int *__restrict__ out, size_t n, const int *__restrict__ tile_off)
{
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) out[g] += tile_off[g / SCAN_TILE];
}

size_t scan_tmp_ints(size_t n)
{
    size_t total = 0;
    size_t m = n;
    while (m > (size_t)SCAN_TILE) {
        m = (m + SCAN_TILE - 1) / SCAN_TILE;
        total += m + 1;
    }
    return total + 1;
}

int exclusive_scan_int(const int *in, int *out, size_t n, int *tmp, cudaStream_t s)
{
    if (n == 0) return FEMD_OK;
    const size_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles == 1) {
        k_scan_tiles<<<1, SCAN_THREADS, 0, counted(s)>>>(in, out, n, nullptr);
        FEMD_TRY_CUDA(cudaGetLastError());
        return FEMD_OK;
    }
    int *sums = tmp;
    k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, counted(s)>>>(in, out, n, sums);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY(exclusive_scan_int(sums, sums, tiles, tmp + tiles + 1, s));
    k_scan_add<<<grid_for(n, 256), 256, 0, counted(s)>>>(out, n, sums);
    FEMD_TRY_CUDA(cudaGetLastError());
    return FEMD_OK;
}

int read_status(femd_ctx ctx, int *flags, int *bad_row)
{
    FEMD_TRY_CUDA(cudaMemcpyAsync(ctx->status_host, ctx->status_dev, 4 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    FEMD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    if (flags) *flags = ctx->status_host[0];
    if (bad_row) *bad_row = ctx->status_host[1];
    return FEMD_OK;
}

__global__ void k_reset_status(int *st)
{
    if (threadIdx.x < 4) st[threadIdx.x] = threadIdx.x == 1 ? 0x7fffffff : 0;
}

int reset_status(femd_ctx ctx)
{
    k_reset_status<<<1, 32, 0, counted(ctx->stream)>>>(ctx->status_dev);
    FEMD_TRY_CUDA(cudaGetLastError());
    return FEMD_OK;
}

}  // namespace femd

using namespace femd;

namespace femd {
void ctx_retain(femd_ctx ctx)
{
    if (ctx) ctx->refs.fetch_add(1);
}

void ctx_release(femd_ctx ctx)
{
    if (!ctx || ctx->refs.fetch_sub(1) != 1) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->status_dev);
    cudaFreeHost(ctx->status_host);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}
}  // namespace femd

extern "C" {

const char *femd_cuda_last_error(void) { return g_last_error.c_str(); }

const char *femd_cuda_version(void) { return "femd_b200 0.1 (sm_100a)"; }

long long femd_cuda_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int femd_cuda_ctx_create(int device, femd_ctx *out)
{
    clear_error();
    FEMD_CHECK_ARG(out != nullptr, "femd_cuda_ctx_create: out is NULL");
    *out = nullptr;
    int dev = device;
    if (dev < 0) FEMD_TRY_CUDA(cudaGetDevice(&dev));
    FEMD_TRY_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    FEMD_TRY_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) {
        set_error(std::string("femd_b200 needs an sm_100a device (B200); device ") + std::to_string(dev) + " is sm_" +
                  std::to_string(prop.major) + std::to_string(prop.minor));
        return FEMD_ECUDA;
    }
    femd_ctx c = new femd_ctx_s();
    c->device = dev;
    c->sm_count = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->status_dev, 4 * sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&c->status_host, 4 * sizeof(int));
    if (e != cudaSuccess) {
        set_error(std::string("femd_cuda_ctx_create: ") + cudaGetErrorString(e));
        if (c->status_dev) cudaFree(c->status_dev);
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return FEMD_ECUDA;
    }
    femd::reset_status(c);
    *out = c;
    return FEMD_OK;
}

int femd_cuda_ctx_destroy(femd_ctx ctx)
{
    femd::ctx_release(ctx);
    return FEMD_OK;
}

void *femd_cuda_ctx_stream(femd_ctx ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int femd_cuda_ctx_sync(femd_ctx ctx)
{
    clear_error();
    FEMD_CHECK_ARG(ctx != nullptr, "femd_cuda_ctx_sync: ctx is NULL");
    FEMD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return FEMD_OK;
}

void femd_cuda_release(void *handle)
{
    if (!handle) return;
    HandleBase *h = static_cast<HandleBase *>(handle);
    if (h->kind == KIND_PATTERN || h->kind == KIND_MATRIX || h->kind == KIND_SOLVER || h->kind == KIND_BATCH ||
        h->kind == KIND_FACETS || h->kind == KIND_PRECOND) {
        h->kind = 0;
        delete h;
    }
}

}  // extern "C"
