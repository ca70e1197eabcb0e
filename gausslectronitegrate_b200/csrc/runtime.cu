// Runtime plumbing: per-thread error status, the device context with its
// non-blocking stream and pooled stream-ordered allocations, and a three-phase
// exclusive prefix sum used by the enumeration and key-compaction kernels.
#include <stdarg.h>
#include <string.h>

#include "gli_internal.cuh"

namespace gli {

static thread_local int t_status = GLI_OK;
static thread_local char t_message[512] = "";
static thread_local int t_device = 0;

void set_error(int code, const char* fmt, ...) {
    t_status = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_message, sizeof(t_message), fmt, ap);
    va_end(ap);
}

void clear_error() {
    t_status = GLI_OK;
    t_message[0] = 0;
}

int last_error() { return t_status; }

void fail(int code, const char* fmt, ...) {
    t_status = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_message, sizeof(t_message), fmt, ap);
    va_end(ap);
    throw Failure{code};
}

const char* last_message() { return t_message; }

static thread_local long long t_launches = 0;
void count_launch() { ++t_launches; }
long long launch_count() { return t_launches; }
void add_launches(long long n) { t_launches += n; }

int set_device(int ordinal) {
    t_device = ordinal;
    return GLI_OK;
}

// One context per (thread, device): the stream is created on first use and the
// device's default memory pool keeps freed blocks cached for later calls.
Context& context() {
    static thread_local Context ctx[16];
    static thread_local bool ready[16] = {false};
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        fail(GLI_ERR_NO_DEVICE, "no CUDA device available (%s)",
             e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
    }
    if (t_device < 0 || t_device >= count || t_device >= 16)
        fail(GLI_ERR_ARGUMENT, "device ordinal %d out of range (%d devices)", t_device, count);
    GLI_CUDA(cudaSetDevice(t_device));
    Context& c = ctx[t_device];
    if (!ready[t_device]) {
        c.device = t_device;
        GLI_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        GLI_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, t_device));
        cudaMemPool_t pool;
        GLI_CUDA(cudaDeviceGetDefaultMemPool(&pool, t_device));
        uint64_t keep = UINT64_MAX;
        GLI_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        ready[t_device] = true;
    }
    return c;
}

GridDesc grid_desc(const struct cartesian_grid_3d* g) {
    GridDesc d;
    for (int a = 0; a < 3; ++a) {
        d.istart[a] = g->coord_range[a].istart;
        d.num[a] = g->coord_range[a].num;
        if (d.num[a] <= 0) fail(GLI_ERR_ARGUMENT, "grid axis %d has %lld points", a, (long long)d.num[a]);
    }
    return d;
}

// The symmetry-reduced paths need the grid (-e, 2e+1) on every axis (the
// reference's python module enforces this, python/pymodule.c:1149-1166).
i64 symmetric_extent(const GridDesc& g) {
    const i64 e = -g.istart[0];
    for (int a = 0; a < 3; ++a)
        if (g.istart[a] != -e || g.num[a] != 2 * e + 1) return -1;
    return e;
}

// ---------------------------------------------------------------------------
// exclusive scan: u32 counts -> u64 offsets
static constexpr int SCAN_BLOCK = 1024;
static constexpr int SCAN_ITEMS = 4;  // items per thread
static constexpr i64 SCAN_TILE = (i64)SCAN_BLOCK * SCAN_ITEMS;

__device__ inline uint64_t block_exclusive_sum(uint64_t v, uint64_t* warp_sums, uint64_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
        uint64_t wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const uint64_t r = warp_sums[warp] + incl - v;
    __syncthreads();
    return r;
}

__global__ void scan_tile_sums(const uint32_t* __restrict__ in, i64 n, uint64_t* __restrict__ tile_sums) {
    __shared__ uint64_t ws[32];
    __shared__ uint64_t tot;
    const i64 base = (i64)blockIdx.x * SCAN_TILE + (i64)threadIdx.x * SCAN_ITEMS;
    uint64_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < n) s += in[base + k];
    block_exclusive_sum(s, ws, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// single block: exclusive scan of the tile sums in place, total at [ntiles]
__global__ void scan_tile_offsets(uint64_t* tile_sums, i64 ntiles) {
    __shared__ uint64_t ws[32];
    __shared__ uint64_t tot;
    uint64_t carry = 0;
    for (i64 base = 0; base < ntiles; base += blockDim.x) {
        const i64 i = base + threadIdx.x;
        const uint64_t v = (i < ntiles) ? tile_sums[i] : 0;
        const uint64_t ex = block_exclusive_sum(v, ws, &tot);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_sums[ntiles] = carry;
}

__global__ void scan_tiles_apply(const uint32_t* __restrict__ in, i64 n, const uint64_t* __restrict__ tile_offsets,
                                 uint64_t* __restrict__ out) {
    __shared__ uint64_t ws[32];
    __shared__ uint64_t tot;
    const i64 base = (i64)blockIdx.x * SCAN_TILE + (i64)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint64_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    uint64_t run = tile_offsets[blockIdx.x] + block_exclusive_sum(s, ws, &tot);
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

// small arrays: one block walks the array in tiles of 4096 (4 consecutive
// items per thread, coalesced), carrying the running total; total at tot[0]
constexpr i64 SCAN_SMALL = 1 << 13;

__global__ void scan_small(const uint32_t* __restrict__ in, i64 n, uint64_t* __restrict__ out,
                           uint64_t* __restrict__ tot) {
    __shared__ uint64_t ws[32];
    __shared__ uint64_t total;
    uint64_t carry = 0;
    for (i64 base = 0; base < n; base += SCAN_TILE) {
        const i64 i0 = base + (i64)threadIdx.x * SCAN_ITEMS;
        uint32_t v[SCAN_ITEMS];
        uint64_t sum = 0;
        for (int k = 0; k < SCAN_ITEMS; ++k) {
            v[k] = i0 + k < n ? in[i0 + k] : 0u;
            sum += v[k];
        }
        uint64_t run = carry + block_exclusive_sum(sum, ws, &total);
        for (int k = 0; k < SCAN_ITEMS; ++k) {
            if (i0 + k < n) out[i0 + k] = run;
            run += v[k];
        }
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) tot[0] = carry;
}

i64 exclusive_scan_u32(const uint32_t* d_in, uint64_t* d_out, i64 n, cudaStream_t s) {
    if (n == 0) return 0;
    if (n <= SCAN_SMALL) {
        DevBuf<uint64_t> tot(1, s);
        scan_small<<<1, SCAN_BLOCK, 0, s>>>(d_in, n, d_out, tot.p);
        GLI_CHECK_LAUNCH();
        uint64_t total = 0;
        GLI_CUDA(cudaMemcpyAsync(&total, tot.p, sizeof(total), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s));
        return (i64)total;
    }
    const i64 ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    DevBuf<uint64_t> tiles(ntiles + 1, s);
    scan_tile_sums<<<(unsigned)ntiles, SCAN_BLOCK, 0, s>>>(d_in, n, tiles.p);
    GLI_CHECK_LAUNCH();
    scan_tile_offsets<<<1, SCAN_BLOCK, 0, s>>>(tiles.p, ntiles);
    GLI_CHECK_LAUNCH();
    scan_tiles_apply<<<(unsigned)ntiles, SCAN_BLOCK, 0, s>>>(d_in, n, tiles.p, d_out);
    GLI_CHECK_LAUNCH();
    uint64_t total = 0;
    GLI_CUDA(cudaMemcpyAsync(&total, tiles.p + ntiles, sizeof(total), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    return (i64)total;
}

// the same scan with its total left in device memory (*d_total), no host sync
__global__ void k_copy_total(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst) { *dst = *src; }

void exclusive_scan_u32_dev(const uint32_t* d_in, uint64_t* d_out, i64 n, uint64_t* d_total, cudaStream_t s) {
    if (n == 0) {
        GLI_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), s));
        return;
    }
    if (n <= SCAN_SMALL) {
        scan_small<<<1, SCAN_BLOCK, 0, s>>>(d_in, n, d_out, d_total);
        GLI_CHECK_LAUNCH();
        return;
    }
    const i64 ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    DevBuf<uint64_t> tiles(ntiles + 1, s);
    scan_tile_sums<<<(unsigned)ntiles, SCAN_BLOCK, 0, s>>>(d_in, n, tiles.p);
    GLI_CHECK_LAUNCH();
    scan_tile_offsets<<<1, SCAN_BLOCK, 0, s>>>(tiles.p, ntiles);
    GLI_CHECK_LAUNCH();
    scan_tiles_apply<<<(unsigned)ntiles, SCAN_BLOCK, 0, s>>>(d_in, n, tiles.p, d_out);
    GLI_CHECK_LAUNCH();
    k_copy_total<<<1, 1, 0, s>>>(tiles.p + ntiles, d_total);
    GLI_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// FP64 throughput probe: independent FMA chains, no memory traffic.  Used to
// state the measured FP64 roofline of the box next to the integral kernels.
__global__ void k_fp64_probe(double seed, int iters, double* __restrict__ sink) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 1e-9 + k;
    const double m = 0.999999999, c = 1e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, c);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678) sink[0] = s;  // keeps the chains live
}

// ... and the FP64 tensor-core path (mma.sync m8n8k4 f64: 256 FMAs per warp
// instruction), 16 independent accumulator tiles per warp
__global__ void k_dmma_probe(double seed, int iters, double* __restrict__ sink) {
    double c[16][2];
#pragma unroll
    for (int k = 0; k < 16; ++k) c[k][0] = c[k][1] = 0.0;
    const double a = seed + threadIdx.x * 1e-9, b = 0.999999999;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(c[k][0]), "+d"(c[k][1])
                         : "d"(a), "d"(b));
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += c[k][0] + c[k][1];
    if (s == 12345.678) sink[0] = s;
}

// FP64 peak of the device: the faster of the FMA and the tensor-core probes
double fp64_probe_tflops() {
    Context& c = context();
    cudaStream_t s = c.stream;
    DevBuf<double> sink(1, s);
    const int blocks = c.num_sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t e0, e1;
    GLI_CUDA(cudaEventCreate(&e0));
    GLI_CUDA(cudaEventCreate(&e1));
    float ms = 0;
    k_fp64_probe<<<blocks, threads, 0, s>>>(1.0, iters / 16, sink.p);  // warm-up
    GLI_CHECK_LAUNCH();
    GLI_CUDA(cudaEventRecord(e0, s));
    k_fp64_probe<<<blocks, threads, 0, s>>>(1.0, iters, sink.p);
    GLI_CHECK_LAUNCH();
    GLI_CUDA(cudaEventRecord(e1, s));
    GLI_CUDA(cudaEventSynchronize(e1));
    GLI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double fma_tf = 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12;
    const int mblocks = c.num_sms * 4, miters = 1 << 11;
    k_dmma_probe<<<mblocks, 128, 0, s>>>(1.0, miters / 16, sink.p);
    GLI_CHECK_LAUNCH();
    GLI_CUDA(cudaEventRecord(e0, s));
    k_dmma_probe<<<mblocks, 128, 0, s>>>(1.0, miters, sink.p);
    GLI_CHECK_LAUNCH();
    GLI_CUDA(cudaEventRecord(e1, s));
    GLI_CUDA(cudaEventSynchronize(e1));
    GLI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double mma_tf = 2.0 * 256.0 * 16.0 * miters * (double)mblocks * 4 / (ms * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return fma_tf > mma_tf ? fma_tf : mma_tf;
}

}  // namespace gli
