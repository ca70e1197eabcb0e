// Kinetic-energy matrix, reference src/kinetic_integrals.c:14-37 (1-D table)
// and :73-121 (dense K x I x I + I x K x I + I x I x K).
//
// The 1-D table is one block reduction per shift.  The dense matrix is a pure
// HBM write (8 bytes per entry, almost all zero): one block row per grid point
// i, threads stride over j with coalesced stores; the table sits in shared
// memory.
#include <math.h>
#include <stdlib.h>

#include <mutex>

#include "gli_internal.cuh"

namespace gli {

// k1[s] = 1/2 sum_ij b_i b_j (3/2) sqrt(pi) (1 - d^2/2) exp(-d^2/4), d = 3s + i - j
__global__ void k_kinetic_1d(const double* __restrict__ b, int nb, double* __restrict__ k1) {
    __shared__ double red[32];
    const int s = blockIdx.x;
    double acc = 0;
    const double c = 1.5 * 1.7724538509055160273;  // 3/2 sqrt(pi)
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        const int i = e / nb, j = e % nb;
        const double d = (double)(3 * s + (i - j));
        const double d2 = d * d;
        acc += 0.5 * b[i] * b[j] * (c * (1 - 0.5 * d2) * exp(-0.25 * d2));
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) k1[s] = acc;
    }
}

__global__ void __launch_bounds__(256) k_kinetic_matrix(const double* __restrict__ k1g, int L, int nx, int ny, int nz,
                                                        double* __restrict__ out) {
    __shared__ double k1[1024];
    for (int s = threadIdx.x; s < L && s < 1024; s += blockDim.x) k1[s] = k1g[s];
    __syncthreads();
    const i64 N = (i64)nx * ny * nz;
    const i64 row = blockIdx.y + (i64)blockIdx.z * gridDim.y;
    if (row >= N) return;
    const int az = (int)(row % nz), ay = (int)((row / nz) % ny), ax = (int)(row / ((i64)nz * ny));
    double* r = out + row * N;
    for (i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x; j < N; j += (i64)gridDim.x * blockDim.x) {
        const int bz = (int)(j % nz), by = (int)((j / nz) % ny), bx = (int)(j / ((i64)nz * ny));
        const int dx = ax - bx, dy = ay - by, dz = az - bz;
        double v = 0;
        if (dy == 0 && dz == 0) v += k1[dx < 0 ? -dx : dx];
        if (dx == 0 && dz == 0) v += k1[dy < 0 ? -dy : dy];
        if (dx == 0 && dy == 0) v += k1[dz < 0 ? -dz : dz];
        r[j] = v;
    }
}

void kinetic_table_device(const double* h_coeffs, i64 nb, i64 L, double* d_k1, cudaStream_t s) {
    DevBuf<double> b(nb, s);
    GLI_CUDA(cudaMemcpyAsync(b.p, h_coeffs, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    k_kinetic_1d<<<(unsigned)L, 256, 0, s>>>(b.p, (int)nb, d_k1);
    GLI_CHECK_LAUNCH();
}

void kinetic_matrix_device(const double* h_coeffs, i64 nb, const GridDesc& g, double* d_out, cudaStream_t s) {
    const i64 L = g.max_range();
    if (L > 1024) fail(GLI_ERR_LIMIT, "kinetic matrix supports axes up to 1024 points");
    DevBuf<double> k1(L, s);
    kinetic_table_device(h_coeffs, nb, L, k1.p, s);
    const i64 N = g.points();
    const i64 yrows = N < 65535 ? N : 65535;
    const i64 zrows = (N + yrows - 1) / yrows;
    const i64 xblocks = (N + 255) / 256 < 8 ? (N + 255) / 256 : 8;
    k_kinetic_matrix<<<dim3((unsigned)xblocks, (unsigned)yrows, (unsigned)zrows), 256, 0, s>>>(
        k1.p, (int)L, (int)g.num[0], (int)g.num[1], (int)g.num[2], d_out);
    GLI_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Kinetic matrix without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need the
// matrix: code that has reserved its whole device-memory budget up front (a
// solver that pre-sizes its arena before the first iteration), code running
// while another framework captures a CUDA graph or owns the allocator, and
// hosts that forbid allocation inside a latency-critical loop.  For them the
// per-axis kinetic table -- the only scratch this computation needs -- lives in
// the file-scope device array below instead of a cudaMalloc'ed buffer; the
// caller supplies the coefficients and the output matrix in device memory.
//
// The array holds one table entry per grid shift, so the largest axis of the
// grid may have at most kNoAllocMaxAxis points.  Every GPU that loads the
// library keeps these 8 KB until the process exits.  The array is shared by all
// calls on a device: each call rewrites the entries it reads before reading
// them (nothing needs clearing), so consecutive calls are independent, but two
// calls whose kernels overlap on the GPU (different streams or threads without
// ordering between them) race on it.
constexpr int kNoAllocMaxAxis = 1024;
static __device__ __align__(256) double g_noalloc_kinetic_table[kNoAllocMaxAxis];

// Host code may not use g_noalloc_kinetic_table directly: on the host that name
// is a host-side stand-in, not a device address.  The device address is looked
// up once per device (with that device current) and remembered.
static std::mutex g_noalloc_mu;
static double* g_noalloc_table_ptr[64] = {};

static double* noalloc_table_address() {
    int device = 0;
    GLI_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= 64) fail(GLI_ERR_LIMIT, "device ordinal %d out of range for the no-alloc table", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_table_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_kinetic_table);
        if (e != cudaSuccess || p == nullptr)
            fail(GLI_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc kinetic table failed: %s", cudaGetErrorString(e));
        g_noalloc_table_ptr[device] = static_cast<double*>(p);
    }
    return g_noalloc_table_ptr[device];
}

static void kinetic_matrix_noalloc(const double* d_coeffs, i64 nb, const GridDesc& g, double* d_out, cudaStream_t s) {
    if (!d_coeffs || !d_out) fail(GLI_ERR_ARGUMENT, "coefficient and matrix pointers must be device memory, not NULL");
    if (nb <= 0 || nb % 2 != 1) fail(GLI_ERR_ARGUMENT, "gausslet coefficient count must be odd, got %lld", (long long)nb);
    const i64 L = g.max_range();
    if (L > kNoAllocMaxAxis)
        fail(GLI_ERR_LIMIT, "the allocation-free kinetic matrix supports axes up to %d points (got %lld)", kNoAllocMaxAxis,
             (long long)L);
    double* table = noalloc_table_address();
    k_kinetic_1d<<<(unsigned)L, 256, 0, s>>>(d_coeffs, (int)nb, table);
    GLI_CHECK_LAUNCH();
    const i64 N = g.points();
    const i64 yrows = N < 65535 ? N : 65535;
    const i64 zrows = (N + yrows - 1) / yrows;
    const i64 xblocks = (N + 255) / 256 < 8 ? (N + 255) / 256 : 8;
    k_kinetic_matrix<<<dim3((unsigned)xblocks, (unsigned)yrows, (unsigned)zrows), 256, 0, s>>>(
        table, (int)L, (int)g.num[0], (int)g.num[1], (int)g.num[2], d_out);
    GLI_CHECK_LAUNCH();
}

}  // namespace gli

extern "C" int gli_b200_kinetic_matrix_noalloc(const double* d_coeffs, glong num_coeffs,
                                               const struct cartesian_grid_3d* grid, double* d_matrix, void* stream) {
    gli::clear_error();
    try {
        if (!grid) gli::fail(GLI_ERR_ARGUMENT, "grid missing");
        const gli::GridDesc g = gli::grid_desc(grid);
        gli::kinetic_matrix_noalloc(d_coeffs, num_coeffs, g, d_matrix, static_cast<cudaStream_t>(stream));
    } catch (const gli::Failure&) {
        if (!getenv("GLI_B200_QUIET")) fprintf(stderr, "gausslectronitegrate_b200: %s\n", gli::last_message());
    }
    return gli::last_error();
}
