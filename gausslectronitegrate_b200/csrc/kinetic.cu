// Kinetic-energy matrix, reference src/kinetic_integrals.c:14-37 (1-D table)
// and :73-121 (dense K x I x I + I x K x I + I x I x K).
//
// The 1-D table is one block reduction per shift.  The dense matrix is a pure
// HBM write (8 bytes per entry, almost all zero).  Row i = (ax, ay, az) has
// its nonzeros on three lines through i: the x line (columns bx P + c, P =
// ny nz, c = ay nz + az), the y line and the z line inside the x block bx = ax.
// A block writes whole rows with 16-byte stores; each thread walks its columns
// with the x block and the in-block offset updated incrementally (no division
// per entry), and only the x block of the row itself decodes (y, z).
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>
#include <vector>

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

// value of column (bx, q) of row (ax, c = ay nz + az)
__device__ __forceinline__ double kinetic_entry(const double* __restrict__ k1, int ax, int ay, int az, int c, int nz,
                                                int bx, int q) {
    double v = q == c ? k1[abs(ax - bx)] : 0.0;  // the x line
    if (bx == ax) {                               // the y and z lines (and the diagonal)
        const int by = q / nz, bz = q - by * nz;
        if (by == ay) v += k1[abs(az - bz)];
        if (bz == az) v += k1[abs(ay - by)];
    }
    return v;
}

__global__ void __launch_bounds__(256) k_kinetic_matrix(const double* __restrict__ k1g, int L, int nx, int ny, int nz,
                                                        double* __restrict__ out) {
    __shared__ double k1[1024];
    for (int s = threadIdx.x; s < L && s < 1024; s += blockDim.x) k1[s] = k1g[s];
    __syncthreads();
    const int P = ny * nz, N = nx * P;
    const int step = 2 * blockDim.x;
    for (int row = blockIdx.x; row < N; row += gridDim.x) {
        const int ax = row / P, c = row - ax * P, ay = c / nz, az = c - ay * nz;
        double* r = out + (i64)row * N;
        // a row starting on an odd double writes its first entry alone, so
        // that the pairs stored as double2 sit on 16-byte boundaries
        const int j0 = (int)(((i64)row * N) & 1);
        if (j0 && threadIdx.x == 0) r[0] = kinetic_entry(k1, ax, ay, az, c, nz, 0, 0);
        int j = j0 + 2 * threadIdx.x;
        int bx = j / P, q = j - bx * P;
        for (; j + 1 < N; j += step) {
            const double v0 = kinetic_entry(k1, ax, ay, az, c, nz, bx, q);
            const int q1 = q + 1 < P ? q + 1 : 0, bx1 = q + 1 < P ? bx : bx + 1;
            const double v1 = kinetic_entry(k1, ax, ay, az, c, nz, bx1, q1);
            *reinterpret_cast<double2*>(r + j) = make_double2(v0, v1);
            q += step;
            while (q >= P) {
                q -= P;
                ++bx;
            }
        }
        if (j < N) r[j] = kinetic_entry(k1, ax, ay, az, c, nz, bx, q);  // an unpaired last entry
    }
}

// blocks of the matrix kernel: rows spread over a few waves of the current
// device's SMs (an attribute query: no context state of the library is made)
static unsigned kinetic_blocks(i64 N) {
    int dev = 0, sms = 148;
    GLI_CUDA(cudaGetDevice(&dev));
    GLI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return (unsigned)std::min<i64>(N, (i64)sms * 8);
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
    if (N >= ((i64)1 << 31)) fail(GLI_ERR_LIMIT, "kinetic matrix of %lld points exceeds the row index range", (long long)N);
    k_kinetic_matrix<<<kinetic_blocks(N), 256, 0, s>>>(k1.p, (int)L, (int)g.num[0], (int)g.num[1], (int)g.num[2],
                                                       d_out);
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
// is a host-side stand-in, not a device address.  The device address belongs to
// the module loaded in the current context, so it is looked up, with the
// device current, on every call made outside a stream capture (cheap once the
// module is loaded; it follows a context made current by the caller and the
// new module after a device reset) and remembered per context.  A call made
// while its stream is being captured uses the address remembered for the
// current context: the first call in a context must come before any capture.
static std::mutex g_noalloc_mu;
struct NoallocAddress {
    void* ctx;
    double* table;
};
static std::vector<NoallocAddress> g_noalloc_addr;

// the current driver context (cuCtxGetCurrent through the runtime's entry
// point lookup, so that the library needs no link to the driver library)
static void* current_context() {
    using Fn = int (*)(void**);
    static const Fn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (Fn) nullptr;
        return (Fn)f;
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0 || !ctx) fail(GLI_ERR_CUDA, "no current CUDA context for the no-alloc kinetic table");
    return ctx;
}

static double* noalloc_table_address(cudaStream_t s) {
    int device = 0;
    GLI_CUDA(cudaGetDevice(&device));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    GLI_CUDA(cudaStreamIsCapturing(s, &cap));
    void* ctx = current_context();
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    auto it = std::find_if(g_noalloc_addr.begin(), g_noalloc_addr.end(),
                           [&](const NoallocAddress& a) { return a.ctx == ctx; });
    if (cap != cudaStreamCaptureStatusNone) {
        if (it == g_noalloc_addr.end())
            fail(GLI_ERR_ARGUMENT, "the first allocation-free kinetic call on device %d must come before stream capture",
                 device);
        return it->table;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_kinetic_table);
    if (e != cudaSuccess || p == nullptr)
        fail(GLI_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc kinetic table failed: %s", cudaGetErrorString(e));
    if (it == g_noalloc_addr.end())
        g_noalloc_addr.push_back({ctx, static_cast<double*>(p)});
    else
        it->table = static_cast<double*>(p);
    return static_cast<double*>(p);
}

// device (or managed) memory, checked outside a capture: a host pointer handed
// to the kernels would fault the GPU instead of failing the call
static void check_device_pointer(const void* p, const char* what, cudaStream_t s) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    GLI_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone) return;
    cudaPointerAttributes a = {};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(GLI_ERR_ARGUMENT, "%s pointer is not CUDA memory", what);
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
        fail(GLI_ERR_ARGUMENT, "%s pointer must be device memory (got %s memory)", what,
             a.type == cudaMemoryTypeHost ? "pinned host" : "unregistered host");
}

static void kinetic_matrix_noalloc(const double* d_coeffs, i64 nb, const GridDesc& g, double* d_out, cudaStream_t s) {
    if (!d_coeffs || !d_out) fail(GLI_ERR_ARGUMENT, "coefficient and matrix pointers must be device memory, not NULL");
    if (nb <= 0 || nb % 2 != 1) fail(GLI_ERR_ARGUMENT, "gausslet coefficient count must be odd, got %lld", (long long)nb);
    if (nb > 46340) fail(GLI_ERR_LIMIT, "gausslet coefficient count %lld too large (nb^2 must fit 32 bits)", (long long)nb);
    const i64 L = g.max_range();
    if (L > kNoAllocMaxAxis)
        fail(GLI_ERR_LIMIT, "the allocation-free kinetic matrix supports axes up to %d points (got %lld)", kNoAllocMaxAxis,
             (long long)L);
    if (g.points() >= ((i64)1 << 31))
        fail(GLI_ERR_LIMIT, "kinetic matrix of %lld points exceeds the row index range", (long long)g.points());
    check_device_pointer(d_coeffs, "coefficient", s);
    check_device_pointer(d_out, "matrix", s);
    double* table = noalloc_table_address(s);
    k_kinetic_1d<<<(unsigned)L, 256, 0, s>>>(d_coeffs, (int)nb, table);
    GLI_CHECK_LAUNCH();
    const i64 N = g.points();
    k_kinetic_matrix<<<kinetic_blocks(N), 256, 0, s>>>(table, (int)L, (int)g.num[0], (int)g.num[1], (int)g.num[2],
                                                       d_out);
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
