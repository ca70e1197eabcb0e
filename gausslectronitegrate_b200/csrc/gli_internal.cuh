// Internal declarations shared by the CUDA translation units of libgli_b200.
//
// Layout of the library:
//   runtime.cu    error state, per-thread streams, device buffers, prefix sums
//   tables.cu     Gaussian-pair factor/product vectors, folded lattice weights,
//                 Coulomb lookup tables, the kinetic 1-D table (all on device)
//   enumerate.cu  symmetry-reduced ERI / ERIDA class enumeration (bit-exact)
//   contract.cu   the staged lattice contraction that evaluates every class
//   kinetic.cu    dense kinetic matrix
//   nuclear.cu    nuclear-attraction matrices (field + staged contraction), batches
//   tc_gemm.cu    int8-sliced tcgen05 GEMM (mixed form, FP64-level products)
//   autotune.cu   launch-configuration autotuner (host)
//   dense.cu      sparse -> dense expansion, ERI apply, projections
//   capi.cu       the extern "C" entry points (reference API + extensions)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "gli_b200.h"

namespace gli {

typedef int64_t i64;

// ---------------------------------------------------------------------------
// error handling: every entry point records a status and message per thread
void set_error(int code, const char* fmt, ...);
void clear_error();
int last_error();

struct Failure {
    int code;
};

// throw a Failure after recording the message; caught by each C entry point
[[noreturn]] void fail(int code, const char* fmt, ...);

#define GLI_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t _e = (call);                                                         \
        if (_e != cudaSuccess)                                                           \
            ::gli::fail(GLI_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                        cudaGetErrorString(_e));                                         \
    } while (0)

// every kernel launch site is followed by GLI_CHECK_LAUNCH(), which also counts
// the launch (per thread) for gli_b200_launch_count()
void count_launch();
#define GLI_CHECK_LAUNCH()            \
    do {                              \
        ::gli::count_launch();        \
        GLI_CUDA(cudaGetLastError()); \
    } while (0)

// one launch on stream s (the arguments converted to the kernel's parameter types)
template <typename... KArgs, typename... Args>
void launch_kernel(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    GLI_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...));
    count_launch();
}

// ---------------------------------------------------------------------------
// device context: the calling thread's device and its non-blocking stream
struct Context {
    int device;
    cudaStream_t stream;
    int num_sms;
};
Context& context();                 // initialises the device on first use (fails loudly without a GPU)

// stream-ordered device buffer (cudaMallocAsync / cudaFreeAsync on the call stream)
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = 0;
    bool owned = true;  // false: memory lent by a longer-lived owner, not freed here
    DevBuf() = default;
    DevBuf(size_t count, cudaStream_t stream) { alloc(count, stream); }
    void alloc(size_t count, cudaStream_t stream) {
        release();
        s = stream;
        n = count;
        owned = true;
        if (count) GLI_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), stream));
    }
    void borrow(T* mem, size_t count, cudaStream_t stream) {
        release();
        s = stream;
        n = count;
        owned = false;
        p = mem;
    }
    void zero() {
        if (n) GLI_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    void release() {
        if (p && owned) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

// exclusive prefix sum of 32-bit counts into 64-bit offsets; returns the total
// (synchronises the stream)
i64 exclusive_scan_u32(const uint32_t* d_in, uint64_t* d_out, i64 n, cudaStream_t s);
// the same, total left in device memory at d_total (no synchronisation)
void exclusive_scan_u32_dev(const uint32_t* d_in, uint64_t* d_out, i64 n, uint64_t* d_total, cudaStream_t s);

// ---------------------------------------------------------------------------
// grids
struct GridDesc {
    i64 istart[3];
    i64 num[3];
    i64 points() const { return num[0] * num[1] * num[2]; }
    i64 max_range() const {
        i64 m = num[0];
        if (num[1] > m) m = num[1];
        if (num[2] > m) m = num[2];
        return m;
    }
};
GridDesc grid_desc(const struct cartesian_grid_3d* g);
// rotationally symmetric grid (-e, 2e+1) on all three axes; returns e or -1
i64 symmetric_extent(const GridDesc& g);

// ---------------------------------------------------------------------------
// O_h: the 48 signed permutation matrices.  Element g = 8 * perm + signs,
// perm indexes the six permutations of (x, y, z), bit a of signs negates axis a.
__host__ __device__ inline void oh_apply(int g, const int p[3], int q[3]) {
    const int perm = g >> 3;
    // permutations in lexicographic order: 012 021 102 120 201 210
    const int a0 = (perm < 2) ? 0 : (perm < 4 ? 1 : 2);
    const int a1 = (perm == 0) ? 1 : (perm == 1) ? 2 : (perm == 2) ? 0 : (perm == 3) ? 2 : (perm == 4) ? 0 : 1;
    const int a2 = 3 - a0 - a1;
    q[0] = (g & 1) ? -p[a0] : p[a0];
    q[1] = (g & 2) ? -p[a1] : p[a1];
    q[2] = (g & 4) ? -p[a2] : p[a2];
}

// ---------------------------------------------------------------------------
// integral forms
enum Form { FORM_FP64 = 0, FORM_MIXED = 1 };

// the staged lattice contraction (contract.cu)
struct ContractStats {
    i64 keys_a = 0, pairs = 0, U = 0;
    i64 keys_used = 0;  // distinct axis keys of the class list
    int product = 0;    // stage C ran as the (pair, key) product GEMM
    i64 products = 0;   // ... and computed this many (pair, key) products
    int tc_a = 0, tc_b = 0;  // stage A / B ran as int8-sliced products on the tcgen05 tensor cores
    int gather = 0;          // the class gather of a product-form stage C: 1 packed keys, 2 decoding
                             // and checking against a kept plan
    double screen_tol = 0;    // the product threshold the tables were built with (mixed form: screened)
    double screen_bound = 0;  // bound on the change of a class value by that screening (grid units)
    float ms_tables = 0, ms_a = 0, ms_b = 0, ms_c = 0;
    // stage C in two parts: the (pair, key) product GEMM (0 when stage C ran
    // per class) and the class-level kernel (the gather, or the per-class dots)
    float ms_c_product = 0, ms_c_class = 0;
};

// drops the calling thread's captured evaluations and every cached table set
// (the next evaluation builds its tables again)
void clear_eval_caches();
void clear_table_cache();

// kind: 0 = ERIDA (two-index classes), 1 = ERI (four-index classes)
void sparse_values_device(int kind, const double* h_coeffs, i64 nb, const GridDesc& g,
                          const int64_t* d_indices, i64 m, double tol, int form,
                          double* d_out, cudaStream_t s, ContractStats* stats);
// the same queued without a host wait: returns a ticket; sparse_values_wait
// reads its status (and that of every evaluation queued before it on this
// thread), evaluating again where a sized graph overflowed
i64 sparse_values_device_async(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* d_indices,
                               i64 m, double tol, int form, double* d_out, cudaStream_t s);
void sparse_values_wait(i64 ticket);
// the same from host buffers (pinned staging, one synchronisation)
void sparse_values_host(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* h_indices, i64 m,
                        double tol, int form, double* h_out, cudaStream_t s);

// enumeration (enumerate.cu); returns a device array (caller frees with cudaFreeAsync)
i64 enumerate_device(int kind, const GridDesc& g, int64_t** d_out, cudaStream_t s);

// kinetic (kinetic.cu): dense N x N matrix on device
void kinetic_matrix_device(const double* h_coeffs, i64 nb, const GridDesc& g, double* d_out, cudaStream_t s);
void kinetic_table_device(const double* h_coeffs, i64 nb, i64 L, double* d_k1, cudaStream_t s);

// tables.cu: per-shift Gaussian-pair factors F[s][m], s = 0..L-1, m = 0..2nb-2
void factors_device(const double* d_b, int nb, int L, double* d_F, cudaStream_t s);

// nuclear.cu: dense nuclear matrix over the product of three axis coordinate lists
void nuclear_matrix_device(const double* h_coeffs, i64 nb, const std::vector<int> axes[3],
                           const struct atomic_nucleus* nuclei, int nn, double tol, double* d_out, cudaStream_t s);

// one instance of a nuclear batch: ascending coordinate lists per axis, its
// nuclei (host memory) and its N x N output (device memory)
struct NuclearJob {
    std::vector<int> axes[3];
    const struct atomic_nucleus* nuclei = nullptr;
    int nn = 0;
    double* d_out = nullptr;
};
struct NuclearBatchStats {
    i64 instances = 0, chunks = 0;
    int streams = 0;
};
// every instance's matrix, one graph per chunk of instances; form FP64 or mixed
void nuclear_batch_device(const double* h_coeffs, i64 nb, const std::vector<NuclearJob>& jobs, double tol, int form,
                          cudaStream_t s);
const NuclearBatchStats& last_nuclear_stats();

// dense.cu
void fill_dense_device(int kind, const GridDesc& sparse, const int64_t* d_idx, const double* d_val, i64 m,
                       const GridDesc& dense, double* d_out, cudaStream_t s);
void grid_perms_device(const GridDesc& g, int64_t* d_perm, cudaStream_t s);
void apply_eri_device(const GridDesc& g, const int64_t* d_idx, const double* d_val, i64 m, const double* d_states,
                      i64 ns, double* d_ret, cudaStream_t s);
void project_device(int kind, const GridDesc& g, const int64_t* d_idx, const double* d_val, i64 m,
                    const double* d_basis, i64 M, double* d_out, cudaStream_t s);

// runtime.cu / contract.cu
double fp64_probe_tflops();
long long launch_count();
// adds n kernels launched as part of a CUDA graph replay
void add_launches(long long n);
const char* last_message();
int set_device(int ordinal);
void set_timing(bool on);
const ContractStats& last_stats();

}  // namespace gli
