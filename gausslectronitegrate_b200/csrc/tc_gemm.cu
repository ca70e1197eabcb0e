// Tensor-core (tcgen05) FP64-accurate GEMM by int8 slicing, for sm_100a.
//
//   C[m][n] (+)= sum_k A[m][k] B[n][k]            (A: M x K, B: N x K, FP64, K-major)
//
// Each operand row r is split as  x = 2^e_r sum_{p=0..S-1} 2^(-7(p+1)) d_p,  d_p
// int8 in [-64, 64] (e_r chosen so |x| 2^-e_r < 1/2; each slice carries 7 bits).
// The product of two rows is then
//   2^(ea+eb) sum_{p,q} 2^(-7(p+q+2)) (A_p . B_q)
// where every A_p . B_q is an exact int8 x int8 -> int32 dot product on the
// tensor cores.  Products with p + q >= R are below the target precision and
// are dropped; all pairs with the same p + q share one int32 accumulator
// region in tensor memory (exact: |sum| <= 8 * 64 * 64 * K < 2^31 for K <= 8192).
// The epilogue converts each region to FP64, scales by 2^(-7(p+q+2)) and sums.
// Two variants are built: S = 5, R = 5 keeps about 2^-36 of max|a| max|b| per
// product term (the mixed form of the integral stages) and S = 7, R = 8 about
// 2^-50 (FP64-level accuracy).
//
// Kernel structure (one CTA = 128 rows of C x 64 columns, 128 threads):
//   * warp 0 allocates 512 tensor-memory columns (R regions of 64), thread 0
//     initialises one mbarrier;
//   * for each slice p of A and each 128-byte K chunk: all threads copy the A_p
//     tile (128 x 128 int8) and the B_q tiles (64 x 128 int8, p + q < R) into
//     shared memory in the canonical K-major core-matrix layout (8 rows x 16
//     bytes per core matrix), fence the async proxy, synchronise; thread 0
//     issues 4 MMAs (K = 32 each) per q into region p+q and commits to the
//     mbarrier; all threads wait on it (bounded), then the next chunk reuses
//     the buffers;
//   * epilogue: warp w reads lanes 32w..32w+31 (its 32 rows) of every region
//     with tcgen05.ld, 16 columns at a time, and accumulates in FP64.
// Every mbarrier wait has an iteration limit; on expiry the CTA records an
// error code, stops issuing, waits (bounded) for its MMAs and frees its tensor
// memory before returning.
#include <stdint.h>
#include <stdlib.h>

#include "tc_gemm.cuh"

namespace gli {

constexpr int TCG_SMAX = 8;               // most slices per operand
constexpr int TCG_BM = 128;               // rows of C per CTA (MMA M)
constexpr int TCG_BN = 64;                // columns of C per CTA (MMA N)
constexpr int TCG_BK = 128;               // K bytes per shared-memory chunk (4 MMAs of K = 32)
constexpr int TCG_TMEM_COLS = 512;
constexpr unsigned TCG_WAIT_LIMIT = 1u << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle (core matrix = 8 rows x 16 B)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: int8 x int8 -> int32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// bounded wait; returns false on expiry
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (unsigned it = 0; it < TCG_WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Sliced operand set: S slices of a matrix with `rows` rows and K (padded to a
// multiple of 32) int8 columns, slice-major: slice p at data + p * slice_stride;
// e[r] the row exponent.  Batched operands add batch_stride (int8) and e_batch.
struct SlicedOp {
    const int8_t* data;
    i64 ld;            // bytes between rows
    i64 slice_stride;  // bytes between slices
    i64 batch_stride;  // bytes between batches
    const int* e;      // exponent per row
    i64 e_batch;       // exponents between batches
    int rows;
    const int* row0;   // optional per-batch first row (then batch_stride/e_batch are unused)
};

struct OutView {
    double* p;
    i64 rs, cs, bs;    // row, column and batch strides (elements)
    const int* col0;   // optional per-batch first column (then bs is unused)
};

constexpr int TCG_SMEM_TILES = TCG_BM * TCG_BK + TCG_SMAX * TCG_BN * TCG_BK;  // 80 KB
// requested dynamic shared memory: more than half of the SM's 228 KB, so that at
// most one CTA (and one owner of the 512 tensor-memory columns) is resident per SM
constexpr int TCG_SMEM_REQUEST = 116 * 1024;

// TCG_S slices per operand; products of slices p + q <= TCG_R - 1 (0-based) are
// kept, one tensor-memory region of 64 int32 columns per value of p + q.
template <int TCG_S, int TCG_R>
__global__ void __launch_bounds__(128, 1) k_tc_gemm_sliced(SlicedOp A, SlicedOp B, int K, OutView C, int accumulate,
                                                            const int* __restrict__ batch_rows_n, int* __restrict__ err) {
    static_assert(TCG_R * TCG_BN <= TCG_TMEM_COLS, "tensor-memory regions exceed 512 columns");
    static_assert(TCG_S <= TCG_SMAX && TCG_R <= 2 * TCG_S - 1, "slice and region counts out of range");
    extern __shared__ __align__(1024) int8_t tcg_smem[];
    int8_t* sA = tcg_smem;
    int8_t* sB0 = tcg_smem + TCG_BM * TCG_BK;  // slice q at sB0 + q * TCG_BN * TCG_BK
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int b = blockIdx.z;
    const int m0 = blockIdx.x * TCG_BM, n0 = blockIdx.y * TCG_BN;
    const int Nb = batch_rows_n ? batch_rows_n[b] : B.rows;   // valid B rows of this batch
    if (n0 >= Nb) return;                                     // uniform across the CTA

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base_sh)),
                     "r"(TCG_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    const int8_t* Ab = A.data + (A.row0 ? (i64)A.row0[b] * A.ld : (i64)b * A.batch_stride);
    const int8_t* Bb = B.data + (B.row0 ? (i64)B.row0[b] * B.ld : (i64)b * B.batch_stride);
    const int* Ae = A.e + (A.row0 ? (i64)A.row0[b] : (i64)b * A.e_batch);
    const int* Be = B.e + (B.row0 ? (i64)B.row0[b] : (i64)b * B.e_batch);
    double* Cb = C.p + (C.col0 ? (i64)C.col0[b] * C.cs : (i64)b * C.bs);
    const uint32_t idesc = idesc_i8(TCG_BM, TCG_BN);
    const uint32_t sA_addr = smem_addr(sA);
    uint32_t phase = 0;
    bool started[TCG_R] = {};  // region has received its first MMA
    int issued = 0;

    for (int p = 0; p < TCG_S && p < TCG_R && !abort_flag; ++p) {
        for (int k0 = 0; k0 < K; k0 += TCG_BK) {
            // A_p tile: 128 rows x 128 bytes = 1024 16-byte pieces
            for (int c = tid; c < TCG_BM * (TCG_BK / 16); c += 128) {
                const int r = c / (TCG_BK / 16), kc = c % (TCG_BK / 16);
                int4 v = make_int4(0, 0, 0, 0);
                if (m0 + r < A.rows && k0 + kc * 16 < K)
                    v = *reinterpret_cast<const int4*>(Ab + p * A.slice_stride + (i64)(m0 + r) * A.ld + k0 + kc * 16);
                *reinterpret_cast<int4*>(sA + ((r >> 3) * (TCG_BK / 16) + kc) * 128 + (r & 7) * 16) = v;
            }
            const int nq = min(TCG_S, TCG_R - p);  // q = 0 .. nq-1 keeps p + q <= R - 1
            for (int q = 0; q < nq; ++q)
                for (int c = tid; c < TCG_BN * (TCG_BK / 16); c += 128) {
                    const int r = c / (TCG_BK / 16), kc = c % (TCG_BK / 16);
                    int4 v = make_int4(0, 0, 0, 0);
                    if (n0 + r < Nb && k0 + kc * 16 < K)
                        v = *reinterpret_cast<const int4*>(Bb + q * B.slice_stride + (i64)(n0 + r) * B.ld + k0 +
                                                          kc * 16);
                    *reinterpret_cast<int4*>(sB0 + q * TCG_BN * TCG_BK + ((r >> 3) * (TCG_BK / 16) + kc) * 128 + (r & 7) * 16) = v;
                }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int kmax = min(TCG_BK, K - k0);
                for (int q = 0; q < nq; ++q) {
                    const int region = p + q;
                    const uint32_t sB_addr = smem_addr(sB0 + q * TCG_BN * TCG_BK);
                    for (int kk = 0; kk < kmax; kk += 32) {
                        // 32 int8 along K = 2 core matrices: LBO = 128 B between them,
                        // SBO = (TCG_BK / 16) * 128 B between 8-row groups
                        const uint64_t da = umma_desc(sA_addr + (kk / 16) * 128, 128, (TCG_BK / 16) * 128);
                        const uint64_t db = umma_desc(sB_addr + (kk / 16) * 128, 128, (TCG_BK / 16) * 128);
                        mma_i8(tmem + (uint32_t)(region * TCG_BN), da, db, idesc, started[region] ? 1u : 0u);
                        started[region] = true;
                    }
                }
                mma_commit(&mbar);
            }
            ++issued;
            if (!mbar_wait_bounded(&mbar, phase)) {
                if (lane == 0) atomicExch(err, 1);
                abort_flag = 1;
                // give the MMAs in flight one more bounded chance to finish
                // before the tensor memory they write is released
                mbar_wait_bounded(&mbar, phase);
            }
            phase ^= 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncthreads();
            if (abort_flag) break;
        }
    }

    if (!abort_flag) {
        // epilogue: region r holds sum_{p+q=r} A_p . B_q (slices 0-based, weight 2^(-7(r+2)))
        const int row = m0 + warp * 32 + lane;
        const double ea = (row < A.rows) ? (double)Ae[row] : 0.0;
        for (int c0 = 0; c0 < TCG_BN; c0 += 16) {
            double acc[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = 0.0;
            for (int r = 0; r < TCG_R; ++r) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(r * TCG_BN + c0), v);
                const double w = ldexp(1.0, -7 * (r + 2));
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[j] = fma((double)(int32_t)v[j], w, acc[j]);
            }
            if (row < A.rows) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < Nb) {
                        const double eb = (double)Be[col];
                        const double val = ldexp(acc[j], (int)(ea + eb));
                        double* out = Cb + (i64)row * C.rs + (i64)col * C.cs;
                        *out = accumulate ? *out + val : val;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCG_TMEM_COLS));
}

// ---------------------------------------------------------------------------
// slicing: rows of an FP64 matrix (row stride ld_src, K columns) into S int8
// slices with K padded to Kp (multiple of 16), plus one exponent per row.
// One warp per row.
__global__ void k_slice_rows(const double* __restrict__ src, i64 rows, int K, i64 ld_src, i64 src_batch_stride,
                             int Kp, int nslices, int8_t* __restrict__ dst, i64 slice_stride, i64 dst_batch_stride,
                             int* __restrict__ e, i64 e_batch, int batches) {
    const i64 gw = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= rows * batches) return;
    const i64 b = gw / rows, r = gw % rows;
    const double* x = src + b * src_batch_stride + r * ld_src;
    double mx = 0;
    for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(x[k]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int ex = 0;
    if (mx > 0) {
        frexp(mx, &ex);  // mx = f 2^ex, f in [0.5, 1)
        ex += 1;         // |x| 2^-ex < 1/2
    }
    if (lane == 0) e[b * e_batch + r] = ex;
    int8_t* d = dst + b * dst_batch_stride + r * (i64)Kp;
    for (int k = lane; k < Kp; k += 32) {
        double v = (k < K && mx > 0) ? ldexp(x[k], -ex) : 0.0;
        for (int p = 0; p < nslices; ++p) {
            const double t = v * 128.0;
            const double dp = rint(t);  // |t| <= 64
            d[p * slice_stride + k] = (int8_t)(int)dp;
            v = t - dp;                 // exact in FP64, |v| <= 1/2
        }
    }
}

// host wrappers ---------------------------------------------------------------
// slice `batches` row blocks (rows x K each, row stride ld, batch stride bs)
void slice_rows(const double* src, i64 rows, int K, i64 ld, i64 bs, int batches, int nslices, SlicedMatrix& out,
                cudaStream_t s) {
    if (nslices < 1 || nslices > TCG_SMAX) fail(GLI_ERR_INTERNAL, "slice count %d out of range", nslices);
    out.rows = rows;
    out.batches = batches;
    out.slices = nslices;
    out.Kp = (K + 31) / 32 * 32;  // whole MMAs of K = 32
    out.data.alloc((size_t)nslices * rows * out.Kp * batches, s);
    out.e.alloc((size_t)rows * batches, s);
    const i64 warps = rows * batches;
    k_slice_rows<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(src, rows, K, ld, bs, (int)out.Kp, nslices, out.data.p,
                                                                      rows * out.Kp * batches, rows * out.Kp, out.e.p,
                                                                      rows, batches);
    GLI_CHECK_LAUNCH();
}

// C[b] (+)= A[b] B[b]^T for sliced operands.  Uniform batches by default; for
// ragged batches of B (rows b_row0[b] .. b_row0[b] + b_rows[b]) and of the
// output columns (c_col0[b]) pass the device arrays (else NULL).  Fails loudly
// if a CTA gave up waiting.
void tc_gemm_sliced(const SlicedMatrix& A, const SlicedMatrix& B, int n_max, double* C, i64 rs, i64 cs, i64 bs,
                    int batches, const int* b_row0, const int* b_rows, const int* c_col0, bool accumulate,
                    cudaStream_t s) {
    if (A.Kp != B.Kp) fail(GLI_ERR_INTERNAL, "sliced GEMM operands disagree on K");
    if (A.Kp <= 0 || A.Kp > 8192) fail(GLI_ERR_LIMIT, "sliced tensor-core GEMM supports 1 <= K <= 8192");
    if (A.slices != B.slices) fail(GLI_ERR_INTERNAL, "sliced GEMM operands disagree on the slice count");
    auto kernel = A.slices == 5 ? k_tc_gemm_sliced<5, 5> : A.slices == 7 ? k_tc_gemm_sliced<7, 8> : nullptr;
    if (!kernel) fail(GLI_ERR_INTERNAL, "no sliced GEMM variant for %d slices", A.slices);
    // the attribute is set on every call: cheap, and correct for every device
    GLI_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TCG_SMEM_REQUEST));
    // SlicedMatrix::rows counts the rows of one batch
    SlicedOp a{A.data.p, A.Kp, A.slice_stride(), A.rows * A.Kp, A.e.p, A.rows, (int)A.rows, nullptr};
    SlicedOp bop{B.data.p, B.Kp, B.slice_stride(), B.rows * B.Kp, B.e.p, B.rows, (int)B.rows, b_row0};
    OutView c{C, rs, cs, bs, c_col0};
    if ((n_max + TCG_BN - 1) / TCG_BN > 65535 || batches > 65535 || (a.rows + TCG_BM - 1) / TCG_BM > (i64)INT32_MAX)
        fail(GLI_ERR_LIMIT, "sliced tensor-core GEMM: launch grid too large");
    DevBuf<int> err(1, s);
    err.zero();
    dim3 grid((unsigned)((a.rows + TCG_BM - 1) / TCG_BM), (unsigned)((n_max + TCG_BN - 1) / TCG_BN), (unsigned)batches);
    kernel<<<grid, 128, TCG_SMEM_REQUEST, s>>>(a, bop, (int)A.Kp, c, accumulate ? 1 : 0, b_rows, err.p);
    GLI_CHECK_LAUNCH();
    int h_err = 0;
    GLI_CUDA(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    if (h_err) fail(GLI_ERR_INTERNAL, "tensor-core GEMM: an mbarrier wait expired");
}

}  // namespace gli

// ---------------------------------------------------------------------------
// Public entry point: C = A B^T with FP64 inputs and output, evaluated by the
// sliced int8 tensor-core GEMM with 7 slices and 8 product classes (about
// 2^-50 of max|a| max|b| per product term: FP64-level accuracy).
extern "C" int gli_b200_dgemm_sliced_dev(const double* d_A, glong lda, const double* d_B, glong ldb, double* d_C,
                                         glong ldc, glong M, glong N, glong K, void* stream) {
    gli::clear_error();
    try {
        if (M <= 0 || N <= 0 || K <= 0) gli::fail(GLI_ERR_ARGUMENT, "matrix sizes must be positive");
        if (!d_A || !d_B || !d_C) gli::fail(GLI_ERR_ARGUMENT, "device pointers must not be NULL");
        if (lda < K || ldb < K || ldc < N) gli::fail(GLI_ERR_ARGUMENT, "leading dimensions too small");
        if (M > (1 << 30) || N > (1 << 30)) gli::fail(GLI_ERR_LIMIT, "matrix too large");
        cudaStream_t s = stream ? (cudaStream_t)stream : gli::context().stream;
        gli::SlicedMatrix As, Bs;
        gli::slice_rows(d_A, M, (int)K, lda, 0, 1, 7, As, s);
        gli::slice_rows(d_B, N, (int)K, ldb, 0, 1, 7, Bs, s);
        gli::tc_gemm_sliced(As, Bs, (int)N, d_C, ldc, 1, 0, 1, nullptr, nullptr, nullptr, false, s);
    } catch (const gli::Failure&) {
        if (!getenv("GLI_B200_QUIET")) fprintf(stderr, "gausslectronitegrate_b200: %s\n", gli::last_message());
    }
    return gli::last_error();
}
