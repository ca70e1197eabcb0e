// Tensor-core (tcgen05) FP64-accurate GEMM by int8 slicing, for sm_100a.
//
//   C[i][j] = sum_k A[i][k] B[j][k]      (A, B: FP64 rows split into S int8 slices)
//
// With a_i = 2^ea sum_p 2^(-7(p+1)) A_p[i] and b_j likewise, the product is
//   2^(ea+eb) sum_{p,q} 2^(-7(p+q+2)) (A_p . B_q)
// where every A_p . B_q is an exact int8 x int8 -> int32 dot product on the
// tensor cores.  Pairs with p + q >= R are below the target precision and are
// dropped; all pairs with the same p + q share one int32 accumulator region in
// tensor memory (exact: |sum| <= 8 * 64 * 64 * K < 2^31 for K <= 8192).  The
// epilogue converts each region to FP64, scales it by 2^(-7(p+q+2)), sums the
// regions and applies the row and column exponents.  Two variants are built:
// S = 5, R = 5 (about 2^-36 of max|a| max|b| per product term: the mixed form of
// the integral stages) and S = 7, R = 8 (about 2^-50: FP64 level).
//
// One CTA computes a 128 x N tile of C (N = tile_n(S): 96 for S = 5, 64 for
// S = 7) with 256 threads:
//   * warp 0 allocates 512 tensor-memory columns (R regions of N used);
//   * lane 0 of warp 0 is the producer: for every K chunk of 64 bytes it
//     issues two bulk copies (all S slices of the A tile, all S slices of the B
//     tile: one contiguous run each in the pre-tiled layout) into a ring of
//     NST shared-memory stages, completing on the stage's `full` mbarrier;
//   * lane 0 of warp 1 issues the MMAs: per chunk, for every kept slice pair
//     (p, q) two MMAs (K = 32 each) of the A_p tile with the B_q tile into
//     region p + q, then commits to the stage's `empty` mbarrier, which hands
//     the stage back to the producer; after the last chunk it commits to `done`;
//   * all eight warps wait on `done`; warp w reads TMEM lanes 32 (w % 4) ..
//     +31 (its rows) of every region for half of the columns with tcgen05.ld,
//     combines the regions exactly in int64 and converts once to FP64.
// Every mbarrier wait is bounded by wall time (1 s).  On expiry the CTA records
// an error, stops issuing, waits (bounded) for the work it issued, frees its
// tensor memory and returns.  The kernel uses no cluster and no multicast.
#include <stdint.h>
#include <stdlib.h>

#include <atomic>

#include "tc_gemm.cuh"

namespace gli {

constexpr int TC_TMEM_COLS = 512;
constexpr uint64_t TC_WAIT_NS = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// shared-memory matrix descriptor: K-major, no swizzle (core matrix = 8 rows x 16 B);
// LBO = byte distance between core matrices along K, SBO = between 8-row groups
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: s8 x s8 -> s32, both operands K-major, M x N
__host__ __device__ constexpr uint32_t idesc_s8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_s8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// bounded wait: false after TC_WAIT_NS of wall time (or 2^30 polls)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    for (unsigned it = 0; it < (1u << 30); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 63u && global_ns() - t0 > TC_WAIT_NS) return false;
    }
    return false;
}

// global -> shared bulk copy (no tensor map, no multicast), completing on bar
__device__ __forceinline__ void bulk_copy(void* dst_smem, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
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

template <int S>
__host__ __device__ constexpr int stages_for() { return S <= 5 ? 3 : 2; }

template <int S>
__host__ __device__ constexpr int smem_bytes() { return stages_for<S>() * S * (TC_BM + tile_n(S)) * TC_BK; }

// first slice p of the pairs (p, q) with p + q = r, p, q < S
__host__ __device__ constexpr int first_p(int r, int S) { return r < S ? 0 : r - (S - 1); }

// 2^e for |e| <= 1000, built from its bit pattern (exact)
__device__ __forceinline__ double pow2(int e) { return __hiloint2double((1023 + e) << 20, 0); }

// the regions of one output, combined exactly in integers and converted once:
// region r carries weight 2^(-7 (r + 2))
template <int R>
__device__ __forceinline__ double combine_regions(const uint32_t (&v)[R][16], int j) {
    if constexpr (R <= 5) {
        long long s = (int32_t)v[0][j];  // |region| < 2^29: R <= 5 regions fit 2^57
#pragma unroll
        for (int r = 1; r < R; ++r) s = s * 128 + (int32_t)v[r][j];
        return (double)s * pow2(-7 * (R + 1));
    } else {
        long long hi = (int32_t)v[0][j], lo = (int32_t)v[4][j];
#pragma unroll
        for (int r = 1; r < 4; ++r) hi = hi * 128 + (int32_t)v[r][j];
#pragma unroll
        for (int r = 5; r < R; ++r) lo = lo * 128 + (int32_t)v[r][j];
        return fma((double)hi, pow2(-35), (double)lo * pow2(-7 * (R + 1)));
    }
}

template <int S, int R>
__global__ void __launch_bounds__(256, 1) k_tc_gemm(TiledOperand A, TiledOperand B, TileWork w, int* __restrict__ err) {
    constexpr int TC_BN = tile_n(S);
    static_assert(R * TC_BN <= TC_TMEM_COLS, "tensor-memory regions exceed 512 columns");
    static_assert(TC_BN % 16 == 0 && TC_BN >= 16 && TC_BN <= 256, "MMA N out of range for M = 128");
    static_assert(R <= 2 * S - 1, "more regions than slice pairs");
    constexpr int NST = stages_for<S>();
    constexpr uint32_t A_BYTES = S * TC_BM * TC_BK, B_BYTES = S * TC_BN * TC_BK;
    constexpr uint32_t STAGE = A_BYTES + B_BYTES;
    extern __shared__ __align__(128) uint8_t tc_smem[];
    __shared__ uint64_t full[NST], empty[NST], done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t = blockIdx.x, mt = blockIdx.y;
    const int batch = w.tile_batch ? w.tile_batch[t] : 0;
    const int col0 = w.tile_batch ? w.tile_col0[t] : t * TC_BN;
    const int n_total = w.n_dev ? (int)*w.n_dev : w.n_total;
    const int ncols = w.tile_batch ? w.tile_ncols[t] : min(TC_BN, n_total - t * TC_BN);
    const int rows_valid = min(TC_BM, w.a_rows - mt * TC_BM);
    if (ncols <= 0 || rows_valid <= 0) return;  // uniform across the CTA
    const i64 a_rb = w.a_batched ? (i64)batch * w.a_blocks + mt : mt;
    const int nkc = A.nkc;
    const int8_t* gA = A.data + a_rb * nkc * (i64)A_BYTES;
    const i64 b_rb = w.tile_bblock ? w.tile_bblock[t] : t;
    const int8_t* gB = B.data + b_rb * nkc * (i64)B_BYTES;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < NST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    if (warp == 0 && lane == 0) {
        // producer
        for (int kc = 0; kc < nkc && !abort_flag; ++kc) {
            const int s = kc % NST, round = kc / NST;
            if (round > 0 && !mbar_wait(&empty[s], (round - 1) & 1)) {
                atomicExch(err, 1);
                abort_flag = 1;
                break;
            }
            uint8_t* st = tc_smem + s * STAGE;
            mbar_expect_tx(&full[s], STAGE);
            bulk_copy(st, gA + (i64)kc * A_BYTES, A_BYTES, &full[s]);
            bulk_copy(st + A_BYTES, gB + (i64)kc * B_BYTES, B_BYTES, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        constexpr uint32_t idesc = idesc_s8(TC_BM, TC_BN);
        constexpr uint32_t SBO = (TC_BK / 16) * 128;
        for (int kc = 0; kc < nkc; ++kc) {
            const int s = kc % NST, round = kc / NST;
            if (abort_flag || !mbar_wait(&full[s], round & 1)) {
                atomicExch(err, 2);
                abort_flag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(tc_smem + s * STAGE);
            const uint32_t sb = sa + A_BYTES;
#pragma unroll
            for (int p = 0; p < S; ++p) {
#pragma unroll
                for (int q = 0; q < S; ++q) {
                    if (p + q >= R) continue;
#pragma unroll
                    for (int kk = 0; kk < TC_BK; kk += 32) {
                        const uint64_t da = umma_desc(sa + p * TC_BM * TC_BK + (kk / 16) * 128, 128, SBO);
                        const uint64_t db = umma_desc(sb + q * TC_BN * TC_BK + (kk / 16) * 128, 128, SBO);
                        // the first MMA into a region (chunk 0, its first pair, k step 0) overwrites
                        const bool overwrite = kc == 0 && kk == 0 && p == first_p(p + q, S);
                        mma_s8(tmem + (uint32_t)((p + q) * TC_BN), da, db, idesc, overwrite ? 0u : 1u);
                    }
                }
            }
            mma_commit(&empty[s]);
        }
        mma_commit(&done);  // arrives once every MMA this thread issued has completed
    }
    __syncwarp();  // lanes 1-31 of warps 0 and 1 wait here for their lane 0

    // everyone: wait for the accumulators (bounded); on expiry skip the epilogue
    if (!mbar_wait(&done, 0)) {
        if (lane == 0) atomicExch(err, 3);
        abort_flag = 1;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();

    if (!abort_flag) {
        // eight warps: warp w reads TMEM lanes 32 (w % 4) .. (its rows) and half
        // of the columns
        const int quarter = warp & 3, half = warp >> 2;
        const int row = quarter * 32 + lane;
        const bool live = row < rows_valid;
        const int ea = live ? A.e[a_rb * TC_BM + row] : 0;
        double* crow = w.C + (i64)(mt * TC_BM + row) * w.rs;
        const int* eb = B.e + b_rb * TC_BN;
        constexpr int HALF = TC_BN / 2;
        static_assert(HALF % 16 == 0, "column halves of whole 16-column loads");
        for (int c0 = half * HALF; c0 < (half + 1) * HALF; c0 += 16) {
            uint32_t v[R][16];
#pragma unroll
            for (int r = 0; r < R; ++r)
                tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(r * TC_BN + c0), v[r]);
            if (live) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int c = c0 + j;
                    if (c < ncols) {
                        const int ex = ea + eb[c];
                        const double acc = combine_regions<R>(v, j);
                        crow[(i64)(col0 + c) * w.cs] = (ex >= -1000 && ex <= 1000) ? acc * pow2(ex) : ldexp(acc, ex);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

// host ---------------------------------------------------------------------------
static std::atomic<unsigned> g_prepared_devices{0};  // bit d: attributes set on device d

void tc_gemm_prepare() {
    int dev = 0;
    GLI_CUDA(cudaGetDevice(&dev));
    if (dev < 32 && (g_prepared_devices.load() >> dev) & 1u) return;
    GLI_CUDA(cudaFuncSetAttribute(k_tc_gemm<MIXED_SLICES, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem_bytes<MIXED_SLICES>()));
    GLI_CUDA(cudaFuncSetAttribute(k_tc_gemm<FP64_SLICES, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem_bytes<FP64_SLICES>()));
    if (dev < 32) g_prepared_devices.fetch_or(1u << dev);
}

template <int S, int R>
static void launch_variant(const TiledOperand& A, const TiledOperand& B, const TileWork& w, int ntiles, int* err,
                           cudaStream_t s) {
    constexpr int smem = smem_bytes<S>();
    dim3 grid((unsigned)ntiles, (unsigned)w.a_blocks);
    launch_kernel(k_tc_gemm<S, R>, grid, dim3(256), smem, s, A, B, w, err);
}

void tc_gemm_tiled(const TiledOperand& A, const TiledOperand& B, const TileWork& w, int ntiles, int* d_err,
                   cudaStream_t s) {
    if (ntiles <= 0 || w.a_blocks <= 0 || w.a_rows <= 0) return;
    if (A.nkc != B.nkc) fail(GLI_ERR_INTERNAL, "sliced GEMM operands disagree on K");
    if (A.S != B.S) fail(GLI_ERR_INTERNAL, "sliced GEMM operands disagree on the slice count");
    if (A.nkc <= 0 || A.nkc * TC_BK > 8192) fail(GLI_ERR_LIMIT, "sliced tensor-core GEMM supports 1 <= K <= 8192");
    if (w.a_blocks > 65535) fail(GLI_ERR_LIMIT, "sliced tensor-core GEMM: more than 65535 row tiles");
    tc_gemm_prepare();
    DevBuf<int> own;
    int* err = d_err;
    if (!err) {
        own.alloc(1, s);
        own.zero();
        err = own.p;
    }
    if (A.S == MIXED_SLICES)
        launch_variant<MIXED_SLICES, 5>(A, B, w, ntiles, err, s);
    else if (A.S == FP64_SLICES)
        launch_variant<FP64_SLICES, 8>(A, B, w, ntiles, err, s);
    else
        fail(GLI_ERR_INTERNAL, "no sliced GEMM variant for %d slices", A.S);
    if (!d_err) {
        int h = 0;
        GLI_CUDA(cudaMemcpyAsync(&h, own.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s));
        if (h) fail(GLI_ERR_INTERNAL, "tensor-core GEMM: an mbarrier wait expired (code %d)", h);
    }
}

}  // namespace gli

// ---------------------------------------------------------------------------
// Public entry point: C = A B^T with FP64 inputs and output (row-major, leading
// dimensions lda, ldb, ldc), evaluated by the sliced int8 tensor-core GEMM with
// 7 slices and 8 product classes: FP64-level accuracy (about 2^-50 of
// max|a_i| max|b_j| per product term).
extern "C" int gli_b200_dgemm_sliced_dev(const double* d_A, glong lda, const double* d_B, glong ldb, double* d_C,
                                         glong ldc, glong M, glong N, glong K, void* stream) {
    gli::clear_error();
    try {
        if (M <= 0 || N <= 0 || K <= 0) gli::fail(GLI_ERR_ARGUMENT, "matrix sizes must be positive");
        if (!d_A || !d_B || !d_C) gli::fail(GLI_ERR_ARGUMENT, "device pointers must not be NULL");
        if (lda < K || ldb < K || ldc < N) gli::fail(GLI_ERR_ARGUMENT, "leading dimensions too small");
        if (K > 8192) gli::fail(GLI_ERR_LIMIT, "K above 8192");
        if (M > (glong)65535 * gli::TC_BM || N > ((glong)1 << 30)) gli::fail(GLI_ERR_LIMIT, "matrix too large");
        cudaStream_t s = stream ? (cudaStream_t)stream : gli::context().stream;
        constexpr int BN = gli::tile_n(gli::FP64_SLICES);
        const gli::i64 mb = (M + gli::TC_BM - 1) / gli::TC_BM, nb = (N + BN - 1) / BN;
        gli::TiledSlices As, Bs;
        As.alloc(mb, gli::TC_BM, (int)K, gli::FP64_SLICES, s);
        Bs.alloc(nb, BN, (int)K, gli::FP64_SLICES, s);
        gli::slice_tiled(gli::DenseRows{d_A, lda}, M, (int)K, As, s);
        gli::slice_tiled(gli::DenseRows{d_B, ldb}, N, (int)K, Bs, s);
        gli::TileWork w;
        w.a_rows = (int)M;
        w.a_blocks = (int)mb;
        w.n_total = (int)N;
        w.C = d_C;
        w.rs = ldc;
        w.cs = 1;
        gli::tc_gemm_tiled(As.view(), Bs.view(), w, (int)nb, nullptr, s);
    } catch (const gli::Failure&) {
        if (!getenv("GLI_B200_QUIET")) fprintf(stderr, "gausslectronitegrate_b200: %s\n", gli::last_message());
    }
    return gli::last_error();
}
