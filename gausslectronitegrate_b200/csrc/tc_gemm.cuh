// Sliced int8 tensor-core GEMM (tc_gemm.cu): FP64-accurate products on the
// tcgen05 tensor cores, used by the mixed form of the integral stages and by
// the FP64-level GEMM entry point.
//
// An FP64 operand row x is split as  x = 2^e sum_{p<S} 2^(-7(p+1)) d_p  with
// int8 slices d_p in [-64, 64] and one exponent e per row (|x| 2^-e < 1/2).
// Operands are stored pre-tiled for the kernel: rows in blocks of RB (128 for
// the A side, tile_n(S) for the B side), K in chunks of TC_BK = 64 bytes, and for each
// (row block, K chunk) the S slices one after another, each an RB x 64 byte
// tile in the tensor cores' K-major core-matrix order (8 rows x 16 bytes per
// core matrix, core matrices along K first).  One (row block, K chunk) is thus
// one contiguous run of S * RB * 64 bytes that a single bulk copy moves into
// shared memory.
#pragma once
#include "gli_internal.cuh"

namespace gli {

constexpr int MIXED_SLICES = 5;  // mixed form: products of slices p + q < 5 (~2^-36 per term)
constexpr int FP64_SLICES = 7;   // FP64 level: products p + q < 8 (~2^-50 per term)
constexpr int TC_BM = 128;       // A rows per tile (MMA M)
constexpr int TC_BK = 64;        // K bytes per chunk (two MMAs of K = 32)

// B rows per tile (MMA N): R accumulator regions of N int32 columns must fit the
// 512 tensor-memory columns, so 96 for the mixed form (5 x 96 = 480) and 64 for
// the FP64-level variant (8 x 64 = 512)
__host__ __device__ constexpr int tile_n(int S) { return S <= MIXED_SLICES ? 96 : 64; }

__host__ __device__ inline i64 tiled_offset(i64 rb, int kc, int p, int r, int k, int nkc, int S, int RB) {
    return ((rb * nkc + kc) * S + p) * (i64)RB * TC_BK + ((r >> 3) * (TC_BK / 16) + (k >> 4)) * 128 + (r & 7) * 16 +
           (k & 15);
}

// device view of a tiled sliced operand; e[] is indexed by padded row
// (row block * RB + row within the block)
struct TiledOperand {
    const int8_t* data = nullptr;
    const int* e = nullptr;
    int nkc = 0;  // K chunks (K padded to nkc * 64)
    int S = 0;    // slices
};

// stream-ordered owner
struct TiledSlices {
    DevBuf<int8_t> data;
    DevBuf<int> e;
    i64 blocks = 0;
    int RB = 0, nkc = 0, S = 0;
    void alloc(i64 row_blocks, int rb, int K, int nslices, cudaStream_t s) {
        blocks = row_blocks;
        RB = rb;
        S = nslices;
        nkc = (K + TC_BK - 1) / TC_BK;
        data.alloc((size_t)(blocks * RB) * nkc * TC_BK * S, s);
        e.alloc((size_t)(blocks * RB), s);
    }
    TiledOperand view() const { return TiledOperand{data.p, e.p, nkc, S}; }
};

// Slicing kernels.  Src is a device functor with
//   Ctx row(i64 r) const                    per-row context of source row r (bases,
//                                           maps: whatever is computed once per row)
//   double at(const Ctx& c, int k) const    value of that row at column k < K
//   i64 dest(i64 r) const                   padded row of source row r
//   i64 source(i64 d, i64 rows) const       source row of padded row d, or -1
//   bool valid(i64 r) const                 false beyond a count in device memory
// Every row x is split as 2^e sum_p 2^(-7(p+1)) d_p (|x| 2^-e < 1/2).

__device__ inline int slice_exponent(double mx) {
    int ex = 0;
    if (mx > 0) {
        frexp(mx, &ex);  // mx = f 2^ex, f in [0.5, 1)
        ex += 1;         // |x| 2^-ex < 1/2
    }
    return ex;
}

// 16 values -> S slices of 16 int8 each (packed in uint4)
__device__ inline void slice_piece(double (&v)[16], int S, uint4* out) {
    for (int p = 0; p < S; ++p) {
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const double t = v[j] * 128.0;
            const double d = rint(t);  // |t| <= 64
            v[j] = t - d;              // exact in FP64, |v| <= 1/2
            w[j >> 2] |= ((uint32_t)(uint8_t)(int8_t)(int)d) << (8 * (j & 3));
        }
        out[p] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

constexpr int SLICE_GROUP_NKC = 8;  // K <= 512 for the grouped kernel
constexpr int SLICE_GROUP_S = 7;

// One block per group of 8 padded rows (8 warps, warp w slices row 8 g + w).
// Lane l holds columns k = l + 32 j (coalesced reads of the source row); each
// value's slices go byte by byte into a shared-memory stage laid out in the
// tiled order, which the block then writes as contiguous 512-byte runs (8 rows
// x 64 bytes of K per slice and chunk).  Padding rows are written as zeros.
template <class Src>
__global__ void __launch_bounds__(256) k_slice_group(Src src, i64 rows, int K, int nkc, int S, int RB,
                                                     int8_t* __restrict__ dst, int* __restrict__ e) {
    __shared__ __align__(16) int8_t stage[SLICE_GROUP_NKC][SLICE_GROUP_S][512];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const i64 d0 = (i64)blockIdx.x * 8, dr = d0 + w;
    i64 sr = src.source(dr, rows);
    if (sr >= 0 && !src.valid(sr)) sr = -1;
    const int Kp = nkc * TC_BK;
    double x[16];
    double mx = 0;
    const auto rc = src.row(sr < 0 ? 0 : sr);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int k = lane + 32 * j;
        x[j] = (sr >= 0 && k < K) ? src.at(rc, k) : 0.0;
        mx = fmax(mx, fabs(x[j]));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const int ex = slice_exponent(mx);
    if (lane == 0) e[dr] = ex;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int k = lane + 32 * j;
        if (k >= Kp) break;
        double v = mx > 0 ? ldexp(x[j], -ex) : 0.0;
        // byte of column k: chunk k / 64, core matrix (k % 64) / 16, row w, byte k % 16
        int8_t* out = &stage[k >> 6][0][((k & 63) >> 4) * 128 + w * 16 + (k & 15)];
        for (int p = 0; p < S; ++p) {
            const double t = v * 128.0;
            const double d = rint(t);  // |t| <= 64
            v = t - d;                 // exact in FP64, |v| <= 1/2
            out[p * 512] = (int8_t)(int)d;
        }
    }
    __syncthreads();
    const i64 rb = d0 / RB;
    const int grp = (int)((d0 % RB) >> 3);
    for (int t = threadIdx.x; t < nkc * S * 32; t += blockDim.x) {
        const int kc = t / (S * 32), p = (t / 32) % S, q = t % 32;
        uint4* out = reinterpret_cast<uint4*>(dst + ((rb * nkc + kc) * S + p) * (i64)RB * TC_BK +
                                              (i64)grp * (TC_BK / 16) * 128);
        out[q] = reinterpret_cast<const uint4*>(&stage[kc][p][0])[q];
    }
}

// Rows of any length: one warp per source row, two passes over the row
// (maximum, then slices), 16-byte stores.  Padding rows are left unwritten.
template <class Src>
__global__ void k_slice_rows_any(Src src, i64 rows, int K, int nkc, int S, int RB, int8_t* __restrict__ dst,
                                 int* __restrict__ e) {
    const i64 r = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows || !src.valid(r)) return;  // uniform across the warp
    const auto rc = src.row(r);
    double mx = 0;
    for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(src.at(rc, k)));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const int ex = slice_exponent(mx);
    const i64 pr = src.dest(r);
    const i64 rb = pr / RB;
    const int rr = (int)(pr % RB);
    if (lane == 0) e[pr] = ex;
    const int pieces = nkc * (TC_BK / 16);
    for (int pc = lane; pc < pieces; pc += 32) {
        double v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int k = pc * 16 + j;
            v[j] = (k < K && mx > 0) ? ldexp(src.at(rc, k), -ex) : 0.0;
        }
        const int kc = pc / (TC_BK / 16), k0 = (pc % (TC_BK / 16)) * 16;
        uint4 sl[8];
        slice_piece(v, S, sl);
        for (int p = 0; p < S; ++p)
            *reinterpret_cast<uint4*>(dst + tiled_offset(rb, kc, p, rr, k0, nkc, S, RB)) = sl[p];
    }
}

// slices of source rows 0 .. rows-1 into a tiled operand with padded_rows rows
template <class Src>
void launch_slice(const Src& src, i64 rows, i64 padded_rows, int K, int nkc, int S, int RB, int8_t* dst, int* e,
                  cudaStream_t s) {
    if (rows <= 0 || padded_rows <= 0) return;
    if (nkc <= SLICE_GROUP_NKC && S <= SLICE_GROUP_S && RB % 8 == 0)
        launch_kernel(k_slice_group<Src>, dim3((unsigned)(padded_rows / 8)), dim3(256), 0, s, src, rows, K, nkc, S, RB,
                   dst, e);
    else
        launch_kernel(k_slice_rows_any<Src>, dim3((unsigned)((rows * 32 + 255) / 256)), dim3(256), 0, s, src, rows, K,
                   nkc, S, RB, dst, e);
}

template <class Src>
void slice_tiled(const Src& src, i64 rows, int K, TiledSlices& out, cudaStream_t s) {
    launch_slice(src, rows, out.blocks * out.RB, K, out.nkc, out.S, out.RB, out.data.p, out.e.p, s);
}

// identity row placement (source row r = padded row r), for the functors below
#define GLI_IDENTITY_ROWS                                          \
    __device__ i64 dest(i64 r) const { return r; }                 \
    __device__ i64 source(i64 d, i64 rows) const { return d < rows ? d : -1; }

// source functors ----------------------------------------------------------------
// context of rows read contiguously from a base pointer
struct RowBase {
    const double* p;
};

struct DenseRows {  // row r at src + r * ld
    const double* src;
    i64 ld;
    __device__ RowBase row(i64 r) const { return {src + r * ld}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k]; }
    __device__ bool valid(i64) const { return true; }
    GLI_IDENTITY_ROWS
};

struct GatheredRows {  // row r at src + rowmap[r] * ld
    const double* src;
    const int* rowmap;
    i64 ld;
    __device__ RowBase row(i64 r) const { return {src + (i64)rowmap[r] * ld}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k]; }
    __device__ bool valid(i64) const { return true; }
    GLI_IDENTITY_ROWS
};

// Work of one launch.  The A side has a_rows valid rows per batch in a_blocks
// row blocks; batched A takes row block batch * a_blocks + m-tile, shared A
// takes the m-tile.  The B side is a list of tile_n(S)-row tiles (tiled row
// block t): tile t belongs to batch tile_batch[t], its columns are tile_col0[t]
// .. tile_col0[t] + tile_ncols[t] - 1 of the output (device arrays), or, with
// tile_batch NULL, one batch whose tile t covers columns tile_n(S) t .. of
// n_total (read from *n_dev in device memory when n_dev is set).
// Output element (row i of the batch, column j) is C[i * rs + j * cs].
struct TileWork {
    int a_rows = 0, a_blocks = 0, a_batched = 0;
    const int* tile_batch = nullptr;
    const int* tile_col0 = nullptr;
    const int* tile_ncols = nullptr;
    const int* tile_bblock = nullptr;  // B row block of tile t (default t: every tile its own rows)
    int n_total = 0;
    const int64_t* n_dev = nullptr;
    double* C = nullptr;
    i64 rs = 0, cs = 0;
};

// sets the kernels' shared-memory attribute on the current device (once per
// device); called before a CUDA graph capture, where it may not run
void tc_gemm_prepare();

// launches the tensor-core GEMM over ntiles B tiles x a_blocks m-tiles; a CTA
// that gives up waiting sets *d_err (with d_err NULL the call checks its own
// flag and synchronises the stream)
void tc_gemm_tiled(const TiledOperand& A, const TiledOperand& B, const TileWork& w, int ntiles, int* d_err,
                   cudaStream_t s);

}  // namespace gli
