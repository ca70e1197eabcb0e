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

// Writes the slices of source rows r = 0 .. rows-1 (src(r, k), k < K) to their
// padded rows src.dest(r); rows with !src.valid(r) (beyond a count that lives
// in device memory) are skipped.  One warp per row; for K <= 512 each lane
// gathers one 16-value piece of the row once into registers, longer rows are
// read twice (maximum, then slices).  Src: device functor with `double
// operator()(i64 r, int k) const`, `i64 dest(i64 r) const` and `bool valid(i64
// r) const`.
template <class Src>
__global__ void k_slice_tiled(Src src, i64 rows, int K, int nkc, int S, int RB, int8_t* __restrict__ dst,
                              int* __restrict__ e) {
    const i64 r = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows || !src.valid(r)) return;  // uniform across the warp
    const int pieces = nkc * (TC_BK / 16);
    const bool one_pass = pieces <= 32;
    double x[16];
    double mx = 0;
    if (one_pass) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int k = lane * 16 + j;
            x[j] = (lane < pieces && k < K) ? src(r, k) : 0.0;
            mx = fmax(mx, fabs(x[j]));
        }
    } else {
        for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(src(r, k)));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int ex = 0;
    if (mx > 0) {
        frexp(mx, &ex);  // mx = f 2^ex, f in [0.5, 1)
        ex += 1;         // |x| 2^-ex < 1/2
    }
    const i64 pr = src.dest(r);
    const i64 rb = pr / RB;
    const int rr = (int)(pr % RB);
    if (lane == 0) e[pr] = ex;
    for (int pc = lane; pc < pieces; pc += 32) {
        double v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int k = pc * 16 + j;
            const double xv = one_pass ? x[j] : (k < K ? src(r, k) : 0.0);
            v[j] = mx > 0 ? ldexp(xv, -ex) : 0.0;
        }
        const int kc = pc / (TC_BK / 16), k0 = (pc % (TC_BK / 16)) * 16;
        for (int p = 0; p < S; ++p) {
            uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const double t = v[j] * 128.0;
                const double d = rint(t);  // |t| <= 64
                v[j] = t - d;              // exact in FP64, |v| <= 1/2
                w[j >> 2] |= ((uint32_t)(uint8_t)(int8_t)(int)d) << (8 * (j & 3));
            }
            *reinterpret_cast<uint4*>(dst + tiled_offset(rb, kc, p, rr, k0, nkc, S, RB)) =
                make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

template <class Src>
void slice_tiled(const Src& src, i64 rows, int K, TiledSlices& out, cudaStream_t s) {
    if (rows <= 0) return;
    k_slice_tiled<Src><<<(unsigned)((rows * 32 + 255) / 256), 256, 0, s>>>(src, rows, K, out.nkc, out.S, out.RB,
                                                                          out.data.p, out.e.p);
    GLI_CHECK_LAUNCH();
}

// source functors ----------------------------------------------------------------
struct DenseRows {  // row r at src + r * ld
    const double* src;
    i64 ld;
    __device__ double operator()(i64 r, int k) const { return src[r * ld + k]; }
    __device__ i64 dest(i64 r) const { return r; }
    __device__ bool valid(i64) const { return true; }
};

struct GatheredRows {  // row r at src + rowmap[r] * ld
    const double* src;
    const int* rowmap;
    i64 ld;
    __device__ double operator()(i64 r, int k) const { return src[(i64)rowmap[r] * ld + k]; }
    __device__ i64 dest(i64 r) const { return r; }
    __device__ bool valid(i64) const { return true; }
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
