// FP64 tensor-core tiles: mma.sync.m8n8k4.f64 over operand tiles that the
// caller gathers into shared memory with 8-byte cp.async copies.
//
// A block (4 warps) computes a 64 x BN tile of C = A B (BN = 32, 64, 80 or 144,
// chosen per Op) over K in chunks of 16, three chunks in flight (two for an Op
// that declares STAGES = 2: the 144-column tiles, so that three blocks still
// fit on an SM; cp.async groups, the waits are the hardware's own group waits,
// no flag spins).  Warp w owns the
// 32 x BN/2 quadrant (w & 1, w >> 1) as 4 x BN/16 m8n8 accumulators; per
// k-step of 4 it reads 4 A and BN/16 B fragments (one double each) for
// 4 BN/16 MMAs of 256 FMAs.  BN = 80 serves 65..80 and 129..160 columns in
// one and two column tiles (129 keys: 2 tiles instead of 3, measured 20%
// faster on the stage A shape); BN = 144 holds 129 keys in one tile (another
// 1.5%: the lattice gathers are made once).
//
// The operand sources are arbitrary: an Op class says, per tile element, where
// the double comes from (a strided matrix, a lattice-table gather, a gather
// through an index map) and where the results go.  Each operand tile is kept
// in shared memory in one of two layouts, chosen so that the thread mapping
// that coalesces the global reads also writes shared memory without bank
// conflicts, and so that the fragment reads (row = lane / 4, k = lane % 4) are
// conflict-free in both:
//   K-major  [k][row], rows + 4 doubles per k (rows are the unit-stride direction)
//   row-major [row][k], 20 doubles per row    (k is the unit-stride direction)
// (rows + 4 and 20 are 4 mod 16 doubles, so the 16 (row, k) pairs of a half
// warp's fragment read fall in distinct bank pairs.)
// Fragment layouts of m8n8k4 (PTX ISA, mma .f64 m8n8k4): A row = lane/4,
// k = lane%4; B k = lane%4, column = lane/4; C row = lane/4, columns
// 2 (lane%4) + {0, 1}.
#pragma once

#include <cooperative_groups.h>

#include <atomic>
#include <type_traits>

#include "gli_internal.cuh"

namespace gli {

constexpr int DM_BM = 64, DM_BN = 64, DM_BK = 16, DM_STAGES = 3, DM_THREADS = 128;
constexpr int DM_LDK = DM_BK + 4;          // row-major tile: doubles per row
constexpr int DM_LDR = DM_BM + 4;          // K-major 64-row tile: doubles per k
constexpr int DM_TILE_A = DM_BM * DM_LDK;  // doubles of the A tile (>= DM_BK * DM_LDR)
static_assert(DM_TILE_A >= DM_BK * DM_LDR, "operand tile too small for the K-major layout");

// doubles of a B tile of BN rows, and the shared memory of a launch
__host__ __device__ constexpr int dm_tile_b(int bn) { return bn * DM_LDK; }
__host__ __device__ constexpr int dm_smem(int bn, int stages = DM_STAGES) {
    return stages * (DM_TILE_A + dm_tile_b(bn)) * (int)sizeof(double);
}

// pipeline stages of an Op: Op::STAGES where it declares one, else DM_STAGES
template <class Op, class = void>
struct dm_stages_of {
    static constexpr int value = DM_STAGES;
};
template <class Op>
struct dm_stages_of<Op, std::void_t<decltype(Op::STAGES)>> {
    static constexpr int value = Op::STAGES;
};

// Thread tid's q-th element of a rows x 16 operand tile:
//   K-major (64 rows):  row = tid & 63,          k = (tid >> 6) + 2 q,  q < 8
//   row-major:          row = (tid >> 4) + 8 q,  k = tid & 15,          q < rows / 8
constexpr int DM_ELEMS = DM_BM * DM_BK / DM_THREADS;  // 8: the 64-row tiles

__device__ __forceinline__ int dm_kmajor_row(int tid) { return tid & 63; }
__device__ __forceinline__ int dm_kmajor_k(int tid, int q) { return (tid >> 6) + 2 * q; }
__device__ __forceinline__ int dm_rowmajor_row(int tid, int q) { return (tid >> 4) + 8 * q; }
__device__ __forceinline__ int dm_rowmajor_k(int tid) { return tid & 15; }
__device__ __forceinline__ int dm_kmajor_at(int row, int k) { return k * DM_LDR + row; }
__device__ __forceinline__ int dm_rowmajor_at(int row, int k) { return row * DM_LDK + k; }

// 8-byte asynchronous copy global -> shared; src-size 0 writes zeros (src must
// still be a valid address)
__device__ __forceinline__ void dm_cp8(double* dst, const double* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0)
                 : "memory");
}
// 16-byte copy of two consecutive doubles; bytes (0, 8 or 16) are read, the
// rest of the 16 written as zeros (src 16-byte aligned, valid even for 0)
__device__ __forceinline__ void dm_cp16(double* dst, const double* src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
// row-major tiles whose rows are contiguous in K: thread tid's q-th pair of
// elements (q < rows / 16) is row (tid >> 3) + 16 q, k = 2 (tid & 7) and k + 1
__device__ __forceinline__ int dm_pair_row(int tid, int q) { return (tid >> 3) + 16 * q; }
__device__ __forceinline__ int dm_pair_k(int tid) { return (tid & 7) * 2; }
// bytes of the pair (k, k + 1) that lie before the end of the K range
__device__ __forceinline__ int dm_pair_bytes(int k, int kend) { return k + 1 < kend ? 16 : (k < kend ? 8 : 0); }
__device__ __forceinline__ void dm_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void dm_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dm_mma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

template <bool KMAJOR>
__device__ __forceinline__ double dm_frag(const double* s, int row0, int k0, int lane) {
    return KMAJOR ? s[dm_kmajor_at(row0 + (lane >> 2), k0 + (lane & 3))]
                  : s[dm_rowmajor_at(row0 + (lane >> 2), k0 + (lane & 3))];
}

// Op interface (all device, const):
//   static constexpr bool A_KMAJOR, B_KMAJOR;  static constexpr int BN (32, 64,
//   80 or 144; K-major B tiles have 64 rows); optionally STAGES (2 or 3)
//   struct Block { int mvalid, nvalid, nk; ... };       the block's work item
//   struct AState; struct BState;                       per-thread cached row data
//   bool begin(Block&)                                  false: nothing to do (uniform)
//   void a_init(const Block&, AState&), b_init(...)
//   void a_issue(const Block&, AState&, int kc, double* tile)   cp.async of chunk kc
//   void b_issue(const Block&, BState&, int kc, double* tile)   (chunks issued in order)
//   void store(const Block&, int m, int n, double v_n, double v_n1)   C[m][n], C[m][n+1]
//
// Op::a_landed(const Block&, AState&, int kc, double* tile) (optional, when
// the Op declares A_LANDED): called by each thread once its own copies of
// chunk kc have landed and before the block's barrier, to adjust the elements
// it copied (in place, in shared memory)
template <class Op, class = void>
struct dm_a_landed {
    static constexpr bool value = false;
};
template <class Op>
struct dm_a_landed<Op, std::void_t<decltype(Op::A_LANDED)>> {
    static constexpr bool value = Op::A_LANDED;
};

// The k loop of one block; FULL: every m8n8 tile of the warp's quadrant holds
// data, so the MMAs run unpredicated (a runtime predicate per MMA costs about
// a fifth of the tensor-pipe throughput).
template <class Op, bool FULL>
__device__ __forceinline__ void dm_mainloop(const Op& op, const typename Op::Block& blk, typename Op::AState& as,
                                            typename Op::BState& bs, double* smem, int wm, int wn, int mt, int nt,
                                            double (&acc)[4][Op::BN / 16][2]) {
    constexpr int NJ = Op::BN / 16, STAGE = DM_TILE_A + dm_tile_b(Op::BN), NS = dm_stages_of<Op>::value;
    const int lane = threadIdx.x & 31;
    const int nk = blk.nk;
    for (int kc = 0; kc < nk; ++kc) {
        dm_wait<NS - 2>();  // chunk kc has landed (this thread's copies)
        if constexpr (dm_a_landed<Op>::value) op.a_landed(blk, as, kc, smem + (kc % NS) * STAGE);
        __syncthreads();    // ... everyone's; and chunk kc - 1 is consumed
        const int nx = kc + NS - 1;
        if (nx < nk) {
            const int st = nx % NS;
            op.a_issue(blk, as, nx, smem + st * STAGE);
            op.b_issue(blk, bs, nx, smem + st * STAGE + DM_TILE_A);
        }
        dm_commit();
        const double* a_s = smem + (kc % NS) * STAGE;
        const double* b_s = a_s + DM_TILE_A;
#pragma unroll
        for (int k0 = 0; k0 < DM_BK; k0 += 4) {
            double af[4], bf[NJ];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = dm_frag<Op::A_KMAJOR>(a_s, wm + 8 * i, k0, lane);
#pragma unroll
            for (int j = 0; j < NJ; ++j) bf[j] = dm_frag<Op::B_KMAJOR>(b_s, wn + 8 * j, k0, lane);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < NJ; ++j)
                    if (FULL || (i < mt && j < nt)) dm_mma(acc[i][j], af[i], bf[j]);
        }
    }
}

// blocks per SM a launch is compiled for: Op::MIN_BLOCKS where declared, else 3
template <class Op, class = void>
struct dm_blocks_of {
    static constexpr int value = 3;
};
template <class Op>
struct dm_blocks_of<Op, std::void_t<decltype(Op::MIN_BLOCKS)>> {
    static constexpr int value = Op::MIN_BLOCKS;
};

// Split K inside a thread-block cluster (CLUSTER = true): the launch's
// gridDim.z chunks of K form one cluster of gridDim.z (<= 8) blocks; each
// block leaves its partial tile in its own shared memory, and after a cluster
// barrier every block sums its share of the tile's rows over the cluster's
// blocks through distributed shared memory, in the order of their ranks (the
// same order on every run), and stores it.  The Op then writes every part to
// the same destination (part stride 0).  Every block of a cluster reaches both
// cluster barriers: a block without work contributes zeros.
constexpr int DM_RED_LD = 2;  // doubles of padding per reduction-tile row

template <class Op, bool CLUSTER>
__device__ __forceinline__ void dm_cluster_reduce(const Op& op, const typename Op::Block& blk, bool active,
                                                  double* smem, int wm, int wn, int mt, int nt,
                                                  const double (&acc)[4][Op::BN / 16][2]) {
    constexpr int NJ = Op::BN / 16, LD = Op::BN + DM_RED_LD;
    namespace cg = cooperative_groups;
    const int lane = threadIdx.x & 31;
    __syncthreads();  // every warp is done with the operand tiles
    // this block's partial tile, zeros where it has none
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const bool has = active && i < mt && j < nt;
            double* d = smem + (wm + 8 * i + (lane >> 2)) * LD + wn + 8 * j + 2 * (lane & 3);
            d[0] = has ? acc[i][j][0] : 0.0;
            d[1] = has ? acc[i][j][1] : 0.0;
        }
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    const int P = (int)cl.num_blocks(), r = (int)cl.block_rank();
    if (active) {
        // block r sums rows [r0, r1) of the tile: per column pair, the P
        // partial pairs are loaded first (16-byte distributed shared-memory
        // loads, all in flight together) and then added in rank order
        constexpr int PAIRS = Op::BN / 2;
        const int r0 = (DM_BM * r) / P, r1 = (DM_BM * (r + 1)) / P;
        const double2* part[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            part[q] = reinterpret_cast<const double2*>(cl.map_shared_rank(smem, q < P ? q : 0));
        for (int e = r0 * PAIRS + threadIdx.x; e < r1 * PAIRS; e += blockDim.x) {
            const int row = e / PAIRS, c = 2 * (e % PAIRS);
            const int off = (row * LD + c) / 2;  // LD and c are even: 16-byte aligned pairs
            double2 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (q < P) v[q] = part[q][off];
            double v0 = v[0].x, v1 = v[0].y;
#pragma unroll
            for (int q = 1; q < 8; ++q)
                if (q < P) {
                    v0 += v[q].x;
                    v1 += v[q].y;
                }
            op.store(blk, row, c, v0, v1);
        }
    }
    cl.sync();  // no block leaves while another still reads its tile
}

// Tail split (an Op that declares TAIL_SPLIT): the last, partial wave of a
// launch would leave most SMs idle, so its m tiles are each computed by two
// blocks over the two halves of K, and the blocks of a full wave's worth of
// tiles run whole before them.  Both halves write their partial tile to
// global scratch in the threads' own fragment order (coalesced, no shared
// memory), then take a ticket for the tile; the second to arrive adds the
// other's partial to its own and stores the sum (a + b = b + a exactly, so
// the result does not depend on which half came second), and resets the
// ticket for the next evaluation.  No block waits on another.
//   Op::split_half()  -1 for a whole tile, else 0 or 1 (uniform in a block)
//   Op::split_slot()  the tile's scratch slot; Op::ws, Op::tickets
template <class Op, class = void>
struct dm_tail_split {
    static constexpr bool value = false;
};
template <class Op>
struct dm_tail_split<Op, std::void_t<decltype(Op::TAIL_SPLIT)>> {
    static constexpr bool value = Op::TAIL_SPLIT;
};

template <class Op>
__device__ __forceinline__ void dm_split_store(const Op& op, const typename Op::Block& blk, int half, int wm, int wn,
                                               int mt, int nt, const double (&acc)[4][Op::BN / 16][2]) {
    constexpr int NJ = Op::BN / 16, TILE = DM_BM * Op::BN;
    const int lane = threadIdx.x & 31, slot = op.split_slot();
    __shared__ unsigned s_ticket;
    double* mine = op.ws + ((i64)slot * 2 + half) * TILE;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j)
            if (i < mt && j < nt) {
                __stcg(mine + ((i * NJ + j) * 2) * DM_THREADS + threadIdx.x, acc[i][j][0]);
                __stcg(mine + ((i * NJ + j) * 2 + 1) * DM_THREADS + threadIdx.x, acc[i][j][1]);
            }
    __threadfence();  // the partial is visible before the ticket is taken
    __syncthreads();
    if (threadIdx.x == 0) s_ticket = atomicAdd(op.tickets + slot, 1u);
    __syncthreads();
    if (s_ticket == 0) return;  // the other half arrives second and sums
    __threadfence();
    const double* other = op.ws + ((i64)slot * 2 + (half ^ 1)) * TILE;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j)
            if (i < mt && j < nt) {
                const double o0 = __ldcg(other + ((i * NJ + j) * 2) * DM_THREADS + threadIdx.x);
                const double o1 = __ldcg(other + ((i * NJ + j) * 2 + 1) * DM_THREADS + threadIdx.x);
                op.store(blk, wm + 8 * i + (lane >> 2), wn + 8 * j + 2 * (lane & 3), acc[i][j][0] + o0,
                         acc[i][j][1] + o1);
            }
    if (threadIdx.x == 0) op.tickets[slot] = 0u;
}

template <class Op, bool CLUSTER = false>
__global__ void __launch_bounds__(DM_THREADS, dm_blocks_of<Op>::value) k_dmma(const Op op) {
    constexpr int NJ = Op::BN / 16, STAGE = DM_TILE_A + dm_tile_b(Op::BN), NS = dm_stages_of<Op>::value;
    static_assert(Op::BN == 64 || ((Op::BN == 80 || Op::BN == 32 || Op::BN == 144) && !Op::B_KMAJOR),
                  "column tiles of 64, or 32, 80 and 144 read row-major");
    static_assert(NS >= 2 && NS <= 3, "two or three stages");
    static_assert(!CLUSTER || DM_BM * (Op::BN + DM_RED_LD) <= NS * STAGE, "reduction tile exceeds the operand ring");
    extern __shared__ __align__(16) double dm_smem[];
    typename Op::Block blk;
    const bool active = op.begin(blk);
    if (!active) {
        if constexpr (CLUSTER) {
            double none[4][NJ][2];
            dm_cluster_reduce<Op, CLUSTER>(op, blk, false, dm_smem, 0, 0, 0, 0, none);
        }
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * (Op::BN / 2);
    typename Op::AState as;
    typename Op::BState bs;
    op.a_init(blk, as);
    op.b_init(blk, bs);
#pragma unroll
    for (int st = 0; st < NS - 1; ++st) {
        if (st < blk.nk) {
            op.a_issue(blk, as, st, dm_smem + st * STAGE);
            op.b_issue(blk, bs, st, dm_smem + st * STAGE + DM_TILE_A);
        }
        dm_commit();
    }
    // m8 / n8 tiles of this warp's quadrant that hold rows / columns (warp-uniform)
    const int mt = min(4, max(0, (blk.mvalid - wm + 7) >> 3));
    const int nt = min(NJ, max(0, (blk.nvalid - wn + 7) >> 3));
    double acc[4][NJ][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    if (mt == 4 && nt == NJ)
        dm_mainloop<Op, true>(op, blk, as, bs, dm_smem, wm, wn, mt, nt, acc);
    else
        dm_mainloop<Op, false>(op, blk, as, bs, dm_smem, wm, wn, mt, nt, acc);
    dm_wait<0>();
    if constexpr (CLUSTER) {
        dm_cluster_reduce<Op, CLUSTER>(op, blk, true, dm_smem, wm, wn, mt, nt, acc);
        return;
    }
    if constexpr (dm_tail_split<Op>::value) {
        const int half = op.split_half();
        if (half >= 0) {
            dm_split_store(op, blk, half, wm, wn, mt, nt, acc);
            return;
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j)
            if (i < mt && j < nt)
                op.store(blk, wm + 8 * i + (lane >> 2), wn + 8 * j + 2 * (lane & 3), acc[i][j][0], acc[i][j][1]);
}

// (three blocks per SM: 3 x 60 or 69 KB of shared memory, at most 170 registers)

// shared memory above the 48 KB default: set once per device and Op type,
// outside any graph capture (cudaFuncSetAttribute is not a stream operation)
template <class Op, bool CLUSTER = false>
void dmma_prepare() {
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    GLI_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
    if (bit && (done.load() & bit)) return;
    GLI_CUDA(cudaFuncSetAttribute(k_dmma<Op, CLUSTER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  dm_smem(Op::BN, dm_stages_of<Op>::value)));
    done.fetch_or(bit);
}

// blocks of k_dmma<Op> resident on one SM (registers and shared memory)
template <class Op>
int dmma_blocks_per_sm() {
    static std::atomic<int> cached{0};
    int v = cached.load();
    if (v > 0) return v;
    dmma_prepare<Op>();
    GLI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_dmma<Op>, DM_THREADS,
                                                           dm_smem(Op::BN, dm_stages_of<Op>::value)));
    v = v > 0 ? v : 1;
    cached.store(v);
    return v;
}

// one launch of k_dmma<Op> on grid `grid`
template <class Op>
void dmma_launch(const Op& op, dim3 grid, cudaStream_t s) {
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
    dmma_prepare<Op>();
    launch_kernel(k_dmma<Op>, grid, dim3(DM_THREADS), dm_smem(Op::BN, dm_stages_of<Op>::value), s, op);
}

// the same with K split over grid.z (2..8) blocks that sum their partial tiles
// in a cluster (the Op's part stride must be 0)
template <class Op>
void dmma_launch_cluster(const Op& op, dim3 grid, cudaStream_t s) {
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
    if (grid.z == 1) return dmma_launch(op, grid, s);
    if (grid.z > 8) fail(GLI_ERR_INTERNAL, "cluster split of %u parts", grid.z);
    dmma_prepare<Op, true>();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(DM_THREADS);
    cfg.dynamicSmemBytes = dm_smem(Op::BN, dm_stages_of<Op>::value);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = grid.z;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    GLI_CUDA(cudaLaunchKernelEx(&cfg, k_dmma<Op, true>, op));
    count_launch();
}

}  // namespace gli
