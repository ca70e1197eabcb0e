// Symmetry-reduced class enumeration on the device, bit-exact with
// enumerate_symmetry_reduced_erida_indices (src/erida_integrals.c:300-410) and
// enumerate_symmetry_reduced_eri_indices (src/eri_integrals.c:382-526).
//
// A candidate tuple is kept when no element of its orbit -- the 48 O_h images
// of the tuple and of its bias-shifted copies (a doubled box centre of +-1 on an
// axis admits the copy moved by that centre), combined with the index
// permutations i<->j (and k<->l, (ij)<->(kl) for ERI) -- has a smaller
// linearised index.  Images are computed arithmetically from the signed
// permutation matrices, so no 48 x N permutation tables are built.
//
// Candidates are generated so that the flat candidate order equals ascending
// index order: a slot is i (ERIDA: partners j ascending) or (i, j, k) (ERI:
// partners l ascending), and slots ascend with the index.
//
// A filter skips most candidates before the orbit test.  A candidate's index
// leads with its first point i, and an image of the tuple whose smallest point
// index lies below i is a smaller index, so no point of a canonical tuple has
// an O_h image below i: with omin[p] the smallest index among the 48 images of
// point p (the unshifted copies are part of every orbit), a canonical tuple has
// omin[i] = i and omin[q] >= i for each other point q.
//
// ERIDA, one pass (k_enum_collect): a thread per slot; each block gathers its
// survivors in shared memory and sorts them (within a block ascending index is
// the (slot, partner) order, and blocks cover increasing index ranges), then
// appends them to a scratch buffer; a scan of the blocks' counts and a copy
// place the runs in block order.  129^3: 1.4 ms.
//
// ERI, live slots: at 7^3, 168,092 of the 40 million slots (i, j, k) hold a
// canonical class, and a thread per slot leaves most lanes of a warp idle
// beside one busy slot.  The slots that pass the filter are compacted first
// (k_enum_live); a warp then takes each live slot's partner candidates 32 at
// a time in ascending order, keeps the survivors (placed in order by its
// ballots) in shared memory and appends them to a scratch buffer, and a scan
// of the slots' counts and a copy place the runs (k_enum_slots_collect).  7^3:
// 25 ms against 146 ms for a thread per slot in two passes.  (The same
// scheme for ERIDA, whose live slots have only 27 cheap candidates each,
// measured slower at 129^3: 3.6 against 1.4 ms; it serves the ERIDA tests of
// the live-slot fallback.)
//
// Fallbacks, when a block's or a slot's survivors exceed its buffer or the
// scratch buffer fills: two passes (count, scan, write), over the live slots
// (k_enum_slots) for ERI and over every slot (k_enum_erida) for ERIDA.  The
// thread-per-slot two passes of ERI (k_enum_eri) remain for the tests.  The
// output is sorted by construction on every path.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>

#include "symmetry.cuh"

namespace gli {

// ---------------------------------------------------------------------------
// ERIDA: slot i; partner coordinates j_a = -i_a - 1 + t_a, t_a in {0,1,2}
// (doubled box centre t_a - 1), ascending in (t_x, t_y, t_z) = ascending j.
template <class Emit>
__device__ inline void erida_candidates(const SymGrid& G, i64 i, Emit&& emit) {
    if (G.omin[i] != (int)i) return;
    int p[2][3];
    point_of(G, i, p[0]);
    for (int tx = 0; tx < 3; ++tx) {
        const int jx = -p[0][0] - 1 + tx;
        if (jx < -G.e || jx > G.e || jx < p[0][0]) continue;
        for (int ty = 0; ty < 3; ++ty) {
            const int jy = -p[0][1] - 1 + ty;
            if (jy < -G.e || jy > G.e) continue;
            for (int tz = 0; tz < 3; ++tz) {
                const int jz = -p[0][2] - 1 + tz;
                if (jz < -G.e || jz > G.e) continue;
                p[1][0] = jx;
                p[1][1] = jy;
                p[1][2] = jz;
                const i64 j = lin3(G, p[1]);
                if (G.omin[j] < (int)i) continue;
                const int bias[3] = {tx - 1, ty - 1, tz - 1};
                const i64 idx = i * G.N + j;
                if (canonical_pair(G, p, bias, idx)) emit(idx);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// ERI: one thread per (i, j, k); admissible l coordinates per axis keep the
// doubled box centre min + max in {-1, 0, 1}.
constexpr int MAX_AXIS = 72;  // room for L <= 63

// ascending admissible partner coordinates l for fixed lo/hi of (i, j, k)
__device__ inline int axis_partners(int lo, int hi, int e, int lmin, signed char* s) {
    int n = 0;
    for (int d = -1; d <= 1; ++d) {  // l < lo: centre l + hi
        const int l = d - hi;
        if (l >= -e && l < lo && l >= lmin) s[n++] = (signed char)l;
    }
    if (lo + hi >= -1 && lo + hi <= 1)  // lo <= l <= hi: centre lo + hi
        for (int l = lo; l <= hi; ++l)
            if (l >= lmin) s[n++] = (signed char)l;
    for (int d = -1; d <= 1; ++d) {  // l > hi: centre lo + l
        const int l = d - lo;
        if (l > hi && l <= e && l >= lmin) s[n++] = (signed char)l;
    }
    return n;
}

// ERI: slot t = (i, j, k)
template <class Emit>
__device__ inline void eri_candidates(const SymGrid& G, i64 t, Emit&& emit) {
    const i64 i = t / (G.N * G.N), j = (t / G.N) % G.N, k = t % G.N;
    if (G.omin[i] != (int)i || G.omin[j] < (int)i || G.omin[k] < (int)i) return;
    int p[4][3];
    point_of(G, i, p[0]);
    point_of(G, j, p[1]);
    point_of(G, k, p[2]);
    // reference x-ordering: i <= j, i <= k (and k <= l below) on the x coordinate
    if (p[0][0] <= p[1][0] && p[0][0] <= p[2][0]) {
        signed char sx[MAX_AXIS], sy[MAX_AXIS], sz[MAX_AXIS];
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(min(p[0][a], p[1][a]), p[2][a]);
            hi[a] = max(max(p[0][a], p[1][a]), p[2][a]);
        }
        const int nx = axis_partners(lo[0], hi[0], G.e, p[2][0], sx);
        const int ny = axis_partners(lo[1], hi[1], G.e, -G.e, sy);
        const int nz = axis_partners(lo[2], hi[2], G.e, -G.e, sz);
        const i64 base = ((i * G.N + j) * G.N + k) * G.N;
        for (int ax = 0; ax < nx; ++ax) {
            p[3][0] = sx[ax];
            const int bx = min(lo[0], p[3][0]) + max(hi[0], p[3][0]);
            for (int ay = 0; ay < ny; ++ay) {
                p[3][1] = sy[ay];
                const int by = min(lo[1], p[3][1]) + max(hi[1], p[3][1]);
                for (int az = 0; az < nz; ++az) {
                    p[3][2] = sz[az];
                    const i64 l = lin3(G, p[3]);
                    if (G.omin[l] < (int)i) continue;
                    const int bz = min(lo[2], p[3][2]) + max(hi[2], p[3][2]);
                    const int bias[3] = {bx, by, bz};
                    const i64 idx = base + l;
                    if (canonical_quad(G, p, bias, idx)) emit(idx);
                }
            }
        }
    }
}

template <int KIND, class Emit>
__device__ inline void slot_candidates(const SymGrid& G, i64 t, Emit&& emit) {
    if (KIND == 0)
        erida_candidates(G, t, emit);
    else
        eri_candidates(G, t, emit);
}

// smallest linear index among the 48 O_h images of each grid point
__global__ void k_orbit_min(SymGrid G, int* __restrict__ omin) {
    const i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= G.N) return;
    int q[3];
    point_of(G, p, q);
    i64 best = p;
    for (int g = 0; g < 48; ++g) {
        int r[3];
        oh_apply(g, q, r);
        best = min(best, lin3(G, r));
    }
    omin[p] = (int)best;
}

// ---------------------------------------------------------------------------
// two passes: survivors per slot, then each slot's survivors at its offset
template <bool WRITE>
__global__ void k_enum_erida(SymGrid G, uint32_t* __restrict__ counts, const uint64_t* __restrict__ offsets,
                             int64_t* __restrict__ out) {
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G.N) return;
    if (WRITE) {
        uint64_t w = offsets[i];
        erida_candidates(G, i, [&](i64 idx) { out[w++] = idx; });
    } else {
        uint32_t c = 0;
        erida_candidates(G, i, [&](i64) { ++c; });
        counts[i] = c;
    }
}

template <bool WRITE>
__global__ void k_enum_eri(SymGrid G, uint32_t* __restrict__ counts, const uint64_t* __restrict__ offsets,
                           int64_t* __restrict__ out) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= G.N * G.N * G.N) return;
    if (WRITE) {
        uint64_t w = offsets[t];
        eri_candidates(G, t, [&](i64 idx) { out[w++] = idx; });
    } else {
        uint32_t c = 0;
        eri_candidates(G, t, [&](i64) { ++c; });
        counts[t] = c;
    }
}

// ---------------------------------------------------------------------------
// one pass (ERIDA: blocks of slots; ERI: live slots)

struct EnumStatus {
    unsigned long long used;  // scratch entries reserved
    int overflow;             // 1: a block's (or slot's) survivors exceeded its buffer; 2: the scratch buffer filled
};

// ERIDA in one pass: a thread per slot, survivors sorted per block
constexpr int ENUM_BLOCK = 128;  // slots per block
constexpr int ENUM_CAP = 2048;   // survivors a block can hold (16 KB)

template <int KIND>
__global__ void __launch_bounds__(ENUM_BLOCK) k_enum_collect(SymGrid G, i64 slots, int64_t* __restrict__ scratch,
                                                             unsigned long long cap, uint32_t* __restrict__ run_n,
                                                             unsigned long long* __restrict__ run_off,
                                                             EnumStatus* __restrict__ st) {
    __shared__ int64_t buf[ENUM_CAP];
    __shared__ int n;
    __shared__ unsigned long long off;
    if (threadIdx.x == 0) n = 0;
    __syncthreads();
    const i64 t = (i64)blockIdx.x * ENUM_BLOCK + threadIdx.x;
    if (t < slots)
        slot_candidates<KIND>(G, t, [&](i64 idx) {
            const int k = atomicAdd(&n, 1);
            if (k < ENUM_CAP) buf[k] = idx;
        });
    __syncthreads();
    const int cnt = n;  // the same for every thread: the returns below are uniform
    if (cnt == 0 || cnt > ENUM_CAP) {
        if (threadIdx.x == 0) {
            run_n[blockIdx.x] = 0;
            if (cnt > ENUM_CAP) atomicOr(&st->overflow, 1);
        }
        return;
    }
    // bitonic sort, padded to a power of two with the largest index
    int np = 1;
    while (np < cnt) np <<= 1;
    for (int k = cnt + threadIdx.x; k < np; k += ENUM_BLOCK) buf[k] = LLONG_MAX;
    __syncthreads();
    for (int k = 2; k <= np; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < np; i += ENUM_BLOCK) {
                const int x = i ^ j;
                if (x > i) {
                    const int64_t a = buf[i], b = buf[x];
                    if ((a > b) == ((i & k) == 0)) {
                        buf[i] = b;
                        buf[x] = a;
                    }
                }
            }
            __syncthreads();
        }
    if (threadIdx.x == 0) {
        off = atomicAdd(&st->used, (unsigned long long)cnt);
        const bool fits = off + cnt <= cap;
        run_n[blockIdx.x] = fits ? (uint32_t)cnt : 0u;
        run_off[blockIdx.x] = off;
        if (!fits) atomicOr(&st->overflow, 2);
    }
    __syncthreads();
    if (off + cnt > cap) return;
    for (int k = threadIdx.x; k < cnt; k += ENUM_BLOCK) scratch[off + k] = buf[k];
}

// each slot's run from the scratch buffer to its place (dest: exclusive scan
// of the run lengths in slot order); one warp per run
__global__ void k_enum_place(const int64_t* __restrict__ scratch, const uint32_t* __restrict__ run_n,
                             const unsigned long long* __restrict__ run_off, const uint64_t* __restrict__ dest,
                             i64 runs, int64_t* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const i64 warps = (i64)gridDim.x * (blockDim.x >> 5);
    for (i64 r = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < runs; r += warps) {
        const uint32_t n = run_n[r];
        if (n == 0) continue;
        const int64_t* src = scratch + run_off[r];
        int64_t* dst = out + dest[r];
        for (uint32_t k = lane; k < n; k += 32) dst[k] = src[k];
    }
}

// scratch entries: ERIDA lists have L (L + 1) (L + 2) / 6 classes; ERI lists
// about N^4 / 3,900 at L = 7 (and a falling fraction beyond), so N^4 / 1024
// with a floor; at most 2^26 entries (512 MB); a list that does not fit takes
// the two passes
static i64 enum_scratch(int kind, const SymGrid& G) {
    const double L = G.L, N = (double)G.N;
    const double want = kind == 0 ? L * (L + 1) * (L + 2) / 6 + 1024 : N * N * N * N / 1024 + (1 << 20);
    return (i64)std::min(want, (double)((i64)1 << 26));
}

// one pass into out (allocated here); false when it did not fit
template <int KIND>
static bool enumerate_one_pass(const SymGrid& G, i64 slots, int64_t** d_out, i64* total, int num_sms,
                               cudaStream_t s) {
    const i64 runs = (slots + ENUM_BLOCK - 1) / ENUM_BLOCK;
    const i64 cap = enum_scratch(KIND, G);
    DevBuf<int64_t> scratch(cap, s);
    DevBuf<uint32_t> run_n(runs, s);
    DevBuf<unsigned long long> run_off(runs, s);
    DevBuf<EnumStatus> st(1, s);
    st.zero();
    k_enum_collect<KIND><<<(unsigned)runs, ENUM_BLOCK, 0, s>>>(G, slots, scratch.p, (unsigned long long)cap, run_n.p,
                                                               run_off.p, st.p);
    GLI_CHECK_LAUNCH();
    DevBuf<uint64_t> dest(runs, s);
    const i64 n = exclusive_scan_u32(run_n.p, dest.p, runs, s);  // synchronises
    EnumStatus h;
    GLI_CUDA(cudaMemcpyAsync(&h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    if (h.overflow) return false;
    int64_t* out = nullptr;
    GLI_CUDA(cudaMallocAsync((void**)&out, (n > 0 ? n : 1) * sizeof(int64_t), s));
    const unsigned grid = (unsigned)std::max<i64>(1, std::min<i64>((runs + 7) / 8, (i64)num_sms * 16));
    k_enum_place<<<grid, 256, 0, s>>>(scratch.p, run_n.p, run_off.p, dest.p, runs, out);
    GLI_CHECK_LAUNCH();
    *d_out = out;
    *total = n;
    return true;
}

// can slot t hold a canonical class: the omin filter (ERIDA: i canonical;
// ERI: also omin[j], omin[k] >= i) and for ERI the reference's x-ordering
// (i_x <= j_x, i_x <= k_x)
template <int KIND>
__device__ inline bool slot_live(const SymGrid& G, i64 t) {
    if (KIND == 0) return G.omin[t] == (int)t;
    const i64 N = G.N;
    const i64 i = t / (N * N), j = (t / N) % N, k = t % N;
    if (G.omin[i] != (int)i || G.omin[j] < (int)i || G.omin[k] < (int)i) return false;
    // x coordinate: the leading digit of the x-major linear index
    const i64 LL = (i64)G.L * G.L;
    const i64 xi = i / LL;
    return xi <= j / LL && xi <= k / LL;
}

// WRITE = false: live slots per block of 256; WRITE = true: their ids at the
// block's offset, in order
template <int KIND, bool WRITE>
__global__ void __launch_bounds__(256) k_enum_live(SymGrid G, i64 slots, uint32_t* __restrict__ block_counts,
                                                   const uint64_t* __restrict__ block_offsets,
                                                   int64_t* __restrict__ slot_ids) {
    __shared__ uint32_t wsum[8];
    const i64 t = (i64)blockIdx.x * 256 + threadIdx.x;
    const bool live = t < slots && slot_live<KIND>(G, t);
    const unsigned b = __ballot_sync(0xffffffffu, live);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wsum[warp] = __popc(b);
    __syncthreads();
    if (!WRITE) {
        if (threadIdx.x == 0) {
            uint32_t tot = 0;
            for (int w = 0; w < 8; ++w) tot += wsum[w];
            block_counts[blockIdx.x] = tot;
        }
        return;
    }
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    if (live) slot_ids[block_offsets[blockIdx.x] + before + __popc(b & ((1u << lane) - 1u))] = t;
}

// The 27 partner candidates j of live ERIDA slot i (lane c = 9 tx + 3 ty + tz,
// ascending j), emit(idx, rank) called by every lane after the ballot (idx < 0
// for a lane without a survivor).  Returns the slot's survivors.
template <class Emit>
__device__ inline uint32_t erida_slot_walk(const SymGrid& G, i64 i, int lane, Emit&& emit) {
    int p[2][3];
    point_of(G, i, p[0]);
    bool keep = false;
    i64 idx = 0;
    if (lane < 27) {
        const int tx = lane / 9, ty = (lane / 3) % 3, tz = lane % 3;
        p[1][0] = -p[0][0] - 1 + tx;
        p[1][1] = -p[0][1] - 1 + ty;
        p[1][2] = -p[0][2] - 1 + tz;
        bool in = p[1][0] >= p[0][0];
        for (int a = 0; a < 3; ++a) in = in && p[1][a] >= -G.e && p[1][a] <= G.e;
        if (in) {
            const i64 j = lin3(G, p[1]);
            if (G.omin[j] >= (int)i) {
                const int bias[3] = {tx - 1, ty - 1, tz - 1};
                idx = i * G.N + j;
                keep = canonical_pair(G, p, bias, idx);
            }
        }
    }
    const unsigned b = __ballot_sync(0xffffffffu, keep);
    emit(keep ? idx : (i64)-1, (uint32_t)__popc(b & ((1u << lane) - 1u)));
    return (uint32_t)__popc(b);
}

// The partner candidates l of live slot t (ascending), 32 at a time, one per
// lane; emit(idx, rank) is called by every lane after each group's ballot
// (rank: the place of the lane's survivor among the slot's survivors; idx < 0
// for a lane without one).  Returns the slot's survivors (the same in every
// lane).
template <class Emit>
__device__ inline uint32_t eri_slot_walk(const SymGrid& G, i64 t, int lane, Emit&& emit) {
    const i64 N = G.N;
    {
        const i64 i = t / (N * N), j = (t / N) % N, k = t % N;
        int p[4][3];
        point_of(G, i, p[0]);
        point_of(G, j, p[1]);
        point_of(G, k, p[2]);
        signed char sx[MAX_AXIS], sy[MAX_AXIS], sz[MAX_AXIS];
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(min(p[0][a], p[1][a]), p[2][a]);
            hi[a] = max(max(p[0][a], p[1][a]), p[2][a]);
        }
        const int nx = axis_partners(lo[0], hi[0], G.e, p[2][0], sx);
        const int ny = axis_partners(lo[1], hi[1], G.e, -G.e, sy);
        const int nz = axis_partners(lo[2], hi[2], G.e, -G.e, sz);
        const int total = nx * ny * nz;  // the same in every lane
        const i64 base = t * N;
        uint32_t c = 0;
        for (int c0 = 0; c0 < total; c0 += 32) {
            const int cand = c0 + lane;
            bool keep = false;
            i64 idx = 0;
            if (cand < total) {
                const int az = cand % nz, r = cand / nz, ay = r % ny, ax = r / ny;
                p[3][0] = sx[ax];
                p[3][1] = sy[ay];
                p[3][2] = sz[az];
                const i64 l = lin3(G, p[3]);
                if (G.omin[l] >= (int)i) {
                    const int bias[3] = {min(lo[0], p[3][0]) + max(hi[0], p[3][0]),
                                         min(lo[1], p[3][1]) + max(hi[1], p[3][1]),
                                         min(lo[2], p[3][2]) + max(hi[2], p[3][2])};
                    idx = base + l;
                    keep = canonical_quad(G, p, bias, idx);
                }
            }
            const unsigned b = __ballot_sync(0xffffffffu, keep);
            emit(keep ? idx : (i64)-1, c + __popc(b & ((1u << lane) - 1u)));
            c += __popc(b);
        }
        return c;
    }
}

template <int KIND, class Emit>
__device__ inline uint32_t slot_walk(const SymGrid& G, i64 t, int lane, Emit&& emit) {
    if (KIND == 0) return erida_slot_walk(G, t, lane, emit);
    return eri_slot_walk(G, t, lane, emit);
}

// one warp per live slot; WRITE = false: survivors per slot; WRITE = true:
// survivors at the slot's offset, in order
template <int KIND, bool WRITE>
__global__ void __launch_bounds__(256) k_enum_slots(SymGrid G, const int64_t* __restrict__ slot_ids, i64 nlive,
                                                    uint32_t* __restrict__ counts,
                                                    const uint64_t* __restrict__ offsets, int64_t* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const i64 warps = (i64)gridDim.x * (blockDim.x >> 5);
    for (i64 sl = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); sl < nlive; sl += warps) {
        const uint64_t w = WRITE ? offsets[sl] : 0;
        const uint32_t c = slot_walk<KIND>(G, slot_ids[sl], lane, [&](i64 idx, uint32_t rank) {
            if (WRITE && idx >= 0) out[w + rank] = idx;
        });
        if (!WRITE && lane == 0) counts[sl] = c;
    }
}

// one pass over the live slots: each warp keeps its slot's survivors in shared
// memory, then appends them to the scratch buffer (run_n, run_off per slot);
// a slot with more than ENUM_SLOT_CAP survivors or a full scratch buffer sets
// the overflow status
constexpr int ENUM_SLOT_CAP = 512;

template <int KIND>
__global__ void __launch_bounds__(256) k_enum_slots_collect(SymGrid G, const int64_t* __restrict__ slot_ids,
                                                            i64 nlive, int64_t* __restrict__ scratch,
                                                            unsigned long long cap, uint32_t* __restrict__ run_n,
                                                            unsigned long long* __restrict__ run_off,
                                                            EnumStatus* __restrict__ st) {
    __shared__ int64_t buf[8][ENUM_SLOT_CAP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 warps = (i64)gridDim.x * (blockDim.x >> 5);
    int64_t* mine = buf[warp];
    for (i64 sl = (i64)blockIdx.x * (blockDim.x >> 5) + warp; sl < nlive; sl += warps) {
        const uint32_t c = slot_walk<KIND>(G, slot_ids[sl], lane, [&](i64 idx, uint32_t rank) {
            if (idx >= 0 && rank < ENUM_SLOT_CAP) mine[rank] = idx;
        });
        __syncwarp();
        unsigned long long off = 0;
        if (c > 0 && c <= ENUM_SLOT_CAP && lane == 0) off = atomicAdd(&st->used, (unsigned long long)c);
        off = __shfl_sync(0xffffffffu, off, 0);
        const bool fits = c <= ENUM_SLOT_CAP && off + c <= cap;
        if (lane == 0) {
            run_n[sl] = fits ? c : 0u;
            run_off[sl] = off;
            if (!fits) atomicOr(&st->overflow, c > ENUM_SLOT_CAP ? 1 : 2);
        }
        if (fits)
            for (uint32_t q = lane; q < c; q += 32) scratch[off + q] = mine[q];
        __syncwarp();
    }
}

// collect = false: the count and write passes over the live slots (the
// fallback of a slot with more survivors than a warp's buffer)
template <int KIND>
static i64 enumerate_live(const SymGrid& G, bool collect, int64_t** d_out, int num_sms, cudaStream_t s) {
    const i64 slots = KIND == 0 ? G.N : G.N * G.N * G.N;
    const i64 nb = (slots + 255) / 256;
    DevBuf<uint32_t> bc(nb, s);
    DevBuf<uint64_t> bo(nb, s);
    k_enum_live<KIND, false><<<(unsigned)nb, 256, 0, s>>>(G, slots, bc.p, nullptr, nullptr);
    GLI_CHECK_LAUNCH();
    const i64 nlive = exclusive_scan_u32(bc.p, bo.p, nb, s);
    int64_t* out = nullptr;
    if (nlive == 0) {
        GLI_CUDA(cudaMallocAsync((void**)&out, sizeof(int64_t), s));
        *d_out = out;
        return 0;
    }
    DevBuf<int64_t> ids(nlive, s);
    k_enum_live<KIND, true><<<(unsigned)nb, 256, 0, s>>>(G, slots, nullptr, bo.p, ids.p);
    GLI_CHECK_LAUNCH();
    const unsigned grid = (unsigned)std::max<i64>(1, std::min<i64>((nlive + 7) / 8, (i64)num_sms * 16));
    if (collect) {
        // one pass: survivors kept per warp, appended to scratch, placed in slot order
        const i64 cap = enum_scratch(KIND, G);
        DevBuf<int64_t> scratch(cap, s);
        DevBuf<uint32_t> run_n(nlive, s);
        DevBuf<unsigned long long> run_off(nlive, s);
        DevBuf<EnumStatus> st(1, s);
        st.zero();
        k_enum_slots_collect<KIND><<<grid, 256, 0, s>>>(G, ids.p, nlive, scratch.p, (unsigned long long)cap,
                                                        run_n.p, run_off.p, st.p);
        GLI_CHECK_LAUNCH();
        DevBuf<uint64_t> dest(nlive, s);
        const i64 n = exclusive_scan_u32(run_n.p, dest.p, nlive, s);  // synchronises
        EnumStatus h;
        GLI_CUDA(cudaMemcpyAsync(&h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s));
        if (!h.overflow) {
            GLI_CUDA(cudaMallocAsync((void**)&out, (n > 0 ? n : 1) * sizeof(int64_t), s));
            k_enum_place<<<grid, 256, 0, s>>>(scratch.p, run_n.p, run_off.p, dest.p, nlive, out);
            GLI_CHECK_LAUNCH();
            *d_out = out;
            return n;
        }
    }
    DevBuf<uint32_t> counts(nlive, s);
    DevBuf<uint64_t> offsets(nlive, s);
    k_enum_slots<KIND, false><<<grid, 256, 0, s>>>(G, ids.p, nlive, counts.p, nullptr, nullptr);
    GLI_CHECK_LAUNCH();
    const i64 total = exclusive_scan_u32(counts.p, offsets.p, nlive, s);
    GLI_CUDA(cudaMallocAsync((void**)&out, (total > 0 ? total : 1) * sizeof(int64_t), s));
    k_enum_slots<KIND, true><<<grid, 256, 0, s>>>(G, ids.p, nlive, nullptr, offsets.p, out);
    GLI_CHECK_LAUNCH();
    *d_out = out;
    return total;
}

i64 enumerate_device(int kind, const GridDesc& g, int64_t** d_out, cudaStream_t s) {
    const i64 e = symmetric_extent(g);
    if (e < 0) fail(GLI_ERR_ARGUMENT, "specified grid is not rotationally symmetric");
    SymGrid G;
    G.e = (int)e;
    G.L = (int)(2 * e + 1);
    G.N = (i64)G.L * G.L * G.L;
    // (ERI: N^3 slots in blocks of 128, fewer than 2^31 blocks)
    if (kind == 1 && G.L > 17) fail(GLI_ERR_LIMIT, "ERI enumeration supports grids up to 17^3 (got %d^3)", G.L);
    if (kind == 0 && G.L > 1025) fail(GLI_ERR_LIMIT, "ERIDA enumeration supports grids up to 1025^3");
    const i64 slots = kind == 0 ? G.N : G.N * G.N * G.N;
    DevBuf<int> omin(G.N, s);
    k_orbit_min<<<(unsigned)((G.N + 255) / 256), 256, 0, s>>>(G, omin.p);
    GLI_CHECK_LAUNCH();
    G.omin = omin.p;
    // live slots in one pass.  For their tests, GLI_B200_ENUM_TWO_PASS selects
    // the thread-per-slot two passes, and the value "live" the count and write
    // passes over the live slots.
    const char* two = getenv("GLI_B200_ENUM_TWO_PASS");
    const bool live_two = two && strcmp(two, "live") == 0;
    if (!two || live_two) {
        const int sms = context().num_sms;
        if (kind == 1) return enumerate_live<1>(G, !live_two, d_out, sms, s);
        if (live_two) return enumerate_live<0>(G, false, d_out, sms, s);
        i64 total = 0;
        if (enumerate_one_pass<0>(G, slots, d_out, &total, sms, s)) return total;
    }
    DevBuf<uint32_t> counts(slots, s);
    DevBuf<uint64_t> offsets(slots, s);
    const unsigned blocks = (unsigned)((slots + 127) / 128);
    if (kind == 0)
        k_enum_erida<false><<<blocks, 128, 0, s>>>(G, counts.p, nullptr, nullptr);
    else
        k_enum_eri<false><<<blocks, 128, 0, s>>>(G, counts.p, nullptr, nullptr);
    GLI_CHECK_LAUNCH();
    const i64 total = exclusive_scan_u32(counts.p, offsets.p, slots, s);
    int64_t* out = nullptr;
    GLI_CUDA(cudaMallocAsync((void**)&out, (total > 0 ? total : 1) * sizeof(int64_t), s));
    if (kind == 0)
        k_enum_erida<true><<<blocks, 128, 0, s>>>(G, nullptr, offsets.p, out);
    else
        k_enum_eri<true><<<blocks, 128, 0, s>>>(G, nullptr, offsets.p, out);
    GLI_CHECK_LAUNCH();
    *d_out = out;
    return total;
}

}  // namespace gli
