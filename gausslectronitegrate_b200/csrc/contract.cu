// Staged lattice contraction: every ERI / ERIDA class value in one pass.
//
// Reference: compute_sparse_eri_gausslet_integrals (src/eri_integrals.c:544-678)
// and compute_sparse_erida_gausslet_integrals (src/erida_integrals.c:429-542)
// evaluate each class on its own as
//   val = sum_{x,y,z} Px[x] Py[y] Pz[z] T[(cx+x)^2 + (cy+y)^2 + (cz+z)^2]
// (a 2-D scatter into rho bins followed by a z pass per bin).  The weights are
// separable and T depends only on the squared lattice distance, so with the
// folded per-axis weights W[k][u] (tables.cu) the same sum reads
//   val = sum_u W[kx][u] sum_v W[ky][v] sum_t W[kz][t] T[u^2+v^2+t^2].
// Classes share per-axis keys heavily (3.57M ERI classes on 7^3 use 364 keys
// and ~4e4 key pairs), so the sum is staged over the whole class list:
//   stage A  H[a][s]     = sum_t W[key_a][t] T[s + t^2]               per distinct A key, s = u^2+v^2
//   stage B  H2[p][u]    = sum_v W[key_b][v] H[a(p)][u^2+v^2]         per distinct (A, B) key pair
//   stage C  val[n]      = sum_u W[key_c][u] H2[p(n)][u]              per class: warp dot + shuffles
// The value is symmetric under permuting the three axes (T is), so each class's
// key triple is sorted (k1 <= k2 <= k3) and assigned A = k2, B = k1, C = k3.
// Stage A runs over the distinct s = u^2 + v^2 (H depends on u, v only through
// s); stage C is a per-class warp dot product, or -- when the (pair, key)
// combinations are few against the classes -- one small GEMM plus a gather.
#include <math.h>

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <list>
#include <memory>
#include <thread>

#include "dmma.cuh"
#include "tables.cuh"

namespace gli {

// ---------------------------------------------------------------------------
// Device bounds checks of the debug build (built with -DGLI_B200_DEBUG, python
// -m gausslectronitegrate_b200.build --debug: libgli_b200_debug.so).  A failed
// check records its site and the offending index in a device word (the first
// failure wins) and the access it guards is skipped, so that nothing is read
// or written out of bounds and the GPU does not fault; the host reads the word
// after every evaluation and fails the call with GLI_ERR_INTERNAL naming the
// site.  Release builds compile the checks away.
//   site 1: a decoded axis key outside the key space      (k_mark)
//   site 2: an s index outside the distinct-s list        (stage B gathers)
//   site 3: a (pair, key) product outside Q               (k_gather_q)
//   site 4: a pair row or key outside H2 / W              (k_stage_c)
#ifdef GLI_B200_DEBUG
static __device__ unsigned long long g_debug_fault;
__device__ __forceinline__ bool dcheck(bool cond, int site, long long index) {
    if (!cond) atomicCAS(&g_debug_fault, 0ull, ((unsigned long long)site << 56) | ((unsigned long long)index & ((1ull << 56) - 1)));
    return cond;
}
#else
__device__ __forceinline__ constexpr bool dcheck(bool, int, long long) { return true; }
#endif

// ---------------------------------------------------------------------------
// class decoding
struct ClassDecode {
    int kind;
    i64 N;          // grid points
    i64 L;          // table range (largest axis length)
    i64 istart[3];
    i64 num[3];
    i64 nkeys;
    // device decode: 32-bit point arithmetic (N < 2^31; ERI N^2 < 2^32), the
    // 64-bit quotient by a double estimate when the index is below 2^53, and
    // for ERI a table of point coordinates
    uint32_t n32, n1, n2;
    int is[3];
    uint64_t N2;
    double invN, invN2;
    int fast;
    const short4* pt;
    // ERI point pairs (p, q), index p N + q: per axis |x_p - x_q| and
    // x_p + x_q - 2 istart, 8 bits each (axes of at most 128 points), so that a
    // class decodes with one quotient and two loads; null: point table route
    const uint2* pd;
    void finish() {
        n32 = (uint32_t)N;
        n1 = (uint32_t)num[1];
        n2 = (uint32_t)num[2];
        for (int a = 0; a < 3; ++a) is[a] = (int)istart[a];
        N2 = (uint64_t)N * (uint64_t)N;
        invN = 1.0 / (double)N;
        invN2 = 1.0 / (double)N2;
        // largest class index + 1: N^2 (ERIDA), N^4 (ERI)
        const double top = kind == 0 ? (double)N2 : (double)N2 * (double)N2;
        fast = top <= 9007199254740992.0 ? 1 : 0;  // 2^53
    }
};

// floor(u / d) for u < 2^53: the double estimate u * (1/d) is within one of
// the quotient, and one correction step lands on it
__device__ inline uint64_t div_est(uint64_t u, uint64_t d, double inv) {
    uint64_t q = (uint64_t)((double)u * inv);
    const int64_t r = (int64_t)(u - q * d);
    if (r < 0)
        --q;
    else if (r >= (int64_t)d)
        ++q;
    return q;
}

// the same for 32-bit operands, in 32-bit arithmetic (d < 2^31): the
// remainder of a quotient one too large wraps to at least 2^32 - d
__device__ inline uint32_t div32_est(uint32_t u, uint32_t d, double inv) {
    uint32_t q = (uint32_t)((double)u * inv);
    const uint32_t r = u - q * d;
    if (r >= 0x80000000u)
        --q;
    else if (r >= d)
        ++q;
    return q;
}

// grid point lin (x-major) -> coordinates; 32-bit arithmetic
__device__ inline void decode_pt(const ClassDecode& d, uint32_t lin, int p[3]) {
    const uint32_t r = lin / d.n2;
    p[2] = d.is[2] + (int)(lin - r * d.n2);
    const uint32_t x = r / d.n1;
    p[1] = d.is[1] + (int)(r - x * d.n1);
    p[0] = d.is[0] + (int)x;
}

// coordinates of every grid point (ERI decoding)
__global__ void k_point_table(ClassDecode d, short4* __restrict__ pt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n32) return;
    int p[3];
    decode_pt(d, i, p);
    pt[i] = make_short4((short)p[0], (short)p[1], (short)p[2], 0);
}

// Axis field of one ERI pair descriptor word: bits 0-7 |x_p - x_q|, 8-15
// x_p + x_q - 2 istart of axis 2a (word .x: axes 0, 1; word .y: axis 2).
__device__ __forceinline__ uint32_t pd_field(int dax, int sax) {
    return (uint32_t)abs(dax) | ((uint32_t)sax << 8);
}

// descriptor of every point pair h = p N + q (N^2 entries); skip (sized
// replays): when *skip is set the table kept with the replay's saved plan is
// current (a function of the grid alone, made by the replay that made the plan)
__global__ void k_pair_desc(ClassDecode d, uint2* __restrict__ pd, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if ((uint64_t)h >= d.N2) return;
    const uint32_t p = h / d.n32, q = h - p * d.n32;
    int a[3], b[3];
    decode_pt(d, p, a);
    decode_pt(d, q, b);
    uint32_t f[3];
    for (int x = 0; x < 3; ++x) f[x] = pd_field(a[x] - b[x], a[x] + b[x] - 2 * d.is[x]);
    pd[h] = make_uint2(f[0] | (f[1] << 16), f[2]);
}

// key of one axis from the two pair fields (|d01| | s01 << 8, |d23| | s23 << 8):
// the unordered shift pair and |(i+j) - (k+l)| of that axis, as eri_axis_key32
__device__ __forceinline__ int pd_axis_key(uint32_t f01, uint32_t f23, int L2m1) {
    const int d01 = (int)(f01 & 0xffu), d23 = (int)(f23 & 0xffu);
    const int c = abs((int)(f01 >> 8) - (int)(f23 >> 8));
    const int a = min(d01, d23), b = max(d01, d23);
    return ((b * (b + 1) >> 1) + a) * L2m1 + c;
}

// The pair-descriptor decode covers ERI grids whose axes have at most 128
// points, whose N^2 descriptors take at most 32 MB, and whose class indices
// lie below 2^53 (the quotient estimate is exact there).
inline bool pair_desc_applies(const ClassDecode& d) {
    return d.kind == 1 && d.fast && d.L <= 128 && d.N2 <= ((uint64_t)1 << 22);
}

// sorted axis keys of class idx; false for an index outside the tensor
__device__ inline bool class_keys(const ClassDecode& d, i64 idx, int k[3]) {
    if (idx < 0) return false;
    const uint64_t u = (uint64_t)idx;
    if (d.kind == 0) {
        if (u >= d.N2) return false;
        const uint64_t pi = d.fast ? div_est(u, d.n32, d.invN) : u / d.n32;
        int a[3], b[3];
        decode_pt(d, (uint32_t)pi, a);
        decode_pt(d, (uint32_t)(u - pi * d.n32), b);
        for (int x = 0; x < 3; ++x) k[x] = abs(a[x] - b[x]);
    } else if (d.pd) {
        // (d.pd is set only where N^4 < 2^53: the quotient estimate is exact)
        const uint64_t hi = div_est(u, d.N2, d.invN2);  // point pair (p0, p1)
        if (hi >= d.N2) return false;
        const uint32_t lo = (uint32_t)u - (uint32_t)hi * (uint32_t)d.N2;  // (p2, p3): the remainder is below 2^32
        const uint2 a = __ldg(&d.pd[hi]), b = __ldg(&d.pd[lo]);
        const int L2m1 = 2 * (int)d.L - 1;
        k[0] = pd_axis_key(a.x & 0xffffu, b.x & 0xffffu, L2m1);
        k[1] = pd_axis_key(a.x >> 16, b.x >> 16, L2m1);
        k[2] = pd_axis_key(a.y, b.y, L2m1);
    } else {
        const uint64_t hi = d.fast ? div_est(u, d.N2, d.invN2) : u / d.N2;  // point pair (p0, p1)
        if (hi >= d.N2) return false;
        const uint32_t h = (uint32_t)hi, lo = (uint32_t)(u - hi * d.N2);  // point pair (p2, p3); N^2 < 2^32
        const uint32_t i0 = div32_est(h, d.n32, d.invN), i2 = div32_est(lo, d.n32, d.invN);
        const short4 p0 = d.pt[i0], p1 = d.pt[h - i0 * d.n32], p2 = d.pt[i2], p3 = d.pt[lo - i2 * d.n32];
        const int L = (int)d.L;
        k[0] = eri_axis_key32(p0.x - p1.x, p2.x - p3.x, (p0.x + p1.x) - (p2.x + p3.x), L);
        k[1] = eri_axis_key32(p0.y - p1.y, p2.y - p3.y, (p0.y + p1.y) - (p2.y + p3.y), L);
        k[2] = eri_axis_key32(p0.z - p1.z, p2.z - p3.z, (p0.z + p1.z) - (p2.z + p3.z), L);
    }
    // sort ascending
    if (k[0] > k[1]) { const int t = k[0]; k[0] = k[1]; k[1] = t; }
    if (k[1] > k[2]) { const int t = k[1]; k[1] = k[2]; k[2] = t; }
    if (k[0] > k[1]) { const int t = k[0]; k[0] = k[1]; k[1] = t; }
    return true;
}

// a class's sorted key triple, packed 21 bits per key (keys < 2^21, checked
// on the host); all ones for an index outside the tensor
constexpr uint64_t BAD_KEYS = ~(uint64_t)0;
__device__ inline uint64_t pack_keys(const int k[3]) {
    return (uint64_t)k[0] | ((uint64_t)k[1] << 21) | ((uint64_t)k[2] << 42);
}
__device__ inline void unpack_keys(uint64_t p, int k[3]) {
    k[0] = (int)(p & 0x1fffff);
    k[1] = (int)((p >> 21) & 0x1fffff);
    k[2] = (int)(p >> 42);
}

// counts of one evaluation, kept in device memory so that kernels can size their
// work without a host round trip
struct PlanCounts {
    uint64_t key_total;  // used keys + used A keys (joint scan total)
    uint64_t nP;         // distinct (A, B) key pairs
    int64_t nku, nA;     // used keys, used A keys
    // an evaluation queued with the sizes of an earlier one found more keys or
    // pairs than those sizes hold: the counts are zeroed (every later pass
    // then has nothing to do) and the host evaluates again with exact sizes
    int64_t overflow;
};

// The counts of a trusted replay: those of the kept plan when it is valid,
// else none and the overflow flag (the host then evaluates again, exactly)
__device__ __forceinline__ void restore_counts(bool valid, const PlanCounts* __restrict__ saved,
                                               PlanCounts* __restrict__ cnt) {
    if (valid) {
        const PlanCounts c = *saved;
        cnt->key_total = c.key_total;
        cnt->nku = c.nku;
        cnt->nA = c.nA;
        cnt->nP = c.nP;
        cnt->overflow = 0;
    } else {
        cnt->key_total = 0;
        cnt->nku = 0;
        cnt->nA = 0;
        cnt->nP = 0;
        cnt->overflow = 1;
    }
}

// an evaluation's status block: its counts and its flags
struct EvalStatus {
    PlanCounts cnt;
    int bad;                      // a class index outside the tensor
    int tc_err;                   // a tensor-core CTA gave up waiting
    unsigned long long products;  // (pair, key) products that stage C's product GEMM computed
};

// The status block of a trusted replay, written whole by its first kernel
// (such a replay queues no memset of the block): the restored counts, no
// flags raised and no products counted yet
__device__ __forceinline__ void restore_status(bool valid, const PlanCounts* __restrict__ saved,
                                               EvalStatus* __restrict__ st) {
    restore_counts(valid, saved, &st->cnt);
    st->bad = 0;
    st->tc_err = 0;
    st->products = 0ull;
}

// Decodes every class once (its packed keys are kept for the later passes)
// and marks the keys it uses (any role: usedKey; as A = k2: usedA) and its
// (A, B) = (k2, k1) key pair (bit k2 * nk + k1 of pairBits).  Millions of
// classes share a few hundred keys and a few thousand pairs, so writes of the
// same flag from every block would queue on a few cache lines: with `local`
// set each block collects its key flags and pair bits in shared memory and
// merges them once.  used = [usedKey | usedA], 2 nk flags.  keys may be null:
// the later passes then decode the classes again (the pair-descriptor decode
// costs less than writing and re-reading 8 bytes per class).
// skip: as in k_mark_eri_pd (replays whose gather decodes and checks the
// classes against a saved plan).
__global__ void __launch_bounds__(256) k_mark(ClassDecode d, const int64_t* __restrict__ idx, i64 m,
                                              uint32_t* __restrict__ used, uint32_t* __restrict__ pairBits,
                                              uint64_t* __restrict__ keys, int* __restrict__ bad, int local,
                                              const int* __restrict__ skip) {
    if (skip && *skip) return;
    extern __shared__ uint32_t sflag[];
    const int nk = (int)d.nkeys;
    const int words = (nk * nk + 31) >> 5;
    uint32_t* sbits = sflag + 2 * nk;
    if (local) {
        for (int i = threadIdx.x; i < 2 * nk + words; i += blockDim.x) sflag[i] = 0;
        __syncthreads();
    }
    uint32_t* flags = local ? sflag : used;
    uint32_t* bits = local ? sbits : pairBits;
    // four classes per thread and step, their index loads issued together
    constexpr int V = 4;
    const i64 step = (i64)gridDim.x * blockDim.x;
    for (i64 n0 = (i64)blockIdx.x * blockDim.x + threadIdx.x; n0 < m; n0 += V * step) {
        i64 cls[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const i64 n = n0 + v * step;
            cls[v] = n < m ? __ldg(&idx[n]) : -1;
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const i64 n = n0 + v * step;
            if (n >= m) break;
            int k[3];
            if (!class_keys(d, cls[v], k)) {
                if (keys) keys[n] = BAD_KEYS;
                atomicOr(bad, 1);
                continue;
            }
            if (!dcheck(k[0] >= 0 && k[2] < nk, 1, k[0] < 0 ? k[0] : k[2])) continue;
            if (keys) keys[n] = pack_keys(k);
            flags[k[0]] = 1;
            flags[k[1]] = 1;
            flags[k[2]] = 1;
            flags[nk + k[1]] = 1;
            // neighbouring classes share their pair: a read first, so that the
            // serialising atomic runs only for a new bit
            const int slot = k[1] * nk + k[0];
            const uint32_t bit = 1u << (slot & 31);
            if (!(bits[slot >> 5] & bit)) atomicOr(&bits[slot >> 5], bit);
        }
    }
    if (local) {
        __syncthreads();
        for (int i = threadIdx.x; i < 2 * nk; i += blockDim.x)
            if (sflag[i]) used[i] = 1;
        for (int w = threadIdx.x; w < words; w += blockDim.x)
            if (sbits[w]) atomicOr(&pairBits[w], sbits[w]);
    }
}

// packed keys of class n: from the keys buffer, or decoded from the class
// index when the evaluation keeps none
__device__ __forceinline__ uint64_t class_packed(const uint64_t* __restrict__ keys, const ClassDecode& d,
                                                 const int64_t* __restrict__ idx, i64 n) {
    if (keys) return keys[n];
    int k[3];
    return class_keys(d, __ldg(&idx[n]), k) ? pack_keys(k) : BAD_KEYS;
}

// Sorted axis keys s0 <= s1 <= s2 of ERI class x through the pair
// descriptors; (base, da) carry the first index of the point pair (i, j) of
// the previous class of the same thread (its quotient by N^2 times N^2;
// PD_NO_BASE: none) and that pair's descriptor, reused while the remainder
// stays below N^2.  False for an index outside the tensor.
constexpr uint64_t PD_NO_BASE = (uint64_t)1 << 63;  // u - PD_NO_BASE >= 2^63 > N^2 for every index u < 2^63
__device__ __forceinline__ bool pd_class_keys(const ClassDecode& d, int64_t x, uint64_t& base, uint2& da, int& s0,
                                              int& s1, int& s2) {
    if (x < 0) return false;
    const uint64_t u = (uint64_t)x, N2 = d.N2;
    if (u - base >= N2) {
        const uint64_t hi = div_est(u, N2, d.invN2);
        if (hi >= N2) {
            base = PD_NO_BASE;
            return false;
        }
        base = hi * N2;
        da = __ldg(&d.pd[hi]);
    }
    const uint32_t lo = (uint32_t)(u - base);
    const uint2 db = __ldg(&d.pd[lo]);
    const int L2m1 = 2 * (int)d.L - 1;
    const int k0 = pd_axis_key(da.x & 0xffffu, db.x & 0xffffu, L2m1);
    const int k1 = pd_axis_key(da.x >> 16, db.x >> 16, L2m1);
    const int k2 = pd_axis_key(da.y, db.y, L2m1);
    const int a = min(k0, k1), b = max(k0, k1);
    s0 = min(a, k2);
    s2 = max(b, k2);
    s1 = a + b + k2 - s0 - s2;
    return true;
}

// The decode pass for ERI classes through the pair descriptors.  A thread
// takes four consecutive classes (16-byte loads of the indices and stores of
// the packed keys when the arrays are 16-byte aligned): a sorted list keeps the
// point pair (i, j) of neighbouring classes, so the quotient by N^2 and the
// first descriptor are reused while the remainder stays below N^2 (any order
// is still decoded correctly: an out-of-range remainder takes the quotient
// again), and a pair bit already set by the thread's previous class is not
// tested again.  Flags and pair bits as in k_mark.
// skip (non-null in replays that may reuse their plan): when *skip is
// set, the saved plan stands for this replay unless the class gather finds a
// class outside it, so the classes are not marked here (the gather decodes
// and checks them).  keys may be null (such replays do not read them).
__global__ void __launch_bounds__(256) k_mark_eri_pd(ClassDecode d, const int64_t* __restrict__ idx, i64 m,
                                                     uint32_t* __restrict__ used, uint32_t* __restrict__ pairBits,
                                                     uint64_t* __restrict__ keys, int* __restrict__ bad, int local,
                                                     const int* __restrict__ skip) {
    if (skip && *skip) return;
    extern __shared__ uint32_t sflag[];
    const int nk = (int)d.nkeys;
    const int words = (nk * nk + 31) >> 5;
    uint32_t* sbits = sflag + 2 * nk;
    if (local) {
        for (int i = threadIdx.x; i < 2 * nk + words; i += blockDim.x) sflag[i] = 0;
        __syncthreads();
    }
    uint32_t* flags = local ? sflag : used;
    uint32_t* bits = local ? sbits : pairBits;
    const bool vec = ((uintptr_t)idx & 15) == 0 && ((uintptr_t)keys & 15) == 0;
    const i64 groups = (m + 3) / 4;
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += (i64)gridDim.x * blockDim.x) {
        const i64 n0 = 4 * g;
        const bool full = n0 + 3 < m;
        int64_t c[4];
        if (vec && full) {
            const longlong2 a = __ldg(reinterpret_cast<const longlong2*>(idx + n0));
            const longlong2 b = __ldg(reinterpret_cast<const longlong2*>(idx + n0 + 2));
            c[0] = a.x, c[1] = a.y, c[2] = b.x, c[3] = b.y;
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) c[v] = n0 + v < m ? __ldg(&idx[n0 + v]) : 0;
        }
        uint64_t base = PD_NO_BASE;
        uint2 da = make_uint2(0, 0);
        int last_slot = -1;
        uint64_t kv[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            kv[v] = BAD_KEYS;
            if (n0 + v >= m) continue;
            int s0, s1, s2;
            if (!pd_class_keys(d, c[v], base, da, s0, s1, s2)) {
                atomicOr(bad, 1);
                continue;
            }
            if (!dcheck(s0 >= 0 && s2 < nk, 1, s2)) continue;
            const int k[3] = {s0, s1, s2};
            kv[v] = pack_keys(k);
            flags[s0] = 1;
            flags[s1] = 1;
            flags[s2] = 1;
            flags[nk + s1] = 1;
            const int slot = s1 * nk + s0;
            if (slot != last_slot) {
                last_slot = slot;
                const uint32_t bit = 1u << (slot & 31);
                if (!(bits[slot >> 5] & bit)) atomicOr(&bits[slot >> 5], bit);
            }
        }
        if (!keys) continue;
        if (vec && full) {
            reinterpret_cast<ulonglong2*>(keys + n0)[0] = make_ulonglong2(kv[0], kv[1]);
            reinterpret_cast<ulonglong2*>(keys + n0)[1] = make_ulonglong2(kv[2], kv[3]);
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (n0 + v < m) keys[n0 + v] = kv[v];
        }
    }
    if (local) {
        __syncthreads();
        for (int i = threadIdx.x; i < 2 * nk; i += blockDim.x)
            if (sflag[i]) used[i] = 1;
        for (int w = threadIdx.x; w < words; w += blockDim.x)
            if (sbits[w]) atomicOr(&pairBits[w], sbits[w]);
    }
}

// id of the pair in bit `slot` of the pair bitmap: the set bits before it
__device__ inline i64 pair_id(const uint32_t* __restrict__ bits, const uint64_t* __restrict__ pre, i64 slot) {
    const i64 w = slot >> 5;
    return (i64)pre[w] + __popc(bits[w] & ((1u << (slot & 31)) - 1u));
}

// dynamic shared memory of k_mark's local variant, 0 when it does not fit
static size_t mark_local_bytes(i64 nk) {
    const i64 bytes = (2 * nk + (nk * nk + 31) / 32) * (i64)sizeof(uint32_t);  // key flags + pair bits
    return bytes <= 48 * 1024 ? (size_t)bytes : 0;
}

// After the joint scan of (usedKey | usedA): compact key id kid[k] = ids[k],
// A id = ids[nk + k] - nku.  Records both inverse maps and the counts.
__global__ void k_plan_keys(i64 nk, const uint32_t* __restrict__ used, const uint64_t* __restrict__ ids,
                            int* __restrict__ keyOf, int* __restrict__ aId, int* __restrict__ aKey,
                            PlanCounts* __restrict__ cnt) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nku = ids[nk];  // exclusive scan at nk = number of used keys
    if (k == 0) {
        cnt->nku = (int64_t)nku;
        cnt->nA = (int64_t)(cnt->key_total - nku);
    }
    if (k >= nk) return;
    if (used[k]) keyOf[ids[k]] = (int)k;
    if (used[nk + k]) {
        const int a = (int)(ids[nk + k] - nku);
        aId[k] = a;
        aKey[a] = (int)k;
    }
}

// block-wide exclusive sum of one value per thread (blockDim.x = 1024)
__device__ inline uint32_t block_scan_1024(uint32_t v, uint32_t* warp_sums, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warp_sums[lane];
        uint32_t wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    return warp_sums[warp] + incl - v;
}

// Bounded plans (at most 512 key flags, 65,536 pair slots): one block scans the
// key flags and records the key maps and counts -- the joint scan and
// k_plan_keys in one launch.
__global__ void __launch_bounds__(1024) k_plan_keys_small(i64 nk, const uint32_t* __restrict__ used,
                                                          uint64_t* __restrict__ ids, int* __restrict__ keyOf,
                                                          int* __restrict__ aId, int* __restrict__ aKey,
                                                          PlanCounts* __restrict__ cnt) {
    __shared__ uint32_t ws[32], total, nku_s;
    const int k = threadIdx.x;  // flag k of 2 nk (<= 512)
    const uint32_t f = k < 2 * nk ? used[k] : 0u;
    const uint32_t ex = block_scan_1024(f, ws, &total);
    if (k < 2 * nk) ids[k] = ex;
    if (k == nk) nku_s = ex;  // exclusive count at nk = used keys
    __syncthreads();
    const uint32_t nku = nk > 0 ? nku_s : 0u;
    if (k == 0) {
        cnt->key_total = total;
        cnt->nku = nku;
        cnt->nA = (int64_t)total - nku;
    }
    if (k < nk && f) keyOf[ex] = k;
    if (k >= nk && k < 2 * nk && f) {
        const int a = (int)(ex - nku);
        aId[k - nk] = a;
        aKey[a] = (int)(k - nk);
    }
}

// ... and the pair bitmap (bit k2 * nk + k1): the exclusive count of set bits
// before every word, the pair lists in bit order (sorted by A key, then B
// key), and the pair count.  Tiles of 1024 words, scanned with a running carry.
__global__ void __launch_bounds__(1024) k_pairs_small(i64 words, int nk, const uint32_t* __restrict__ bits,
                                                      const int* __restrict__ aId, uint64_t* __restrict__ pre,
                                                      int* __restrict__ pairA, int* __restrict__ pairB,
                                                      PlanCounts* __restrict__ cnt) {
    __shared__ uint32_t ws[32], total;
    uint32_t carry = 0;
    for (i64 base = 0; base < words; base += 1024) {
        const i64 w = base + threadIdx.x;
        uint32_t b = w < words ? bits[w] : 0u;
        uint32_t id = carry + block_scan_1024(__popc(b), ws, &total);
        if (w < words) pre[w] = id;
        while (b) {
            const int bit = __ffs(b) - 1;
            b &= b - 1;
            const i64 slot = w * 32 + bit;
            pairA[id] = aId[slot / nk];
            pairB[id] = (int)(slot % nk);
            ++id;
        }
        carry += total;
        __syncthreads();  // total and ws are rewritten by the next tile's scan
    }
    if (threadIdx.x == 0) cnt->nP = carry;
}

// set bits per word of the pair bitmap (the exclusive scan of which gives pre)
__global__ void k_word_counts(i64 words, const uint32_t* __restrict__ bits, uint32_t* __restrict__ counts) {
    const i64 w = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (w < words) counts[w] = __popc(bits[w]);
}

__global__ void k_pair_lists(i64 words, int nk, const uint32_t* __restrict__ bits, const uint64_t* __restrict__ pre,
                             const int* __restrict__ aId, int* __restrict__ pairA, int* __restrict__ pairB) {
    const i64 w = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    uint32_t b = bits[w];
    i64 id = (i64)pre[w];
    while (b) {
        const int bit = __ffs(b) - 1;
        b &= b - 1;
        const i64 slot = w * 32 + bit;
        pairA[id] = aId[slot / nk];
        pairB[id] = (int)(slot % nk);
        ++id;
    }
}

// ---------------------------------------------------------------------------
// stage A: H[a][j] = sum_t W[aKey[a]][t] T[S[j] + t^2]
// H depends on (u, v) only through s = u^2 + v^2, so it is evaluated once per
// distinct s (S, ascending; 10,823 values instead of 31,329 (u, v) at U = 177).
// As a GEMM: C[j][a] = sum_t G[j][t] W[aKey[a]][t] with G[j][t] = T[S[j] + t^2]
// gathered tile by tile into shared memory (consecutive j read neighbouring
// table entries, so a warp's 32 gathers touch a few cache lines), and the
// FP64 tensor-core tiles of dmma.cuh.  blockIdx.z selects a chunk of t: the
// split blocks of small problems sum their partial tiles in a cluster; the
// 144-column tiles split only the m tiles of a partial last wave, in two
// halves of t (dm_split_store).
template <int BN_>
struct StageAOp {
    static constexpr bool A_KMAJOR = true, B_KMAJOR = false;
    static constexpr int BN = BN_;
    static constexpr int STAGES = BN_ > 80 ? 2 : DM_STAGES;  // 144 columns: three blocks per SM
    static constexpr int NB = BN / 16;  // B element pairs per thread (rows of W are contiguous in t)
    // W row offsets: 32-bit for the 144-column tiles, whose registers are
    // scarce (aKey * Up < 2^31 with at most 8,192 keys)
    using Off = std::conditional_t<(BN_ > 80), int, i64>;
    const double* W;
    const double* T;
    const int* S;
    const int* aKey;
    const PlanCounts* cnt;
    int nS, U, Up, t_chunk;
    i64 part_stride;
    double* H;
    // tail split (k_dmma's dm_split_store; ws null: none): blocks from nfull on
    // are the two K halves of the m tiles nfull, nfull + 1, ...
    int nfull = 0;
    double* ws = nullptr;
    unsigned* tickets = nullptr;
    static constexpr bool TAIL_SPLIT = true;
    // trusted replays (restore_valid non-null; 64- and 80-column tiles): the
    // first block restores the kept plan's counts into cnt for the later
    // kernels (k_restore_plan's work, one launch fewer), and every block reads
    // the kept counts
    const int* restore_valid = nullptr;
    const PlanCounts* restore_from = nullptr;
    EvalStatus* restore_to = nullptr;
    __device__ int split_half() const {
        return ws && (int)blockIdx.x >= nfull ? (int)((blockIdx.x - nfull) & 1) : -1;
    }
    __device__ int split_slot() const { return (int)(blockIdx.x - nfull) >> 1; }
    struct Block {
        int mvalid, nvalid, nk;
        int m0, n0, t0, t1;
        double* H;
    };
    struct AState {
        const double* base;  // T + S[j] of this thread's row j
        bool ok;
    };
    struct BState {
        Off off[NB];  // aKey * Up of this thread's rows, -1 past nA
    };
    __device__ bool begin(Block& b) const {
        const PlanCounts* c = cnt;
        if (BN_ <= 80 && restore_valid) {
            const bool valid = *restore_valid != 0;
            if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0)
                restore_status(valid, restore_from, restore_to);
            if (!valid) return false;
            c = restore_from;
        }
        const int nA = (int)c->nA;
        b.n0 = blockIdx.y * BN;
        if (b.n0 >= nA) return false;  // grids are sized by a bound on nA
        const int half = split_half();
        b.m0 = (half < 0 ? (int)blockIdx.x : nfull + split_slot()) * DM_BM;
        b.mvalid = min(DM_BM, nS - b.m0);
        b.nvalid = min(BN, nA - b.n0);
        if (half < 0) {
            b.t0 = blockIdx.z * t_chunk;
            b.t1 = min(U, b.t0 + t_chunk);
        } else {  // (the host splits only K ranges of at least two chunks)
            const int hc = ((U + DM_BK - 1) / DM_BK + 1) / 2 * DM_BK;
            b.t0 = half ? hc : 0;
            b.t1 = half ? U : min(U, hc);
        }
        b.nk = (b.t1 - b.t0 + DM_BK - 1) / DM_BK;
        b.H = H + (i64)blockIdx.z * part_stride;
        return b.nk > 0;
    }
    __device__ void a_init(const Block& b, AState& st) const {
        const int r = dm_kmajor_row(threadIdx.x);
        st.ok = r < b.mvalid;
        st.base = T + (st.ok ? S[b.m0 + r] : 0);
    }
    __device__ void a_issue(const Block& b, AState& st, int kc, double* tile) const {
        const int r = dm_kmajor_row(threadIdx.x);
#pragma unroll
        for (int q = 0; q < DM_ELEMS; ++q) {
            const int k = dm_kmajor_k(threadIdx.x, q), t = b.t0 + kc * DM_BK + k;
            const bool v = st.ok && t < b.t1;
            dm_cp8(tile + dm_kmajor_at(r, k), v ? st.base + t * t : T, v);
        }
    }
    __device__ void b_init(const Block& b, BState& st) const {
#pragma unroll
        for (int q = 0; q < NB; ++q) {
            const int r = dm_pair_row(threadIdx.x, q);
            st.off[q] = r < b.nvalid ? (Off)aKey[b.n0 + r] * (Off)Up : (Off)-1;
        }
    }
    // pairs (t, t + 1), t even: W rows start at multiples of Up (a multiple of
    // 4) and chunks at multiples of 16, so every pair is 16-byte aligned
    __device__ void b_issue(const Block& b, BState& st, int kc, double* tile) const {
        const int k = dm_pair_k(threadIdx.x), t = b.t0 + kc * DM_BK + k;
        const int bytes = dm_pair_bytes(t, b.t1);
#pragma unroll
        for (int q = 0; q < NB; ++q) {
            const int n = st.off[q] >= 0 ? bytes : 0;
            dm_cp16(tile + dm_rowmajor_at(dm_pair_row(threadIdx.x, q), k), n ? W + st.off[q] + t : W, n);
        }
    }
    __device__ void store(const Block& b, int m, int n, double v0, double v1) const {
        if (m >= b.mvalid) return;
        double* h = b.H + (i64)(b.n0 + n) * nS + b.m0 + m;
        if (n < b.nvalid) h[0] = v0;
        if (n + 1 < b.nvalid) h[nS] = v1;
    }
};

// ---------------------------------------------------------------------------
// stage B: H2[p][u] = sum_v W[pairB[p]][v] Hf[a(p)][v][u],  Hf[a][v][u] = H[a][sidx[v U + u]]
// Pairs are ordered by their A key and cut into tiles of 64 pairs of one A key
// (k_pair_tiles); block (pair tile, 64 u, chunk of v) is one GEMM tile with the
// pair weights as A (rows read along v) and the expanded H of the tile's A key
// as B, gathered through sidx straight from H (no expanded copy in memory).
// The sidx values of the next chunk are loaded one chunk ahead, so the
// dependent gathers do not wait on them.
// DEEP = false: two pipeline stages and four blocks per SM (at most 128
// registers), for grids of several waves (ERIDA 129^3: 199 against 213 us);
// small grids keep three stages (ERIDA 33^3: 20.5 against 22.5 us)
template <bool DEEP>
struct StageBOp {
    static constexpr bool A_KMAJOR = false, B_KMAJOR = true;
    static constexpr int BN = DM_BN;
    static constexpr int STAGES = DEEP ? 3 : 2, MIN_BLOCKS = DEEP ? 3 : 4;
    const double* W;
    const double* H;
    const int* sidx;
    const int* rowKey;   // weight key of each tile row
    const int* rowPair;  // H2 row (pair id) of each tile row
    const int* tile_batch;
    const int* tile_col0;
    const int* tile_ncols;
    int nS, U, Up, v_chunk;
    i64 part_stride;
    double* H2;
    struct Block {
        int mvalid, nvalid, nk;
        int p0, u0, v0, v1;
        const double* h;  // H row of the tile's A key
        double* H2;
    };
    struct AState {
        i64 off[DM_BM / 16];  // weight key * Up of this thread's rows, -1 past the tile
    };
    struct BState {
        int sv[DM_ELEMS];  // sidx of the next chunk's elements (-1: zero fill)
    };
    __device__ bool begin(Block& b) const {
        const int tile = blockIdx.x;
        b.mvalid = tile_ncols[tile];
        if (b.mvalid <= 0) return false;  // tiles past the last one
        b.p0 = tile_col0[tile];
        b.h = H + (i64)tile_batch[tile] * nS;
        b.u0 = blockIdx.y * DM_BN;
        b.nvalid = min(DM_BN, U - b.u0);
        b.v0 = blockIdx.z * v_chunk;
        b.v1 = min(U, b.v0 + v_chunk);
        b.nk = (b.v1 - b.v0 + DM_BK - 1) / DM_BK;
        b.H2 = H2 + (i64)blockIdx.z * part_stride;
        return b.nk > 0;
    }
    __device__ void a_init(const Block& b, AState& st) const {
#pragma unroll
        for (int q = 0; q < DM_BM / 16; ++q) {
            const int r = dm_pair_row(threadIdx.x, q);
            st.off[q] = r < b.mvalid ? (i64)rowKey[b.p0 + r] * Up : -1;
        }
    }
    // pairs (v, v + 1), v even: 16-byte aligned in the W rows
    __device__ void a_issue(const Block& b, AState& st, int kc, double* tile) const {
        const int k = dm_pair_k(threadIdx.x), v = b.v0 + kc * DM_BK + k;
        const int bytes = dm_pair_bytes(v, b.v1);
#pragma unroll
        for (int q = 0; q < DM_BM / 16; ++q) {
            const int n = st.off[q] >= 0 ? bytes : 0;
            dm_cp16(tile + dm_rowmajor_at(dm_pair_row(threadIdx.x, q), k), n ? W + st.off[q] + v : W, n);
        }
    }
    __device__ void b_load(const Block& b, BState& st, int kc) const {
        const int n = dm_kmajor_row(threadIdx.x), u = b.u0 + n;
#pragma unroll
        for (int q = 0; q < DM_ELEMS; ++q) {
            const int v = b.v0 + kc * DM_BK + dm_kmajor_k(threadIdx.x, q);
            st.sv[q] = (n < b.nvalid && v < b.v1) ? __ldg(&sidx[v * U + u]) : -1;
            if (!dcheck(st.sv[q] < nS, 2, st.sv[q])) st.sv[q] = -1;
        }
    }
    __device__ void b_init(const Block& b, BState& st) const { b_load(b, st, 0); }
    __device__ void b_issue(const Block& b, BState& st, int kc, double* tile) const {
        const int n = dm_kmajor_row(threadIdx.x);
#pragma unroll
        for (int q = 0; q < DM_ELEMS; ++q) {
            const int sv = st.sv[q];
            dm_cp8(tile + dm_kmajor_at(n, dm_kmajor_k(threadIdx.x, q)), sv >= 0 ? b.h + sv : b.h, sv >= 0);
        }
        if (kc + 1 < b.nk) b_load(b, st, kc + 1);
    }
    __device__ void store(const Block& b, int m, int n, double v0, double v1) const {
        if (m >= b.mvalid) return;
        double* h2 = b.H2 + (i64)__ldg(&rowPair[b.p0 + m]) * Up + b.u0 + n;
        if (n + 1 < b.nvalid)
            *reinterpret_cast<double2*>(h2) = make_double2(v0, v1);  // Up, u0 and n are even
        else if (n < b.nvalid)
            h2[0] = v0;
    }
};

// Splits of a reduction loop of length U into P chunks (chunk a multiple of
// `grain`) so that a launch of `blocks` blocks reaches about `target` blocks:
// small problems otherwise leave most SMs idle while each block walks the
// whole loop.
// The split minimises waves x time per block: `target` blocks run in one
// wave, and a block's time grows with the K chunks it walks (ERIDA 33^3 stage
// A: 170 tiles, three parts took two waves of 4 chunks, two parts one wave of
// 6; ERI 7^3 stage A likewise two parts instead of three: 25 -> 21 us).
// A block also pays a fixed cost of about three chunks (pipeline fill, drain
// and store), and a split block two more for the cluster sum (measured: ERI
// 7^3 stage B 27 us unsplit, 37 us in two parts, 48 us in five).
static int split_count(i64 blocks, int U, int grain, i64 target, int* chunk) {
    const int most = (int)std::min<i64>(8, (U + grain - 1) / grain);
    int best = 1;
    i64 best_cost = -1;
    for (int P = 1; P <= std::max(1, most); ++P) {
        const int c = ((U + P - 1) / P + grain - 1) / grain * grain;
        const int parts = (U + c - 1) / c;
        const i64 waves = (blocks * parts + target - 1) / target;
        const i64 cost = waves * (c / grain + 3 + (parts > 1 ? 2 : 0));
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = parts;
        }
    }
    *chunk = ((U + best - 1) / best + grain - 1) / grain * grain;
    return (U + *chunk - 1) / *chunk;
}

// column-tile width of the FP64 tensor-core GEMM for n columns: 80 where it
// needs fewer tiles than 64 (129 keys: two tiles instead of three)
static int col_tile(i64 n) { return (n + 79) / 80 < (n + 63) / 64 ? 80 : 64; }

// blocks per SM that the split aims at for the FP64 tensor-core tiles: one
// wave (three fit on an SM by shared memory)
constexpr int DM_SPLIT_TARGET = 3;

// ---------------------------------------------------------------------------
// stage C, per class: one warp per class, lanes stride over u, shuffle reduction
// Stage C computes either every class's dot product (k_stage_c)
// or every (pair, used key) product as one GEMM and gathers the classes from it
// (ProductOp + k_gather_q): the GEMM reuses each H2 row across keys at
// tensor-core rate, the per-class dots re-read an H2 row per class from L2 at
// about a tenth of that rate.  The product wins while it computes at most
// eight times as many dot products as there are classes, and the class list
// is long enough (65,536) for the GEMM's latency not to dominate.  With bounded plans
// the counts are known on the device only, so both paths are queued and each
// kernel checks the choice (`choice`: 0 run, 1 run if the product is chosen,
// 2 run if it is not).
__device__ __host__ inline bool product_pays(double pairs, double keys, i64 m) {
    return m >= 65536 && pairs * keys <= 8.0 * (double)m;
}
__device__ inline bool product_chosen(const PlanCounts* c, i64 m) {
    return product_pays((double)c->nP, (double)c->nku, m);
}
__device__ inline bool choice_runs(int choice, const PlanCounts* c, i64 m) {
    return choice == 0 || (choice == 1) == product_chosen(c, m);
}

// per class: one warp per class (its pair and C key found from the packed
// keys), lanes stride over u, shuffle reduction
__global__ void __launch_bounds__(256) k_stage_c(const double* __restrict__ W, const double* __restrict__ H2,
                                                  const uint64_t* __restrict__ keys, ClassDecode dec,
                                                  const int64_t* __restrict__ idx, int nk,
                                                  const uint32_t* __restrict__ pairBits,
                                                  const uint64_t* __restrict__ pairPre, i64 m, int U, int Up,
                                                  const PlanCounts* __restrict__ cnt, int choice,
                                                  double* __restrict__ out) {
    if (cnt->overflow || !choice_runs(choice, cnt, m)) return;
    const int lane = threadIdx.x & 31;
    const i64 warps = (i64)gridDim.x * (blockDim.x >> 5);
    for (i64 n = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); n < m; n += warps) {
        const uint64_t p = class_packed(keys, dec, idx, n);
        double acc = 0;
        if (p != BAD_KEYS) {
            int k[3];
            unpack_keys(p, k);
            const i64 pid = pair_id(pairBits, pairPre, (i64)k[1] * nk + k[0]);
            const double* w = W + (i64)k[2] * Up;
            const double* h = H2 + pid * Up;
            if (dcheck(pid < (i64)cnt->nP && k[2] < nk, 4, pid))
                for (int u = lane; u < U; u += 32) acc = fma(w[u], h[u], acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[n] = acc;
    }
}

// Q[p][j] = sum_u H2[p][u] W[keyOf[j]][u] over the pairs and used keys (their
// counts read on the device: blocks past them return at once).  A class reads
// Q at its pair (A key a, B key) and its largest key c >= a, and pairs are
// ordered by A key, so the column tiles of a row tile start at the key of its
// first A key: keys below it are never read (129 ERIDA keys: 166 blocks
// instead of 396).  blockIdx.z selects a chunk of u; the chunks' partial
// products go to separate slices of Q, summed by k_gather_q.
template <int BN_>
struct ProductOp {
    static constexpr bool A_KMAJOR = false, B_KMAJOR = false;
    static constexpr int BN = BN_;
    static constexpr int STAGES = 2, MIN_BLOCKS = 4;  // four blocks per SM: a grid under a wave splits u in three
    static constexpr int NB = BN / 16;  // B element pairs per thread
    const double* H2;
    const double* W;
    const int* keyOf;
    const int* pairA;
    const int* aKey;
    const uint64_t* kid;  // dense id of each used key
    const PlanCounts* cnt;
    i64 m;
    int choice, U, Up, ldq, u_chunk;
    double* Q;
    unsigned long long* products;  // count of the products computed (one add per tile)
    struct Block {
        int mvalid, nvalid, nk;
        int m0, n0, u0, u1;
        double* Q;
    };
    struct AState {
        i64 off[DM_BM / 16];
    };
    struct BState {
        i64 off[NB];
    };
    __device__ bool begin(Block& b) const {
        if (!choice_runs(choice, cnt, m)) return false;
        b.m0 = blockIdx.x * DM_BM;
        b.mvalid = min(DM_BM, (int)cnt->nP - b.m0);
        if (b.mvalid <= 0) return false;
        b.n0 = (int)kid[aKey[pairA[b.m0]]] + blockIdx.y * BN;
        b.nvalid = min(BN, (int)cnt->nku - b.n0);
        if (b.nvalid <= 0) return false;
        b.u0 = blockIdx.z * u_chunk;
        b.u1 = min(U, b.u0 + u_chunk);
        b.nk = (b.u1 - b.u0 + DM_BK - 1) / DM_BK;
        b.Q = Q;
        if (threadIdx.x == 0 && blockIdx.z == 0) atomicAdd(products, (unsigned long long)b.mvalid * b.nvalid);
        return b.nk > 0;
    }
    __device__ void a_init(const Block& b, AState& st) const {
#pragma unroll
        for (int q = 0; q < DM_BM / 16; ++q) {
            const int r = dm_pair_row(threadIdx.x, q);
            st.off[q] = r < b.mvalid ? (i64)(b.m0 + r) * Up : -1;
        }
    }
    __device__ void b_init(const Block& b, BState& st) const {
#pragma unroll
        for (int q = 0; q < NB; ++q) {
            const int r = dm_pair_row(threadIdx.x, q);
            st.off[q] = r < b.nvalid ? (i64)keyOf[b.n0 + r] * Up : -1;
        }
    }
    // pairs (u, u + 1), u even: H2 and W rows start at multiples of Up (a
    // multiple of 4), so every pair is 16-byte aligned
    __device__ void a_issue(const Block& b, AState& st, int kc, double* tile) const {
        const int k = dm_pair_k(threadIdx.x), u = b.u0 + kc * DM_BK + k;
        const int bytes = dm_pair_bytes(u, b.u1);
#pragma unroll
        for (int q = 0; q < DM_BM / 16; ++q) {
            const int n = st.off[q] >= 0 ? bytes : 0;
            dm_cp16(tile + dm_rowmajor_at(dm_pair_row(threadIdx.x, q), k), n ? H2 + st.off[q] + u : H2, n);
        }
    }
    __device__ void b_issue(const Block& b, BState& st, int kc, double* tile) const {
        const int k = dm_pair_k(threadIdx.x), u = b.u0 + kc * DM_BK + k;
        const int bytes = dm_pair_bytes(u, b.u1);
#pragma unroll
        for (int q = 0; q < NB; ++q) {
            const int n = st.off[q] >= 0 ? bytes : 0;
            dm_cp16(tile + dm_rowmajor_at(dm_pair_row(threadIdx.x, q), k), n ? W + st.off[q] + u : W, n);
        }
    }
    __device__ void store(const Block& b, int mm, int n, double v0, double v1) const {
        if (mm >= b.mvalid) return;
        double* q = b.Q + (i64)(b.m0 + mm) * ldq + b.n0 + n;
        if (n < b.nvalid) q[0] = v0;
        if (n + 1 < b.nvalid) q[1] = v1;
    }
};

// val[n] = Q[pair(n)][kid(k3)], the class's (pair, key) found from its packed
// keys
__global__ void __launch_bounds__(256) k_gather_q(const double* __restrict__ Q, i64 nq,
                                                   const uint64_t* __restrict__ keys, ClassDecode dec,
                                                   const int64_t* __restrict__ idx, i64 m,
                                                   const uint64_t* __restrict__ kid, int nk,
                                                   const uint32_t* __restrict__ pairBits,
                                                   const uint64_t* __restrict__ pairPre, int ldq,
                                                   const PlanCounts* __restrict__ cnt, int choice,
                                                   double* __restrict__ out) {
    if (cnt->overflow || !choice_runs(choice, cnt, m)) return;
    // four consecutive classes per group, two groups per thread and step
    // (16-byte loads and stores where the arrays allow): each class is a chain
    // of dependent loads (keys, then pair id and key id, then Q); the eight
    // chains run side by side, and a pair id equal to the previous class's is
    // not looked up again
    const bool vec = keys && ((uintptr_t)keys & 15) == 0 && ((uintptr_t)out & 15) == 0;
    const i64 groups = (m + 3) / 4, stride = (i64)gridDim.x * blockDim.x;
    constexpr int G = 2;
    for (i64 g0 = (i64)blockIdx.x * blockDim.x + threadIdx.x; g0 < groups; g0 += G * stride) {
        uint64_t p[G][4];
#pragma unroll
        for (int h = 0; h < G; ++h) {
            const i64 n0 = 4 * (g0 + h * stride);
            if (vec && n0 + 3 < m) {
                const ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2*>(keys + n0));
                const ulonglong2 b = __ldg(reinterpret_cast<const ulonglong2*>(keys + n0 + 2));
                p[h][0] = a.x, p[h][1] = a.y, p[h][2] = b.x, p[h][3] = b.y;
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) p[h][v] = n0 + v < m ? class_packed(keys, dec, idx, n0 + v) : BAD_KEYS;
            }
        }
        i64 q[G][4];
#pragma unroll
        for (int h = 0; h < G; ++h) {
            i64 last_slot = -1, last_pid = 0;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                q[h][v] = -1;
                if (p[h][v] != BAD_KEYS) {
                    int k[3];
                    unpack_keys(p[h][v], k);
                    const i64 slot = (i64)k[1] * nk + k[0];
                    if (slot != last_slot) {
                        last_slot = slot;
                        last_pid = pair_id(pairBits, pairPre, slot);
                    }
                    q[h][v] = last_pid * ldq + (i64)kid[k[2]];
                }
            }
        }
        double acc[G][4];
#pragma unroll
        for (int h = 0; h < G; ++h)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                acc[h][v] = 0.0;
                if (q[h][v] >= 0 && dcheck(q[h][v] < nq, 3, q[h][v])) acc[h][v] = Q[q[h][v]];
            }
#pragma unroll
        for (int h = 0; h < G; ++h) {
            const i64 n0 = 4 * (g0 + h * stride);
            if (n0 >= m) continue;
            if (vec && n0 + 3 < m) {
                reinterpret_cast<double2*>(out + n0)[0] = make_double2(acc[h][0], acc[h][1]);
                reinterpret_cast<double2*>(out + n0)[1] = make_double2(acc[h][2], acc[h][3]);
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    if (n0 + v < m) out[n0 + v] = acc[h][v];
            }
        }
    }
}

// The class gather of replays that reuse their plan without marking the
// classes (the mark pass skipped): each class is decoded here from its index
// (through the pair descriptors where PD, else class_keys) and checked against
// the plan -- its (A, B) pair set in the plan's pair bitmap and its third key
// a used key (bit 31 of kk[k2]), which the marks of the list that made the
// plan guarantee for every class of that list.  A class outside the plan
// (the list was rewritten in place since) or outside the tensor sets the
// overflow flag, and the host evaluates the list again with a new plan.  This
// saves the mark pass's read of the indices and the write and re-read of the
// packed keys (24 bytes per class).
template <bool PD>
__global__ void __launch_bounds__(256, PD ? 8 : 6) k_gather_q_plan(const double* __restrict__ Q, int nq,
                                                        ClassDecode dec, const int64_t* __restrict__ idx, i64 m,
                                                        const uint32_t* __restrict__ kk, int nk,
                                                        const uint2* __restrict__ bitpre, int ldq,
                                                        PlanCounts* __restrict__ cnt, double* __restrict__ out) {
    if (cnt->overflow) return;
    const bool vec = ((uintptr_t)idx & 15) == 0 && ((uintptr_t)out & 15) == 0;
    const i64 groups = (m + 3) / 4, stride = (i64)gridDim.x * blockDim.x;
    // one group of four classes per thread and step, at most 32 registers:
    // eight blocks per SM hide the dependent loads better than two groups
    // at four blocks (ERI 7^3 stage C 45 against 49 us)
    constexpr int G = 1;
    bool miss = false;
    for (i64 g0 = (i64)blockIdx.x * blockDim.x + threadIdx.x; g0 < groups; g0 += G * stride) {
        int64_t c[G][4];
#pragma unroll
        for (int h = 0; h < G; ++h) {
            const i64 n0 = 4 * (g0 + h * stride);
            if (vec && n0 + 3 < m) {
                const longlong2 a = __ldg(reinterpret_cast<const longlong2*>(idx + n0));
                const longlong2 b = __ldg(reinterpret_cast<const longlong2*>(idx + n0 + 2));
                c[h][0] = a.x, c[h][1] = a.y, c[h][2] = b.x, c[h][3] = b.y;
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) c[h][v] = n0 + v < m ? __ldg(&idx[n0 + v]) : 0;
            }
        }
        int q[G][4];
#pragma unroll
        for (int h = 0; h < G; ++h) {
            const i64 n0 = 4 * (g0 + h * stride);
            uint64_t base = PD_NO_BASE;
            uint2 da = make_uint2(0, 0);
            int last_slot = -1, last_pid = -1;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                q[h][v] = -1;
                if (n0 + v >= m) continue;
                int s0, s1, s2;
                if constexpr (PD) {
                    if (!pd_class_keys(dec, c[h][v], base, da, s0, s1, s2)) {
                        miss = true;
                        continue;
                    }
                } else {
                    int k[3];
                    if (!class_keys(dec, c[h][v], k)) {
                        miss = true;
                        continue;
                    }
                    s0 = k[0], s1 = k[1], s2 = k[2];
                }
                if (!dcheck(s0 >= 0 && s2 < nk, 1, s2)) continue;
                const int slot = s1 * nk + s0;
                if (slot != last_slot) {
                    last_slot = slot;
                    const uint2 bp = __ldg(&bitpre[slot >> 5]);  // (bits, pairs before the word)
                    const uint32_t bit = (uint32_t)(slot & 31);
                    last_pid = (bp.x >> bit) & 1u ? (int)(bp.y + __popc(bp.x & ((1u << bit) - 1u))) : -1;
                }
                const uint32_t k0 = __ldg(&kk[s2]);  // key id, bit 31: a key the list uses
                if (last_pid < 0 || !(k0 >> 31)) {
                    miss = true;
                    continue;
                }
                q[h][v] = last_pid * ldq + (int)(k0 & 0x7fffffffu);  // (Q has fewer than 2^31 entries)
            }
        }
        double acc[G][4];
#pragma unroll
        for (int h = 0; h < G; ++h)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                acc[h][v] = 0.0;
                if (q[h][v] >= 0 && dcheck(q[h][v] < nq, 3, q[h][v])) acc[h][v] = Q[q[h][v]];
            }
#pragma unroll
        for (int h = 0; h < G; ++h) {
            const i64 n0 = 4 * (g0 + h * stride);
            if (n0 >= m) continue;
            if (vec && n0 + 3 < m) {
                reinterpret_cast<double2*>(out + n0)[0] = make_double2(acc[h][0], acc[h][1]);
                reinterpret_cast<double2*>(out + n0)[1] = make_double2(acc[h][2], acc[h][3]);
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    if (n0 + v < m) out[n0 + v] = acc[h][v];
            }
        }
    }
    if (miss) atomicExch(reinterpret_cast<unsigned long long*>(&cnt->overflow), 1ull);
}

// ---------------------------------------------------------------------------
// mixed form: stages A and B as int8-sliced products on the tensor cores
//   stage A:  H^T[j][a] = sum_t G[j][t] W[aKey[a]][t],   G[j][t] = T[S[j] + t^2]
//   stage B:  H2[p][u]  = sum_v Hf[a][u][v] W[pairB[p]][v]  for the pairs p of A key a
// (Hf[a] is symmetric, so its rows serve as the K-major operand); stage C
// stays FP64 (its product form is a small DMMA GEMM).
struct LatticeGRows {
    const double* T;
    const int* S;
    __device__ RowBase row(i64 r) const { return {T + S[r]}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k * k]; }
    __device__ bool valid(i64) const { return true; }
    GLI_IDENTITY_ROWS
};

struct AKeyRows {  // A key a: row W[aKey[a]]
    const double* W;
    const int* aKey;
    const PlanCounts* cnt;
    i64 Up;
    __device__ RowBase row(i64 a) const { return {W + (i64)aKey[a] * Up}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k]; }
    __device__ bool valid(i64 a) const { return a < cnt->nA; }
    GLI_IDENTITY_ROWS
};

struct ExpandedHRows {  // row r = a * U + u of the stacked Hf[a], batch a padded to whole tiles
    const double* H;
    const int* sidx;
    const PlanCounts* cnt;
    i64 nS;
    int U, blocks;
    struct Ctx {
        const double* h;  // H row of the A key
        const int* map;   // sidx row u
    };
    __device__ Ctx row(i64 r) const {
        const i64 a = r / U, u = r - a * U;
        return {H + a * nS, sidx + u * U};
    }
    __device__ double at(const Ctx& c, int k) const { return c.h[c.map[k]]; }
    __device__ i64 dest(i64 r) const { return (r / U) * blocks * TC_BM + r % U; }
    __device__ i64 source(i64 d, i64 rows) const {
        const i64 a = d / ((i64)blocks * TC_BM), u = d % ((i64)blocks * TC_BM);
        return (u < U && a * U + u < rows) ? a * U + u : -1;
    }
    __device__ bool valid(i64 r) const { return r < cnt->nA * U; }
};

struct PairRows {  // pair p: row W[pairB[p]], placed in the tiles of its A key
    const double* W;
    const int* pairA;
    const int* pairB;
    const int* first;       // first pair of each A key
    const int* tile0;       // first tile of each A key
    const int* tile_col0;   // first pair of each tile
    const int* tile_ncols;  // pairs in each tile
    const PlanCounts* cnt;
    i64 Up;
    int bn;  // rows per tile
    __device__ RowBase row(i64 p) const { return {W + (i64)pairB[p] * Up}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k]; }
    __device__ i64 dest(i64 p) const {
        const int a = pairA[p];
        return (i64)tile0[a] * bn + (p - first[a]);
    }
    __device__ i64 source(i64 d, i64 rows) const {
        const i64 t = d / bn;
        const int j = (int)(d % bn);
        const i64 p = j < tile_ncols[t] ? (i64)tile_col0[t] + j : -1;
        return p < rows ? p : -1;
    }
    __device__ bool valid(i64 p) const { return p < (i64)cnt->nP; }
};

// Balanced hosts of a full pair triangle.  A pair's stage-B row is symmetric
// in its two keys (sum_v sum_t W_b[v] W_a[t] T[u^2 + v^2 + t^2]), so either
// key's H row can host it.  Hosting by the larger key gives key a a + 1 rows
// (ragged tiles: 67% full at 129 keys); when every pair {a, b} of n A keys is
// present the hosts are chosen instead so that most keys fill whole tiles:
// keys below y = min(n, 2 bn - 1) form a regular tournament (key i hosts its
// own pair and i + j mod y for j < reg_count(i, y): at most bn rows), and the
// keys from y up host every pair with a key below y plus a regular tournament
// among themselves (129 keys: 132 tiles of 64 instead of 195).
__host__ __device__ __forceinline__ int reg_count(int i, int y) { return (y & 1) ? (y + 1) / 2 : y / 2 + (i < y / 2); }
__host__ __device__ __forceinline__ int reg_prefix(int i, int y) {  // rows of the members below i
    if (y & 1) return i * ((y + 1) / 2);
    const int h = y / 2;
    return i <= h ? i * (h + 1) : h * (h + 1) + (i - h) * h;
}
__host__ __device__ __forceinline__ int bal_count(int h, int n, int y) {
    return h < y ? reg_count(h, y) : y + reg_count(h - y, n - y);
}
__device__ __forceinline__ int bal_offset(int h, int n, int y) {
    return h < y ? reg_prefix(h, y) : y * (y + 1) / 2 + (h - y) * y + reg_prefix(h - y, n - y);
}
// the partner key of host h's j-th row
__device__ __forceinline__ int bal_partner(int h, int j, int n, int y) {
    if (h < y) return (h + j) % y;
    return j < y ? j : y + (h - y + j - y) % (n - y);
}

// One block: first pair, pair count and first tile of every A key (pairs are
// ordered by A key), and the tile list of stage B (tiles of bn rows, each in
// one host A key); tiles past the last one get no columns.  With row lists
// (rowPair, rowKey: the H2 row and the weight key of each tile row) a full
// pair triangle of more than bn keys gets balanced hosts; otherwise the rows
// are the pairs in order, each hosted by its A key.
// (pairA, pairB and aKey may have been written earlier in the same kernel:
// plain coherent loads, no __restrict__)
__device__ void pair_tiles_block(bool first_ready, const int* pairA, const int* pairB, const int* aKey, int nP, int nA, int nku, int bn, int max_tiles,
                                 int* __restrict__ first, int* __restrict__ tile0, int* __restrict__ tile_batch,
                                 int* __restrict__ tile_col0, int* __restrict__ tile_ncols, int* __restrict__ rowPair,
                                 int* __restrict__ rowKey) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    for (int t = threadIdx.x; t < max_tiles; t += blockDim.x) tile_ncols[t] = 0;
    // every A key has at least one pair, and pairs are sorted by A key: the
    // first pair of each key is where the key changes (unless the caller
    // filled first[] already)
    if (!first_ready)
        for (int p = threadIdx.x; p < nP; p += blockDim.x)
            if (p == 0 || pairA[p] != pairA[p - 1]) first[pairA[p]] = p;
    const bool balanced = rowPair && nA > bn && nku == nA && (i64)nP == (i64)nA * (nA + 1) / 2;
    const int y = min(nA, 2 * bn - 1);
    if (rowPair) {
        if (balanced) {
            // host h's rows in stripes of 8 threads
            for (int item = threadIdx.x; item < nA * 8; item += blockDim.x) {
                const int h = item >> 3, d = bal_count(h, nA, y), o = bal_offset(h, nA, y);
                for (int j = item & 7; j < d; j += 8) {
                    const int g = bal_partner(h, j, nA, y), hi = max(h, g), lo = min(h, g);
                    rowPair[o + j] = hi * (hi + 1) / 2 + lo;  // the pair id of (hi, lo) in a full triangle
                    rowKey[o + j] = aKey[g];
                }
            }
        } else {
            for (int p = threadIdx.x; p < nP; p += blockDim.x) {
                rowPair[p] = p;
                rowKey[p] = pairB[p];
            }
        }
    }
    __syncthreads();
    for (int base = 0; base < nA; base += blockDim.x) {
        const int a = base + threadIdx.x;
        int lo = 0, npairs = 0;
        if (a < nA) {
            if (balanced) {
                lo = bal_offset(a, nA, y);
                npairs = bal_count(a, nA, y);
            } else {
                lo = first[a];
                npairs = (a + 1 < nA ? first[a + 1] : nP) - lo;
            }
        }
        const int nt = (npairs + bn - 1) / bn;
        // block exclusive scan of nt
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        int incl = nt;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const int ws = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
            int wi = ws;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += v;
            }
            warp_sums[lane] = wi - ws;
        }
        __syncthreads();
        const int t0 = carry + warp_sums[warp] + incl - nt;
        if (a < nA) {
            tile0[a] = t0;
            for (int k = 0; k < nt; ++k) {
                tile_batch[t0 + k] = a;
                tile_col0[t0 + k] = lo + k * bn;
                tile_ncols[t0 + k] = min(bn, npairs - k * bn);
            }
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = t0 + nt;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) k_pair_tiles(const int* __restrict__ pairA, const int* __restrict__ pairB,
                                                      const int* __restrict__ aKey, const PlanCounts* __restrict__ cnt,
                                                      int bn, int max_tiles, int* __restrict__ first,
                                                      int* __restrict__ tile0, int* __restrict__ tile_batch,
                                                      int* __restrict__ tile_col0, int* __restrict__ tile_ncols,
                                                      int* __restrict__ rowPair, int* __restrict__ rowKey) {
    pair_tiles_block(false, pairA, pairB, aKey, (int)cnt->nP, (int)cnt->nA, (int)cnt->nku, bn, max_tiles, first,
                     tile0, tile_batch, tile_col0, tile_ncols, rowPair, rowKey);
}

// the tile arrays of one stage B launch: first pair and first tile of every A
// key, then batch (host A key), first row and row count of every tile, and
// (FP64 stage B: `rows`) the H2 row and weight key of every tile row
struct PairTiles {
    DevBuf<int> buf;
    int bn = 0;
    i64 max_tiles = 0;
    int *first = nullptr, *tile0 = nullptr, *batch = nullptr, *col0 = nullptr, *ncols = nullptr;
    int *rowPair = nullptr, *rowKey = nullptr;
    bool built = false;
    static i64 ints(i64 nA, i64 nP, int tile_pairs, bool rows) {
        return 2 * nA + 3 * (nP / tile_pairs + nA + 1) + (rows ? 2 * nP : 0);
    }
    // mem: nullptr to allocate on the stream, or ints(...) ints lent by an owner
    void alloc(i64 nA, i64 nP, int tile_pairs, bool rows, cudaStream_t s, int* mem = nullptr) {
        bn = tile_pairs;
        max_tiles = nP / bn + nA + 1;
        if (mem)
            buf.borrow(mem, ints(nA, nP, tile_pairs, rows), s);
        else
            buf.alloc(ints(nA, nP, tile_pairs, rows), s);
        first = buf.p;
        tile0 = buf.p + nA;
        batch = buf.p + 2 * nA;
        col0 = batch + max_tiles;
        ncols = col0 + max_tiles;
        rowPair = rows ? ncols + max_tiles : nullptr;
        rowKey = rows ? rowPair + nP : nullptr;
    }
};

// The plan of a captured evaluation (bounded or sized), kept between the
// replays of its graph: the key and pair lists, word prefixes and stage-B
// tiles, plus the key flags, the pair bitmap and the counts they were made
// from.  A replay that marks its classes compares its key flags and pair
// bitmap with the saved ones on the device: when they are equal, the plan
// they determine is the saved one and the plan kernel only restores its
// counts; otherwise it plans anew and saves.  (The plan is a function of those
// flags and bits alone.)  Replays of the product form do not mark at all while
// the saved plan is valid: their gather checks every class instead
// (k_gather_q_plan).
struct PlanReuse {
    uint32_t* saved_used = nullptr;
    uint32_t* saved_bits = nullptr;
    PlanCounts* saved_cnt = nullptr;
    int* valid = nullptr;  // null: no reuse (bounded plans)
    // the plan in the form the plan-checking gather reads: per pair-bitmap
    // word its bits and the pairs before it, per key its id with bit 31 set
    // when the list uses it (one load each instead of two)
    uint2* bitpre = nullptr;
    uint32_t* kk = nullptr;
    // set: the replay did not mark its classes (the mark pass skipped them and
    // k_gather_q_plan checks each against the plan), so a valid saved plan is
    // restored without the comparison
    int trust = 0;
};
struct PlanStore {
    DevMem<uint64_t> ids, pairPre;
    DevMem<int> keyOf, aId, aKey, pairA, pairB, tiles;
    DevMem<uint32_t> saved_used, saved_bits;
    DevMem<PlanCounts> saved_cnt;
    DevMem<int> valid;
    DevMem<uint2> bitpre;
    DevMem<uint32_t> kk;
    DevMem<uint2> pd;  // the ERI pair descriptors, when the decode uses them
    // the (pair, key) products of a product-form stage C, kept with the graph
    // so that a class gather launched apart from it can read them
    DevMem<double> Q;
    void alloc(i64 nk, i64 words, i64 capA, i64 capP, i64 tile_ints, i64 pairs, i64 q_entries) {
        if (pairs > 0) pd.alloc((size_t)pairs);
        if (q_entries > 0) Q.alloc((size_t)q_entries);
        ids.alloc((size_t)(2 * nk));
        pairPre.alloc((size_t)words);
        keyOf.alloc((size_t)nk);
        aId.alloc((size_t)nk);
        aKey.alloc((size_t)nk);
        pairA.alloc((size_t)std::max<i64>(capP, 1));
        pairB.alloc((size_t)std::max<i64>(capP, 1));
        tiles.alloc((size_t)tile_ints);
        saved_used.alloc((size_t)(2 * nk));
        saved_bits.alloc((size_t)words);
        bitpre.alloc((size_t)words);
        kk.alloc((size_t)nk);
        saved_cnt.alloc(1);
        valid.alloc(1);
        GLI_CUDA(cudaMemset(valid.p, 0, sizeof(int)));
    }
    PlanReuse reuse(bool trust) {
        PlanReuse r;
        r.saved_used = saved_used.p;
        r.saved_bits = saved_bits.p;
        r.saved_cnt = saved_cnt.p;
        r.valid = valid.p;
        r.bitpre = bitpre.p;
        r.kk = kk.p;
        r.trust = trust ? 1 : 0;
        return r;
    }
};

// Bounded plans (at most 256 keys: 512 key flags, 2,048 pair-bitmap words):
// the key plan, the pair plan and the stage-B tiles in one single-block launch
// (three phases separated by block barriers; the global writes of a phase
// are visible to the next).  The pair bitmap, its word prefixes and the A ids
// stay in shared memory for the pair placement (a thread per slot) and for the
// first pair of each A key (the count of set bits before its row).
//
// capA, capP: the A keys and pairs the buffers hold.  Bounded plans pass
// bounds that cannot be exceeded; plans sized by an earlier evaluation of the
// same list pass its counts, and a list that needs more sets the overflow
// flag and zeroes the counts before anything is written past the buffers.
constexpr int PLAN_SMALL_KEYS = 384, PLAN_SMALL_WORDS = PLAN_SMALL_KEYS * PLAN_SMALL_KEYS / 32;
__global__ void __launch_bounds__(1024) k_plan_small(i64 nk, i64 capA, i64 capP, const uint32_t* __restrict__ used,
                                                     uint64_t* __restrict__ ids, int* __restrict__ keyOf,
                                                     int* __restrict__ aId, int* __restrict__ aKey, i64 words,
                                                     const uint32_t* __restrict__ bits, uint64_t* __restrict__ pre,
                                                     int* __restrict__ pairA, int* __restrict__ pairB, int bn,
                                                     int max_tiles, int* __restrict__ first, int* __restrict__ tile0,
                                                     int* __restrict__ tile_batch, int* __restrict__ tile_col0,
                                                     int* __restrict__ tile_ncols, int* __restrict__ rowPair,
                                                     int* __restrict__ rowKey, PlanCounts* __restrict__ cnt,
                                                     PlanReuse reuse) {
    __shared__ uint32_t ws[32], total, nku_s;
    __shared__ uint32_t s_bits[PLAN_SMALL_WORDS], s_pre[PLAN_SMALL_WORDS];
    __shared__ int s_aId[PLAN_SMALL_KEYS], s_aKey[PLAN_SMALL_KEYS];
    if (reuse.valid && *reuse.valid) {
        // the saved plan stands if this list marked the same keys and pairs
        // (or was not marked: the gather checks its classes instead)
        bool same = true;
        if (!reuse.trust) {
            for (i64 i = threadIdx.x; i < 2 * nk; i += blockDim.x) same = same && used[i] == reuse.saved_used[i];
            for (i64 w = threadIdx.x; w < words; w += blockDim.x) same = same && bits[w] == reuse.saved_bits[w];
        }
        if (__syncthreads_and(same)) {
            if (threadIdx.x == 0) {
                const PlanCounts c = *reuse.saved_cnt;
                cnt->key_total = c.key_total;
                cnt->nku = c.nku;
                cnt->nA = c.nA;
                cnt->nP = c.nP;
                cnt->overflow = 0;
            }
            return;
        }
    }
    // keys: joint scan of [usedKey | usedA]
    const int k = threadIdx.x;  // flag k of 2 nk (<= 512)
    const uint32_t f = k < 2 * nk ? used[k] : 0u;
    const uint32_t ex = block_scan_1024(f, ws, &total);
    if (k < 2 * nk) ids[k] = ex;
    if (k == nk) nku_s = ex;  // exclusive count at nk = used keys
    __syncthreads();
    const uint32_t nku = nk > 0 ? nku_s : 0u;
    const uint32_t key_total = total;  // (total is reused by the pair scan below)
    const int nA = (int)(key_total - nku);
    if (k < nk && f) keyOf[ex] = k;
    if (k >= nk && k < 2 * nk && f) {
        const int a = (int)(ex - nku);
        aId[k - nk] = a;
        aKey[a] = (int)(k - nk);
        s_aId[k - nk] = a;
        s_aKey[a] = (int)(k - nk);
    }
    __syncthreads();
    // pairs: per-word exclusive counts, then every set bit placed in parallel
    uint32_t carry = 0;
    for (i64 base = 0; base < words; base += 1024) {
        const i64 w = base + threadIdx.x;
        const uint32_t b = w < words ? bits[w] : 0u;
        const uint32_t id = carry + block_scan_1024(__popc(b), ws, &total);
        if (w < words) {
            pre[w] = id;
            s_bits[w] = b;
            s_pre[w] = id;
        }
        carry += total;
        __syncthreads();  // total and ws are rewritten by the next tile's scan
    }
    const int nP = (int)carry;
    const bool over = nA > capA || (i64)nP > capP;  // the same on every thread
    if (over && tile_ncols)
        for (int t = threadIdx.x; t < max_tiles; t += blockDim.x) tile_ncols[t] = 0;  // stage B: no tiles
    if (over && reuse.valid && threadIdx.x == 0) *reuse.valid = 0;
    if (threadIdx.x == 0) {
        cnt->key_total = over ? 0 : key_total;
        cnt->nku = over ? 0 : nku;
        cnt->nA = over ? 0 : nA;
        cnt->nP = over ? 0 : nP;
        cnt->overflow = over ? 1 : 0;
    }
    if (over) return;
    const int slots = (int)(nk * nk);
    for (int slot = threadIdx.x; slot < slots; slot += blockDim.x) {
        const uint32_t b = s_bits[slot >> 5];
        if (!((b >> (slot & 31)) & 1u)) continue;
        const int id = (int)s_pre[slot >> 5] + __popc(b & ((1u << (slot & 31)) - 1u));
        const int k2 = slot / (int)nk;
        pairA[id] = s_aId[k2];
        pairB[id] = slot - k2 * (int)nk;
    }
    // the first pair of A key a: the set bits before row aKey[a]
    if (first)
        for (int a = threadIdx.x; a < nA; a += blockDim.x) {
            const int slot = s_aKey[a] * (int)nk, w = slot >> 5;
            first[a] = (int)s_pre[w] + __popc(s_bits[w] & ((1u << (slot & 31)) - 1u));
        }
    __syncthreads();
    if (first)
        pair_tiles_block(true, pairA, pairB, aKey, nP, nA, (int)nku, bn, max_tiles, first, tile0, tile_batch,
                         tile_col0, tile_ncols, rowPair, rowKey);
    if (reuse.valid) {
        // save what this plan was made from, for the next replay's check
        for (i64 i = threadIdx.x; i < 2 * nk; i += blockDim.x) reuse.saved_used[i] = used[i];
        for (i64 w = threadIdx.x; w < words; w += blockDim.x) {
            reuse.saved_bits[w] = s_bits[w];
            reuse.bitpre[w] = make_uint2(s_bits[w], s_pre[w]);
        }
        if (k < nk) reuse.kk[k] = ex | (f ? 0x80000000u : 0u);
        if (threadIdx.x == 0) {
            PlanCounts c;
            c.key_total = key_total;
            c.nku = nku;
            c.nA = nA;
            c.nP = nP;
            c.overflow = 0;
            *reuse.saved_cnt = c;
            *reuse.valid = 1;
        }
    }
}

// The first kernel of a replay that trusts its kept plan (the host has seen an
// earlier replay of the graph complete): the plan's counts, or, should no
// valid plan be kept, an overflow (the host then evaluates anew).  Such a
// replay launches neither the mark pass nor the plan kernel; its class gather
// checks every class against the kept plan (k_gather_q_plan).
__global__ void k_restore_plan(PlanReuse reuse, EvalStatus* __restrict__ st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    restore_status(*reuse.valid != 0, reuse.saved_cnt, st);
}

// G sliced once per table set (cached with the tables); the build synchronises
// the stream so that the slices are ready for any stream that uses them later
static TiledOperand lattice_g_slices(const LatticeTables& t, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(t.g_mu);
    if (!t.g_sliced) {
        auto g = std::make_unique<TiledTable>();
        const int nkc = (int)((t.U + TC_BK - 1) / TC_BK);
        const i64 rows = (t.nS + TC_BM - 1) / TC_BM * TC_BM;
        g->data.alloc((size_t)MIXED_SLICES * rows * nkc * TC_BK);
        g->e.alloc((size_t)rows);
        g->view = TiledOperand{g->data.p, g->e.p, nkc, MIXED_SLICES};
        launch_slice(LatticeGRows{t.T.p, t.S.p}, t.nS, rows, (int)t.U, nkc, MIXED_SLICES, TC_BM, g->data.p, g->e.p, s);
        GLI_CUDA(cudaStreamSynchronize(s));
        t.g_sliced = std::move(g);
    }
    return t.g_sliced->view;
}

void dgemm_prepare();  // dense.cu: attributes of the strided FP64 GEMM

static thread_local bool t_timing = false;
static thread_local ContractStats t_last;
static thread_local int t_paths = 0;  // tensor-core stages of the evaluation being completed
// product threshold of the evaluation being completed and its screening bound
static thread_local double t_screen_tol = 0.0, t_screen_bound = 0.0;
// the stage marks of the timed graph the evaluation being completed replayed
static thread_local struct StageTimer* t_graph_timer = nullptr;

void set_timing(bool on) { t_timing = on; }
const ContractStats& last_stats() { return t_last; }

// (external: the marks are recorded inside a graph capture, as event record
// nodes of the graph, so that every replay of the graph records them)
struct StageTimer {
    static constexpr int kMax = 8;
    bool on;
    cudaStream_t s;
    bool external;
    cudaEvent_t ev[kMax];
    int n = 0;
    StageTimer(bool enabled, cudaStream_t st, bool in_graph = false) : on(enabled), s(st), external(in_graph) {
        if (on)
            for (auto& e : ev) GLI_CUDA(cudaEventCreate(&e));
    }
    void mark() {
        if (!on) return;
        if (n >= kMax) fail(GLI_ERR_INTERNAL, "stage timer overflow");
        GLI_CUDA(external ? cudaEventRecordWithFlags(ev[n++], s, cudaEventRecordExternal) : cudaEventRecord(ev[n++], s));
    }
    StageTimer(const StageTimer&) = delete;
    StageTimer& operator=(const StageTimer&) = delete;
    ~StageTimer() {
        if (on)
            for (auto& e : ev) cudaEventDestroy(e);
    }
    float between(int a, int b) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[a], ev[b]);
        return ms;
    }
};

// status of one evaluation, read back by the host after the last kernel
struct EvalArgs {
    bool mixed = false;
    const LatticeTables* t = nullptr;
    TiledOperand G;
    ClassDecode d;
    const int64_t* idx = nullptr;
    i64 m = 0;
    double* out = nullptr;
    int num_sms = 148;
};

// Sizes that the host must know to allocate and launch: either bounds derived
// from the key space (no host synchronisation: the whole evaluation can be
// queued, and captured in a CUDA graph) or the exact counts (two host round
// trips; used when the key space is too large for bounds to be cheap).
struct EvalSizes {
    i64 nku = 0, nA = 0, nP = 0;
};

// A key space of at most this many dense keys is planned with bounds: every
// ERIDA grid up to 256 points per axis and ERI grids up to 5 points per axis
// (135 keys).  Larger ERI key spaces (364 keys at 7 points) keep exact sizes:
// their pair count is far below the bound, and the exact count selects the
// product form of stage C.
constexpr i64 BOUNDED_KEYS = 256;

// stage A runs on the tensor cores (mixed form) from this many outputs nA nS
// (GLI_B200_TC_A_OUTPUTS overrides it, for measurements)
constexpr i64 TC_A_OUTPUTS = 1000000;
static i64 tc_a_outputs() {
    static const i64 v = [] {
        const char* e = getenv("GLI_B200_TC_A_OUTPUTS");
        return e && *e ? (i64)atoll(e) : TC_A_OUTPUTS;
    }();
    return v;
}

// the tensor-core stages of the last evaluation queued by this thread (bit 0:
// stage A, bit 1: stage B) and its class gather (bits 2-3: 1 k_gather_q, 2
// k_gather_q_plan; 0 none, the per-class stage C)
static thread_local int t_enq_paths = 0;

// Stage B on the tensor cores slices every row of the expanded Hf (nA U^2
// gathered values) against an FP64 product of nP U^2 FMAs: measured at ERIDA
// 129^3 (nP = 65 nA) the two cost the same, so the sliced form is taken only
// when the pairs per A key are clearly more.
// (GLI_B200_TC_B_PAIRS_PER_KEY and GLI_B200_TC_B_OUTPUTS override the two
// thresholds, for measurements)
static i64 env_i64(const char* name, i64 dflt) {
    const char* e = getenv(name);
    return e && *e ? (i64)atoll(e) : dflt;
}
static bool stage_b_sliced(bool mixed, i64 nA, i64 nP, int U) {
    static const i64 per_key = env_i64("GLI_B200_TC_B_PAIRS_PER_KEY", 80);
    static const i64 outputs = env_i64("GLI_B200_TC_B_OUTPUTS", 4000000);
    return mixed && nA * (i64)U * U >= outputs && nP >= per_key * nA;
}

static void read_status(EvalStatus* d_st, EvalStatus& h, cudaStream_t s) {
    GLI_CUDA(cudaMemcpyAsync(&h, d_st, sizeof(EvalStatus), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
}

// How the host sizes an evaluation's buffers and grids:
//   PLAN_BOUNDED  bounds derived from the key space (small key spaces);
//   PLAN_EXACT    the exact counts, read back once after the plan (a host
//                 round trip in the middle of the evaluation);
//   PLAN_SIZED    the counts of an earlier evaluation of the same list, passed
//                 in `sz`: nothing is read back; the plan kernel checks the
//                 list against these sizes and flags an overflow instead of
//                 writing past them (the host then evaluates again, exactly).
enum PlanMode { PLAN_BOUNDED = 0, PLAN_EXACT = 1, PLAN_SIZED = 2 };

// key spaces that the sized plan's single-block plan kernel holds
static bool sized_plan_fits(i64 nk) { return nk <= PLAN_SMALL_KEYS && (nk * nk + 31) / 32 <= 8 * 1024; }

// What a plan-checking class gather needs, for a gather launched apart from
// the graph of its stages (the pipelined host-buffer path gathers the class
// list range by range as it arrives): all of it lives with the graph (its
// kept plan, its products Q, its status block).
struct GatherLaunch {
    const double* Q = nullptr;
    i64 nq = 0;  // entries of Q
    ClassDecode dec;
    const uint32_t* kk = nullptr;
    int nk = 0;
    const uint2* bitpre = nullptr;
    int ldq = 0;
    PlanCounts* cnt = nullptr;
};

// the plan-checking gather of classes idx[0, m) into out[0, m)
static void launch_gather(const GatherLaunch& gl, const int64_t* idx, i64 m, double* out, int num_sms,
                          cudaStream_t s) {
    if (m <= 0) return;
    if (gl.nq >= ((i64)1 << 31)) fail(GLI_ERR_INTERNAL, "class gather over %lld products", (long long)gl.nq);
    const unsigned gq = (unsigned)std::min<i64>(((m + 3) / 4 + 255) / 256, (i64)num_sms * 8);
    if (gl.dec.pd)
        launch_kernel(k_gather_q_plan<true>, dim3(gq), dim3(256), 0, s, gl.Q, (int)gl.nq, gl.dec, idx, m,
                      gl.kk, gl.nk, gl.bitpre, gl.ldq, gl.cnt, out);
    else
        launch_kernel(k_gather_q_plan<false>, dim3(gq), dim3(256), 0, s, gl.Q, (int)gl.nq, gl.dec, idx,
                      m, gl.kk, gl.nk, gl.bitpre, gl.ldq, gl.cnt, out);
}

// the u split of the stage-C product: 64-column tiles (the product's grid is
// small, and wider tiles cost it parallelism: ERIDA 129^3 73 us with 80
// columns, 66 us with 64).  A grid under a wave (four blocks per SM; about half
// the column tiles are active after the A-key shift) splits u over up to four
// blocks of a cluster, which sum their partial tiles in distributed shared
// memory, so Q holds one product per (pair, key).  (Summing slices of Q in the
// gather instead made ERI 7^3's 3.57 million classes read several values
// each.)  Returns the blocks per tile; *u_chunk their length of u.
static int product_split(i64 nP, i64 nku, int U, int num_sms, int* u_chunk) {
    const i64 mt = (nP + DM_BM - 1) / DM_BM, nt = (nku + DM_BN - 1) / DM_BN;
    *u_chunk = U;
    const int P = std::min(4, split_count(mt * ((nt + 1) / 2), U, DM_BK, 4 * (i64)num_sms, u_chunk));
    *u_chunk = ((U + P - 1) / P + DM_BK - 1) / DM_BK * DM_BK;
    return (U + *u_chunk - 1) / *u_chunk;
}

// Stage A with 129..144 A keys holds them in one 144-column tile and does not
// split the whole K range (the partial 144-column tiles would not fit the
// operand ring for the cluster sum, and summing them through HBM measured
// slower, ERIDA 129^3 0.439 against 0.410 ms).  Only a last wave under half
// full is split in K, two blocks per m tile (ERIDA 129^3: 1,072 m tiles on 444
// block slots, 2.41 waves).  Returns the m tiles split so (0: none).
static i64 stage_a_tail(i64 nA, int nS, int U, int num_sms) {
    if (!(nA > 128 && nA <= 144)) return 0;
    const i64 mb = (nS + DM_BM - 1) / DM_BM;
    const i64 slots = (i64)dmma_blocks_per_sm<StageAOp<144>>() * num_sms;
    const i64 tail = mb % slots;
    return tail > 0 && 2 * tail <= slots && (U + DM_BK - 1) / DM_BK >= 2 ? tail : 0;
}

// Buffers of the three stages, sized by the plan's counts
struct StageBufs {
    DevBuf<double> H, H2, Q;
    DevBuf<double> split_ws;  // stage A's tail split: two partial tiles per split m tile
    DevBuf<unsigned> tickets;
    int q_parts = 0, u_chunk = 0;
    i64 tail = 0;
    void alloc(const EvalArgs& a, const EvalSizes& sz, bool tc_a, bool product, cudaStream_t s,
               const PlanStore* keep = nullptr) {
        const LatticeTables& t = *a.t;
        const int U = (int)t.U, Up = (int)t.Up, nS = (int)t.nS;
        if (sz.nA * (i64)U * U > ((i64)1 << 31))
            fail(GLI_ERR_LIMIT, "stage buffers exceed 16 GB (%lld A keys, lattice extent %d)", (long long)sz.nA, U);
        H.alloc(sz.nA * (i64)nS, s);
        H2.alloc(sz.nP * (i64)Up, s);
        if (product) {
            q_parts = product_split(sz.nP, sz.nku, U, a.num_sms, &u_chunk);
            const i64 q = sz.nP * sz.nku;
            if (keep && keep->Q.p && keep->Q.n >= (size_t)q)
                Q.borrow(keep->Q.p, q, s);  // a graph's own products, kept between its replays
            else
                Q.alloc(q, s);
        }
        tail = tc_a ? 0 : stage_a_tail(sz.nA, nS, U, a.num_sms);
        if (tail) {
            split_ws.alloc(tail * 2 * DM_BM * 144, s);
            tickets.alloc(tail, s);
            tickets.zero();
        }
    }
};

// Queues one evaluation on stream s.  Kernels read the counts from st->cnt;
// the host sizes buffers and grids by `sz` (an input for PLAN_SIZED, an output
// otherwise).
// trusted: a replay that launches neither the mark pass nor the plan (the
// plan kept in pstore stands; k_restore_plan): for evaluations whose class
// gather checks every class (product form, kept plan).  split (trusted
// only): the class gather is not launched; *split receives its arguments.
static void enqueue_eval(const EvalArgs& a, PlanMode mode, EvalStatus* st, StageTimer& timer, EvalSizes& sz,
                         cudaStream_t s, PlanStore* pstore = nullptr, bool trusted = false,
                         GatherLaunch* split = nullptr) {
    const bool bounded = mode == PLAN_BOUNDED;
    const LatticeTables& t = *a.t;
    const i64 nk = t.nkeys, m = a.m;
    const int U = (int)t.U, Up = (int)t.Up, nS = (int)t.nS;
    // A trusted replay of a small plan starts with the kernel that restores
    // the kept plan, which writes the whole status block (k_restore_plan, or
    // stage A's first block): no memset node ahead of it
    const bool restores = trusted && (bounded || mode == PLAN_SIZED) && (nk * nk + 31) / 32 <= 8 * 1024 &&
                          nk <= PLAN_SMALL_KEYS;
    if (!restores) GLI_CUDA(cudaMemsetAsync(st, 0, sizeof(EvalStatus), s));
    PlanCounts* cnt = &st->cnt;
    if (bounded) {
        sz.nku = nk;
        sz.nA = nk;
        // pairs (A, B) have A >= B; every class has one pair
        sz.nP = std::min(nk * (nk + 1) / 2, m);
    }
    // Bounded and sized evaluations know every size here: all their buffers
    // are allocated and zeroed before the first kernel, so that a captured
    // graph has its allocation and memset nodes at the root and its kernels
    // follow one another directly
    const bool known = mode != PLAN_EXACT;
    // usedKey and usedA side by side so that one scan serves both; pair flags
    // over all key pairs (slot k2 * nk + k1)
    const i64 words = (nk * nk + 31) / 32;
    DevBuf<uint32_t> used, pairBits;
    if (!trusted) {
        used.alloc(2 * nk, s);
        pairBits.alloc(words, s);
        used.zero();
        pairBits.zero();
    }
    const unsigned cb = (unsigned)((m + 255) / 256);
    const unsigned kb = (unsigned)((nk + 255) / 256);
    DevBuf<short4> pts;
    DevBuf<uint2> pdesc;
    ClassDecode dec = a.d;
    dec.pd = nullptr;
    const int* pd_skip = nullptr;
    if (dec.kind == 1 && pair_desc_applies(dec)) {
        // the pair-descriptor decode of the ERI classes (a sized replay keeps
        // the table with its plan, and remakes it only with the plan)
        if (pstore && pstore->pd.p) {
            pdesc.borrow(pstore->pd.p, dec.N2, s);
            pd_skip = pstore->valid.p;
        } else {
            pdesc.alloc(dec.N2, s);
        }
        dec.pd = pdesc.p;
    } else if (dec.kind == 1) {
        pts.alloc(dec.N, s);
        dec.pt = pts.p;
    }
    // Replays of the product form (the host's choice) mark their classes only
    // when the saved plan is not valid: otherwise the plan is restored and the
    // gather decodes and checks every class (the list may have been rewritten
    // in place since the plan was made).
    const bool fused = pstore && mode != PLAN_EXACT && product_pays((double)sz.nP, (double)sz.nku, m);
    if (trusted && !(fused && pstore->pd.p == dec.pd))
        fail(GLI_ERR_INTERNAL, "a trusted replay needs a kept plan and the product form");
    if (split && !(trusted && pstore->Q.p))
        fail(GLI_ERR_INTERNAL, "a gather launched apart needs a trusted replay with kept products");
    // packed key triple per class, written by the decode pass and read by the
    // gather (decoding a class twice, in the mark pass and again in the gather,
    // measured slower than re-reading its 8 bytes: ERI 7^3 stage C 52 against
    // 32 us)
    DevBuf<uint64_t> keys;
    if (!fused) keys.alloc(m, s);
    DevBuf<uint64_t> ids, pairPre;
    DevBuf<int> keyOf, aId, aKey;
    DevBuf<int> pairA, pairB;
    PairTiles tiles;
    if (pstore) {  // a sized graph's plan, kept between its replays
        ids.borrow(pstore->ids.p, 2 * nk, s);
        keyOf.borrow(pstore->keyOf.p, nk, s);
        aId.borrow(pstore->aId.p, nk, s);
        aKey.borrow(pstore->aKey.p, nk, s);
        pairPre.borrow(pstore->pairPre.p, words, s);
    } else {
        ids.alloc(2 * nk, s);
        keyOf.alloc(nk, s);
        aId.alloc(nk, s);
        aKey.alloc(nk, s);
        pairPre.alloc(words, s);
    }
    const bool small_pairs = (bounded || mode == PLAN_SIZED) && words <= 8 * 1024;
    if (mode == PLAN_SIZED && !(small_pairs && nk <= PLAN_SMALL_KEYS))
        fail(GLI_ERR_INTERNAL, "sized plan for a key space of %lld keys", (long long)nk);
    // the whole plan and stage B's tiles in one launch (bounded and sized
    // plans; for exact plans, whose counts are read back half way, the single
    // block's pass over nk^2 pair slots measured no faster than the multi-block
    // path: ERI 7^3 0.206 against 0.200 ms)
    const bool plan_small = small_pairs && nk <= PLAN_SMALL_KEYS;
    if (plan_small) {
        const bool sliced = stage_b_sliced(a.mixed, sz.nA, sz.nP, U);
        const int tbn = sliced ? tile_n(MIXED_SLICES) : DM_BM;
        if (pstore) {
            pairA.borrow(pstore->pairA.p, sz.nP, s);
            pairB.borrow(pstore->pairB.p, sz.nP, s);
            tiles.alloc(sz.nA, sz.nP, tbn, !sliced, s, pstore->tiles.p);
        } else {
            pairA.alloc(sz.nP, s);
            pairB.alloc(sz.nP, s);
            tiles.alloc(sz.nA, sz.nP, tbn, !sliced, s);
        }
    }
    // the mixed form runs a stage on the tensor cores when it is large enough
    // for them to pay off; smaller stages (latency-bound either way) stay FP64
    // (decided on the sizes: bounds for bounded plans, counts otherwise)
    StageBufs sb;
    auto stage_bufs = [&]() {
        const bool tc = a.mixed && sz.nA * (i64)nS >= tc_a_outputs();
        const bool prod = product_pays((double)sz.nP, (double)sz.nku, m) || (bounded && m >= 65536);
        sb.alloc(a, sz, tc, prod, s, pstore);
    };
    if (known) stage_bufs();

    if (dec.pd && !trusted)
        launch_kernel(k_pair_desc, dim3((unsigned)((dec.N2 + 255) / 256)), dim3(256), 0, s, dec, pdesc.p, pd_skip);
    else if (!dec.pd && dec.kind == 1)
        launch_kernel(k_point_table, dim3((unsigned)((dec.N + 255) / 256)), dim3(256), 0, s, dec, pts.p);
    if (!trusted) {
        const size_t lb = mark_local_bytes(nk);
        if (dec.pd) {
            const i64 groups = (m + 3) / 4;
            const unsigned mb = (unsigned)std::min<i64>((groups + 255) / 256, (i64)a.num_sms * 8);
            launch_kernel(k_mark_eri_pd, dim3(mb), dim3(256), lb, s, dec, a.idx, m, used.p, pairBits.p, keys.p,
                          &st->bad, lb ? 1 : 0, fused ? (const int*)pstore->valid.p : (const int*)nullptr);
        } else {
            const unsigned mb = (unsigned)std::min<i64>(cb, (i64)a.num_sms * 8);
            launch_kernel(k_mark, dim3(mb), dim3(256), lb, s, dec, a.idx, m, used.p, pairBits.p, keys.p, &st->bad,
                          lb ? 1 : 0, fused ? (const int*)pstore->valid.p : (const int*)nullptr);
        }
    }
    // (a trusted replay whose stage A runs on the FP64 tensor-core GEMM in 64-
    // or 80-column tiles restores the kept counts in that kernel; the
    // 144-column tiles have no registers to spare for it)
    const bool restore_in_a = plan_small && trusted && !(a.mixed && sz.nA * (i64)nS >= tc_a_outputs()) &&
                              !(sz.nA > 128 && sz.nA <= 144);
    if (restores != (plan_small && trusted)) fail(GLI_ERR_INTERNAL, "trusted replay without its restoring kernel");
    if (plan_small && trusted) {
        if (!restore_in_a) launch_kernel(k_restore_plan, dim3(1), dim3(32), 0, s, pstore->reuse(true), st);
        tiles.built = true;
    } else if (plan_small) {
        launch_kernel(k_plan_small, dim3(1), dim3(1024), 0, s, nk, sz.nA, sz.nP, used.p, ids.p, keyOf.p, aId.p, aKey.p, words,
                   pairBits.p, pairPre.p, pairA.p, pairB.p, tiles.bn, (int)tiles.max_tiles, tiles.first, tiles.tile0,
                   tiles.batch, tiles.col0, tiles.ncols, tiles.rowPair, tiles.rowKey, cnt,
                   pstore ? pstore->reuse(fused) : PlanReuse{});
        tiles.built = true;
    } else {
        if (2 * nk <= 1024) {
            launch_kernel(k_plan_keys_small, dim3(1), dim3(1024), 0, s, nk, used.p, ids.p, keyOf.p, aId.p, aKey.p, cnt);
        } else {
            exclusive_scan_u32_dev(used.p, ids.p, 2 * nk, &cnt->key_total, s);
            launch_kernel(k_plan_keys, dim3(kb), dim3(256), 0, s, nk, used.p, ids.p, keyOf.p, aId.p, aKey.p, cnt);
        }
        DevBuf<uint32_t> counts;
        if (!small_pairs) {
            counts.alloc(words, s);
            launch_kernel(k_word_counts, dim3((unsigned)((words + 255) / 256)), dim3(256), 0, s, words, pairBits.p,
                       counts.p);
            exclusive_scan_u32_dev(counts.p, pairPre.p, words, &cnt->nP, s);
        }
        if (mode == PLAN_EXACT) {
            EvalStatus h;
            read_status(st, h, s);
            if (h.bad)
                fail(GLI_ERR_ARGUMENT, "class index outside the %s tensor of the grid", t.kind ? "ERI" : "ERIDA");
            sz.nku = h.cnt.nku;
            sz.nA = h.cnt.nA;
            sz.nP = (i64)h.cnt.nP;
        }
        pairA.alloc(sz.nP, s);
        pairB.alloc(sz.nP, s);
        if (small_pairs)
            launch_kernel(k_pairs_small, dim3(1), dim3(1024), 0, s, words, (int)nk, pairBits.p, aId.p, pairPre.p,
                       pairA.p, pairB.p, cnt);
        else
            launch_kernel(k_pair_lists, dim3((unsigned)((words + 255) / 256)), dim3(256), 0, s, words, (int)nk,
                       pairBits.p, pairPre.p, aId.p, pairA.p, pairB.p);
    }
    if (!known) stage_bufs();

    const i64 nA = sz.nA, nP = sz.nP, nku = sz.nku;
    DevBuf<double>& H = sb.H;
    // the mixed form runs a stage on the tensor cores when it is large enough for
    // them to pay off; smaller stages (latency-bound either way) stay FP64
    const bool tc_a = a.mixed && nA * (i64)nS >= tc_a_outputs();
    if (restore_in_a && (tc_a || (nA > 128 && nA <= 144)))
        fail(GLI_ERR_INTERNAL, "trusted replay: stage A changed path after the plan");
    const bool tc_b = stage_b_sliced(a.mixed, nA, nP, U);
    DevBuf<double>& H2 = sb.H2;
    t_enq_paths = (tc_a ? 1 : 0) | (tc_b ? 2 : 0);
    timer.mark();
    // ---- stage A
    if (tc_a) {
        constexpr int BN = tile_n(MIXED_SLICES);
        TiledSlices Wa;
        const int nbt = (int)((nA + BN - 1) / BN);
        Wa.alloc(nbt, BN, U, MIXED_SLICES, s);
        slice_tiled(AKeyRows{t.W.p, aKey.p, cnt, Up}, nA, U, Wa, s);
        TileWork w;
        w.a_rows = nS;
        w.a_blocks = (nS + TC_BM - 1) / TC_BM;
        w.n_total = (int)nA;
        w.n_dev = &cnt->nA;
        w.C = H.p;
        w.rs = 1;
        w.cs = nS;
        tc_gemm_tiled(a.G, Wa.view(), w, nbt, &st->tc_err, s);
    } else {
        // small problems split the t loop so that enough blocks exist (the
        // partial tiles summed in a cluster)
        const unsigned mb = (unsigned)((nS + DM_BM - 1) / DM_BM);
        const int bn = (nA > 128 && nA <= 144) ? 144 : col_tile(nA);
        const unsigned nb = (unsigned)((nA + bn - 1) / bn);
        int t_chunk = U;
        const int P = bn == 144 ? 1 : split_count((i64)mb * nb, U, DM_BK, DM_SPLIT_TARGET * a.num_sms, &t_chunk);
        const dim3 grid(mb, nb, (unsigned)P);
        if (restore_in_a && (mb == 0 || nb == 0))  // (no stage-A block would restore the counts)
            launch_kernel(k_restore_plan, dim3(1), dim3(32), 0, s, pstore->reuse(true), st);
        auto restoring = [&](auto op) {
            if (restore_in_a && mb > 0 && nb > 0) {
                op.restore_valid = pstore->valid.p;
                op.restore_from = pstore->saved_cnt.p;
                op.restore_to = st;
            }
            return op;
        };
        if (bn == 144) {
            // one 144-column tile; a last wave under half full split in K
            // (stage_a_tail)
            StageAOp<144> op{t.W.p, t.T.p, t.S.p, aKey.p, cnt, nS, U, Up, U, 0, H.p};
            dim3 g = grid;
            if (sb.tail) {
                op.nfull = (int)(mb - sb.tail);
                op.ws = sb.split_ws.p;
                op.tickets = sb.tickets.p;
                g.x = (unsigned)(mb + sb.tail);
            }
            dmma_launch(op, g, s);
        } else if (bn == 80) {
            // a split sums its parts inside a cluster of the P blocks of a tile
            dmma_launch_cluster(restoring(StageAOp<80>{t.W.p, t.T.p, t.S.p, aKey.p, cnt, nS, U, Up, t_chunk, 0, H.p}),
                                grid, s);
        } else {
            dmma_launch_cluster(restoring(StageAOp<64>{t.W.p, t.T.p, t.S.p, aKey.p, cnt, nS, U, Up, t_chunk, 0, H.p}),
                                grid, s);
        }
    }
    timer.mark();
    // ---- stage B
    if (tiles.built && tiles.bn != (tc_b ? tile_n(MIXED_SLICES) : DM_BM)) tiles.built = false;
    if (tc_b) {
        constexpr int BN = tile_n(MIXED_SLICES);
        const int mb = (U + TC_BM - 1) / TC_BM;
        TiledSlices Hs, Wb;
        Hs.alloc(nA * mb, TC_BM, U, MIXED_SLICES, s);
        slice_tiled(ExpandedHRows{H.p, t.sidx.p, cnt, nS, U, mb}, nA * U, U, Hs, s);
        if (!tiles.built) {
            tiles.alloc(nA, nP, BN, false, s);
            launch_kernel(k_pair_tiles, dim3(1), dim3(1024), 0, s, pairA.p, pairB.p, aKey.p, cnt, BN,
                       (int)tiles.max_tiles, tiles.first, tiles.tile0, tiles.batch, tiles.col0, tiles.ncols,
                       (int*)nullptr, (int*)nullptr);
        }
        const i64 max_tiles = tiles.max_tiles;
        Wb.alloc(max_tiles, BN, U, MIXED_SLICES, s);
        slice_tiled(PairRows{t.W.p, pairA.p, pairB.p, tiles.first, tiles.tile0, tiles.col0, tiles.ncols, cnt, Up, BN},
                    nP, U, Wb, s);
        TileWork w;
        w.a_rows = U;
        w.a_blocks = mb;
        w.a_batched = 1;
        w.tile_batch = tiles.batch;
        w.tile_col0 = tiles.col0;
        w.tile_ncols = tiles.ncols;
        w.C = H2.p;
        w.rs = 1;
        w.cs = Up;
        tc_gemm_tiled(Hs.view(), Wb.view(), w, (int)max_tiles, &st->tc_err, s);
    } else {
        // tiles of 64 rows of one host A key, then (tile, 64 u, chunk of v) blocks
        if (!tiles.built) {
            tiles.alloc(nA, nP, DM_BM, true, s);
            launch_kernel(k_pair_tiles, dim3(1), dim3(1024), 0, s, pairA.p, pairB.p, aKey.p, cnt, DM_BM,
                       (int)tiles.max_tiles, tiles.first, tiles.tile0, tiles.batch, tiles.col0, tiles.ncols,
                       tiles.rowPair, tiles.rowKey);
        }
        const i64 max_tiles = tiles.max_tiles;
        // the tile list is built on the device; the grid follows its bound and
        // the split follows the tiles that hold pairs: with exact counts (exact
        // and sized plans) those are known -- a full pair triangle with
        // balanced hosts fills sum_h ceil(rows_h / 64) tiles, other pair sets
        // about nP / 64 + nA / 2 -- with bounded plans the bound stands in
        // (64 u per tile: 80-row K-major gathers measured slower, ERIDA 129^3
        // stage B 0.32 against 0.21 ms)
        i64 active = max_tiles;
        if (!bounded) {
            if (nku == nA && nP == nA * (nA + 1) / 2 && nA > DM_BM) {
                const int y = (int)std::min<i64>(nA, 2 * DM_BM - 1);
                active = 0;
                for (int h = 0; h < (int)nA; ++h) active += (bal_count(h, (int)nA, y) + DM_BM - 1) / DM_BM;
            } else {
                active = std::min<i64>(max_tiles, (nP + DM_BM - 1) / DM_BM + nA / 2);
            }
        }
        const unsigned ub = (unsigned)((U + DM_BN - 1) / DM_BN);
        int v_chunk = U;
        const int P = split_count(active * ub, U, DM_BK, DM_SPLIT_TARGET * a.num_sms, &v_chunk);
        // a split sums its parts inside a cluster of the P blocks of a tile
        const dim3 grid((unsigned)max_tiles, ub, (unsigned)P);
        if (active * ub * P >= 4 * (i64)DM_SPLIT_TARGET * a.num_sms)
            dmma_launch_cluster(StageBOp<false>{t.W.p, H.p, t.sidx.p, tiles.rowKey, tiles.rowPair, tiles.batch,
                                                tiles.col0, tiles.ncols, nS, U, Up, v_chunk, 0, H2.p},
                                grid, s);
        else
            dmma_launch_cluster(StageBOp<true>{t.W.p, H.p, t.sidx.p, tiles.rowKey, tiles.rowPair, tiles.batch,
                                               tiles.col0, tiles.ncols, nS, U, Up, v_chunk, 0, H2.p},
                                grid, s);
    }
    timer.mark();
    // ---- stage C: the product form computes every (pair, key) dot product --
    // up to 16x more than the classes need on the tensor cores, as many as the
    // classes in FP64 -- but as a GEMM it reuses each H2 row across keys instead
    // of re-reading it per class; small class lists keep the per-class kernel
    // exact plans choose here; bounded plans (whose counts are upper bounds)
    // queue both paths and let the device choose, unless the bounds decide
    const bool product_host = product_pays((double)nP, (double)nku, m);
    const bool undecided = bounded && !product_host && m >= 65536;
    const int c_prod = undecided ? 1 : 0, c_class = undecided ? 2 : 0;
    if (undecided || product_host) {
        // (Q and its u split sized with the stage buffers: product_split)
        const i64 mt = (nP + DM_BM - 1) / DM_BM, nt = (nku + DM_BN - 1) / DM_BN;
        const int P = sb.q_parts, u_chunk = sb.u_chunk;
        const i64 ps = nP * nku;
        const DevBuf<double>& Q = sb.Q;
        if (P < 1 || !Q.p) fail(GLI_ERR_INTERNAL, "stage C product without its buffer");
        // (a split sums its parts inside a cluster of the P blocks of a tile)
        dmma_launch_cluster(ProductOp<64>{H2.p, t.W.p, keyOf.p, pairA.p, aKey.p, ids.p, cnt, m, c_prod, U, Up,
                                          (int)nku, u_chunk, Q.p, &st->products},
                            dim3((unsigned)mt, (unsigned)nt, (unsigned)P), s);
        timer.mark();  // (the class-level kernels of stage C start here)
        t_enq_paths |= (fused ? 2 : 1) << 2;  // the class gather that ran
        if (fused) {
            // (the kept plan's packed lookups: this replay's pair bitmap stays
            // empty when the mark pass skipped)
            GatherLaunch gl;
            gl.Q = Q.p;
            gl.nq = ps;
            gl.dec = dec;
            gl.kk = pstore->kk.p;
            gl.nk = (int)nk;
            gl.bitpre = pstore->bitpre.p;
            gl.ldq = (int)nku;
            gl.cnt = cnt;
            if (split)
                *split = gl;
            else
                launch_gather(gl, a.idx, m, a.out, a.num_sms, s);
        } else {
            const unsigned gq = (unsigned)std::min<i64>(((m + 3) / 4 + 255) / 256, (i64)a.num_sms * 8);
            launch_kernel(k_gather_q, dim3(gq), dim3(256), 0, s, Q.p, ps, keys.p, dec, a.idx, m, ids.p, (int)nk,
                          pairBits.p, pairPre.p, (int)nku, cnt, c_prod, a.out);
        }
    }
    if (undecided || !product_host) {
        if (!undecided) timer.mark();  // (no product GEMM: the class-level kernel starts stage C)
        const i64 want = (m + 7) / 8;
        const unsigned gc = (unsigned)(want < (i64)a.num_sms * 16 ? want : (i64)a.num_sms * 16);
        launch_kernel(k_stage_c, dim3(gc), dim3(256), 0, s, t.W.p, H2.p, keys.p, dec, a.idx, (int)nk, pairBits.p, pairPre.p, m, U, Up,
                   cnt, c_class, a.out);
    }
    timer.mark();
}

// ---------------------------------------------------------------------------
// CUDA graphs of evaluations.  A bounded or sized evaluation issues no host
// synchronisation, so the whole launch sequence (allocations, memsets and about
// 15 kernels) is captured once and replayed: every replay recomputes everything
// from the class list in device memory; only the launch overhead is saved.
// A graph is keyed by what fixes its launch sequence and its pointers: the
// table set (kept alive by the entry), the grid, the class-list pointer and
// length, the output pointer and the form.  A sized graph also carries the
// counts of the exact evaluation that sized it; a list that needs more (the
// caller rewrote the list in place) is flagged by the plan, and the host drops
// the graph and evaluates exactly.
struct GraphEntry {
    const LatticeTables* tables = nullptr;
    std::shared_ptr<const LatticeTables> keep;
    int device = 0, mixed = 0;
    const int64_t* idx = nullptr;
    double* out = nullptr;
    i64 m = 0;
    i64 istart[3] = {}, num[3] = {};
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;  // kernels in the graph
    // the trusted variant (no mark pass, no plan kernel; k_restore_plan), for
    // product-form evaluations, replayed once the host has seen a replay of
    // `exec` complete (planned), which leaves a valid plan kept
    cudaGraphExec_t exec_trust = nullptr;
    long long launches_trust = 0;
    bool planned = false;
    // the trusted variant without its class gather, and the gather's launch
    // (the pipelined host-buffer path gathers range by range)
    cudaGraphExec_t exec_stages = nullptr;
    long long launches_stages = 0;
    GatherLaunch gather;
    PlanMode mode = PLAN_BOUNDED;
    EvalSizes sz;            // the sizes a PLAN_SIZED graph was captured with
    std::unique_ptr<PlanStore> plan;  // the graph's plan, kept between replays
    // timed graphs (evaluations while stage timing is on): the stage marks
    // recorded by every replay, before stage A and after stages A, B and C
    bool timed = false;
    std::unique_ptr<StageTimer> timer, timer_trust;
    int paths = 0;           // tensor-core stages of the captured evaluation
    DevMem<EvalStatus> status;
    ~GraphEntry() {
        // (an entry may be evicted or dropped while a queued replay of it --
        // a stream-ordered call not yet waited for -- is still running)
        cudaDeviceSynchronize();
        if (exec) cudaGraphExecDestroy(exec);
        if (exec_trust) cudaGraphExecDestroy(exec_trust);
        if (exec_stages) cudaGraphExecDestroy(exec_stages);
    }
};

static thread_local std::list<std::unique_ptr<GraphEntry>> t_graphs;
static constexpr size_t kGraphEntries = 8;
static const bool g_graphs_enabled = getenv("GLI_B200_NO_GRAPHS") == nullptr;

static GraphEntry* find_graph(const EvalArgs& a, int device, bool timed) {
    for (auto it = t_graphs.begin(); it != t_graphs.end(); ++it) {
        GraphEntry& e = **it;
        if (e.tables == a.t && e.device == device && e.timed == timed && e.mixed == (int)a.mixed && e.idx == a.idx &&
            e.out == a.out &&
            e.m == a.m && e.istart[0] == a.d.istart[0] && e.istart[1] == a.d.istart[1] &&
            e.istart[2] == a.d.istart[2] && e.num[0] == a.d.num[0] && e.num[1] == a.d.num[1] &&
            e.num[2] == a.d.num[2]) {
            t_graphs.splice(t_graphs.begin(), t_graphs, it);  // most recently used first
            return t_graphs.front().get();
        }
    }
    return nullptr;
}

void clear_eval_caches() { t_graphs.clear(); }

// a replay of the graph completed without overflow: its plan is kept and
// valid, and later replays may trust it (e may have been dropped since: it is
// looked up, not dereferenced)
static void graph_replayed(const GraphEntry* e) {
    for (auto& g : t_graphs)
        if (g.get() == e) {
            g->planned = true;
            return;
        }
}

static void drop_graph(const GraphEntry* e) {
    for (auto it = t_graphs.begin(); it != t_graphs.end(); ++it)
        if (it->get() == e) {
            t_graphs.erase(it);
            return;
        }
}

static GraphEntry* capture_graph(const EvalArgs& a, const std::shared_ptr<const LatticeTables>& tp, int device,
                                 cudaStream_t s, PlanMode mode, const EvalSizes& sized, bool timed) {
    auto e = std::make_unique<GraphEntry>();
    e->timed = timed;
    if (timed) e->timer = std::make_unique<StageTimer>(true, s, true);
    e->mode = mode;
    e->sz = sized;
    e->tables = a.t;
    e->keep = tp;
    e->device = device;
    e->mixed = a.mixed;
    e->idx = a.idx;
    e->out = a.out;
    e->m = a.m;
    for (int k = 0; k < 3; ++k) {
        e->istart[k] = a.d.istart[k];
        e->num[k] = a.d.num[k];
    }
    e->status.alloc(1);
    // function attributes are set outside the capture
    tc_gemm_prepare();
    dgemm_prepare();
    dmma_prepare<StageAOp<64>>();
    dmma_prepare<StageAOp<80>>();
    dmma_prepare<StageAOp<144>>();
    dmma_blocks_per_sm<StageAOp<144>>();
    dmma_prepare<StageBOp<true>>();
    dmma_prepare<StageBOp<false>>();
    dmma_prepare<ProductOp<64>>();
    dmma_prepare<ProductOp<64>, true>();
    dmma_prepare<StageAOp<64>, true>();
    dmma_prepare<StageAOp<80>, true>();
    dmma_prepare<StageBOp<true>, true>();
    dmma_prepare<StageBOp<false>, true>();
    // the sizes of the plan: the sized counts, or the bounds of a bounded plan
    const i64 nk = a.t->nkeys;
    EvalSizes szb = sized;
    if (mode == PLAN_BOUNDED) {
        szb.nA = nk;
        szb.nku = nk;
        szb.nP = std::min(nk * (nk + 1) / 2, a.m);
    }
    // the product form (its gather checks every class against the kept plan)
    // has trusted variants, and keeps its products with the graph
    const bool product = product_pays((double)szb.nP, (double)szb.nku, a.m);
    {
        const i64 words = (nk * nk + 31) / 32;
        i64 q_entries = 0;
        if (product) {
            int u_chunk = 0;
            q_entries = szb.nP * szb.nku;
        }
        e->plan = std::make_unique<PlanStore>();
        e->plan->alloc(nk, words, szb.nA, szb.nP, PairTiles::ints(szb.nA, szb.nP, 64, true),
                       pair_desc_applies(a.d) ? (i64)a.d.N2 : 0, q_entries);
    }
    auto capture = [&](bool trusted, StageTimer* tm, cudaGraphExec_t* exec, long long* launches,
                       GatherLaunch* split) {
        const long long l0 = launch_count();
        GLI_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t graph = nullptr;
        try {
            StageTimer untimed(false, s);
            EvalSizes sz = sized;
            enqueue_eval(a, mode, e->status.p, tm ? *tm : untimed, sz, s, e->plan.get(), trusted, split);
        } catch (...) {
            cudaStreamEndCapture(s, &graph);
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            throw;
        }
        GLI_CUDA(cudaStreamEndCapture(s, &graph));
        *launches = launch_count() - l0;
        const cudaError_t ie = cudaGraphInstantiate(exec, graph, 0);
        cudaGraphDestroy(graph);
        GLI_CUDA(ie);
    };
    capture(false, e->timer.get(), &e->exec, &e->launches, nullptr);
    e->paths = t_enq_paths;
    if (product) {
        if (timed) e->timer_trust = std::make_unique<StageTimer>(true, s, true);
        capture(true, e->timer_trust.get(), &e->exec_trust, &e->launches_trust, nullptr);
        // the stages alone, for the pipelined host-buffer path
        if (!timed) capture(true, nullptr, &e->exec_stages, &e->launches_stages, &e->gather);
    }
    t_graphs.push_front(std::move(e));
    while (t_graphs.size() > kGraphEntries) t_graphs.pop_back();
    return t_graphs.front().get();
}

// pinned host memory that grows on demand (per thread)
struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void* get(size_t need) {
        if (need > bytes) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            bytes = 0;
            GLI_CUDA(cudaHostAlloc(&p, need, cudaHostAllocDefault));
            bytes = need;
        }
        return p;
    }
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
};

// The arguments of one evaluation: checks, the (cached) tables of its form and
// the class decoder of its grid.  tp keeps the tables alive.
static EvalArgs eval_args(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* d_indices,
                          i64 m, double tol, int form, double* d_out, cudaStream_t s,
                          std::shared_ptr<const LatticeTables>& tp, StageTimer& timer) {
    if (form != FORM_FP64 && form != FORM_MIXED)
        fail(GLI_ERR_ARGUMENT, "form %d is not a sparse evaluation form (0 = FP64, 1 = mixed)", form);
    if (!(tol >= 0)) fail(GLI_ERR_ARGUMENT, "tol must be non-negative");
    const Context& ctx = context();
    timer.mark();
    // the mixed form screens the products within its error budget
    // (mixed_screen_tol: a first-order bound of MIXED_SCREEN_BOUND grid units)
    double screen_bound = 0.0;
    const double ttol = form == FORM_MIXED ? mixed_screen_tol(kind, h_coeffs, nb, g.max_range(), tol, &screen_bound, s)
                                           : tol;
    t_screen_tol = ttol;
    t_screen_bound = screen_bound;
    tp = lattice_tables(kind, h_coeffs, nb, g.max_range(), ttol, s);
    const LatticeTables& t = *tp;
    EvalArgs a;
    a.mixed = form == FORM_MIXED;
    a.t = &t;
    // the G slices exist for stage A on the tensor cores, which needs at least
    // 1e6 stage-A outputs (nA <= nkeys A keys); built once per table set
    if (a.mixed && t.nkeys * t.nS >= tc_a_outputs()) a.G = lattice_g_slices(t, s);
    timer.mark();
    a.d.kind = kind;
    a.d.N = g.points();
    a.d.L = t.L;
    for (int k = 0; k < 3; ++k) {
        a.d.istart[k] = g.istart[k];
        a.d.num[k] = g.num[k];
    }
    a.d.nkeys = t.nkeys;
    bool decodable = a.d.N < ((i64)1 << 31);
    if (kind == 1)  // ERI: N^2 < 2^32, coordinates in 16 bits
        for (int k = 0; k < 3; ++k)
            decodable = decodable && a.d.N <= 65535 && std::llabs(g.istart[k]) + g.num[k] < 32767;
    if (!decodable) fail(GLI_ERR_LIMIT, "grid of %lld points is beyond the class decoder's range", (long long)a.d.N);
    if (t.nkeys > 8192)
        fail(GLI_ERR_LIMIT, "grid spans %lld axis keys (limit 8192)", (long long)t.nkeys);
    a.d.finish();
    a.idx = d_indices;
    a.m = m;
    a.out = d_out;
    a.num_sms = ctx.num_sms;
    return a;
}

// Queues one evaluation on stream s and an asynchronous copy of its status
// block into h_status (pinned); the caller synchronises and checks it.
// *sized receives the graph that was replayed (null otherwise): when its
// status reports an overflow (a sized plan outgrown, or a class outside a
// reused plan), the caller drops it and calls again, which plans anew.
static void sparse_values_enqueue(int kind, const double* h_coeffs, i64 nb, const GridDesc& g,
                                  const int64_t* d_indices, i64 m, double tol, int form, double* d_out, cudaStream_t s,
                                  EvalStatus* h_status, std::shared_ptr<const LatticeTables>& tp, StageTimer& timer,
                                  const GraphEntry** sized) {
    *sized = nullptr;
    const Context& ctx = context();
    EvalArgs a = eval_args(kind, h_coeffs, nb, g, d_indices, m, tol, form, d_out, s, tp, timer);
    const LatticeTables& t = *tp;
    const bool bounded = t.nkeys <= BOUNDED_KEYS;
    const bool graphs = g_graphs_enabled;
    // (stage timing replays graphs of its own, whose stage marks are nodes)
    GraphEntry* e = graphs && (bounded || sized_plan_fits(t.nkeys)) ? find_graph(a, ctx.device, t_timing) : nullptr;
    if (!e && graphs && bounded) e = capture_graph(a, tp, ctx.device, s, PLAN_BOUNDED, EvalSizes{}, t_timing);
    const bool trust = e && e->exec_trust && e->planned;
    t_graph_timer = e ? (trust ? e->timer_trust.get() : e->timer.get()) : nullptr;
    if (e) {
        GLI_CUDA(cudaGraphLaunch(trust ? e->exec_trust : e->exec, s));
        add_launches(trust ? e->launches_trust : e->launches);
        t_paths = e->paths;
        GLI_CUDA(cudaMemcpyAsync(h_status, e->status.p, sizeof(EvalStatus), cudaMemcpyDeviceToHost, s));
        *sized = e;
        return;
    }
    DevBuf<EvalStatus> st(1, s);
    EvalSizes sz;
    enqueue_eval(a, bounded ? PLAN_BOUNDED : PLAN_EXACT, st.p, timer, sz, s);
    t_paths = t_enq_paths;
    GLI_CUDA(cudaMemcpyAsync(h_status, st.p, sizeof(EvalStatus), cudaMemcpyDeviceToHost, s));
    // the exact counts of this list size the graph that its next evaluations replay
    if (graphs && !bounded && sized_plan_fits(t.nkeys)) capture_graph(a, tp, ctx.device, s, PLAN_SIZED, sz, t_timing);
}

// debug builds: a device bounds check that failed during the evaluation
static void check_debug_fault() {
#ifdef GLI_B200_DEBUG
    unsigned long long f = 0;
    GLI_CUDA(cudaMemcpyFromSymbol(&f, g_debug_fault, sizeof(f)));
    if (f) {
        const unsigned long long zero = 0;
        GLI_CUDA(cudaMemcpyToSymbol(g_debug_fault, &zero, sizeof(zero)));
        fail(GLI_ERR_INTERNAL, "device bounds check failed: site %llu, index %lld", f >> 56,
             (long long)(f & ((1ull << 56) - 1)));
    }
#endif
}

// after the stream synchronised: errors of the evaluation, and the statistics
static void check_status(int kind, i64 m, const EvalStatus& h, const LatticeTables& t, StageTimer& timer,
                         ContractStats* stats) {
    check_debug_fault();
    if (h.bad) fail(GLI_ERR_ARGUMENT, "class index outside the %s tensor of the grid", kind ? "ERI" : "ERIDA");
    if (h.tc_err) fail(GLI_ERR_INTERNAL, "tensor-core stage: an mbarrier wait expired (code %d)", h.tc_err);
    ContractStats st;
    st.keys_a = h.cnt.nA;
    st.pairs = (i64)h.cnt.nP;
    st.U = t.U;
    st.keys_used = h.cnt.nku;
    st.product = product_pays((double)h.cnt.nP, (double)h.cnt.nku, m) ? 1 : 0;
    st.products = st.product ? (i64)h.products : 0;
    st.tc_a = t_paths & 1;
    st.tc_b = (t_paths >> 1) & 1;
    st.gather = (t_paths >> 2) & 3;
    st.screen_tol = t_screen_tol;
    st.screen_bound = t_screen_bound;
    if (t_timing) {
        st.ms_tables = timer.between(0, 1);
        // a replayed graph's own marks, else those of the uncaptured evaluation
        StageTimer& g = t_graph_timer ? *t_graph_timer : timer;
        const int b = t_graph_timer ? 0 : 2;
        st.ms_a = g.between(b, b + 1);
        st.ms_b = g.between(b + 1, b + 2);
        st.ms_c = g.between(b + 2, b + 4);
        st.ms_c_product = g.between(b + 2, b + 3);
        st.ms_c_class = g.between(b + 3, b + 4);
    }
    t_last = st;
    if (stats) *stats = st;
}

static thread_local PinnedBuf t_pin_status, t_pin_idx, t_pin_val;

void sparse_values_device(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* d_indices,
                          i64 m, double tol, int form, double* d_out, cudaStream_t s, ContractStats* stats) {
    if (m == 0) return;
    EvalStatus* h = (EvalStatus*)t_pin_status.get(sizeof(EvalStatus));
    std::shared_ptr<const LatticeTables> tp;
    StageTimer timer(t_timing, s);
    const GraphEntry* sized = nullptr;
    sparse_values_enqueue(kind, h_coeffs, nb, g, d_indices, m, tol, form, d_out, s, h, tp, timer, &sized);
    GLI_CUDA(cudaStreamSynchronize(s));
    if (h->cnt.overflow) {  // the list outgrew the sizes of its graph: evaluate exactly
        drop_graph(sized);
        sparse_values_enqueue(kind, h_coeffs, nb, g, d_indices, m, tol, form, d_out, s, h, tp, timer, &sized);
        GLI_CUDA(cudaStreamSynchronize(s));
    }
    check_status(kind, m, *h, *tp, timer, stats);
    if (!h->cnt.overflow) graph_replayed(sized);
}

// Stream-ordered evaluations: queued without a host wait, their status read
// when the caller waits for them.  A pending evaluation keeps what it needs to
// be evaluated again (the coefficients, the grid, the device pointers) and its
// own page-locked status slot; the tables stay alive with it.  Waiting for a
// ticket waits for that evaluation and every one queued before it on this
// thread, in order; one whose sized graph overflowed (its list outgrew the
// plan the graph was sized for) is evaluated again there, exactly.
struct PendingEval {
    i64 ticket = 0;
    int kind = 0;
    std::vector<double> coeffs;
    GridDesc g;
    const int64_t* idx = nullptr;
    i64 m = 0;
    double tol = 0.0;
    int form = 0;
    double* out = nullptr;
    cudaStream_t s = nullptr;
    EvalStatus* h_status = nullptr;  // page-locked slot (from t_status_slots)
    cudaEvent_t done = nullptr;
    std::shared_ptr<const LatticeTables> tp;
    const GraphEntry* sized = nullptr;
};

struct StatusSlots {  // page-locked status blocks, reused
    std::vector<EvalStatus*> free;
    EvalStatus* get() {
        if (free.empty()) {
            void* p = nullptr;
            GLI_CUDA(cudaHostAlloc(&p, sizeof(EvalStatus), cudaHostAllocDefault));
            return (EvalStatus*)p;
        }
        EvalStatus* p = free.back();
        free.pop_back();
        return p;
    }
    ~StatusSlots() {
        for (EvalStatus* p : free) cudaFreeHost(p);
    }
};
static thread_local StatusSlots t_status_slots;
static thread_local std::list<PendingEval> t_pending;
static thread_local i64 t_next_ticket = 1;
constexpr size_t MAX_PENDING = 256;

static void finish_pending(PendingEval& e) {
    struct Recycle {
        PendingEval& e;
        ~Recycle() {
            if (e.done) cudaEventDestroy(e.done);
            e.done = nullptr;
            if (e.h_status) t_status_slots.free.push_back(e.h_status);
            e.h_status = nullptr;
        }
    } recycle{e};
    if (e.m == 0) return;
    GLI_CUDA(cudaEventSynchronize(e.done));
    if (e.h_status->cnt.overflow) {
        drop_graph(e.sized);
        sparse_values_device(e.kind, e.coeffs.data(), (i64)e.coeffs.size(), e.g, e.idx, e.m, e.tol, e.form, e.out,
                             e.s, nullptr);
        return;
    }
    StageTimer timer(false, e.s);
    check_status(e.kind, e.m, *e.h_status, *e.tp, timer, nullptr);
    graph_replayed(e.sized);
}

void sparse_values_wait(i64 ticket) {
    bool found = false;
    for (const PendingEval& e : t_pending) found = found || e.ticket == ticket;
    if (!found) fail(GLI_ERR_ARGUMENT, "no pending evaluation %lld on this thread", (long long)ticket);
    // in order: every evaluation up to this one (the first error ends the wait
    // and is reported; the evaluations after it stay pending)
    while (!t_pending.empty()) {
        PendingEval e = std::move(t_pending.front());
        t_pending.pop_front();
        const bool last = e.ticket == ticket;
        finish_pending(e);
        if (last) break;
    }
}

i64 sparse_values_device_async(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* d_indices,
                               i64 m, double tol, int form, double* d_out, cudaStream_t s) {
    if (t_pending.size() >= MAX_PENDING) sparse_values_wait(t_pending.front().ticket);
    PendingEval e;
    e.ticket = t_next_ticket++;
    e.kind = kind;
    e.coeffs.assign(h_coeffs, h_coeffs + nb);
    e.g = g;
    e.idx = d_indices;
    e.m = m;
    e.tol = tol;
    e.form = form;
    e.out = d_out;
    e.s = s;
    if (m > 0) {
        e.h_status = t_status_slots.get();
        try {
            StageTimer timer(false, s);
            sparse_values_enqueue(kind, h_coeffs, nb, g, d_indices, m, tol, form, d_out, s, e.h_status, e.tp, timer,
                                  &e.sized);
            GLI_CUDA(cudaEventCreateWithFlags(&e.done, cudaEventDisableTiming));
            GLI_CUDA(cudaEventRecord(e.done, s));
        } catch (...) {
            if (e.done) cudaEventDestroy(e.done);
            t_status_slots.free.push_back(e.h_status);
            throw;
        }
    }
    t_pending.push_back(std::move(e));
    return t_pending.back().ticket;
}

// Device copies of a host class list and its values, kept per thread and
// device between calls (grown on demand), so that repeated calls reuse the
// same device pointers and therefore the same captured evaluation.
struct HostCallBuffers {
    int device = -1;
    std::unique_ptr<DevMem<int64_t>> idx;
    std::unique_ptr<DevMem<double>> val;
    i64 cap = 0;
    void ensure(int dev, i64 m) {
        if (dev != device || m > cap) {
            idx.reset();
            val.reset();
            idx = std::make_unique<DevMem<int64_t>>();
            val = std::make_unique<DevMem<double>>();
            idx->alloc((size_t)m);
            val->alloc((size_t)m);
            cap = m;
            device = dev;
        }
    }
};
static thread_local HostCallBuffers t_host_call;

// Host copies of long class lists: a pageable <-> pinned memcpy runs at a
// fraction of the host's memory bandwidth on one core, so copies of several MB
// are split over a few threads.
static void host_copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kSplit = (size_t)1 << 20;  // at least 1 MB per thread
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::min<size_t>(std::min<size_t>(8, hw > 1 ? hw / 2 : 1), bytes / kSplit);
    if (nt <= 1) {
        memcpy(dst, src, bytes);
        return;
    }
    const size_t part = (bytes / nt + 63) / 64 * 64;
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) {
        const size_t b0 = std::min(bytes, k * part), b1 = std::min(bytes, (k + 1) * part);
        if (b1 > b0) th.emplace_back([=] { memcpy((char*)dst + b0, (const char*)src + b0, b1 - b0); });
    }
    memcpy(dst, src, std::min(bytes, part));
    for (auto& t : th) t.join();
}

// The evaluation from and into host arrays: the class list goes to the device
// in chunks, each chunk's DMA overlapping the host copy of the next into the
// pinned staging buffer; the values come back the same way in reverse.
// true for page-locked host memory the DMA engines can read and write directly
static bool is_pinned(const void* p) {
    cudaPointerAttributes a = {};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// the two copy streams of the page-locked host path (per thread and device)
struct CopyStreams {
    int device = -1;
    cudaStream_t in = nullptr, out = nullptr;
    void ensure(int dev) {
        if (dev == device) return;
        GLI_CUDA(cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking));
        GLI_CUDA(cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking));
        device = dev;
    }
    ~CopyStreams() {
        if (in) cudaStreamDestroy(in);
        if (out) cudaStreamDestroy(out);
    }
};
static thread_local CopyStreams t_copy_streams;

// Page-locked class list and value arrays: the copies go straight between them
// and the device buffers (no staging).  Once a list's graph has completed a
// replay (its plan is kept and valid), a list of a million classes or more is
// pipelined: the stages, which need only the kept plan, run while the class
// list streams in on one copy stream in PIPE_CHUNKS ranges; each range is
// gathered as soon as it has arrived (the plan-checking gather), and its values
// stream out on a second copy stream while later ranges arrive.  The stages run
// once for the whole list, so the values equal those of the other paths.  A
// list that no longer fits the kept plan (rewritten since: a class of it fails
// the gather's check) is evaluated again, whole and exactly.  Before that (the
// first calls for a list) and for smaller lists, the list is copied in,
// evaluated and copied out.
constexpr i64 PIPE_CHUNKS = 8;

struct PipeEvents {  // the pipeline's events, created once per thread and device
    int device = -1;
    cudaEvent_t start = nullptr, in[PIPE_CHUNKS] = {}, gathered[PIPE_CHUNKS] = {};
    void ensure(int dev) {
        if (dev == device) return;
        release();
        GLI_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
        for (i64 c = 0; c < PIPE_CHUNKS; ++c) {
            GLI_CUDA(cudaEventCreateWithFlags(&in[c], cudaEventDisableTiming));
            GLI_CUDA(cudaEventCreateWithFlags(&gathered[c], cudaEventDisableTiming));
        }
        device = dev;
    }
    void release() {
        if (start) cudaEventDestroy(start);
        for (i64 c = 0; c < PIPE_CHUNKS; ++c) {
            if (in[c]) cudaEventDestroy(in[c]);
            if (gathered[c]) cudaEventDestroy(gathered[c]);
            in[c] = gathered[c] = nullptr;
        }
        start = nullptr;
        device = -1;
    }
    ~PipeEvents() { release(); }
};
static thread_local PipeEvents t_pipe_events;

static void sparse_values_pinned(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* h_indices,
                                 i64 m, double tol, int form, double* h_out, cudaStream_t s) {
    const Context& ctx = context();
    t_host_call.ensure(ctx.device, m);
    EvalStatus* hs = (EvalStatus*)t_pin_status.get(sizeof(EvalStatus));
    std::shared_ptr<const LatticeTables> tp;
    StageTimer timer(t_timing, s);
    int64_t* d_idx = t_host_call.idx->p;
    double* d_val = t_host_call.val->p;
    GraphEntry* e = nullptr;
    if (!t_timing && g_graphs_enabled && m >= ((i64)1 << 20)) {
        const EvalArgs a = eval_args(kind, h_coeffs, nb, g, d_idx, m, tol, form, d_val, s, tp, timer);
        e = find_graph(a, ctx.device, false);
        if (e && !(e->planned && e->exec_stages)) e = nullptr;
    }
    if (e) {
        t_copy_streams.ensure(ctx.device);
        t_pipe_events.ensure(ctx.device);
        cudaStream_t s_in = t_copy_streams.in, s_out = t_copy_streams.out;
        PipeEvents& ev = t_pipe_events;
        const i64 per = (m + PIPE_CHUNKS - 1) / PIPE_CHUNKS;
        // the copy streams start after the work already queued on s
        GLI_CUDA(cudaEventRecord(ev.start, s));
        GLI_CUDA(cudaStreamWaitEvent(s_in, ev.start, 0));
        GLI_CUDA(cudaStreamWaitEvent(s_out, ev.start, 0));
        GLI_CUDA(cudaGraphLaunch(e->exec_stages, s));
        add_launches(e->launches_stages);
        for (i64 c = 0; c < PIPE_CHUNKS; ++c) {
            const i64 b = c * per, n = std::max<i64>(0, std::min(m, b + per) - b);
            if (n > 0)
                GLI_CUDA(cudaMemcpyAsync(d_idx + b, h_indices + b, (size_t)n * sizeof(int64_t),
                                         cudaMemcpyHostToDevice, s_in));
            GLI_CUDA(cudaEventRecord(ev.in[c], s_in));
        }
        for (i64 c = 0; c < PIPE_CHUNKS; ++c) {
            const i64 b = c * per, n = std::max<i64>(0, std::min(m, b + per) - b);
            GLI_CUDA(cudaStreamWaitEvent(s, ev.in[c], 0));
            launch_gather(e->gather, d_idx + b, n, d_val + b, ctx.num_sms, s);
            GLI_CUDA(cudaEventRecord(ev.gathered[c], s));
            GLI_CUDA(cudaStreamWaitEvent(s_out, ev.gathered[c], 0));
            if (n > 0)
                GLI_CUDA(cudaMemcpyAsync(h_out + b, d_val + b, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                                         s_out));
        }
        GLI_CUDA(cudaMemcpyAsync(hs, e->status.p, sizeof(EvalStatus), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s_out));
        GLI_CUDA(cudaStreamSynchronize(s));
        t_paths = e->paths;
        t_graph_timer = nullptr;
        if (hs->cnt.overflow) {
            // a class outside the kept plan: the list (already in device
            // memory) once more, whole, with a new plan
            drop_graph(e);
            const GraphEntry* sized = nullptr;
            sparse_values_enqueue(kind, h_coeffs, nb, g, d_idx, m, tol, form, d_val, s, hs, tp, timer, &sized);
            GLI_CUDA(cudaMemcpyAsync(h_out, d_val, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
            GLI_CUDA(cudaStreamSynchronize(s));
            if (hs->cnt.overflow) fail(GLI_ERR_INTERNAL, "a new plan overflowed");
        }
        check_status(kind, m, *hs, *tp, timer, nullptr);
        return;
    }
    const GraphEntry* sized = nullptr;
    GLI_CUDA(cudaMemcpyAsync(d_idx, h_indices, (size_t)m * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    for (int attempt = 0; attempt < 2; ++attempt) {
        sparse_values_enqueue(kind, h_coeffs, nb, g, d_idx, m, tol, form, d_val, s, hs, tp, timer, &sized);
        GLI_CUDA(cudaMemcpyAsync(h_out, d_val, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s));
        if (!hs->cnt.overflow) break;
        drop_graph(sized);  // the list outgrew its graph's sizes: once more, exactly
    }
    check_status(kind, m, *hs, *tp, timer, nullptr);
    if (!hs->cnt.overflow) graph_replayed(sized);
}

void sparse_values_host(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* h_indices, i64 m,
                        double tol, int form, double* h_out, cudaStream_t s) {
    if (m == 0) return;
    if (is_pinned(h_indices) && is_pinned(h_out))
        return sparse_values_pinned(kind, h_coeffs, nb, g, h_indices, m, tol, form, h_out, s);
    const Context& ctx = context();
    EvalStatus* hs = (EvalStatus*)t_pin_status.get(sizeof(EvalStatus));
    int64_t* pin_idx = (int64_t*)t_pin_idx.get((size_t)m * sizeof(int64_t));
    double* pin_val = (double*)t_pin_val.get((size_t)m * sizeof(double));
    t_host_call.ensure(ctx.device, m);
    const i64 chunks = m >= ((i64)1 << 20) ? 2 : 1, per = (m + chunks - 1) / chunks;
    for (i64 c = 0; c < chunks; ++c) {
        const i64 b = c * per, n = std::min(m, b + per) - b;
        if (n <= 0) break;
        host_copy(pin_idx + b, h_indices + b, (size_t)n * sizeof(int64_t));
        GLI_CUDA(cudaMemcpyAsync(t_host_call.idx->p + b, pin_idx + b, (size_t)n * sizeof(int64_t),
                                 cudaMemcpyHostToDevice, s));
    }
    std::shared_ptr<const LatticeTables> tp;
    StageTimer timer(t_timing, s);
    const GraphEntry* sized = nullptr;
    sparse_values_enqueue(kind, h_coeffs, nb, g, t_host_call.idx->p, m, tol, form, t_host_call.val->p, s, hs, tp,
                          timer, &sized);
    // a replayed sized graph whose list outgrew its sizes (status read back
    // with or before the values): evaluate exactly and copy the values again
    auto redo_if_overflow = [&]() {
        if (!hs->cnt.overflow) return false;
        GLI_CUDA(cudaStreamSynchronize(s));
        drop_graph(sized);
        sparse_values_enqueue(kind, h_coeffs, nb, g, t_host_call.idx->p, m, tol, form, t_host_call.val->p, s, hs, tp,
                              timer, &sized);
        GLI_CUDA(cudaMemcpyAsync(pin_val, t_host_call.val->p, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s));
        check_status(kind, m, *hs, *tp, timer, nullptr);
        host_copy(h_out, pin_val, (size_t)m * sizeof(double));
        return true;
    };
    if (chunks == 1) {
        GLI_CUDA(cudaMemcpyAsync(pin_val, t_host_call.val->p, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s));
        if (redo_if_overflow()) return;
        check_status(kind, m, *hs, *tp, timer, nullptr);
        graph_replayed(sized);
        host_copy(h_out, pin_val, (size_t)m * sizeof(double));
        return;
    }
    cudaEvent_t ev[2];
    for (auto& e : ev) GLI_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    struct Release {
        cudaEvent_t* e;
        ~Release() {
            for (int k = 0; k < 2; ++k) cudaEventDestroy(e[k]);
        }
    } release{ev};
    for (i64 c = 0; c < chunks; ++c) {
        const i64 b = c * per, n = std::max<i64>(0, std::min(m, b + per) - b);
        if (n > 0)
            GLI_CUDA(cudaMemcpyAsync(pin_val + b, t_host_call.val->p + b, (size_t)n * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaEventRecord(ev[c], s));
    }
    GLI_CUDA(cudaEventSynchronize(ev[0]));  // the status copy came before the values
    if (redo_if_overflow()) return;
    check_status(kind, m, *hs, *tp, timer, nullptr);
    graph_replayed(sized);
    for (i64 c = 0; c < chunks; ++c) {
        const i64 b = c * per, n = std::min(m, b + per) - b;
        GLI_CUDA(cudaEventSynchronize(ev[c]));
        if (n > 0) host_copy(h_out + b, pin_val + b, (size_t)n * sizeof(double));
    }
}

}  // namespace gli
