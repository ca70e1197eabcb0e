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

#include "tables.cuh"

namespace gli {

// ---------------------------------------------------------------------------
// class decoding
struct ClassDecode {
    int kind;
    i64 N;          // grid points
    i64 L;          // table range (largest axis length)
    i64 istart[3];
    i64 num[3];
    i64 nkeys;
};

__device__ inline void decode_pt(const ClassDecode& d, i64 lin, i64 p[3]) {
    const i64 z = lin % d.num[2];
    lin /= d.num[2];
    const i64 y = lin % d.num[1];
    const i64 x = lin / d.num[1];
    p[0] = d.istart[0] + x;
    p[1] = d.istart[1] + y;
    p[2] = d.istart[2] + z;
}

// returns false for an index outside the tensor
__device__ inline bool class_keys(const ClassDecode& d, i64 idx, i64 k[3]) {
    if (d.kind == 0) {
        if (idx < 0 || idx >= d.N * d.N) return false;
        i64 pi[3], pj[3];
        decode_pt(d, idx / d.N, pi);
        decode_pt(d, idx % d.N, pj);
        for (int a = 0; a < 3; ++a) {
            const i64 dd = pi[a] - pj[a];
            k[a] = dd < 0 ? -dd : dd;
        }
    } else {
        const i64 N2 = d.N * d.N;
        if (idx < 0 || idx / N2 >= N2) return false;
        i64 r = idx;
        const i64 il = r % d.N; r /= d.N;
        const i64 ik = r % d.N; r /= d.N;
        const i64 ij = r % d.N; r /= d.N;
        i64 p0[3], p1[3], p2[3], p3[3];
        decode_pt(d, r, p0);
        decode_pt(d, ij, p1);
        decode_pt(d, ik, p2);
        decode_pt(d, il, p3);
        for (int a = 0; a < 3; ++a)
            k[a] = eri_axis_key(p0[a] - p1[a], p2[a] - p3[a], (p0[a] + p1[a]) - (p2[a] + p3[a]), d.L);
    }
    // sort ascending
    if (k[0] > k[1]) { i64 t = k[0]; k[0] = k[1]; k[1] = t; }
    if (k[1] > k[2]) { i64 t = k[1]; k[1] = k[2]; k[2] = t; }
    if (k[0] > k[1]) { i64 t = k[0]; k[0] = k[1]; k[1] = t; }
    return true;
}

// counts of one evaluation, kept in device memory so that kernels can size their
// work without a host round trip
struct PlanCounts {
    uint64_t key_total;  // used keys + used A keys (joint scan total)
    uint64_t nP;         // distinct (A, B) key pairs
    int64_t nku, nA;     // used keys, used A keys
};

// mark every key the class list uses (any role) and the A keys (k2)
__global__ void k_mark_keys(ClassDecode d, const int64_t* __restrict__ idx, i64 m, uint32_t* __restrict__ usedKey,
                            uint32_t* __restrict__ usedA, int* __restrict__ bad) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    i64 k[3];
    if (!class_keys(d, idx[n], k)) {
        atomicOr(bad, 1);
        return;
    }
    usedKey[k[0]] = 1;
    usedKey[k[1]] = 1;
    usedKey[k[2]] = 1;
    usedA[k[1]] = 1;
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

// ... and the pair flags: exclusive ids of the used slots, the pair lists in
// slot order, and the pair count.  Thread t owns slots [t * per, (t + 1) * per).
__global__ void __launch_bounds__(1024) k_pairs_small(i64 slots, i64 stride, const uint32_t* __restrict__ usedPair,
                                                      const int* __restrict__ keyOf, const int* __restrict__ aId,
                                                      uint64_t* __restrict__ pairId, int* __restrict__ pairA,
                                                      int* __restrict__ pairB, PlanCounts* __restrict__ cnt) {
    __shared__ uint32_t ws[32], total;
    const i64 per = (slots + blockDim.x - 1) / blockDim.x;
    const i64 b = (i64)threadIdx.x * per, e = b + per < slots ? b + per : slots;
    uint32_t c = 0;
    for (i64 q = b; q < e; ++q) c += usedPair[q];
    uint32_t run = block_scan_1024(c, ws, &total);
    for (i64 q = b; q < e; ++q) {
        pairId[q] = run;
        if (usedPair[q]) {
            pairA[run] = aId[keyOf[q / stride]];
            pairB[run] = keyOf[q % stride];
            ++run;
        }
    }
    if (threadIdx.x == 0) cnt->nP = total;
}

// (A, B) pairs over the compacted key ids: slot = kid(k2) * stride + kid(k1)
__global__ void k_mark_pairs(ClassDecode d, const int64_t* __restrict__ idx, i64 m, const uint64_t* __restrict__ kid,
                             i64 stride, uint32_t* __restrict__ usedPair) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    i64 k[3];
    if (!class_keys(d, idx[n], k)) return;
    usedPair[(i64)kid[k[1]] * stride + (i64)kid[k[0]]] = 1;
}

__global__ void k_pair_lists(i64 slots, i64 stride, const uint32_t* __restrict__ usedPair,
                             const uint64_t* __restrict__ pairId, const int* __restrict__ keyOf,
                             const int* __restrict__ aId, int* __restrict__ pairA, int* __restrict__ pairB) {
    const i64 slot = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= slots || !usedPair[slot]) return;
    const i64 ka = keyOf[slot / stride], kb = keyOf[slot % stride];
    pairA[pairId[slot]] = aId[ka];
    pairB[pairId[slot]] = (int)kb;
}

__global__ void k_class_pairs(ClassDecode d, const int64_t* __restrict__ idx, i64 m, const uint64_t* __restrict__ kid,
                              i64 stride, const uint64_t* __restrict__ pairId, int2* __restrict__ cls) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    i64 k[3];
    if (!class_keys(d, idx[n], k)) {
        cls[n] = make_int2(-1, 0);
        return;
    }
    cls[n] = make_int2((int)pairId[(i64)kid[k[1]] * stride + (i64)kid[k[0]]], (int)kid[k[2]]);
}

// ---------------------------------------------------------------------------
// stage A: H[a][j] = sum_t W[aKey[a]][t] T[S[j] + t^2]
// H depends on (u, v) only through s = u^2 + v^2, so it is evaluated once per
// distinct s (S, ascending; 10,823 values instead of 31,329 (u, v) at U = 177).
// Block: 64 threads x 2 s-values, KT keys held in registers per thread; the
// keys' weights for a chunk of t sit in shared memory, read as double2
// broadcasts.  Per t a thread issues 2 table gathers and KT/2 shared loads for
// 2*KT FMAs.
constexpr int A_THREADS = 128;
constexpr int A_SPT = 2;                  // s-values per thread
constexpr int A_STILE = A_THREADS * A_SPT;
constexpr int A_TC = 32;                  // t chunk

template <int KT>
__global__ void __launch_bounds__(A_THREADS) k_stage_a(const double* __restrict__ W, const double* __restrict__ T,
                                                        const int* __restrict__ S, const int* __restrict__ aKey,
                                                        const PlanCounts* __restrict__ cnt, int nS, int U, int Up,
                                                        int t_chunk, i64 part_stride, double* __restrict__ H) {
    __shared__ __align__(16) double ws[A_TC][KT];
    // blockIdx.z: chunk of t (partial sums of small problems, summed afterwards)
    const int t_begin = blockIdx.z * t_chunk, t_end = min(U, t_begin + t_chunk);
    H += (i64)blockIdx.z * part_stride;
    const int j0 = blockIdx.x * A_STILE + threadIdx.x;
    const int j1 = j0 + A_THREADS;
    const int a0 = blockIdx.y * KT;
    const int nA = (int)cnt->nA;
    if (a0 >= nA) return;  // grids are sized by a bound on nA
    const int s0 = j0 < nS ? S[j0] : 0;
    const int s1 = j1 < nS ? S[j1] : 0;
    double acc0[KT], acc1[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) acc0[k] = acc1[k] = 0;
    for (int t0 = t_begin; t0 < t_end; t0 += A_TC) {
        __syncthreads();
        for (int e = threadIdx.x; e < A_TC * KT; e += A_THREADS) {
            const int k = e / A_TC, tt = e % A_TC, t = t0 + tt;
            ws[tt][k] = (a0 + k < nA && t < t_end) ? W[(i64)aKey[a0 + k] * Up + t] : 0.0;
        }
        __syncthreads();
        const int tmax = min(A_TC, t_end - t0);
        // the table gathers of t + 1 are issued before the FMAs of t
        double g0n = __ldg(&T[s0 + t0 * t0]);
        double g1n = __ldg(&T[s1 + t0 * t0]);
        for (int tt = 0; tt < tmax; ++tt) {
            const double g0 = g0n, g1 = g1n;
            if (tt + 1 < tmax) {
                const int t2n = (t0 + tt + 1) * (t0 + tt + 1);
                g0n = __ldg(&T[s0 + t2n]);
                g1n = __ldg(&T[s1 + t2n]);
            }
            const double2* w2 = reinterpret_cast<const double2*>(&ws[tt][0]);
#pragma unroll
            for (int k = 0; k < KT / 2; ++k) {
                const double2 w = w2[k];
                acc0[2 * k] = fma(w.x, g0, acc0[2 * k]);
                acc0[2 * k + 1] = fma(w.y, g0, acc0[2 * k + 1]);
                acc1[2 * k] = fma(w.x, g1, acc1[2 * k]);
                acc1[2 * k + 1] = fma(w.y, g1, acc1[2 * k + 1]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        if (a0 + k >= nA) break;
        double* h = H + (i64)(a0 + k) * nS;
        if (j0 < nS) h[j0] = acc0[k];
        if (j1 < nS) h[j1] = acc1[k];
    }
}

// ---------------------------------------------------------------------------
// stage B: H2[p][u] = sum_v W[pairB[p]][v] Hf[pairA[p]][v][u]
// Hf is H expanded back to the full (v, u) square (coalesced reads over u).
// Pairs are ordered by their A key; block (A key, chunk of 16 of its pairs,
// 128 u) keeps 16 accumulators per thread, so each Hf value feeds 16 FMAs and
// the 16 B-key weights are double2 shared-memory broadcasts (32 pairs per block
// measured slower: 0.66 against 0.615 ms at ERIDA 129^3).
constexpr int B_THREADS = 128;
constexpr int B_PAIRS = 16;
constexpr int B_VC = 64;                  // v chunk staged in shared memory

__global__ void k_expand_h(const double* __restrict__ H, const int* __restrict__ sidx,
                           const PlanCounts* __restrict__ cnt, int nS, int U, double* __restrict__ Hf) {
    const i64 plane = (i64)U * U;
    const i64 total = cnt->nA * plane;
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
        const i64 a = e / plane, vu = e % plane;
        Hf[e] = H[a * nS + sidx[vu]];
    }
}

__global__ void __launch_bounds__(B_THREADS) k_stage_b(const double* __restrict__ W, const double* __restrict__ Hf,
                                                        const int* __restrict__ pairA, const int* __restrict__ pairB,
                                                        const PlanCounts* __restrict__ cnt, int U, int Up, int nub,
                                                        int v_chunk, i64 part_stride, double* __restrict__ H2) {
    __shared__ __align__(16) double wb[B_VC][B_PAIRS];
    __shared__ int range[2];
    const int a = blockIdx.x;
    // blockIdx.z = u block + nub * (chunk of v): partial sums of small problems
    const int ub = blockIdx.z % nub, vz = blockIdx.z / nub;
    const int v_begin = vz * v_chunk, v_end = min(U, v_begin + v_chunk);
    H2 += (i64)vz * part_stride;
    if (a >= cnt->nA) return;  // grids are sized by a bound on nA
    const int nP = (int)cnt->nP;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nP;  // first pair with pairA >= a
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (pairA[mid] < a) lo = mid + 1; else hi = mid;
        }
        int lo2 = lo, hi2 = nP;  // first pair with pairA > a
        while (lo2 < hi2) {
            const int mid = (lo2 + hi2) >> 1;
            if (pairA[mid] <= a) lo2 = mid + 1; else hi2 = mid;
        }
        range[0] = lo;
        range[1] = lo2;
    }
    __syncthreads();
    const int pc = range[0] + blockIdx.y * B_PAIRS;
    if (pc >= range[1]) return;  // uniform across the block
    const int np = min(B_PAIRS, range[1] - pc);
    const int u = ub * B_THREADS + threadIdx.x;
    const bool live = u < U;
    const double* h = Hf + (i64)a * U * U + u;
    double acc[B_PAIRS];
#pragma unroll
    for (int k = 0; k < B_PAIRS; ++k) acc[k] = 0;
    for (int v0 = v_begin; v0 < v_end; v0 += B_VC) {
        __syncthreads();
        for (int e = threadIdx.x; e < B_VC * B_PAIRS; e += B_THREADS) {
            const int k = e / B_VC, vv = e % B_VC, v = v0 + vv;
            wb[vv][k] = (k < np && v < v_end) ? W[(i64)pairB[pc + k] * Up + v] : 0.0;
        }
        __syncthreads();
        if (live) {
            const int vmax = min(B_VC, v_end - v0);
            for (int vv = 0; vv < vmax; ++vv) {
                const double g = h[(i64)(v0 + vv) * U];
                const double2* w2 = reinterpret_cast<const double2*>(&wb[vv][0]);
#pragma unroll
                for (int k = 0; k < B_PAIRS / 2; ++k) {
                    const double2 w = w2[k];
                    acc[2 * k] = fma(w.x, g, acc[2 * k]);
                    acc[2 * k + 1] = fma(w.y, g, acc[2 * k + 1]);
                }
            }
        }
    }
    if (live)
#pragma unroll
        for (int k = 0; k < B_PAIRS; ++k)
            if (k < np) H2[(i64)(pc + k) * Up + u] = acc[k];
}

// out[i] = sum_p parts[p n + i], in order of p (deterministic)
__global__ void k_sum_parts(const double* __restrict__ parts, int P, i64 n, double* __restrict__ out) {
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double acc = parts[i];
        for (int p = 1; p < P; ++p) acc += parts[(i64)p * n + i];
        out[i] = acc;
    }
}

// Splits of a reduction loop of length U into P chunks (chunk a multiple of
// `grain`) so that a launch of `blocks` blocks reaches about eight blocks per
// SM: small problems otherwise leave most SMs idle while each block walks the
// whole loop.
static int split_count(i64 blocks, int U, int grain, int num_sms, int* chunk) {
    int P = (int)std::min<i64>((8LL * num_sms + blocks - 1) / blocks, (U + grain - 1) / grain);
    P = std::max(1, std::min(P, 8));
    *chunk = ((U + P - 1) / P + grain - 1) / grain * grain;
    P = (U + *chunk - 1) / *chunk;
    return P;
}

// ---------------------------------------------------------------------------
// stage C, per class: one warp per class, lanes stride over u, shuffle reduction
__global__ void __launch_bounds__(256) k_stage_c(const double* __restrict__ W, const double* __restrict__ H2,
                                                  const int2* __restrict__ cls, const int* __restrict__ keyOf, i64 m,
                                                  int U, int Up, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const i64 warps = (i64)gridDim.x * (blockDim.x >> 5);
    for (i64 n = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); n < m; n += warps) {
        const int2 c = cls[n];
        double acc = 0;
        if (c.x >= 0) {
            const double* w = W + (i64)keyOf[c.y] * Up;
            const double* h = H2 + (i64)c.x * Up;
            for (int u = lane; u < U; u += 32) acc = fma(w[u], h[u], acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[n] = (c.x >= 0) ? acc : 0.0;
    }
}

// stage C as a product: Q[p][j] = sum_u H2[p][u] Wu[j][u] for every (pair, used key),
// then a gather val[n] = Q[p(n)][j(n)].  Chosen when nP * nku is small against m.
__global__ void k_gather_rows(const double* __restrict__ W, const int* __restrict__ keyOf,
                              const PlanCounts* __restrict__ cnt, int Up, double* __restrict__ Wu) {
    const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= cnt->nku * Up) return;
    Wu[e] = W[(i64)keyOf[e / Up] * Up + e % Up];
}

__global__ void k_gather_q(const double* __restrict__ Q, const int2* __restrict__ cls, i64 m, int nku,
                           double* __restrict__ out) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    const int2 c = cls[n];
    out[n] = c.x >= 0 ? Q[(i64)c.x * nku + c.y] : 0.0;
}

// ---------------------------------------------------------------------------
// mixed form: stages A and B as int8-sliced products on the tensor cores
//   stage A:  H^T[j][a] = sum_t G[j][t] W[aKey[a]][t],   G[j][t] = T[S[j] + t^2]
//   stage B:  H2[p][u]  = sum_v Hf[a][u][v] W[pairB[p]][v]  for the pairs p of A key a
// (Hf[a] is symmetric, so its rows serve as the K-major operand), and stage C
// in its product form Q = H2 Wu^T with the FP64-level slicing.
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

// used key j: row W[keyOf[j]], for j below the used-key count in device memory
struct UsedKeyRows {
    const double* W;
    const int* keyOf;
    const PlanCounts* cnt;
    i64 Up;
    __device__ RowBase row(i64 j) const { return {W + (i64)keyOf[j] * Up}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k]; }
    __device__ bool valid(i64 j) const { return j < cnt->nku; }
    GLI_IDENTITY_ROWS
};

// dense rows whose count lives in device memory (PlanCounts::nP)
struct PairCountedRows {
    const double* src;
    const PlanCounts* cnt;
    i64 ld;
    __device__ RowBase row(i64 r) const { return {src + r * ld}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k]; }
    __device__ bool valid(i64 r) const { return r < (i64)cnt->nP; }
    GLI_IDENTITY_ROWS
};

// One block: first pair, pair count and first tile of every A key (pairs are
// ordered by A key), and the tile list of stage B (tiles of bn pairs, each in
// one A key); tiles past the last one get no columns.
__global__ void __launch_bounds__(1024) k_pair_tiles(const int* __restrict__ pairA, const PlanCounts* __restrict__ cnt,
                                                      int bn, int max_tiles, int* __restrict__ first,
                                                      int* __restrict__ tile0, int* __restrict__ tile_batch,
                                                      int* __restrict__ tile_col0, int* __restrict__ tile_ncols) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    const int nP = (int)cnt->nP, nA = (int)cnt->nA;
    if (threadIdx.x == 0) carry = 0;
    for (int t = threadIdx.x; t < max_tiles; t += blockDim.x) tile_ncols[t] = 0;
    __syncthreads();
    for (int base = 0; base < nA; base += blockDim.x) {
        const int a = base + threadIdx.x;
        int lo = 0, npairs = 0;
        if (a < nA) {
            int hi = nP;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (pairA[mid] < a) lo = mid + 1; else hi = mid;
            }
            int lo2 = lo, hi2 = nP;
            while (lo2 < hi2) {
                const int mid = (lo2 + hi2) >> 1;
                if (pairA[mid] <= a) lo2 = mid + 1; else hi2 = mid;
            }
            npairs = lo2 - lo;
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
            first[a] = lo;
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

void dgemm_strided(int M, int N, int K, const double* A, i64 asb, i64 ar, i64 ac, const double* B, i64 bsb, i64 br,
                   i64 bc, double* C, i64 csb, i64 cr, i64 cc, int batch, bool accumulate, cudaStream_t s);

static thread_local bool t_timing = false;
static thread_local ContractStats t_last;

void set_timing(bool on) { t_timing = on; }
const ContractStats& last_stats() { return t_last; }

struct StageTimer {
    static constexpr int kMax = 8;
    bool on;
    cudaStream_t s;
    cudaEvent_t ev[kMax];
    int n = 0;
    StageTimer(bool enabled, cudaStream_t st) : on(enabled), s(st) {
        if (on)
            for (auto& e : ev) GLI_CUDA(cudaEventCreate(&e));
    }
    void mark() {
        if (!on) return;
        if (n >= kMax) fail(GLI_ERR_INTERNAL, "stage timer overflow");
        GLI_CUDA(cudaEventRecord(ev[n++], s));
    }
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
struct EvalStatus {
    PlanCounts cnt;
    int bad;     // a class index outside the tensor
    int tc_err;  // a tensor-core CTA gave up waiting
};

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

static void read_status(EvalStatus* d_st, EvalStatus& h, cudaStream_t s) {
    GLI_CUDA(cudaMemcpyAsync(&h, d_st, sizeof(EvalStatus), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
}

// Queues one evaluation on stream s.  Kernels read the counts from st->cnt;
// the host sizes buffers and grids by `sz`.
static void enqueue_eval(const EvalArgs& a, bool bounded, EvalStatus* st, StageTimer& timer, EvalSizes& sz,
                         cudaStream_t s) {
    const LatticeTables& t = *a.t;
    const i64 nk = t.nkeys, m = a.m;
    const int U = (int)t.U, Up = (int)t.Up, nS = (int)t.nS;
    GLI_CUDA(cudaMemsetAsync(st, 0, sizeof(EvalStatus), s));
    PlanCounts* cnt = &st->cnt;
    // usedKey and usedA side by side so that one scan serves both
    DevBuf<uint32_t> used(2 * nk, s);
    used.zero();
    const unsigned cb = (unsigned)((m + 255) / 256);
    const unsigned kb = (unsigned)((nk + 255) / 256);
    k_mark_keys<<<cb, 256, 0, s>>>(a.d, a.idx, m, used.p, used.p + nk, &st->bad);
    GLI_CHECK_LAUNCH();
    DevBuf<uint64_t> ids(2 * nk, s);
    DevBuf<int> keyOf(nk, s), aId(nk, s), aKey(nk, s);
    const bool small = 2 * nk <= 1024;
    if (small) {
        k_plan_keys_small<<<1, 1024, 0, s>>>(nk, used.p, ids.p, keyOf.p, aId.p, aKey.p, cnt);
        GLI_CHECK_LAUNCH();
    } else {
        exclusive_scan_u32_dev(used.p, ids.p, 2 * nk, &cnt->key_total, s);
        k_plan_keys<<<kb, 256, 0, s>>>(nk, used.p, ids.p, keyOf.p, aId.p, aKey.p, cnt);
        GLI_CHECK_LAUNCH();
    }
    if (bounded) {
        sz.nku = nk;
        sz.nA = nk;
    } else {
        EvalStatus h;
        read_status(st, h, s);
        if (h.bad) fail(GLI_ERR_ARGUMENT, "class index outside the %s tensor of the grid", t.kind ? "ERI" : "ERIDA");
        sz.nku = h.cnt.nku;
        sz.nA = h.cnt.nA;
        if (sz.nku > 16384)
            fail(GLI_ERR_LIMIT, "class list uses %lld distinct axis keys (limit 16384)", (long long)sz.nku);
    }
    const i64 stride = sz.nku, slots = sz.nku * sz.nku;
    DevBuf<uint32_t> usedPair(slots, s);
    usedPair.zero();
    k_mark_pairs<<<cb, 256, 0, s>>>(a.d, a.idx, m, ids.p, stride, usedPair.p);
    GLI_CHECK_LAUNCH();
    DevBuf<uint64_t> pairId(slots, s);
    const bool small_pairs = bounded && slots <= 65536;
    if (!small_pairs) exclusive_scan_u32_dev(usedPair.p, pairId.p, slots, &cnt->nP, s);
    if (bounded) {
        // pairs (A, B) have kid(A) >= kid(B); every class has one pair
        sz.nP = std::min(sz.nku * (sz.nku + 1) / 2, m);
    } else {
        EvalStatus h;
        read_status(st, h, s);
        sz.nP = (i64)h.cnt.nP;
    }
    DevBuf<int> pairA(sz.nP, s), pairB(sz.nP, s);
    if (small_pairs)
        k_pairs_small<<<1, 1024, 0, s>>>(slots, stride, usedPair.p, keyOf.p, aId.p, pairId.p, pairA.p, pairB.p, cnt);
    else
        k_pair_lists<<<(unsigned)((slots + 255) / 256), 256, 0, s>>>(slots, stride, usedPair.p, pairId.p, keyOf.p,
                                                                      aId.p, pairA.p, pairB.p);
    GLI_CHECK_LAUNCH();
    DevBuf<int2> cls(m, s);
    k_class_pairs<<<cb, 256, 0, s>>>(a.d, a.idx, m, ids.p, stride, pairId.p, cls.p);
    GLI_CHECK_LAUNCH();

    const i64 nA = sz.nA, nP = sz.nP, nku = sz.nku;
    if (nA * (i64)U * U > ((i64)1 << 31))
        fail(GLI_ERR_LIMIT, "stage buffers exceed 16 GB (%lld A keys, lattice extent %d)", (long long)nA, U);
    DevBuf<double> H(nA * (i64)nS, s);
    // the mixed form runs a stage on the tensor cores when it is large enough for
    // them to pay off; smaller stages (latency-bound either way) stay FP64
    const bool tc_a = a.mixed && nA * (i64)nS >= 1000000;
    const bool tc_b = a.mixed && nA * (i64)U * U >= 4000000;
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
        // keys per thread: fewer when the problem is small, so that enough
        // warps exist to hide the table-gather latency; small problems also
        // split the t loop (partial sums, then one summing pass)
        const i64 outputs = nA * (i64)nS;
        const unsigned sb = (unsigned)((nS + A_STILE - 1) / A_STILE);
        const int KT = (outputs >= 4000000 && nA >= 32) ? 32 : outputs >= 1000000 ? 16 : 4;
        const unsigned kb = (unsigned)((nA + KT - 1) / KT);
        int t_chunk = U;
        const int P = split_count((i64)sb * kb, U, A_TC, a.num_sms, &t_chunk);
        DevBuf<double> parts;
        double* dst = H.p;
        if (P > 1) {
            parts.alloc((i64)P * nA * nS, s);
            dst = parts.p;
        }
        const dim3 grid(sb, kb, (unsigned)P);
        const i64 ps = nA * (i64)nS;
        if (KT == 32)
            k_stage_a<32><<<grid, A_THREADS, 0, s>>>(t.W.p, t.T.p, t.S.p, aKey.p, cnt, nS, U, Up, t_chunk, ps, dst);
        else if (KT == 16)
            k_stage_a<16><<<grid, A_THREADS, 0, s>>>(t.W.p, t.T.p, t.S.p, aKey.p, cnt, nS, U, Up, t_chunk, ps, dst);
        else
            k_stage_a<4><<<grid, A_THREADS, 0, s>>>(t.W.p, t.T.p, t.S.p, aKey.p, cnt, nS, U, Up, t_chunk, ps, dst);
        GLI_CHECK_LAUNCH();
        if (P > 1) {
            k_sum_parts<<<(unsigned)std::min<i64>((ps + 255) / 256, (i64)a.num_sms * 16), 256, 0, s>>>(parts.p, P, ps,
                                                                                                      H.p);
            GLI_CHECK_LAUNCH();
        }
    }
    timer.mark();
    // ---- stage B
    DevBuf<double> H2(nP * (i64)Up, s);
    if (tc_b) {
        constexpr int BN = tile_n(MIXED_SLICES);
        const int mb = (U + TC_BM - 1) / TC_BM;
        TiledSlices Hs, Wb;
        Hs.alloc(nA * mb, TC_BM, U, MIXED_SLICES, s);
        slice_tiled(ExpandedHRows{H.p, t.sidx.p, cnt, nS, U, mb}, nA * U, U, Hs, s);
        const i64 max_tiles = nP / BN + nA + 1;
        DevBuf<int> grp(2 * nA + 3 * max_tiles, s);
        int* first = grp.p;
        int* tile0 = grp.p + nA;
        int* tile_batch = grp.p + 2 * nA;
        int* tile_col0 = tile_batch + max_tiles;
        int* tile_ncols = tile_col0 + max_tiles;
        k_pair_tiles<<<1, 1024, 0, s>>>(pairA.p, cnt, BN, (int)max_tiles, first, tile0, tile_batch, tile_col0,
                                        tile_ncols);
        GLI_CHECK_LAUNCH();
        Wb.alloc(max_tiles, BN, U, MIXED_SLICES, s);
        slice_tiled(PairRows{t.W.p, pairA.p, pairB.p, first, tile0, tile_col0, tile_ncols, cnt, Up, BN}, nP, U, Wb,
                    s);
        TileWork w;
        w.a_rows = U;
        w.a_blocks = mb;
        w.a_batched = 1;
        w.tile_batch = tile_batch;
        w.tile_col0 = tile_col0;
        w.tile_ncols = tile_ncols;
        w.C = H2.p;
        w.rs = 1;
        w.cs = Up;
        tc_gemm_tiled(Hs.view(), Wb.view(), w, (int)max_tiles, &st->tc_err, s);
    } else {
        DevBuf<double> Hf(nA * (i64)U * U, s);
        const i64 ework = nA * (i64)U * U;
        const i64 eb = std::min<i64>((ework + 255) / 256, (i64)a.num_sms * 32);
        k_expand_h<<<(unsigned)eb, 256, 0, s>>>(H.p, t.sidx.p, cnt, nS, U, Hf.p);
        GLI_CHECK_LAUNCH();
        // chunk slots per A key: at most nku pairs share one A key
        const unsigned chunks = (unsigned)((nku + B_PAIRS - 1) / B_PAIRS);
        const int nub = (U + B_THREADS - 1) / B_THREADS;
        int v_chunk = U;
        const int P = split_count(nA * (i64)chunks * nub, U, 32, a.num_sms, &v_chunk);
        const i64 ps = nP * (i64)Up;
        DevBuf<double> parts;
        double* dst = H2.p;
        if (P > 1) {
            parts.alloc(P * ps, s);
            dst = parts.p;
        }
        k_stage_b<<<dim3((unsigned)nA, chunks, (unsigned)(nub * P)), B_THREADS, 0, s>>>(
            t.W.p, Hf.p, pairA.p, pairB.p, cnt, U, Up, nub, v_chunk, ps, dst);
        GLI_CHECK_LAUNCH();
        if (P > 1) {
            k_sum_parts<<<(unsigned)std::min<i64>((ps + 255) / 256, (i64)a.num_sms * 16), 256, 0, s>>>(parts.p, P, ps,
                                                                                                      H2.p);
            GLI_CHECK_LAUNCH();
        }
    }
    timer.mark();
    // ---- stage C: the product form computes every (pair, key) dot product --
    // up to 16x more than the classes need on the tensor cores, as many as the
    // classes in FP64 -- but as a GEMM it reuses each H2 row across keys instead
    // of re-reading it per class; small class lists keep the per-class kernel
    const bool product = a.mixed ? (m >= 65536 && nP * nku <= 16 * m) : (nP * nku <= m);
    if (product) {
        DevBuf<double> Q(nP * nku, s);
        if (a.mixed) {
            constexpr int BN = tile_n(FP64_SLICES);
            TiledSlices Hs2, Wus;
            const i64 pb = (nP + TC_BM - 1) / TC_BM, kb2 = (nku + BN - 1) / BN;
            Hs2.alloc(pb, TC_BM, U, FP64_SLICES, s);
            slice_tiled(PairCountedRows{H2.p, cnt, Up}, nP, U, Hs2, s);
            Wus.alloc(kb2, BN, U, FP64_SLICES, s);
            slice_tiled(UsedKeyRows{t.W.p, keyOf.p, cnt, Up}, nku, U, Wus, s);
            TileWork w;
            w.a_rows = (int)nP;
            w.a_blocks = (int)pb;
            w.n_total = (int)nku;
            w.C = Q.p;
            w.rs = nku;
            w.cs = 1;
            tc_gemm_tiled(Hs2.view(), Wus.view(), w, (int)kb2, &st->tc_err, s);
        } else {
            DevBuf<double> Wu(nku * (i64)Up, s);
            k_gather_rows<<<(unsigned)((nku * Up + 255) / 256), 256, 0, s>>>(t.W.p, keyOf.p, cnt, Up, Wu.p);
            GLI_CHECK_LAUNCH();
            dgemm_strided((int)nP, (int)nku, U, H2.p, 0, Up, 1, Wu.p, 0, 1, Up, Q.p, 0, nku, 1, 1, false, s);
        }
        k_gather_q<<<cb, 256, 0, s>>>(Q.p, cls.p, m, (int)nku, a.out);
        GLI_CHECK_LAUNCH();
    } else {
        const i64 want = (m + 7) / 8;
        const unsigned gc = (unsigned)(want < (i64)a.num_sms * 16 ? want : (i64)a.num_sms * 16);
        k_stage_c<<<gc, 256, 0, s>>>(t.W.p, H2.p, cls.p, keyOf.p, m, U, Up, a.out);
        GLI_CHECK_LAUNCH();
    }
    timer.mark();
}

// ---------------------------------------------------------------------------
// CUDA graphs of bounded evaluations.  A bounded evaluation issues no host
// synchronisation, so the whole launch sequence (allocations, memsets and about
// 15 kernels) is captured once and replayed: every replay recomputes everything
// from the class list in device memory; only the launch overhead is saved.
// A graph is keyed by what fixes its launch sequence and its pointers: the
// table set (kept alive by the entry), the grid, the class-list pointer and
// length, the output pointer and the form.
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
    DevMem<EvalStatus> status;
    ~GraphEntry() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

static thread_local std::list<std::unique_ptr<GraphEntry>> t_graphs;
static constexpr size_t kGraphEntries = 8;
static const bool g_graphs_enabled = getenv("GLI_B200_NO_GRAPHS") == nullptr;

static GraphEntry* find_graph(const EvalArgs& a, int device) {
    for (auto it = t_graphs.begin(); it != t_graphs.end(); ++it) {
        GraphEntry& e = **it;
        if (e.tables == a.t && e.device == device && e.mixed == (int)a.mixed && e.idx == a.idx && e.out == a.out &&
            e.m == a.m && e.istart[0] == a.d.istart[0] && e.istart[1] == a.d.istart[1] &&
            e.istart[2] == a.d.istart[2] && e.num[0] == a.d.num[0] && e.num[1] == a.d.num[1] &&
            e.num[2] == a.d.num[2]) {
            t_graphs.splice(t_graphs.begin(), t_graphs, it);  // most recently used first
            return t_graphs.front().get();
        }
    }
    return nullptr;
}

static GraphEntry* capture_graph(const EvalArgs& a, const std::shared_ptr<const LatticeTables>& tp, int device,
                                 cudaStream_t s) {
    auto e = std::make_unique<GraphEntry>();
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
    tc_gemm_prepare();  // function attributes are set outside the capture
    const long long l0 = launch_count();
    GLI_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
        StageTimer timer(false, s);
        EvalSizes sz;
        enqueue_eval(a, true, e->status.p, timer, sz, s);
    } catch (...) {
        cudaStreamEndCapture(s, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
    }
    GLI_CUDA(cudaStreamEndCapture(s, &graph));
    e->launches = launch_count() - l0;
    const cudaError_t ie = cudaGraphInstantiate(&e->exec, graph, 0);
    cudaGraphDestroy(graph);
    GLI_CUDA(ie);
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

// Queues one evaluation on stream s and an asynchronous copy of its status
// block into h_status (pinned); the caller synchronises and checks it.
static void sparse_values_enqueue(int kind, const double* h_coeffs, i64 nb, const GridDesc& g,
                                  const int64_t* d_indices, i64 m, double tol, int form, double* d_out, cudaStream_t s,
                                  EvalStatus* h_status, std::shared_ptr<const LatticeTables>& tp, StageTimer& timer) {
    if (form != FORM_FP64 && form != FORM_MIXED)
        fail(GLI_ERR_ARGUMENT, "form %d is not a sparse evaluation form (0 = FP64, 1 = mixed)", form);
    if (!(tol >= 0)) fail(GLI_ERR_ARGUMENT, "tol must be non-negative");
    const Context& ctx = context();
    timer.mark();
    tp = lattice_tables(kind, h_coeffs, nb, g.max_range(), tol, s);
    const LatticeTables& t = *tp;
    EvalArgs a;
    a.mixed = form == FORM_MIXED;
    a.t = &t;
    if (a.mixed) a.G = lattice_g_slices(t, s);
    timer.mark();
    a.d.kind = kind;
    a.d.N = g.points();
    a.d.L = t.L;
    for (int k = 0; k < 3; ++k) {
        a.d.istart[k] = g.istart[k];
        a.d.num[k] = g.num[k];
    }
    a.d.nkeys = t.nkeys;
    a.idx = d_indices;
    a.m = m;
    a.out = d_out;
    a.num_sms = ctx.num_sms;
    const bool bounded = t.nkeys <= BOUNDED_KEYS;
    if (bounded && !t_timing && g_graphs_enabled) {
        GraphEntry* e = find_graph(a, ctx.device);
        if (!e) e = capture_graph(a, tp, ctx.device, s);
        GLI_CUDA(cudaGraphLaunch(e->exec, s));
        add_launches(e->launches);
        GLI_CUDA(cudaMemcpyAsync(h_status, e->status.p, sizeof(EvalStatus), cudaMemcpyDeviceToHost, s));
    } else {
        DevBuf<EvalStatus> st(1, s);
        EvalSizes sz;
        enqueue_eval(a, bounded, st.p, timer, sz, s);
        GLI_CUDA(cudaMemcpyAsync(h_status, st.p, sizeof(EvalStatus), cudaMemcpyDeviceToHost, s));
    }
}

// after the stream synchronised: errors of the evaluation, and the statistics
static void check_status(int kind, const EvalStatus& h, const LatticeTables& t, StageTimer& timer,
                         ContractStats* stats) {
    if (h.bad) fail(GLI_ERR_ARGUMENT, "class index outside the %s tensor of the grid", kind ? "ERI" : "ERIDA");
    if (h.tc_err) fail(GLI_ERR_INTERNAL, "tensor-core stage: an mbarrier wait expired (code %d)", h.tc_err);
    if (h.cnt.nku > 16384)
        fail(GLI_ERR_LIMIT, "class list uses %lld distinct axis keys (limit 16384)", (long long)h.cnt.nku);
    ContractStats st;
    st.keys_a = h.cnt.nA;
    st.pairs = (i64)h.cnt.nP;
    st.U = t.U;
    if (t_timing) {
        st.ms_tables = timer.between(0, 1);
        st.ms_a = timer.between(2, 3);
        st.ms_b = timer.between(3, 4);
        st.ms_c = timer.between(4, 5);
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
    sparse_values_enqueue(kind, h_coeffs, nb, g, d_indices, m, tol, form, d_out, s, h, tp, timer);
    GLI_CUDA(cudaStreamSynchronize(s));
    check_status(kind, *h, *tp, timer, stats);
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

void sparse_values_host(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* h_indices, i64 m,
                        double tol, int form, double* h_out, cudaStream_t s) {
    if (m == 0) return;
    const Context& ctx = context();
    EvalStatus* hs = (EvalStatus*)t_pin_status.get(sizeof(EvalStatus));
    int64_t* pin_idx = (int64_t*)t_pin_idx.get((size_t)m * sizeof(int64_t));
    double* pin_val = (double*)t_pin_val.get((size_t)m * sizeof(double));
    t_host_call.ensure(ctx.device, m);
    memcpy(pin_idx, h_indices, (size_t)m * sizeof(int64_t));
    GLI_CUDA(cudaMemcpyAsync(t_host_call.idx->p, pin_idx, (size_t)m * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    std::shared_ptr<const LatticeTables> tp;
    StageTimer timer(t_timing, s);
    sparse_values_enqueue(kind, h_coeffs, nb, g, t_host_call.idx->p, m, tol, form, t_host_call.val->p, s, hs, tp,
                          timer);
    GLI_CUDA(cudaMemcpyAsync(pin_val, t_host_call.val->p, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    check_status(kind, *hs, *tp, timer, nullptr);
    memcpy(h_out, pin_val, (size_t)m * sizeof(double));
}

}  // namespace gli
