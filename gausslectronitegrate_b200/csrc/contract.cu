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
//   stage A  H[a][v][u]  = sum_t W[key_a][t] T[u^2 + v^2 + t^2]      per distinct A key
//   stage B  H2[p][u]    = sum_v W[key_b][v] H[a(p)][v][u]            per distinct (A, B) key pair
//   stage C  val[n]      = sum_u W[key_c][u] H2[p(n)][u]              per class: warp dot + shuffles
// The value is symmetric under permuting the three axes (T is), so each class's
// key triple is sorted (k1 <= k2 <= k3) and assigned A = k2, B = k1, C = k3.
#include <math.h>

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

// (A, B) pairs over the compacted key ids: slot = kid(k2) * nku + kid(k1)
__global__ void k_mark_pairs(ClassDecode d, const int64_t* __restrict__ idx, i64 m, const uint64_t* __restrict__ kid,
                             i64 nku, uint32_t* __restrict__ usedPair) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    i64 k[3];
    if (!class_keys(d, idx[n], k)) return;
    usedPair[(i64)kid[k[1]] * nku + (i64)kid[k[0]]] = 1;
}

// compact id -> original key
__global__ void k_key_of(i64 nkeys, const uint32_t* __restrict__ used, const uint64_t* __restrict__ id,
                         int* __restrict__ keyOf) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nkeys && used[k]) keyOf[id[k]] = (int)k;
}

__global__ void k_pair_lists(i64 nku, const uint32_t* __restrict__ usedPair, const uint64_t* __restrict__ pairId,
                             const int* __restrict__ keyOf, const uint64_t* __restrict__ aId, int* __restrict__ pairA,
                             int* __restrict__ pairB) {
    const i64 slot = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nku * nku || !usedPair[slot]) return;
    const i64 ka = keyOf[slot / nku], kb = keyOf[slot % nku];
    pairA[pairId[slot]] = (int)aId[ka];
    pairB[pairId[slot]] = (int)kb;
}

__global__ void k_class_pairs(ClassDecode d, const int64_t* __restrict__ idx, i64 m, const uint64_t* __restrict__ kid,
                              i64 nku, const uint64_t* __restrict__ pairId, int2* __restrict__ cls) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    i64 k[3];
    if (!class_keys(d, idx[n], k)) {
        cls[n] = make_int2(-1, 0);
        return;
    }
    cls[n] = make_int2((int)pairId[(i64)kid[k[1]] * nku + (i64)kid[k[0]]], (int)k[2]);
}

// ---------------------------------------------------------------------------
// stage A: H[a][v][u] = sum_t W[aKey[a]][t] T[u^2 + v^2 + t^2]
// block: 16 x 16 (u, v) tile, KA keys; each thread owns one (u, v) and KA sums.
constexpr int A_TILE = 16;
constexpr int A_KEYS = 16;
constexpr int A_TCHUNK = 32;

__global__ void __launch_bounds__(256) k_stage_a(const double* __restrict__ W, const double* __restrict__ T,
                                                  const int* __restrict__ aKey, int nA, int U, int Up,
                                                  double* __restrict__ H) {
    __shared__ double ws[A_KEYS][A_TCHUNK];
    const int u = blockIdx.x * A_TILE + (threadIdx.x & (A_TILE - 1));
    const int v = blockIdx.y * A_TILE + (threadIdx.x / A_TILE);
    const int a0 = blockIdx.z * A_KEYS;
    const bool live = (u < U) && (v < U);
    const int uv2 = u * u + v * v;
    double acc[A_KEYS];
#pragma unroll
    for (int k = 0; k < A_KEYS; ++k) acc[k] = 0;
    for (int t0 = 0; t0 < U; t0 += A_TCHUNK) {
        __syncthreads();
        for (int e = threadIdx.x; e < A_KEYS * A_TCHUNK; e += blockDim.x) {
            const int k = e / A_TCHUNK, t = t0 + e % A_TCHUNK;
            ws[k][e % A_TCHUNK] = (a0 + k < nA && t < U) ? W[(i64)aKey[a0 + k] * Up + t] : 0.0;
        }
        __syncthreads();
        if (live) {
            const int tmax = min(A_TCHUNK, U - t0);
            for (int tt = 0; tt < tmax; ++tt) {
                const int t = t0 + tt;
                const double g = __ldg(&T[uv2 + t * t]);
#pragma unroll
                for (int k = 0; k < A_KEYS; ++k) acc[k] = fma(ws[k][tt], g, acc[k]);
            }
        }
    }
    if (!live) return;
    const i64 plane = (i64)U * U;
#pragma unroll
    for (int k = 0; k < A_KEYS; ++k)
        if (a0 + k < nA) H[(i64)(a0 + k) * plane + (i64)v * U + u] = acc[k];
}

// ---------------------------------------------------------------------------
// stage B: H2[p][u] = sum_v W[pairB[p]][v] H[pairA[p]][v][u]; one block per pair
__global__ void __launch_bounds__(128) k_stage_b(const double* __restrict__ W, const double* __restrict__ H,
                                                  const int* __restrict__ pairA, const int* __restrict__ pairB, int U,
                                                  int Up, double* __restrict__ H2) {
    extern __shared__ double wb[];
    const int p = blockIdx.x;
    const double* w = W + (i64)pairB[p] * Up;
    for (int v = threadIdx.x; v < U; v += blockDim.x) wb[v] = w[v];
    __syncthreads();
    const double* h = H + (i64)pairA[p] * U * U;
    for (int u = threadIdx.x; u < U; u += blockDim.x) {
        double acc = 0;
        for (int v = 0; v < U; ++v) acc = fma(wb[v], h[(i64)v * U + u], acc);
        H2[(i64)p * Up + u] = acc;
    }
}

// ---------------------------------------------------------------------------
// stage C: one warp per class, lanes stride over u, shuffle reduction
__global__ void __launch_bounds__(256) k_stage_c(const double* __restrict__ W, const double* __restrict__ H2,
                                                  const int2* __restrict__ cls, i64 m, int U, int Up,
                                                  double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const i64 warps = (i64)gridDim.x * (blockDim.x >> 5);
    for (i64 n = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); n < m; n += warps) {
        const int2 c = cls[n];
        double acc = 0;
        if (c.x >= 0) {
            const double* w = W + (i64)c.y * Up;
            const double* h = H2 + (i64)c.x * Up;
            for (int u = lane; u < U; u += 32) acc = fma(w[u], h[u], acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[n] = (c.x >= 0) ? acc : 0.0;
    }
}

static thread_local bool t_timing = false;
static thread_local ContractStats t_last;

void set_timing(bool on) { t_timing = on; }
const ContractStats& last_stats() { return t_last; }

struct StageTimer {
    bool on;
    cudaStream_t s;
    cudaEvent_t ev[5];
    int n = 0;
    StageTimer(bool enabled, cudaStream_t st) : on(enabled), s(st) {
        if (on)
            for (auto& e : ev) GLI_CUDA(cudaEventCreate(&e));
    }
    void mark() {
        if (on) GLI_CUDA(cudaEventRecord(ev[n++], s));
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

void sparse_values_device(int kind, const double* h_coeffs, i64 nb, const GridDesc& g, const int64_t* d_indices,
                          i64 m, double tol, int form, double* d_out, cudaStream_t s, ContractStats* stats) {
    if (form != FORM_FP64 && form != FORM_MIXED) fail(GLI_ERR_ARGUMENT, "unknown form %d", form);
    if (!(tol >= 0)) fail(GLI_ERR_ARGUMENT, "tol must be non-negative");
    if (m == 0) return;
    StageTimer timer(t_timing, s);
    timer.mark();
    LatticeTables t;
    build_lattice_tables(kind, h_coeffs, nb, g.max_range(), tol, t, s);
    timer.mark();

    ClassDecode d;
    d.kind = kind;
    d.N = g.points();
    d.L = t.L;
    for (int a = 0; a < 3; ++a) {
        d.istart[a] = g.istart[a];
        d.num[a] = g.num[a];
    }
    d.nkeys = t.nkeys;
    const i64 nk = t.nkeys;
    DevBuf<uint32_t> usedKey(nk, s), usedA(nk, s);
    usedKey.zero();
    usedA.zero();
    DevBuf<int> bad(1, s);
    bad.zero();
    const unsigned cb = (unsigned)((m + 255) / 256);
    const unsigned kb = (unsigned)((nk + 255) / 256);
    k_mark_keys<<<cb, 256, 0, s>>>(d, d_indices, m, usedKey.p, usedA.p, bad.p);
    GLI_CHECK_LAUNCH();
    DevBuf<uint64_t> kid(nk, s), aId(nk, s);
    const i64 nku = exclusive_scan_u32(usedKey.p, kid.p, nk, s);
    const i64 nA = exclusive_scan_u32(usedA.p, aId.p, nk, s);
    int h_bad = 0;
    GLI_CUDA(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    if (h_bad) fail(GLI_ERR_ARGUMENT, "class index outside the %s tensor of the grid", kind ? "ERI" : "ERIDA");
    if (nku > 16384) fail(GLI_ERR_LIMIT, "class list uses %lld distinct axis keys (limit 16384)", (long long)nku);

    DevBuf<int> keyOf(nku, s), aKey(nA, s);
    k_key_of<<<kb, 256, 0, s>>>(nk, usedKey.p, kid.p, keyOf.p);
    GLI_CHECK_LAUNCH();
    k_key_of<<<kb, 256, 0, s>>>(nk, usedA.p, aId.p, aKey.p);
    GLI_CHECK_LAUNCH();
    DevBuf<uint32_t> usedPair(nku * nku, s);
    usedPair.zero();
    k_mark_pairs<<<cb, 256, 0, s>>>(d, d_indices, m, kid.p, nku, usedPair.p);
    GLI_CHECK_LAUNCH();
    DevBuf<uint64_t> pairId(nku * nku, s);
    const i64 nP = exclusive_scan_u32(usedPair.p, pairId.p, nku * nku, s);
    DevBuf<int> pairA(nP, s), pairB(nP, s);
    k_pair_lists<<<(unsigned)((nku * nku + 255) / 256), 256, 0, s>>>(nku, usedPair.p, pairId.p, keyOf.p, aId.p,
                                                                      pairA.p, pairB.p);
    GLI_CHECK_LAUNCH();
    DevBuf<int2> cls(m, s);
    k_class_pairs<<<cb, 256, 0, s>>>(d, d_indices, m, kid.p, nku, pairId.p, cls.p);
    GLI_CHECK_LAUNCH();

    const int U = (int)t.U, Up = (int)t.Up;
    DevBuf<double> H(nA * (i64)U * U, s);
    dim3 ga((U + A_TILE - 1) / A_TILE, (U + A_TILE - 1) / A_TILE, (unsigned)((nA + A_KEYS - 1) / A_KEYS));
    timer.mark();
    k_stage_a<<<ga, 256, 0, s>>>(t.W.p, t.T.p, aKey.p, (int)nA, U, Up, H.p);
    GLI_CHECK_LAUNCH();
    timer.mark();
    DevBuf<double> H2(nP * (i64)Up, s);
    k_stage_b<<<(unsigned)nP, 128, U * sizeof(double), s>>>(t.W.p, H.p, pairA.p, pairB.p, U, Up, H2.p);
    GLI_CHECK_LAUNCH();
    timer.mark();
    const Context& ctx = context();
    const i64 want = (m + 7) / 8;
    const unsigned gc = (unsigned)(want < (i64)ctx.num_sms * 16 ? want : (i64)ctx.num_sms * 16);
    k_stage_c<<<gc, 256, 0, s>>>(t.W.p, H2.p, cls.p, m, U, Up, d_out);
    GLI_CHECK_LAUNCH();
    timer.mark();
    ContractStats st;
    st.keys_a = nA;
    st.pairs = nP;
    st.U = U;
    if (t_timing) {
        GLI_CUDA(cudaStreamSynchronize(s));
        st.ms_tables = timer.between(0, 1);
        st.ms_a = timer.between(2, 3);
        st.ms_b = timer.between(3, 4);
        st.ms_c = timer.between(4, 5);
    }
    t_last = st;
    if (stats) *stats = st;
}

}  // namespace gli
