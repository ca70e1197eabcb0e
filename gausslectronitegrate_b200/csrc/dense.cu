// Sparse -> dense expansion, the ERI two-particle apply and the projections
// onto an orbital basis.
//
// Reference counterparts:
//   fill_dense_eri_tensor            src/eri_integrals.c:850-967
//   fill_dense_erida_matrix          src/erida_integrals.c:683-765
//   apply_sparse_eri_tensor          src/eri_integrals.c:974-1100
//   project_sparse_eri_gausslet_integrals    src/eri_integrals.c:714-843
//   project_sparse_erida_gausslet_integrals  src/erida_integrals.c:580-676
//   evaluate_octahedral_grid_permutations    src/symmetry.c:120-150
//
// Every dense entry is canonicalised in the sparse grid (box centre moved to
// the origin, minimum over bias shifts x O_h x index swaps) and looked up by
// binary search in the sorted class list, 0 when absent -- the reference's
// semantics for arbitrary (also loaded or hand-made) sparse lists.  The
// projections contract one tensor axis at a time (the factored form the
// reference tests use as their check, test/test_eri_integrals.c:188-212)
// instead of the O(N^4 M^4) atomic loop, over slabs of the first index (or
// batches of index pairs) so that the dense tensor is never held whole.
//
// Complete class lists.  When an ERI list holds every canonical class of its
// grid (the count matches the enumeration, the indices increase strictly and
// each is its orbit's minimum), an entry needs no canonicalisation: each class
// value is a function of the sorted triple of per-axis keys of its four points
// (the staged contraction computes it from exactly that), and every entry has
// the key triple of its class.  The values are then scattered once into a
// table indexed by the sorted key triple, and dense entries are generated by
// key arithmetic and one table read.  The projection's first contraction (the
// O(N^4 M) one) computes its slab that way inside the FP64 tensor-core GEMM
// as it stages the operand tiles (KeyedSlabOp, at most 32 orbitals), or fills
// the slab first (k_fill_slab_keyed) and contracts it.
#include <algorithm>
#include <map>
#include <mutex>

#include "dmma.cuh"
#include "symmetry.cuh"
#include "tables.cuh"

namespace gli {

__device__ inline double lookup_sorted(const int64_t* __restrict__ idx, const double* __restrict__ val, i64 m, i64 key) {
    i64 lo = 0, hi = m;
    while (lo < hi) {
        const i64 mid = (lo + hi) >> 1;
        const i64 v = idx[mid];
        if (key < v) hi = mid;
        else if (key > v) lo = mid + 1;
        else return val[mid];
    }
    return 0.0;
}

struct DenseGrid {
    int istart[3];
    int num[3];
    i64 N;
};

__device__ inline void dense_point(const DenseGrid& D, i64 lin, int p[3]) {
    p[2] = D.istart[2] + (int)(lin % D.num[2]);
    lin /= D.num[2];
    p[1] = D.istart[1] + (int)(lin % D.num[1]);
    p[0] = D.istart[0] + (int)(lin / D.num[1]);
}

__device__ inline double erida_entry(const SymGrid& G, const DenseGrid& D, i64 a, i64 b, const int64_t* idx,
                                     const double* val, i64 m) {
    int p[2][3], bias[3];
    dense_point(D, a, p[0]);
    dense_point(D, b, p[1]);
    centre_points<2>(p, bias);
    return lookup_sorted(idx, val, m, orbit_min_pair(G, p, bias));
}

__device__ inline double eri_entry(const SymGrid& G, const DenseGrid& D, i64 a, i64 b, i64 c, i64 d,
                                   const int64_t* idx, const double* val, i64 m) {
    int p[4][3], bias[3];
    dense_point(D, a, p[0]);
    dense_point(D, b, p[1]);
    dense_point(D, c, p[2]);
    dense_point(D, d, p[3]);
    centre_points<4>(p, bias);
    return lookup_sorted(idx, val, m, orbit_min_quad(G, p, bias));
}

__global__ void k_fill_erida(SymGrid G, DenseGrid D, const int64_t* __restrict__ idx, const double* __restrict__ val,
                             i64 m, double* __restrict__ out) {
    const i64 total = D.N * D.N;
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x)
        out[e] = erida_entry(G, D, e / D.N, e % D.N, idx, val, m);
}

// rows [row0, row0 + nrows) of the (ij) x (kl) flattening: out[(r - row0) * N^2 + kl]
__global__ void k_fill_eri_rows(SymGrid G, DenseGrid D, const int64_t* __restrict__ idx,
                                const double* __restrict__ val, i64 m, i64 row0, i64 nrows,
                                double* __restrict__ out) {
    const i64 N2 = D.N * D.N;
    const i64 total = nrows * N2;
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
        const i64 r = row0 + e / N2, kl = e % N2;
        out[e] = eri_entry(G, D, r / D.N, r % D.N, kl / D.N, kl % D.N, idx, val, m);
    }
}

// ---------------------------------------------------------------------------
// complete class lists: values by sorted per-axis key triple
__host__ __device__ inline i64 tetra_index(i64 k1, i64 k2, i64 k3) {  // k1 <= k2 <= k3
    return k3 * (k3 + 1) * (k3 + 2) / 6 + k2 * (k2 + 1) / 2 + k1;
}
// the same in 32-bit arithmetic, for key tables of at most 2^29 slots (the
// only ones built): then k3 (k3 + 1) (k3 + 2) <= 6 * 2^29 < 2^32
__device__ __forceinline__ uint32_t tetra_index32(uint32_t k1, uint32_t k2, uint32_t k3) {
    return k3 * (k3 + 1) * (k3 + 2) / 6u + k2 * (k2 + 1) / 2u + k1;
}

__device__ inline i64 eri_key_slot(const int p[4][3], i64 L) {
    i64 k[3];
    for (int a = 0; a < 3; ++a)
        k[a] = eri_axis_key(p[0][a] - p[1][a], p[2][a] - p[3][a], (p[0][a] + p[1][a]) - (p[2][a] + p[3][a]), L);
    if (k[0] > k[1]) { i64 t = k[0]; k[0] = k[1]; k[1] = t; }
    if (k[1] > k[2]) { i64 t = k[1]; k[1] = k[2]; k[2] = t; }
    if (k[0] > k[1]) { i64 t = k[0]; k[0] = k[1]; k[1] = t; }
    return tetra_index(k[0], k[1], k[2]);
}

__device__ inline void eri_points(const SymGrid& G, i64 idx, int p[4][3]) {
    const i64 l = idx % G.N;
    idx /= G.N;
    const i64 k = idx % G.N;
    idx /= G.N;
    const i64 j = idx % G.N;
    point_of(G, idx / G.N, p[0]);
    point_of(G, j, p[1]);
    point_of(G, k, p[2]);
    point_of(G, l, p[3]);
}

// bad = 1 unless every index is canonical and the list increases strictly
__global__ void k_check_complete(SymGrid G, const int64_t* __restrict__ idx, i64 m, int* __restrict__ bad) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    const i64 v = idx[n];
    if (v < 0 || v / (G.N * G.N) >= G.N * G.N || (n + 1 < m && v >= idx[n + 1])) {
        atomicOr(bad, 1);
        return;
    }
    int p[4][3], bias[3];
    eri_points(G, v, p);
    centre_points<4>(p, bias);
    if (orbit_min_quad(G, p, bias) != v) atomicOr(bad, 1);
}

__global__ void k_key_table(SymGrid G, const int64_t* __restrict__ idx, const double* __restrict__ val, i64 m,
                            double* __restrict__ table) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    int p[4][3];
    eri_points(G, idx[n], p);
    table[eri_key_slot(p, G.L)] = val[n];
}

// rows [row0, row0 + nrows) of the (ij) x (kl) flattening of the dense grid D,
// from the key table of the sparse grid (range L)
__global__ void k_fill_eri_rows_keyed(DenseGrid D, const double* __restrict__ table, i64 L, i64 row0, i64 nrows,
                                      double* __restrict__ out) {
    const i64 N2 = D.N * D.N;
    const i64 total = nrows * N2;
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
        const i64 r = row0 + e / N2, kl = e % N2;
        int p[4][3];
        dense_point(D, r / D.N, p[0]);
        dense_point(D, r % D.N, p[1]);
        dense_point(D, kl / D.N, p[2]);
        dense_point(D, kl % D.N, p[3]);
        out[e] = table[eri_key_slot(p, L)];
    }
}

// points of a dense grid (x-major), for the slab fill
__global__ void k_dense_points(DenseGrid D, short4* __restrict__ pt) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= D.N) return;
    int p[3];
    dense_point(D, n, p);
    pt[n] = make_short4((short)p[0], (short)p[1], (short)p[2], 0);
}

// slab i of the (i j k l) tensor, S[(j N + k) N + l] = V[i j k l], its first
// `total` entries (rows j < total / N^2), from the key table (range L) of a
// complete list: 32-bit index arithmetic (N^3 < 2^32), the points from a
// table, 32-bit axis keys, one entry per thread
__global__ void __launch_bounds__(256) k_fill_slab_keyed(const short4* __restrict__ pt, uint32_t N, int L, short4 pi,
                                                         const double* __restrict__ table, uint32_t total,
                                                         double* __restrict__ S) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const uint32_t row = e / N, l = e - row * N, j = row / N, k = row - j * N;
        const short4 pj = pt[j], pk = pt[k], pl = pt[l];
        int a = eri_axis_key32(pi.x - pj.x, pk.x - pl.x, (pi.x + pj.x) - (pk.x + pl.x), L);
        int b = eri_axis_key32(pi.y - pj.y, pk.y - pl.y, (pi.y + pj.y) - (pk.y + pl.y), L);
        int c = eri_axis_key32(pi.z - pj.z, pk.z - pl.z, (pi.z + pj.z) - (pk.z + pl.z), L);
        if (a > b) { const int t = a; a = b; b = t; }
        if (b > c) { const int t = b; b = c; c = t; }
        if (a > b) { const int t = a; a = b; b = t; }
        S[e] = table[tetra_index32(a, b, c)];
    }
}

// A1[(j k)][s] = sum_l U[k][l] B[l][s] for slab i of a complete list, where U
// is the upper triangle (l >= k) of the symmetric V[i j k .] with its diagonal
// halved, so that B^T V[i j] B = Y + Y^T for Y = B^T A1[j]: half of the
// entries are generated.  The slab is never written out: each A element is
// computed from the key table as the tile is staged (K-major A tiles: a
// thread keeps its row (j, k) and walks l), B (the basis, at most 32 columns)
// read row-major.  A row tile (rows of one j) starts its K loop at the chunk
// of its smallest k, the elements below each row's k staged as zeros.
//
// One launch covers the pairs g0 <= g < g1 of the packed order
// g = i (i + 1) / 2 + j (j <= i), several slabs at once: slab by slab, the
// launches of the small slabs (a few tiles) left most of the GPU idle and
// every launch ended on a partial wave.  Rows of pair g are
// A1[(g - g0) N + k].
struct KeyedSlabOp {
    static constexpr bool A_KMAJOR = true, B_KMAJOR = false;
    static constexpr int BN = 32;
    const short4* pt;  // points of the grid
    const double* table;
    const double* basis;  // N x M row-major
    double* C;            // (g1 - g0) N x M row-major
    int N, L, M;
    int g0, g1;  // packed pairs (i, j <= i) of this launch
    struct Block {
        int mvalid, nvalid, nk;
        int m0, kc0;
        int j, k0;
        short4 pi;
    };
    struct AState {
        int d[3], s[3], k[3];  // pi - pj, pi + pj, pk per axis of this thread's row
        int kr;                // the row's k
        bool ok;
    };
    struct BState {};
    // row tiles never straddle two pairs: tile t holds rows (k0 .. k0 + 63) of
    // pair g = g0 + t / tpj, k0 = 64 (t % tpj), tpj = ceil(N / 64) tiles per pair
    __device__ bool begin(Block& b) const {
        const int tpj = (N + DM_BM - 1) / DM_BM, t = (int)(blockIdx.x / tpj);
        const int g = g0 + t;
        if (g >= g1) return false;
        // i = the largest integer with i (i + 1) / 2 <= g
        int i = (int)((sqrt(8.0 * (double)g + 1.0) - 1.0) * 0.5);
        while ((i64)(i + 1) * (i + 2) / 2 <= g) ++i;
        while ((i64)i * (i + 1) / 2 > g) --i;
        b.j = g - i * (i + 1) / 2;
        b.pi = pt[i];
        b.k0 = (blockIdx.x - t * tpj) * DM_BM;
        b.m0 = t * N + b.k0;
        b.mvalid = min(DM_BM, N - b.k0);
        if (b.mvalid <= 0) return false;
        b.kc0 = b.k0 / DM_BK;  // l >= k >= k0: the chunks below are zero
        b.nvalid = min(BN, M);
        b.nk = (N + DM_BK - 1) / DM_BK - b.kc0;
        return true;
    }
    __device__ void a_init(const Block& b, AState& st) const {
        const int r = dm_kmajor_row(threadIdx.x);
        st.ok = r < b.mvalid;
        const int k = st.ok ? b.k0 + r : 0;
        const short4 pi = b.pi, pj = pt[b.j], pk = pt[k];
        st.d[0] = pi.x - pj.x, st.d[1] = pi.y - pj.y, st.d[2] = pi.z - pj.z;
        st.s[0] = pi.x + pj.x, st.s[1] = pi.y + pj.y, st.s[2] = pi.z + pj.z;
        st.k[0] = pk.x, st.k[1] = pk.y, st.k[2] = pk.z;
        st.kr = k;
    }
    __device__ void a_issue(const Block& b, AState& st, int kc, double* tile) const {
        const int r = dm_kmajor_row(threadIdx.x);
#pragma unroll
        for (int q = 0; q < DM_ELEMS; ++q) {
            const int kq = dm_kmajor_k(threadIdx.x, q), l = (b.kc0 + kc) * DM_BK + kq;
            const bool v = st.ok && l < N && l >= st.kr;
            const double* src = table;
            if (v) {
                const short4 pl = pt[l];
                int a = eri_axis_key32(st.d[0], st.k[0] - pl.x, st.s[0] - (st.k[0] + pl.x), L);
                int c = eri_axis_key32(st.d[1], st.k[1] - pl.y, st.s[1] - (st.k[1] + pl.y), L);
                int e = eri_axis_key32(st.d[2], st.k[2] - pl.z, st.s[2] - (st.k[2] + pl.z), L);
                if (a > c) { const int t = a; a = c; c = t; }
                if (c > e) { const int t = c; c = e; e = t; }
                if (a > c) { const int t = a; a = c; c = t; }
                src = table + tetra_index32(a, c, e);
            }
            dm_cp8(tile + dm_kmajor_at(r, kq), src, v);
        }
    }
    // the diagonal element of the row, halved once it has landed
    static constexpr bool A_LANDED = true;
    __device__ void a_landed(const Block& b, AState& st, int kc, double* tile) const {
        const int r = dm_kmajor_row(threadIdx.x), kq = st.kr - (b.kc0 + kc) * DM_BK;
        if (!st.ok || kq < 0 || kq >= DM_BK || ((kq - (threadIdx.x >> 6)) & 1)) return;  // not this thread's element
        tile[dm_kmajor_at(r, kq)] *= 0.5;
    }
    __device__ void b_init(const Block&, BState&) const {}
    __device__ void b_issue(const Block& b, BState&, int kc, double* tile) const {
#pragma unroll
        for (int q = 0; q < BN * DM_BK / DM_THREADS; ++q) {
            const int n = dm_rowmajor_row(threadIdx.x, q), kq = dm_rowmajor_k(threadIdx.x);
            const int l = (b.kc0 + kc) * DM_BK + kq;
            const bool v = n < b.nvalid && l < N;
            dm_cp8(tile + dm_rowmajor_at(n, kq), v ? basis + (i64)l * M + n : basis, v);
        }
    }
    __device__ void store(const Block& b, int m, int n, double v0, double v1) const {
        if (m >= b.mvalid) return;
        double* c = C + (i64)(b.m0 + m) * M + n;
        if (n < b.nvalid) c[0] = v0;
        if (n + 1 < b.nvalid) c[1] = v1;
    }
};

// 48 x N permutation tables: perm[g][i] = linear index of O_h element g applied to point i
__global__ void k_grid_perms(SymGrid G, int64_t* __restrict__ perm) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 48 * G.N) return;
    const int g = (int)(t / G.N);
    const i64 i = t % G.N;
    int p[3], q[3];
    point_of(G, i, p);
    oh_apply(g, p, q);
    perm[t] = lin3(G, q);
}

// ---------------------------------------------------------------------------
// FP64 strided batched GEMM: C[b] = A[b] * B[b] (+ C[b] when accumulate).
// Element (i, k) of A sits at A + b*sa + i*ar + k*ac (likewise B, C), so
// transposed operands are expressed through strides.  The FP64 tensor-core
// tiles of dmma.cuh; each operand tile is staged in the shared-memory layout
// whose thread mapping reads its unit-stride direction contiguously.
struct MatView {
    const double* p;
    i64 sb, r, c;
};

// BN_ = 32: products of at most 32 columns (B read row-major), whose 64-column
// tiles would leave half the warps without columns
template <bool AK, bool BK, int BN_ = DM_BN>
struct StridedOp {
    static constexpr bool A_KMAJOR = AK, B_KMAJOR = BK;
    static constexpr int BN = BN_;
    static_assert(BN == DM_BN || (BN == 32 && !BK), "32-column tiles read B row-major");
    int M, N, K;
    MatView A, B;
    double* C;
    i64 csb, cr, cc;
    int accumulate;
    struct Block {
        int mvalid, nvalid, nk;
        int m0, n0;
        const double* a;
        const double* b;
        double* c;
    };
    struct AState {};
    struct BState {};
    __device__ bool begin(Block& b) const {
        b.m0 = blockIdx.y * DM_BM;
        b.n0 = blockIdx.x * BN;
        b.mvalid = min(DM_BM, M - b.m0);
        b.nvalid = min(BN, N - b.n0);
        b.nk = (K + DM_BK - 1) / DM_BK;
        b.a = A.p + (i64)blockIdx.z * A.sb + (i64)b.m0 * A.r;
        b.b = B.p + (i64)blockIdx.z * B.sb + (i64)b.n0 * B.c;
        b.c = C + (i64)blockIdx.z * csb + (i64)b.m0 * cr + (i64)b.n0 * cc;
        return b.mvalid > 0 && b.nvalid > 0;
    }
    __device__ void a_init(const Block&, AState&) const {}
    __device__ void b_init(const Block&, BState&) const {}
    __device__ void a_issue(const Block& b, AState&, int kc, double* tile) const {
#pragma unroll
        for (int q = 0; q < DM_ELEMS; ++q) {
            const int r = AK ? dm_kmajor_row(threadIdx.x) : dm_rowmajor_row(threadIdx.x, q);
            const int k = AK ? dm_kmajor_k(threadIdx.x, q) : dm_rowmajor_k(threadIdx.x);
            const int kk = kc * DM_BK + k;
            const bool v = r < b.mvalid && kk < K;
            dm_cp8(tile + (AK ? dm_kmajor_at(r, k) : dm_rowmajor_at(r, k)), v ? b.a + r * A.r + kk * A.c : A.p, v);
        }
    }
    __device__ void b_issue(const Block& b, BState&, int kc, double* tile) const {
#pragma unroll
        for (int q = 0; q < BN * DM_BK / DM_THREADS; ++q) {
            const int r = BK ? dm_kmajor_row(threadIdx.x) : dm_rowmajor_row(threadIdx.x, q);
            const int k = BK ? dm_kmajor_k(threadIdx.x, q) : dm_rowmajor_k(threadIdx.x);
            const int kk = kc * DM_BK + k;
            const bool v = r < b.nvalid && kk < K;
            dm_cp8(tile + (BK ? dm_kmajor_at(r, k) : dm_rowmajor_at(r, k)), v ? b.b + r * B.c + kk * B.r : B.p, v);
        }
    }
    __device__ void store(const Block& b, int m, int n, double v0, double v1) const {
        if (m >= b.mvalid) return;
        double* c = b.c + (i64)m * cr + (i64)n * cc;
        if (n < b.nvalid) c[0] = accumulate ? c[0] + v0 : v0;
        if (n + 1 < b.nvalid) c[cc] = accumulate ? c[cc] + v1 : v1;
    }
};

static void dgemm(int M, int N, int K, MatView A, MatView B, double* C, i64 csb, i64 cr, i64 cc, int batch,
                  bool accumulate, cudaStream_t s) {
    if (M <= 0 || N <= 0 || batch <= 0) return;
    const dim3 grid((N + DM_BN - 1) / DM_BN, (M + DM_BM - 1) / DM_BM, batch);
    // stage an operand K-major when its row index is the unit-stride direction
    const bool ak = A.r == 1 && A.c != 1, bk = B.c == 1 && B.r != 1;
    const int acc = accumulate ? 1 : 0;
    if (N <= 32) {
        // one 32-column tile (the ERI projection's products onto 32 orbitals);
        // B is small and read row-major
        const dim3 g32(1, grid.y, batch);
        if (ak)
            dmma_launch(StridedOp<true, false, 32>{M, N, K, A, B, C, csb, cr, cc, acc}, g32, s);
        else
            dmma_launch(StridedOp<false, false, 32>{M, N, K, A, B, C, csb, cr, cc, acc}, g32, s);
        return;
    }
    if (ak && bk)
        dmma_launch(StridedOp<true, true>{M, N, K, A, B, C, csb, cr, cc, acc}, grid, s);
    else if (ak)
        dmma_launch(StridedOp<true, false>{M, N, K, A, B, C, csb, cr, cc, acc}, grid, s);
    else if (bk)
        dmma_launch(StridedOp<false, true>{M, N, K, A, B, C, csb, cr, cc, acc}, grid, s);
    else
        dmma_launch(StridedOp<false, false>{M, N, K, A, B, C, csb, cr, cc, acc}, grid, s);
}

void dgemm_prepare() {
    dmma_prepare<StridedOp<true, true>>();
    dmma_prepare<StridedOp<true, false>>();
    dmma_prepare<StridedOp<false, true>>();
    dmma_prepare<StridedOp<false, false>>();
    dmma_prepare<StridedOp<true, false, 32>>();
    dmma_prepare<StridedOp<false, false, 32>>();
}

void dgemm_strided(int M, int N, int K, const double* A, i64 asb, i64 ar, i64 ac, const double* B, i64 bsb, i64 br,
                   i64 bc, double* C, i64 csb, i64 cr, i64 cc, int batch, bool accumulate, cudaStream_t s) {
    dgemm(M, N, K, MatView{A, asb, ar, ac}, MatView{B, bsb, br, bc}, C, csb, cr, cc, batch, accumulate, s);
}

// ---------------------------------------------------------------------------
static SymGrid sym_of(const GridDesc& g) {
    const i64 e = symmetric_extent(g);
    if (e < 0) fail(GLI_ERR_ARGUMENT, "sparse grid is not rotationally symmetric");
    SymGrid G;
    G.e = (int)e;
    G.L = (int)(2 * e + 1);
    G.N = (i64)G.L * G.L * G.L;
    return G;
}

static DenseGrid dense_of(const GridDesc& g) {
    DenseGrid D;
    for (int a = 0; a < 3; ++a) {
        D.istart[a] = (int)g.istart[a];
        D.num[a] = (int)g.num[a];
    }
    D.N = g.points();
    return D;
}

// every dense point must stay inside the sparse grid after the box-centre
// translation: the dense grid's largest |coordinate| may not exceed e
// (python/pymodule.c:876-888 enforces the same before calling the C routine)
static void check_extent(const GridDesc& dense, const SymGrid& G) {
    i64 ext = 0;
    for (int a = 0; a < 3; ++a) {
        const i64 lo = dense.istart[a], hi = dense.istart[a] + dense.num[a] - 1;
        ext = std::max(ext, std::max(lo < 0 ? -lo : lo, hi < 0 ? -hi : hi));
    }
    if (ext > G.e)
        fail(GLI_ERR_ARGUMENT, "sparse grid too small to fill all values for the provided grid (extent %lld)",
             (long long)ext);
}

static unsigned grid_for(i64 work, int per_block = 256) {
    const Context& c = context();
    const i64 want = (work + per_block - 1) / per_block;
    const i64 cap = (i64)c.num_sms * 32;
    return (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
}

// The canonical ERI class list of a symmetric grid of extent e (the
// enumeration, sorted), kept on the device once made: a list is the complete
// canonical list exactly when it equals this one.  Lists above
// ENUM_KEEP_CLASSES are not kept (their count is): the per-class orbit test
// decides for them.
constexpr i64 ENUM_KEEP_CLASSES = (i64)1 << 27;  // 1 GB of indices
struct CanonicalList {
    i64 count = 0;
    int64_t* d = nullptr;  // null: not kept
};
static CanonicalList canonical_eri_list(const GridDesc& g, i64 e, cudaStream_t s) {
    static std::mutex mu;
    static std::map<std::pair<int, i64>, CanonicalList> cache;  // (device, extent)
    int dev = 0;
    GLI_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find({dev, e});
        if (it != cache.end()) return it->second;
    }
    int64_t* d = nullptr;
    CanonicalList c;
    c.count = enumerate_device(1, g, &d, s);
    if (d && c.count <= ENUM_KEEP_CLASSES) {
        c.d = d;  // kept for the process (one list per device and extent)
    } else if (d) {
        GLI_CUDA(cudaFreeAsync(d, s));
    }
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({dev, e});
    if (it != cache.end()) {  // another thread made it meanwhile
        if (c.d) GLI_CUDA(cudaFreeAsync(c.d, s));
        return it->second;
    }
    cache[{dev, e}] = c;
    return c;
}

// bad = 1 where the list differs from the canonical list
__global__ void k_equal_lists(const int64_t* __restrict__ a, const int64_t* __restrict__ b, i64 m,
                              int* __restrict__ bad) {
    bool differ = false;
    for (i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x; n < m; n += (i64)gridDim.x * blockDim.x)
        differ = differ || a[n] != b[n];
    if (differ) atomicOr(bad, 1);
}

// Key table of a complete ERI class list, or an empty buffer when the list is
// not the complete canonical list of its grid (then entries are looked up).
struct KeyTable {
    DevBuf<double> t;
    bool ok = false;
};

static void build_key_table(const SymGrid& G, const GridDesc& g, const int64_t* d_idx, const double* d_val, i64 m,
                            KeyTable& kt, cudaStream_t s) {
    kt.ok = false;
    if (m <= 0) return;
    const i64 L = G.L;
    const i64 nk = L * (L + 1) / 2 * (2 * L - 1);
    const i64 slots = nk * (nk + 1) * (nk + 2) / 6;
    if (slots > ((i64)1 << 29)) return;  // above 4 GB: keep the lookups
    const CanonicalList canon = canonical_eri_list(g, G.e, s);
    if (canon.count != m) return;
    DevBuf<int> bad(1, s);
    bad.zero();
    if (canon.d)
        k_equal_lists<<<grid_for(m), 256, 0, s>>>(d_idx, canon.d, m, bad.p);
    else
        k_check_complete<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(G, d_idx, m, bad.p);
    GLI_CHECK_LAUNCH();
    int h = 0;
    GLI_CUDA(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    if (h) return;
    kt.t.alloc(slots, s);
    k_key_table<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(G, d_idx, d_val, m, kt.t.p);
    GLI_CHECK_LAUNCH();
    kt.ok = true;
}

void fill_dense_device(int kind, const GridDesc& sparse, const int64_t* d_idx, const double* d_val, i64 m,
                       const GridDesc& dense, double* d_out, cudaStream_t s) {
    const SymGrid G = sym_of(sparse);
    check_extent(dense, G);
    const DenseGrid D = dense_of(dense);
    if (kind == 0) {
        k_fill_erida<<<grid_for(D.N * D.N), 256, 0, s>>>(G, D, d_idx, d_val, m, d_out);
    } else {
        const i64 rows = D.N * D.N;
        KeyTable kt;
        build_key_table(G, sparse, d_idx, d_val, m, kt, s);
        if (kt.ok)
            k_fill_eri_rows_keyed<<<grid_for(rows * rows), 256, 0, s>>>(D, kt.t.p, G.L, 0, rows, d_out);
        else
            k_fill_eri_rows<<<grid_for(rows * rows), 256, 0, s>>>(G, D, d_idx, d_val, m, 0, rows, d_out);
        GLI_CHECK_LAUNCH();
        // the key table is released on the stream after the fill
        return;
    }
    GLI_CHECK_LAUNCH();
}

void grid_perms_device(const GridDesc& g, int64_t* d_perm, cudaStream_t s) {
    const SymGrid G = sym_of(g);
    k_grid_perms<<<(unsigned)((48 * G.N + 255) / 256), 256, 0, s>>>(G, d_perm);
    GLI_CHECK_LAUNCH();
}

// ret[(i k), s] = sum_{j l} V[i j k l] states[(j l), s], rows expanded in chunks
void apply_eri_device(const GridDesc& g, const int64_t* d_idx, const double* d_val, i64 m, const double* d_states,
                      i64 ns, double* d_ret, cudaStream_t s) {
    const SymGrid G = sym_of(g);
    const DenseGrid D = dense_of(g);
    const i64 N = D.N, N2 = N * N;
    // chunk of rows i of V[i][j][k][l]: for one i, the (j, k, l) block is N^3
    const i64 per_i = N2 * N;
    i64 ci = (i64)(256 << 20) / (per_i * 8);
    if (ci < 1) ci = 1;
    if (ci > N) ci = N;
    DevBuf<double> V(ci * per_i, s);
    KeyTable kt;
    build_key_table(G, g, d_idx, d_val, m, kt, s);
    for (i64 i0 = 0; i0 < N; i0 += ci) {
        const i64 ni = std::min(ci, N - i0);
        // V rows (i, j) for i in [i0, i0 + ni): layout [i][j][k][l]
        if (kt.ok)
            k_fill_eri_rows_keyed<<<grid_for(ni * per_i), 256, 0, s>>>(D, kt.t.p, G.L, i0 * N, ni * N, V.p);
        else
            k_fill_eri_rows<<<grid_for(ni * per_i), 256, 0, s>>>(G, D, d_idx, d_val, m, i0 * N, ni * N, V.p);
        GLI_CHECK_LAUNCH();
        // for each (i, k): ret[i*N + k][s] = sum_j sum_l V[i][j][k][l] states[j*N + l][s]
        // batch over i (ni) and j-contributions accumulate: for fixed i, j:
        //   C[k][s] += V[i][j][k][:] (N x N, row k) * states[j*N : j*N+N][s] (N x ns)
        for (i64 j = 0; j < N; ++j) {
            MatView A{V.p + j * N2, per_i, N, 1};           // batch i: rows k, cols l
            MatView B{d_states + j * N * ns, 0, ns, 1};       // rows l, cols s
            dgemm((int)N, (int)ns, (int)N, A, B, d_ret + i0 * N * ns, N * ns, ns, 1, (int)ni, j > 0, s);
        }
    }
}

// E[p,q,r,s] = sum V[i j k l] B[i p] B[j q] B[k r] B[l s] (chemists' order).
// kind 1: V = ERI tensor; kind 0: V[i i j j] = ERIDA matrix (Khatri-Rao form).
// W[j][i] = W[i][j] for j > i (blocks of `mm` doubles of an n x n array of blocks)
__global__ void k_mirror_pairs(double* __restrict__ W, i64 n, i64 mm) {
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < n * n * mm; e += (i64)gridDim.x * blockDim.x) {
        const i64 blk = e / mm, r = e - blk * mm, i = blk / n, j = blk - i * n;
        if (j > i) W[e] = W[(j * n + i) * mm + r];
    }
}

// W[i][j] = Y + Y^T for the M x M blocks Y (M <= 32) of the pairs j <= i
// (packed: Y[i (i + 1) / 2 + j]), and W[j][i] = W[i][j]: one block per pair
// (blockIdx.y = i, blockIdx.x = j), Y read once into shared memory, the sums
// written row by row (coalesced)
__global__ void __launch_bounds__(256) k_symmetrize_pairs(const double* __restrict__ Y, double* __restrict__ W, i64 n,
                                                          int M) {
    __shared__ double y[32 * 33];
    const i64 i = blockIdx.y, j = blockIdx.x;
    if (j > i) return;
    const i64 mm = (i64)M * M;
    const double* yg = Y + (i * (i + 1) / 2 + j) * mm;
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) y[(e / M) * 33 + e % M] = yg[e];
    __syncthreads();
    double* blk = W + (i * n + j) * mm;
    double* mir = W + (j * n + i) * mm;
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) {
        const int r = e / M, c = e - r * M;
        const double v = y[r * 33 + c] + y[c * 33 + r];
        blk[e] = v;
        if (j < i) mir[e] = v;
    }
}

void project_device(int kind, const GridDesc& g, const int64_t* d_idx, const double* d_val, i64 m,
                    const double* d_basis, i64 M, double* d_out, cudaStream_t s) {
    const SymGrid G = sym_of(g);
    const DenseGrid D = dense_of(g);
    const i64 N = D.N, N2 = N * N;
    if (kind == 0) {
        // dense ERIDA matrix V (N x N), then E[p,q,r,s] = sum_ij B[i p] B[i q] V[i j] B[j r] B[j s]
        DevBuf<double> V(N2, s), K(N * M * M, s), X(N * M * M, s);
        k_fill_erida<<<grid_for(N2), 256, 0, s>>>(G, D, d_idx, d_val, m, V.p);
        GLI_CHECK_LAUNCH();
        // K[j][(r s)] = B[j r] B[j s]: a batched outer product as a GEMM with K = 1
        dgemm((int)M, (int)M, 1, MatView{d_basis, M, 1, 1}, MatView{d_basis, M, 1, 1}, K.p, M * M, M, 1, (int)N,
              false, s);
        // X[i][(r s)] = sum_j V[i j] K[j][(r s)]
        dgemm((int)N, (int)(M * M), (int)N, MatView{V.p, 0, N, 1}, MatView{K.p, 0, M * M, 1}, X.p, 0, M * M, 1, 1,
              false, s);
        // E[(p q)][(r s)] = sum_i K[i][(p q)] X[i][(r s)]
        dgemm((int)(M * M), (int)(M * M), (int)N, MatView{K.p, 0, 1, M * M}, MatView{X.p, 0, M * M, 1}, d_out, 0,
              M * M, 1, 1, false, s);
        return;
    }
    // slab by slab over i: S[j][k][l] = V[i j k l], filled from the key table
    // of a complete list (key arithmetic and one table read per entry) or by
    // canonical lookups, then contracted on the FP64 tensor-core GEMM (ERI
    // 7^3 onto 32 orbitals: the slab as FP64-level int8 slices on the tcgen05
    // tensor cores took 0.44 s, dominated by writing the slices)
    KeyTable kt;
    build_key_table(G, g, d_idx, d_val, m, kt, s);
    const bool slab32 = kt.ok && N2 * N < ((i64)1 << 32);
    DevBuf<short4> pt;
    std::vector<short4> hpt;
    // Rows of the basis that are zero contribute nothing: with the key table
    // (entries computed from point coordinates) the contraction runs over the
    // points whose rows are nonzero only -- a basis on a sub-grid of the sparse
    // grid (the 6^3 orbitals of a 7^3 class list: (216/343)^4 of the work).
    i64 Nx = N;
    const double* bx = d_basis;
    DevBuf<double> bcomp;
    if (slab32) {
        pt.alloc(N, s);
        k_dense_points<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(D, pt.p);
        GLI_CHECK_LAUNCH();
        hpt.resize(N);
        std::vector<double> hb((size_t)(N * M));
        GLI_CUDA(cudaMemcpyAsync(hpt.data(), pt.p, N * sizeof(short4), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaMemcpyAsync(hb.data(), d_basis, N * M * sizeof(double), cudaMemcpyDeviceToHost, s));
        GLI_CUDA(cudaStreamSynchronize(s));
        std::vector<i64> act;
        for (i64 i = 0; i < N; ++i)
            for (i64 c = 0; c < M; ++c)
                if (hb[(size_t)(i * M + c)] != 0.0) {
                    act.push_back(i);
                    break;
                }
        if (act.empty()) {
            GLI_CUDA(cudaMemsetAsync(d_out, 0, M * M * M * M * sizeof(double), s));
            return;
        }
        if ((i64)act.size() < N) {
            Nx = (i64)act.size();
            std::vector<short4> hp((size_t)Nx);
            std::vector<double> hbc((size_t)(Nx * M));
            for (i64 a = 0; a < Nx; ++a) {
                hp[(size_t)a] = hpt[(size_t)act[(size_t)a]];
                for (i64 c = 0; c < M; ++c) hbc[(size_t)(a * M + c)] = hb[(size_t)(act[(size_t)a] * M + c)];
            }
            hpt.swap(hp);
            GLI_CUDA(cudaMemcpyAsync(pt.p, hpt.data(), Nx * sizeof(short4), cudaMemcpyHostToDevice, s));
            bcomp.alloc(Nx * M, s);
            GLI_CUDA(cudaMemcpyAsync(bcomp.p, hbc.data(), Nx * M * sizeof(double), cudaMemcpyHostToDevice, s));
            GLI_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
            bx = bcomp.p;
        }
    }
    // V[i j k l] = V[j i k l]: the two first contractions run over the pairs
    // j <= i only, W[i][j] = B^T V[i j] B (M x M), and W[j][i] = W[i][j] is
    // copied; then A3[i] = B^T W[i] and E = B^T A3.  The generated entries and
    // the dominant first contraction are halved.
    const i64 Nx2 = Nx * Nx, MM = M * M;
    DevBuf<double> W(Nx2 * MM, s), A3(Nx * MM * M, s);
    // the first contraction with its slab computed as the GEMM stages it (at
    // most 32 orbitals), or from a filled slab
    const bool fused = slab32 && M <= 32;
    if (fused) {
        // The pairs (i, j <= i) in packed order g = i (i + 1) / 2 + j, split
        // evenly over launches of as many pairs as a 1 GB A1 holds (at least
        // Nx, at most 65,535: the batched GEMM's grid.z): the first
        // contraction A1[g] = U[i j] B, then Y[g] = B^T A1[g], one batched GEMM
        // per launch (the 216-point projection: two launches of each instead
        // of one per slab).
        const i64 pairs = Nx * (Nx + 1) / 2, tpj = (Nx + DM_BM - 1) / DM_BM;
        const i64 cap = std::min<i64>(65535, std::max<i64>(Nx, ((i64)1 << 30) / (Nx * M * (i64)sizeof(double))));
        const i64 launches = (pairs + cap - 1) / cap, per = (pairs + launches - 1) / launches;
        if (pairs >= ((i64)1 << 31) || per * tpj >= ((i64)1 << 31) || per * Nx * M >= ((i64)1 << 31))
            fail(GLI_ERR_LIMIT, "projection over %lld points exceeds the slab launch range", (long long)Nx);
        DevBuf<double> A1(per * Nx * M, s), Y(pairs * MM, s);
        for (i64 g0 = 0; g0 < pairs; g0 += per) {
            const i64 g1 = std::min(pairs, g0 + per);
            dmma_launch(KeyedSlabOp{pt.p, kt.t.p, bx, A1.p, (int)Nx, (int)G.L, (int)M, (int)g0, (int)g1},
                        dim3((unsigned)((g1 - g0) * tpj)), s);
            // Y[g] = B^T A1[g]   (batch g0 <= g < g1)
            dgemm((int)M, (int)M, (int)Nx, MatView{bx, 0, 1, M}, MatView{A1.p, Nx * M, M, 1}, Y.p + g0 * MM, MM, M, 1,
                  (int)(g1 - g0), false, s);
        }
        // W[i][j] = Y + Y^T, and the mirror W[j][i]
        k_symmetrize_pairs<<<dim3((unsigned)Nx, (unsigned)Nx), 256, 0, s>>>(Y.p, W.p, Nx, (int)M);
        GLI_CHECK_LAUNCH();
    } else {
        // slab by slab: S = V[i j k l] for j <= i filled, then contracted
        DevBuf<double> A1(Nx2 * M, s), S(Nx2 * Nx, s);
        for (i64 i = 0; i < Nx; ++i) {
            const i64 rows = (i + 1) * Nx;  // (j k) with j <= i
            if (slab32)
                k_fill_slab_keyed<<<grid_for(rows * Nx), 256, 0, s>>>(pt.p, (uint32_t)Nx, (int)G.L, hpt[i], kt.t.p,
                                                                      (uint32_t)(rows * Nx), S.p);
            else if (kt.ok)
                k_fill_eri_rows_keyed<<<grid_for(rows * Nx), 256, 0, s>>>(D, kt.t.p, G.L, i * N, i + 1, S.p);
            else
                k_fill_eri_rows<<<grid_for(rows * Nx), 256, 0, s>>>(G, D, d_idx, d_val, m, i * N, i + 1, S.p);
            GLI_CHECK_LAUNCH();
            // A1[(j k)][s] = sum_l S[(j k)][l] B[l][s]
            dgemm((int)rows, (int)M, (int)Nx, MatView{S.p, 0, Nx, 1}, MatView{bx, 0, M, 1}, A1.p, 0, M, 1, 1, false,
                  s);
            // W[i][j][r][s] = sum_k B[k][r] A1[j][k][s]   (batch j <= i)
            dgemm((int)M, (int)M, (int)Nx, MatView{bx, 0, 1, M}, MatView{A1.p, Nx * M, M, 1}, W.p + i * Nx * MM, MM,
                  M, 1, (int)(i + 1), false, s);
        }
        k_mirror_pairs<<<grid_for(Nx2 * MM), 256, 0, s>>>(W.p, Nx, MM);
        GLI_CHECK_LAUNCH();
    }
    // A3[i][q][(r s)] = sum_j B[j][q] W[i][j][(r s)]   (batch i)
    dgemm((int)M, (int)MM, (int)Nx, MatView{bx, 0, 1, M}, MatView{W.p, Nx * MM, MM, 1}, A3.p, MM * M, MM, 1,
          (int)Nx, false, s);
    // E[p][(q r s)] = sum_i B[i][p] A3[i][(q r s)]
    dgemm((int)M, (int)(MM * M), (int)Nx, MatView{bx, 0, 1, M}, MatView{A3.p, 0, MM * M, 1}, d_out, 0, MM * M, 1, 1,
          false, s);
}

}  // namespace gli
