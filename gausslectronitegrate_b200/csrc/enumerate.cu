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
// Ordering without a sort: candidates are generated so that the flat candidate
// order equals ascending index order -- for ERIDA one thread per i scans its j
// slots in ascending j; for ERI one thread per (i, j, k) scans l ascending --
// then a count pass, an exclusive scan and a write pass place each thread's
// survivors at its offset.  The output is sorted by construction.
#include "symmetry.cuh"

namespace gli {

// ---------------------------------------------------------------------------
// ERIDA: one thread per i; partner coordinates j_a = -i_a - 1 + t_a, t_a in {0,1,2}
// (doubled box centre t_a - 1), ascending in (t_x, t_y, t_z) = ascending j.
template <bool WRITE>
__global__ void k_enum_erida(SymGrid G, uint32_t* __restrict__ counts, const uint64_t* __restrict__ offsets,
                             int64_t* __restrict__ out) {
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G.N) return;
    int p[2][3];
    point_of(G, i, p[0]);
    uint64_t w = WRITE ? offsets[i] : 0;
    uint32_t c = 0;
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
                const int bias[3] = {tx - 1, ty - 1, tz - 1};
                const i64 idx = i * G.N + lin3(G, p[1]);
                if (canonical_pair(G, p, bias, idx)) {
                    if (WRITE) out[w++] = idx;
                    ++c;
                }
            }
        }
    }
    if (!WRITE) counts[i] = c;
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

template <bool WRITE>
__global__ void k_enum_eri(SymGrid G, uint32_t* __restrict__ counts, const uint64_t* __restrict__ offsets,
                           int64_t* __restrict__ out) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 N3 = G.N * G.N * G.N;
    if (t >= N3) return;
    const i64 i = t / (G.N * G.N), j = (t / G.N) % G.N, k = t % G.N;
    int p[4][3];
    point_of(G, i, p[0]);
    point_of(G, j, p[1]);
    point_of(G, k, p[2]);
    uint32_t c = 0;
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
        uint64_t w = WRITE ? offsets[t] : 0;
        const i64 base = ((i * G.N + j) * G.N + k) * G.N;
        for (int ax = 0; ax < nx; ++ax) {
            p[3][0] = sx[ax];
            const int bx = min(lo[0], p[3][0]) + max(hi[0], p[3][0]);
            for (int ay = 0; ay < ny; ++ay) {
                p[3][1] = sy[ay];
                const int by = min(lo[1], p[3][1]) + max(hi[1], p[3][1]);
                for (int az = 0; az < nz; ++az) {
                    p[3][2] = sz[az];
                    const int bz = min(lo[2], p[3][2]) + max(hi[2], p[3][2]);
                    const int bias[3] = {bx, by, bz};
                    const i64 idx = base + lin3(G, p[3]);
                    if (canonical_quad(G, p, bias, idx)) {
                        if (WRITE) out[w++] = idx;
                        ++c;
                    }
                }
            }
        }
    }
    if (!WRITE) counts[t] = c;
}

i64 enumerate_device(int kind, const GridDesc& g, int64_t** d_out, cudaStream_t s) {
    const i64 e = symmetric_extent(g);
    if (e < 0) fail(GLI_ERR_ARGUMENT, "specified grid is not rotationally symmetric");
    SymGrid G;
    G.e = (int)e;
    G.L = (int)(2 * e + 1);
    G.N = (i64)G.L * G.L * G.L;
    if (kind == 1 && G.L > 63) fail(GLI_ERR_LIMIT, "ERI enumeration supports grids up to 63^3 (got %d^3)", G.L);
    if (kind == 0 && G.L > 1025) fail(GLI_ERR_LIMIT, "ERIDA enumeration supports grids up to 1025^3");
    const i64 slots = kind == 0 ? G.N : G.N * G.N * G.N;
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
