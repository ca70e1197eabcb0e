// Device-built tables: Gaussian-pair factors and products, folded lattice
// weights and the Coulomb lookup table.
//
// Reference counterparts:
//   factors         src/gausslet_factors.c:12-81   F_s[i+j] = sqrt(pi)/3 b_i b_j exp(-(0.5 (3s+i-j))^2)
//   ERI products    src/eri_integrals.c:46-110     P_kl[a-b] = sum F_k[a] F_l[b], trimmed at tol
//   ERIDA products  src/erida_integrals.c:44-100   P[i-j] = 2 pi/9 sum b_i b_j, trimmed at tol
//   Coulomb tables  src/eri_integrals.c:18-27,569-574 and src/erida_integrals.c:17-26,446-451
//
// The reference trims each vector to the outermost entries with |P| > tol and
// skips interior entries with |P| <= tol; zeroing every entry with |P| <= tol is
// the same selection, so the masked vectors below carry the truncation exactly.
//
// Symmetries used to fold the tables (all exact in real arithmetic):
//   F_{-s} = F_s and F_s[-m] = F_s[m] (swap i <-> j, b_{-j} = b_j), hence
//   P_{k,l} = P_{|k|,|l|} = P_{|l|,|k|} and P[-x] = P[x]; the lattice weight of a
//   key then depends only on |position|, so the three axis sums fold onto
//   positions u >= 0 and T is read at u^2 + v^2 + t^2.
#include <math.h>

#include <algorithm>
#include <list>
#include <vector>
#include <mutex>

#include "tables.cuh"

namespace gli {

__global__ void k_erida_products(const double* __restrict__ b, int nb, double tol, double* __restrict__ P,
                                 int* __restrict__ maxabs) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x - (nb - 1);
    if (s > nb - 1) return;
    const double prefac = 0.69813170079773183077;  // 2 pi / 9
    double acc = 0;
    for (int i = 0; i < nb; ++i) {
        const int j = i - s;
        if (j >= 0 && j < nb) acc += prefac * b[i] * b[j];
    }
    if (!(fabs(acc) > tol)) acc = 0;
    P[s + nb - 1] = acc;
    if (acc != 0) atomicMax(maxabs, s < 0 ? -s : s);
}

// F[s][m], s = 0..L-1, m = 0..2nb-2 (logical factor index m - (nb-1))
__global__ void k_factors(const double* __restrict__ b, int nb, int L, double* __restrict__ F) {
    const int nf = 2 * nb - 1;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (m >= nf) return;
    const double prefac = 0.590817950301838675766;  // sqrt(pi) / 3
    double acc = 0;
    const int ilo = m - (nb - 1) > 0 ? m - (nb - 1) : 0;
    const int ihi = m < nb - 1 ? m : nb - 1;
    for (int i = ilo; i <= ihi; ++i) {
        const int j = m - i;
        const double e = 0.5 * (double)(3 * s + (i - j));
        acc += prefac * b[i] * b[j] * exp(-e * e);
    }
    F[(i64)s * nf + m] = acc;
}

// Pr[pair][x + 2nb-2] for pairs (sa <= sb) in triangular order, masked at tol
__global__ void k_eri_products(const double* __restrict__ F, int nb, double tol, double* __restrict__ Pr,
                               int* __restrict__ maxabs) {
    const int nf = 2 * nb - 1;
    const int xl = 4 * nb - 3;
    const int xi = blockIdx.x * blockDim.x + threadIdx.x;
    const int pair = blockIdx.y;
    if (xi >= xl) return;
    int sb = 0;
    while ((sb + 1) * (sb + 2) / 2 <= pair) ++sb;
    const int sa = pair - sb * (sb + 1) / 2;
    const int x = xi - (2 * nb - 2);
    const double* fa = F + (i64)sa * nf;
    const double* fb = F + (i64)sb * nf;
    double acc = 0;
    const int alo = x > 0 ? x : 0;
    const int ahi = x < 0 ? nf - 1 + x : nf - 1;
    for (int a = alo; a <= ahi; ++a) acc += fa[a] * fb[a - x];
    if (!(fabs(acc) > tol)) acc = 0;
    Pr[(i64)pair * xl + xi] = acc;
    if (acc != 0) atomicMax(maxabs, x < 0 ? -x : x);
}

// W[key][m] = sum over u in {+m, -m} of the masked product at position u
__global__ void k_fold_weights(int kind, const double* __restrict__ P, int nb, int L, i64 nkeys, int U, int Up,
                               double* __restrict__ W) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const i64 key = blockIdx.y;
    if (m >= Up || key >= nkeys) return;
    double v = 0;
    if (m < U) {
        int centre;       // 3 * displacement (ERIDA) or 3 * |(i+j)-(k+l)| (ERI)
        const double* vec;
        int half;         // entries -half .. half
        if (kind == 0) {
            centre = 3 * (int)key;
            vec = P;
            half = nb - 1;
        } else {
            const int ncc = 2 * L - 1;
            const int tri = (int)(key / ncc);
            centre = 3 * (int)(key % ncc);
            vec = P + (i64)tri * (4 * nb - 3);
            half = 2 * nb - 2;
        }
        const int x1 = m - centre;
        if (x1 >= -half && x1 <= half) v += vec[x1 + half];
        if (m != 0) {
            const int x2 = -m - centre;
            if (x2 >= -half && x2 <= half) v += vec[x2 + half];
        }
    }
    W[key * Up + m] = v;
}

// T[n]: Coulomb interaction of two normalised Gaussians of width w at distance
// sqrt(n)/den, erf(dist / (sqrt2 w)) / dist, with limit sqrt(2/pi)/w at n = 0.
//   ERI   (kind 1): w = 1/3,       den = 6  ->  erf(sqrt(n)/(2 sqrt2)) * 6/sqrt(n)
//   ERIDA (kind 0): w = sqrt(2)/3, den = 3  ->  erf(sqrt(n)/2)        * 3/sqrt(n)
__global__ void k_coulomb_table(int kind, i64 n_entries, double* __restrict__ T) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_entries) return;
    double v;
    if (n == 0) {
        v = kind ? 2.3936536824085962 : 1.6925687506432689;  // 3 sqrt(2/pi), 3/sqrt(pi)
    } else {
        const double r = sqrt((double)n);
        v = kind ? erf(r * 0.35355339059327376220) * 6.0 / r : erf(r * 0.5) * 3.0 / r;
    }
    T[n] = v;
}

void factors_device(const double* d_b, int nb, int L, double* d_F, cudaStream_t s) {
    const int nf = 2 * nb - 1;
    k_factors<<<dim3((nf + 127) / 128, L), 128, 0, s>>>(d_b, nb, L, d_F);
    GLI_CHECK_LAUNCH();
}

// distinct s = u^2 + v^2 (u, v < U): mark, scan, list, and the U x U index
__global__ void k_mark_s(int U, uint32_t* __restrict__ mark) {
    const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (i64)U * U) return;
    const int u = (int)(e / U), v = (int)(e % U);
    mark[u * u + v * v] = 1;
}

__global__ void k_s_list(i64 n, const uint32_t* __restrict__ mark, const uint64_t* __restrict__ pos,
                         int* __restrict__ S) {
    const i64 s = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n && mark[s]) S[pos[s]] = (int)s;
}

__global__ void k_s_index(int U, const uint64_t* __restrict__ pos, int* __restrict__ sidx) {
    const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (i64)U * U) return;
    const int u = (int)(e / U), v = (int)(e % U);
    sidx[e] = (int)pos[u * u + v * v];
}

static void build_lattice_tables(int kind, const double* h_coeffs, i64 nb, i64 L, double tol, LatticeTables& t,
                                 cudaStream_t s) {
    t.kind = kind;
    t.L = L;
    DevBuf<double> b(nb, s);
    GLI_CUDA(cudaMemcpyAsync(b.p, h_coeffs, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    DevBuf<int> maxabs(1, s);
    GLI_CUDA(cudaMemsetAsync(maxabs.p, 0xff, sizeof(int), s));  // -1: nothing above tol

    DevBuf<double> prod;
    if (kind == 0) {
        prod.alloc(2 * nb - 1, s);
        k_erida_products<<<(unsigned)((2 * nb - 1 + 127) / 128), 128, 0, s>>>(b.p, (int)nb, tol, prod.p, maxabs.p);
        GLI_CHECK_LAUNCH();
        t.nkeys = L;
    } else {
        const i64 nf = 2 * nb - 1, xl = 4 * nb - 3, npairs = L * (L + 1) / 2;
        DevBuf<double> F(L * nf, s);
        k_factors<<<dim3((unsigned)((nf + 127) / 128), (unsigned)L), 128, 0, s>>>(b.p, (int)nb, (int)L, F.p);
        GLI_CHECK_LAUNCH();
        prod.alloc(npairs * xl, s);
        k_eri_products<<<dim3((unsigned)((xl + 127) / 128), (unsigned)npairs), 128, 0, s>>>(F.p, (int)nb, tol, prod.p,
                                                                                              maxabs.p);
        GLI_CHECK_LAUNCH();
        t.nkeys = npairs * (2 * L - 1);
    }
    int h_max = -1;
    GLI_CUDA(cudaMemcpyAsync(&h_max, maxabs.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    const i64 centre_max = kind == 0 ? 3 * (L - 1) : 6 * (L - 1);
    if (t.nkeys > 65535) fail(GLI_ERR_LIMIT, "grid too large for the per-axis key table (%lld keys)", (long long)t.nkeys);
    t.U = h_max < 0 ? 1 : centre_max + h_max + 1;
    if (t.U > 4096) fail(GLI_ERR_LIMIT, "lattice extent %lld exceeds 4096", (long long)t.U);
    t.Up = (t.U + 3) / 4 * 4;
    t.tlen = 3 * (t.U - 1) * (t.U - 1) + 1;

    t.W.alloc(t.nkeys * t.Up);
    k_fold_weights<<<dim3((unsigned)((t.Up + 127) / 128), (unsigned)t.nkeys), 128, 0, s>>>(
        kind, prod.p, (int)nb, (int)L, t.nkeys, (int)t.U, (int)t.Up, t.W.p);
    GLI_CHECK_LAUNCH();
    t.T.alloc(t.tlen);
    k_coulomb_table<<<(unsigned)((t.tlen + 255) / 256), 256, 0, s>>>(kind, t.tlen, t.T.p);
    GLI_CHECK_LAUNCH();

    const i64 U = t.U, smax = 2 * (U - 1) * (U - 1) + 1;
    DevBuf<uint32_t> mark(smax, s);
    mark.zero();
    k_mark_s<<<(unsigned)((U * U + 255) / 256), 256, 0, s>>>((int)U, mark.p);
    GLI_CHECK_LAUNCH();
    DevBuf<uint64_t> pos(smax, s);
    t.nS = exclusive_scan_u32(mark.p, pos.p, smax, s);
    t.S.alloc(t.nS);
    k_s_list<<<(unsigned)((smax + 255) / 256), 256, 0, s>>>(smax, mark.p, pos.p, t.S.p);
    GLI_CHECK_LAUNCH();
    t.sidx.alloc(U * U);
    k_s_index<<<(unsigned)((U * U + 255) / 256), 256, 0, s>>>((int)U, pos.p, t.sidx.p);
    GLI_CHECK_LAUNCH();
    GLI_CUDA(cudaStreamSynchronize(s));
}

namespace {
struct CacheEntry {
    int kind, device;
    i64 L;
    double tol;
    std::vector<double> coeffs;
    std::shared_ptr<const LatticeTables> tables;
};
std::mutex g_cache_mu;
std::list<CacheEntry> g_cache;
constexpr size_t kCacheEntries = 8;
}  // namespace

void clear_table_cache() {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache.clear();
}

std::shared_ptr<const LatticeTables> lattice_tables(int kind, const double* h_coeffs, i64 nb, i64 L, double tol,
                                                    cudaStream_t s) {
    if (nb <= 0 || nb % 2 != 1) fail(GLI_ERR_ARGUMENT, "gausslet coefficient count must be odd, got %lld", (long long)nb);
    if (nb > 4096) fail(GLI_ERR_LIMIT, "gausslet coefficient count %lld exceeds 4096", (long long)nb);
    int device = 0;
    GLI_CUDA(cudaGetDevice(&device));
    std::vector<double> c(h_coeffs, h_coeffs + nb);
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        for (auto it = g_cache.begin(); it != g_cache.end(); ++it) {
            if (it->kind == kind && it->device == device && it->L == L && it->tol == tol && it->coeffs == c) {
                g_cache.splice(g_cache.begin(), g_cache, it);  // most recently used first
                return it->tables;
            }
        }
    }
    auto t = std::make_shared<LatticeTables>();
    t->device = device;
    build_lattice_tables(kind, h_coeffs, nb, L, tol, *t, s);
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache.push_front(CacheEntry{kind, device, L, tol, std::move(c), t});
    while (g_cache.size() > kCacheEntries) g_cache.pop_back();
    return t;
}

namespace {
struct ScreenEntry {
    int kind, device;
    i64 L;
    double tol, tau, bound;
    std::vector<double> coeffs;
};
std::list<ScreenEntry> g_screen;  // (guarded by g_cache_mu)
}  // namespace

double mixed_screen_tol(int kind, const double* h_coeffs, i64 nb, i64 L, double tol, double* bound, cudaStream_t s) {
    if (nb <= 0 || nb % 2 != 1) fail(GLI_ERR_ARGUMENT, "gausslet coefficient count must be odd, got %lld", (long long)nb);
    if (nb > 4096) fail(GLI_ERR_LIMIT, "gausslet coefficient count %lld exceeds 4096", (long long)nb);
    int device = 0;
    GLI_CUDA(cudaGetDevice(&device));
    std::vector<double> c(h_coeffs, h_coeffs + nb);
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        for (const ScreenEntry& e : g_screen)
            if (e.kind == kind && e.device == device && e.L == L && e.tol == tol && e.coeffs == c) {
                *bound = e.bound;
                return e.tau;
            }
    }
    // the product vectors without a mask (the same kernels as the tables)
    DevBuf<double> b(nb, s);
    GLI_CUDA(cudaMemcpyAsync(b.p, h_coeffs, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    DevBuf<int> maxabs(1, s);
    GLI_CUDA(cudaMemsetAsync(maxabs.p, 0xff, sizeof(int), s));
    i64 npairs = 1, xl = 2 * nb - 1;
    DevBuf<double> prod;
    if (kind == 0) {
        prod.alloc(xl, s);
        k_erida_products<<<(unsigned)((xl + 127) / 128), 128, 0, s>>>(b.p, (int)nb, 0.0, prod.p, maxabs.p);
        GLI_CHECK_LAUNCH();
    } else {
        const i64 nf = 2 * nb - 1;
        xl = 4 * nb - 3;
        npairs = L * (L + 1) / 2;
        DevBuf<double> F(L * nf, s);
        k_factors<<<dim3((unsigned)((nf + 127) / 128), (unsigned)L), 128, 0, s>>>(b.p, (int)nb, (int)L, F.p);
        GLI_CHECK_LAUNCH();
        prod.alloc(npairs * xl, s);
        k_eri_products<<<dim3((unsigned)((xl + 127) / 128), (unsigned)npairs), 128, 0, s>>>(F.p, (int)nb, 0.0, prod.p,
                                                                                              maxabs.p);
        GLI_CHECK_LAUNCH();
    }
    std::vector<double> P((size_t)(npairs * xl));
    GLI_CUDA(cudaMemcpyAsync(P.data(), prod.p, P.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    // candidates tau = 10^(-16 + k/4) up to 1e-4, the largest whose bound holds
    const double T0 = kind ? 2.3936536824085962 : 1.6925687506432689;  // T(0), as k_coulomb_table
    double S = 0.0;
    for (i64 p = 0; p < npairs; ++p) {
        double l1 = 0.0;
        for (i64 x = 0; x < xl; ++x)
            if (fabs(P[p * xl + x]) > tol) l1 += fabs(P[p * xl + x]);
        S = std::max(S, l1);
    }
    double tau = tol, tau_bound = 0.0;
    for (int k = 0; k <= 48; ++k) {
        const double cand = pow(10.0, -16.0 + 0.25 * k);
        if (cand <= tol) continue;
        double D = 0.0;
        for (i64 p = 0; p < npairs; ++p) {
            double d = 0.0;
            for (i64 x = 0; x < xl; ++x) {
                const double a = fabs(P[p * xl + x]);
                if (a > tol && a <= cand) d += a;
            }
            D = std::max(D, d);
        }
        const double bnd = 3.0 * T0 * D * S * S;
        if (bnd > MIXED_SCREEN_BOUND) break;
        tau = cand;
        tau_bound = bnd;
    }
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_screen.push_front(ScreenEntry{kind, device, L, tol, tau, tau_bound, std::move(c)});
    while (g_screen.size() > kCacheEntries) g_screen.pop_back();
    *bound = tau_bound;
    return tau;
}

}  // namespace gli
