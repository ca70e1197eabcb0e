// Device-built lookup tables shared by the integral kernels.
#pragma once
#include <memory>
#include <mutex>

#include "gli_internal.cuh"
#include "tc_gemm.cuh"

namespace gli {

// Lattice description of a sparse ERI/ERIDA evaluation.  Every class value is
//   sum_{u,v,t >= 0} W[kx][u] W[ky][v] W[kz][t] T[u^2 + v^2 + t^2]
// where W[k] is the folded (|position|-indexed) product weight of per-axis key k
// and T the Coulomb table on the integer lattice.
// long-lived device allocation (cached tables outlive the stream that built them)
template <class T>
struct DevMem {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        n = count;
        if (count) GLI_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
    }
    ~DevMem() {
        if (p) cudaFree(p);
    }
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
};

// a tiled sliced operand that lives as long as the tables it was made from
struct TiledTable {
    DevMem<int8_t> data;
    DevMem<int> e;
    TiledOperand view;
};

struct LatticeTables {
    int kind = 0;            // 0 = ERIDA, 1 = ERI
    int device = 0;
    i64 L = 0;               // largest axis length of the grid (table sizing as in the reference)
    i64 nkeys = 0;           // size of the dense per-axis key space
    i64 U = 0;               // folded lattice extent: positions 0 .. U-1
    i64 Up = 0;              // U rounded up to a multiple of 4 (row pitch of W)
    i64 tlen = 0;            // T entries: 3 (U-1)^2 + 1
    i64 nS = 0;              // distinct values s = u^2 + v^2, u, v < U
    DevMem<double> W;        // nkeys x Up
    DevMem<double> T;        // tlen
    DevMem<int> S;           // nS distinct s values, ascending
    DevMem<int> sidx;        // U x U: position of u^2 + v^2 in S
    // the mixed form's stage-A operand G[j][t] = T[S[j] + t^2], sliced on first use
    mutable std::mutex g_mu;
    mutable std::unique_ptr<TiledTable> g_sliced;
};

// Builds P (ERIDA) or the shift-pair products (ERI) from the coefficients, masks
// entries with |P| <= tol exactly as the reference's trimming and skipping do,
// folds them into W, evaluates T and the distinct-s index.  Tables depend only
// on (kind, coefficients, L, tol, device) and are cached across calls (a few
// entries, least recently used evicted); a build synchronises the stream.
std::shared_ptr<const LatticeTables> lattice_tables(int kind, const double* h_coeffs, i64 nb, i64 L, double tol,
                                                    cudaStream_t s);

// Screening of the mixed form: the largest threshold tau >= tol at which
// dropping the product entries tol < |P| <= tau changes no class value by
// more than MIXED_SCREEN_BOUND grid units, by the first-order bound
//   |dV| <= 3 T(0) D S^2,  D = max_p sum_{tol<|P_p|<=tau} |P_p|,  S = max_p sum_{|P_p|>tol} |P_p|
// (a class value is sum W_x W_y W_z T over the lattice, each folded weight
// row W takes every entry of its product vector at most once, and 0 < T <=
// T(0)).  *bound receives the bound at the returned tau (0 when tau = tol).
// Cached per (kind, coefficients, L, tol, device).
constexpr double MIXED_SCREEN_BOUND = 1e-9;
double mixed_screen_tol(int kind, const double* h_coeffs, i64 nb, i64 L, double tol, double* bound, cudaStream_t s);

// dense ERI key of one axis: shift pair (|s01|, |s23|) unordered and |c|/3
__host__ __device__ inline i64 eri_axis_key(i64 s01, i64 s23, i64 cc, i64 L) {
    i64 a = s01 < 0 ? -s01 : s01;
    i64 b = s23 < 0 ? -s23 : s23;
    if (a > b) { i64 t = a; a = b; b = t; }
    const i64 c = cc < 0 ? -cc : cc;
    return (b * (b + 1) / 2 + a) * (2 * L - 1) + c;
}

// the same key in 32-bit arithmetic (keys < 2^21)
__host__ __device__ inline int eri_axis_key32(int s01, int s23, int cc, int L) {
    int a = s01 < 0 ? -s01 : s01;
    int b = s23 < 0 ? -s23 : s23;
    if (a > b) { const int t = a; a = b; b = t; }
    const int c = cc < 0 ? -cc : cc;
    return (b * (b + 1) / 2 + a) * (2 * L - 1) + c;
}

}  // namespace gli
