// O_h orbit helpers on a rotationally symmetric grid (-e .. e on every axis),
// shared by the enumeration (enumerate.cu) and the sparse -> dense kernels
// (dense.cu).  Reference: minimum_octahedral_orbit_{eri,erida}_tensor_index
// (src/eri_integrals.c:240-291, src/erida_integrals.c:209-234) with the
// bias-shift loops of the enumerators and fill routines.
#pragma once
#include "gli_internal.cuh"

namespace gli {

struct SymGrid {
    int e;   // extent: coordinates -e .. e
    int L;   // 2e + 1
    i64 N;   // L^3
    const int* omin = nullptr;  // enumeration: smallest linear index among each point's 48 O_h images
};

__device__ inline i64 lin3(const SymGrid& G, const int q[3]) {
    return ((i64)(q[0] + G.e) * G.L + (q[1] + G.e)) * G.L + (q[2] + G.e);
}

__device__ inline int absi(int v) { return v < 0 ? -v : v; }

// ERIDA: is (p0, p1) the smallest index of its orbit?  idx = lin(p0) N + lin(p1)
__device__ inline bool canonical_pair(const SymGrid& G, const int p[2][3], const int bias[3], i64 idx) {
    for (int bx = 0; bx <= absi(bias[0]); ++bx)
        for (int by = 0; by <= absi(bias[1]); ++by)
            for (int bz = 0; bz <= absi(bias[2]); ++bz) {
                const int sft[3] = {bx * bias[0], by * bias[1], bz * bias[2]};
                int q0[3], q1[3];
                for (int a = 0; a < 3; ++a) {
                    q0[a] = p[0][a] - sft[a];
                    q1[a] = p[1][a] - sft[a];
                }
                for (int g = 0; g < 48; ++g) {
                    int r0[3], r1[3];
                    oh_apply(g, q0, r0);
                    oh_apply(g, q1, r1);
                    i64 a = lin3(G, r0), b = lin3(G, r1);
                    if (a > b) { i64 t = a; a = b; b = t; }
                    if (a * G.N + b < idx) return false;
                }
            }
    return true;
}

// ERI: is (p0, p1, p2, p3) the smallest index of its orbit?
__device__ inline bool canonical_quad(const SymGrid& G, const int p[4][3], const int bias[3], i64 idx) {
    const i64 N2 = G.N * G.N;
    for (int bx = 0; bx <= absi(bias[0]); ++bx)
        for (int by = 0; by <= absi(bias[1]); ++by)
            for (int bz = 0; bz <= absi(bias[2]); ++bz) {
                const int sft[3] = {bx * bias[0], by * bias[1], bz * bias[2]};
                int q[4][3];
                for (int k = 0; k < 4; ++k)
                    for (int a = 0; a < 3; ++a) q[k][a] = p[k][a] - sft[a];
                for (int g = 0; g < 48; ++g) {
                    i64 l4[4];
                    for (int k = 0; k < 4; ++k) {
                        int r[3];
                        oh_apply(g, q[k], r);
                        l4[k] = lin3(G, r);
                    }
                    i64 ab = l4[0] <= l4[1] ? l4[0] * G.N + l4[1] : l4[1] * G.N + l4[0];
                    i64 cd = l4[2] <= l4[3] ? l4[2] * G.N + l4[3] : l4[3] * G.N + l4[2];
                    if (ab > cd) { i64 t = ab; ab = cd; cd = t; }
                    if (ab * N2 + cd < idx) return false;
                }
            }
    return true;
}

__device__ inline void point_of(const SymGrid& G, i64 lin, int p[3]) {
    p[2] = (int)(lin % G.L) - G.e;
    lin /= G.L;
    p[1] = (int)(lin % G.L) - G.e;
    p[0] = (int)(lin / G.L) - G.e;
}


// smallest index of the orbit of a pair / quadruple already translated so that
// each axis' doubled box centre is in {-1, 0, 1} (bias = that centre)
__device__ inline i64 orbit_min_pair(const SymGrid& G, const int p[2][3], const int bias[3]) {
    i64 best = INT64_MAX;
    for (int bx = 0; bx <= absi(bias[0]); ++bx)
        for (int by = 0; by <= absi(bias[1]); ++by)
            for (int bz = 0; bz <= absi(bias[2]); ++bz) {
                const int sft[3] = {bx * bias[0], by * bias[1], bz * bias[2]};
                int q0[3], q1[3];
                for (int a = 0; a < 3; ++a) {
                    q0[a] = p[0][a] - sft[a];
                    q1[a] = p[1][a] - sft[a];
                }
                for (int g = 0; g < 48; ++g) {
                    int r0[3], r1[3];
                    oh_apply(g, q0, r0);
                    oh_apply(g, q1, r1);
                    i64 a = lin3(G, r0), b = lin3(G, r1);
                    const i64 v = a <= b ? a * G.N + b : b * G.N + a;
                    if (v < best) best = v;
                }
            }
    return best;
}

__device__ inline i64 orbit_min_quad(const SymGrid& G, const int p[4][3], const int bias[3]) {
    const i64 N2 = G.N * G.N;
    i64 best = INT64_MAX;
    for (int bx = 0; bx <= absi(bias[0]); ++bx)
        for (int by = 0; by <= absi(bias[1]); ++by)
            for (int bz = 0; bz <= absi(bias[2]); ++bz) {
                const int sft[3] = {bx * bias[0], by * bias[1], bz * bias[2]};
                int q[4][3];
                for (int k = 0; k < 4; ++k)
                    for (int a = 0; a < 3; ++a) q[k][a] = p[k][a] - sft[a];
                for (int g = 0; g < 48; ++g) {
                    i64 l4[4];
                    for (int k = 0; k < 4; ++k) {
                        int r[3];
                        oh_apply(g, q[k], r);
                        l4[k] = lin3(G, r);
                    }
                    i64 ab = l4[0] <= l4[1] ? l4[0] * G.N + l4[1] : l4[1] * G.N + l4[0];
                    i64 cd = l4[2] <= l4[3] ? l4[2] * G.N + l4[3] : l4[3] * G.N + l4[2];
                    if (ab > cd) { i64 t = ab; ab = cd; cd = t; }
                    const i64 v = ab * N2 + cd;
                    if (v < best) best = v;
                }
            }
    return best;
}

// move the bounding-box centre of np points to the origin (reference
// src/eri_integrals.c:869-903: trans = (min+max)/2 truncating, bias = remainder)
template <int NP>
__device__ inline void centre_points(int p[NP][3], int bias[3]) {
    for (int a = 0; a < 3; ++a) {
        int lo = p[0][a], hi = p[0][a];
        for (int k = 1; k < NP; ++k) {
            lo = min(lo, p[k][a]);
            hi = max(hi, p[k][a]);
        }
        const int c = lo + hi;
        const int trans = c / 2;
        bias[a] = c - 2 * trans;
        for (int k = 0; k < NP; ++k) p[k][a] -= trans;
    }
}

}  // namespace gli
