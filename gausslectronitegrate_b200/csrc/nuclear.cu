// Nuclear-attraction integrals, reference src/nuclear_integrals.c:16-24 (the
// Gaussian-nucleus kernel erf(r/w)/r, w = 1/3), :31-126 (single entry) and
// :133-266 (matrix).
//
// The reference evaluates, per orbital pair (i, j),
//   V_ij = sum_{x,y,z} Fx[x] Fy[y] Fz[z] sum_k Z_k g(|p - R_k|),
//   p_a = (i_a + j_a)/2 + m_a/6,
// one erf per (primitive point, nucleus).  Every primitive point lies on the
// 1/6 lattice, so the nuclear field is tabulated once on the lattice box that
// the grid's primitives cover,
//   Phi[u][v][t] = sum_k Z_k g(|(u,v,t)/6 + origin - R_k|),
// and the separable weights are contracted against it axis by axis:
//   A   H[kz][u][v]     = sum_t Wz[kz][t] Phi[u][v][t]      (GEMM)
//   B   H2[kz][ky][u]   = sum_v Wy[ky][v] H[kz][u][v]       (batched GEMM)
//   C   Vk[kx][kz,ky]   = sum_u Wx[kx][u] H2[kz][ky][u]     (GEMM)
// where an axis key is the unordered coordinate pair {i_a, j_a} (the factor
// depends on |i_a - j_a|, the position on i_a + j_a).  A final scatter writes
// the dense N x N matrix, V_ij = Vk[kx(i,j)][kz(i,j), ky(i,j)].
#include <math.h>

#include <algorithm>

#include "gli_internal.cuh"

namespace gli {


__global__ void k_mask_factors(double* __restrict__ F, i64 n, int nf, int nb, double tol, int* __restrict__ mmax) {
    const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double v = F[e];
    if (!(fabs(v) > tol)) v = 0;
    F[e] = v;
    if (v != 0) {
        const int m = (int)(e % nf) - (nb - 1);
        atomicMax(mmax, m < 0 ? -m : m);
    }
}

// W[key][u]: key = tri(a <= b) over the axis' coordinate list, u lattice position
__global__ void k_nuclear_weights(const double* __restrict__ F, int nf, int nb, const int* __restrict__ coords,
                                  int u0, int U, double* __restrict__ W) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int key = blockIdx.y;
    if (u >= U) return;
    int hi = 0;
    while ((hi + 1) * (hi + 2) / 2 <= key) ++hi;
    const int lo = key - hi * (hi + 1) / 2;
    const int xa = coords[lo], xb = coords[hi];
    const int s = xa > xb ? xa - xb : xb - xa;
    const int m = u + u0 - 3 * (xa + xb);   // factor logical index
    double v = 0;
    if (m >= -(nb - 1) && m <= nb - 1) v = F[(i64)s * nf + m + (nb - 1)];
    W[(i64)key * U + u] = v;
}

struct NucleiDev {
    int n;
    double pos[3 * 64];
    double charge[64];
};

// Phi[u][v][t] (t fastest), position (u + u0x)/6, (v + u0y)/6, (t + u0z)/6
__global__ void k_nuclear_field(NucleiDev nuc, int u0x, int u0y, int u0z, int Ux, int Uy, int Uz,
                                double* __restrict__ Phi) {
    const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 total = (i64)Ux * Uy * Uz;
    if (e >= total) return;
    const int t = (int)(e % Uz), v = (int)((e / Uz) % Uy), u = (int)(e / ((i64)Uz * Uy));
    const double px = (u + u0x) / 6.0, py = (v + u0y) / 6.0, pz = (t + u0z) / 6.0;
    double acc = 0;
    for (int k = 0; k < nuc.n; ++k) {
        const double dx = px - nuc.pos[3 * k], dy = py - nuc.pos[3 * k + 1], dz = pz - nuc.pos[3 * k + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        // g(r) = erf(r / w) / r with w = 1/3; g(0) = 2 / (sqrt(pi) w)
        const double g = r > 0 ? erf(3.0 * r) / r : 3.3851375012865379;  // 6 / sqrt(pi)
        acc += nuc.charge[k] * g;
    }
    Phi[e] = acc;
}

// V[i][j] for the dense grid from the key-indexed block Vk[kx][kz * nky + ky]
__global__ void k_nuclear_scatter(const double* __restrict__ Vk, int nx, int ny, int nz, int nky, int nkz,
                                  double* __restrict__ V) {
    const i64 N = (i64)nx * ny * nz;
    const i64 total = N * N;
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
        const i64 i = e / N, j = e % N;
        const int iz = (int)(i % nz), iy = (int)((i / nz) % ny), ix = (int)(i / ((i64)nz * ny));
        const int jz = (int)(j % nz), jy = (int)((j / nz) % ny), jx = (int)(j / ((i64)nz * ny));
        const int ax = min(ix, jx), bx = max(ix, jx), ay = min(iy, jy), by = max(iy, jy);
        const int az = min(iz, jz), bz = max(iz, jz);
        const i64 kx = bx * (bx + 1) / 2 + ax, ky = by * (by + 1) / 2 + ay, kz = bz * (bz + 1) / 2 + az;
        V[e] = Vk[kx * ((i64)nkz * nky) + kz * nky + ky];
    }
}

// FP64 strided batched GEMM (dense.cu)
void dgemm_strided(int M, int N, int K, const double* A, i64 asb, i64 ar, i64 ac, const double* B, i64 bsb, i64 br,
                   i64 bc, double* C, i64 csb, i64 cr, i64 cc, int batch, bool accumulate, cudaStream_t s);

void nuclear_matrix_device(const double* h_coeffs, i64 nb, const std::vector<int> axes[3],
                           const struct atomic_nucleus* nuclei, int nn, double tol, double* d_out, cudaStream_t s) {
    if (nn <= 0) fail(GLI_ERR_ARGUMENT, "at least one nucleus is required");
    if (nn > 64) fail(GLI_ERR_LIMIT, "at most 64 nuclei per call (got %d)", nn);
    if (!(tol >= 0)) fail(GLI_ERR_ARGUMENT, "tol must be non-negative");
    int L = 1;  // factor shifts needed: 0 .. max |i_a - j_a|
    for (int a = 0; a < 3; ++a) {
        if (axes[a].empty() || axes[a].size() > 256) fail(GLI_ERR_LIMIT, "axis %d has %zu points (1..256)", a,
                                                           axes[a].size());
        L = std::max(L, axes[a].back() - axes[a].front() + 1);
    }
    const int nf = (int)(2 * nb - 1);
    DevBuf<double> b(nb, s), F((i64)L * nf, s);
    GLI_CUDA(cudaMemcpyAsync(b.p, h_coeffs, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    factors_device(b.p, (int)nb, L, F.p, s);
    DevBuf<int> mmax(1, s);
    GLI_CUDA(cudaMemsetAsync(mmax.p, 0xff, sizeof(int), s));
    k_mask_factors<<<(unsigned)(((i64)L * nf + 255) / 256), 256, 0, s>>>(F.p, (i64)L * nf, nf, (int)nb, tol, mmax.p);
    GLI_CHECK_LAUNCH();
    int h_mmax = -1;
    GLI_CUDA(cudaMemcpyAsync(&h_mmax, mmax.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    const i64 N = (i64)axes[0].size() * axes[1].size() * axes[2].size();
    if (h_mmax < 0) {  // every factor below tol
        GLI_CUDA(cudaMemsetAsync(d_out, 0, N * N * sizeof(double), s));
        return;
    }
    int U[3], u0[3], nk[3];
    DevBuf<double> W[3];
    DevBuf<int> coords[3];
    for (int a = 0; a < 3; ++a) {
        const int n = (int)axes[a].size();
        coords[a].alloc(n, s);
        GLI_CUDA(cudaMemcpyAsync(coords[a].p, axes[a].data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        u0[a] = 6 * axes[a].front() - h_mmax;
        U[a] = 6 * (axes[a].back() - axes[a].front()) + 2 * h_mmax + 1;
        nk[a] = n * (n + 1) / 2;
        W[a].alloc((i64)nk[a] * U[a], s);
        k_nuclear_weights<<<dim3((U[a] + 127) / 128, nk[a]), 128, 0, s>>>(F.p, nf, (int)nb, coords[a].p, u0[a], U[a],
                                                                          W[a].p);
        GLI_CHECK_LAUNCH();
    }
    // the staged buffers must hold the axis coordinate lists until the copies ran
    GLI_CUDA(cudaStreamSynchronize(s));
    NucleiDev nd;
    nd.n = nn;
    for (int k = 0; k < nn; ++k) {
        for (int a = 0; a < 3; ++a) nd.pos[3 * k + a] = nuclei[k].pos[a];
        nd.charge[k] = (double)nuclei[k].charge;
    }
    const i64 cells = (i64)U[0] * U[1] * U[2];
    DevBuf<double> Phi(cells, s);
    k_nuclear_field<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(nd, u0[0], u0[1], u0[2], U[0], U[1], U[2], Phi.p);
    GLI_CHECK_LAUNCH();
    // A: H[kz][(u v)] = sum_t Wz[kz][t] Phi[(u v)][t]
    const i64 UxUy = (i64)U[0] * U[1];
    DevBuf<double> H((i64)nk[2] * UxUy, s);
    dgemm_strided(nk[2], (int)UxUy, U[2], W[2].p, 0, U[2], 1, Phi.p, 0, 1, U[2], H.p, 0, UxUy, 1, 1, false, s);
    // B: H2[kz][ky][u] = sum_v Wy[ky][v] H[kz][u][v]   (batch kz)
    DevBuf<double> H2((i64)nk[2] * nk[1] * U[0], s);
    dgemm_strided(nk[1], U[0], U[1], W[1].p, 0, U[1], 1, H.p, UxUy, 1, U[1], H2.p, (i64)nk[1] * U[0], U[0], 1, nk[2],
                  false, s);
    // C: Vk[kx][(kz ky)] = sum_u Wx[kx][u] H2[(kz ky)][u]
    const i64 nzy = (i64)nk[2] * nk[1];
    DevBuf<double> Vk((i64)nk[0] * nzy, s);
    dgemm_strided(nk[0], (int)nzy, U[0], W[0].p, 0, U[0], 1, H2.p, 0, 1, U[0], Vk.p, 0, nzy, 1, 1, false, s);
    const Context& ctx = context();
    const i64 want = (N * N + 255) / 256, cap = (i64)ctx.num_sms * 32;
    k_nuclear_scatter<<<(unsigned)std::min(want, cap), 256, 0, s>>>(Vk.p, (int)axes[0].size(), (int)axes[1].size(),
                                                                    (int)axes[2].size(), nk[1], nk[2], d_out);
    GLI_CHECK_LAUNCH();
}

}  // namespace gli
