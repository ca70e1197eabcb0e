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
//   B   H2[ky][kz][u]   = sum_v Wy[ky][v] H[kz][u][v]       (batched GEMM)
//   C   Vk[kx][ky,kz]   = sum_u Wx[kx][u] H2[ky][kz][u]     (GEMM)
// where an axis key is the unordered coordinate pair {i_a, j_a} (the factor
// depends on |i_a - j_a|, the position on i_a + j_a).  A final scatter writes
// the dense N x N matrix, V_ij = Vk[kx(i,j)][ky(i,j), kz(i,j)] (the sliced
// tensor-core contractions keep the (kz, ky) order of their batched stage B).
//
// Batches.  Any number of instances (each its own grid and nuclei, all with
// the same coefficients and tol) run as one plan: one upload of every
// instance's descriptor, coordinates and nuclei; one kernel builds every
// instance's weights, one tabulates every instance's field, one scatters every
// instance's matrix; each instance's three contractions run on a ring of
// streams so that small instances overlap.  The plan of a chunk of instances
// is captured as one CUDA graph and launched once.  Forms: FP64 throughout (the
// drop-in), or mixed: the three contractions as int8-sliced products on the
// tensor cores (5 slices), field, weights and scatter in FP64.
#include <math.h>

#include <algorithm>
#include <string>

#include "autotune.cuh"
#include "gli_internal.cuh"
#include "tc_gemm.cuh"

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

// device descriptor of one instance
struct NucInst {
    int n[3];          // axis lengths
    int coord_off[3];  // first coordinate of each axis in the packed coordinate list
    int U[3], u0[3];   // lattice extent and origin (units of 1/6) per axis
    int nk[3];         // axis keys: n (n + 1) / 2
    int nuc0, nnuc;    // nuclei in the packed nucleus arrays
    i64 N;             // grid points
    i64 w_off[3];      // weights of each axis in the packed W buffer
    i64 phi_off;       // field in the packed Phi buffer
    i64 vk_off;        // key-indexed matrix in the packed Vk buffer
    double* out;       // N x N row-major
};

// W[key][u] of every (instance, axis): key = tri(lo <= hi) over the axis'
// coordinate list, u a lattice position.  grid (u blocks, key, 3 * instance)
__global__ void k_nuc_weights(const NucInst* __restrict__ inst, const double* __restrict__ F, int nf, int nb,
                              const int* __restrict__ coords, double* __restrict__ W) {
    const NucInst& in = inst[blockIdx.z / 3];
    const int a = blockIdx.z % 3;
    const int key = blockIdx.y;
    if (key >= in.nk[a]) return;
    int hi = (int)((sqrt(8.0 * key + 1.0) - 1.0) * 0.5);
    while (hi * (hi + 1) / 2 > key) --hi;
    while ((hi + 1) * (hi + 2) / 2 <= key) ++hi;
    const int lo = key - hi * (hi + 1) / 2;
    const int xa = coords[in.coord_off[a] + lo], xb = coords[in.coord_off[a] + hi];
    const int s = xa > xb ? xa - xb : xb - xa;
    const int U = in.U[a];
    double* w = W + in.w_off[a] + (i64)key * U;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < U; u += gridDim.x * blockDim.x) {
        const int m = u + in.u0[a] - 3 * (xa + xb);  // factor logical index
        double v = 0;
        if (m >= -(nb - 1) && m <= nb - 1) v = F[(i64)s * nf + m + (nb - 1)];
        w[u] = v;
    }
}

// the Gaussian-nucleus field at lattice point (u, v, t) of an instance
__device__ inline double nuc_field_at(const NucInst& in, const double* __restrict__ npos,
                                      const double* __restrict__ ncharge, int u, int v, int t) {
    const double px = (u + in.u0[0]) / 6.0, py = (v + in.u0[1]) / 6.0, pz = (t + in.u0[2]) / 6.0;
    double acc = 0;
    for (int k = in.nuc0; k < in.nuc0 + in.nnuc; ++k) {
        const double dx = px - npos[3 * k], dy = py - npos[3 * k + 1], dz = pz - npos[3 * k + 2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        // g(r) = erf(r / w) / r with w = 1/3; g(0) = 2 / (sqrt(pi) w).  For
        // 3 r >= 6, erfc(3 r) <= 2.2e-17 is below a quarter ulp of 1: erf
        // rounds to 1 and g = 1 / r
        double g;
        if (r2 >= 4.0) {
            g = rsqrt(r2);
        } else {
            const double r = sqrt(r2);
            g = r > 0 ? erf(3.0 * r) / r : 3.3851375012865379;  // 6 / sqrt(pi)
        }
        acc += ncharge[k] * g;
    }
    return acc;
}

// Phi[u][v][t] (t fastest) of every instance, position (u + u0x, v + u0y, t + u0z) / 6;
// grid (row blocks, instance): a block fills whole (u, v) rows
__global__ void __launch_bounds__(128) k_nuc_field(const NucInst* __restrict__ inst, const double* __restrict__ npos,
                                                   const double* __restrict__ ncharge, double* __restrict__ Phi) {
    const NucInst& in = inst[blockIdx.y];
    const int Uy = in.U[1], Uz = in.U[2];
    const i64 rows = (i64)in.U[0] * Uy;
    for (i64 row = blockIdx.x; row < rows; row += gridDim.x) {
        const int u = (int)(row / Uy), v = (int)(row - (i64)u * Uy);
        double* phi = Phi + in.phi_off + row * Uz;
        for (int t = threadIdx.x; t < Uz; t += blockDim.x) phi[t] = nuc_field_at(in, npos, ncharge, u, v, t);
    }
}

// V[i][j] of every instance from its key-indexed block: Vk[kx][ky * nkz + kz]
// (zfast: the FP64 contractions) or Vk[kx][kz * nky + ky] (the sliced ones).
// Grid (x pairs, instance): block (ix, jx) writes the (ny nz) x (ny nz)
// sub-block of rows ix nyz + (iy, iz) and columns jx nyz + (jy, jz), whose
// entries all lie in the one slice kx = key(ix, jx) (nky nkz entries, read
// from cache after the first touch; a whole row of V would read every slice,
// more than L2 holds for a 24^3 instance).  A thread owns columns, decoded
// once; rows run as (iy, iz) loops, so the inner loop has no division.
__global__ void __launch_bounds__(256) k_nuc_scatter(const NucInst* __restrict__ inst, const double* __restrict__ Vk,
                                                     int zfast) {
    const NucInst& in = inst[blockIdx.y];
    const int nx = in.n[0], ny = in.n[1], nz = in.n[2], nky = in.nk[1], nkz = in.nk[2];
    const int nyz = ny * nz;
    const i64 N = in.N;
    const i64 sy = zfast ? nkz : 1, sz = zfast ? 1 : nky;  // strides of ky and kz in a slice
    for (int pair = blockIdx.x; pair < nx * nx; pair += gridDim.x) {
        const int ix = pair / nx, jx = pair - ix * nx;
        const int ax = min(ix, jx), bx = max(ix, jx);
        const double* slice = Vk + in.vk_off + (i64)(bx * (bx + 1) / 2 + ax) * ((i64)nky * nkz);
        double* block = in.out + (i64)ix * nyz * N + (i64)jx * nyz;
        for (int c = threadIdx.x; c < nyz; c += blockDim.x) {
            const int jy = c / nz, jz = c - jy * nz;
            double* col = block + c;
            for (int iy = 0; iy < ny; ++iy) {
                const int ay = min(iy, jy), by = max(iy, jy);
                const double* sl = slice + (i64)(by * (by + 1) / 2 + ay) * sy;
                double* out = col + (i64)iy * nz * N;
                for (int iz = 0; iz < nz; ++iz) {
                    const int az = min(iz, jz), bz = max(iz, jz);
                    out[(i64)iz * N] = sl[(i64)(bz * (bz + 1) / 2 + az) * sz];
                }
            }
        }
    }
}

// tiles of a shared-B batched product: batch b, B row block j of nbt
__global__ void k_shared_b_tiles(int batches, int nbt, int nrows, int bn, int* __restrict__ tb, int* __restrict__ tc,
                                 int* __restrict__ tn, int* __restrict__ tbb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= batches * nbt) return;
    const int b = t / nbt, j = t % nbt;
    tb[t] = b;
    tc[t] = b * nrows + j * bn;
    tn[t] = min(bn, nrows - j * bn);
    tbb[t] = j;
}

// rows r = b * rows + i of a batched dense matrix, each batch padded to whole
// 128-row tiles
struct BatchedRows {
    const double* src;
    i64 ld;
    int rows, blocks;
    __device__ RowBase row(i64 r) const { return {src + r * ld}; }
    __device__ double at(const RowBase& c, int k) const { return c.p[k]; }
    __device__ i64 dest(i64 r) const { return (r / rows) * blocks * TC_BM + r % rows; }
    __device__ i64 source(i64 d, i64 total) const {
        const i64 b = d / ((i64)blocks * TC_BM), i = d % ((i64)blocks * TC_BM);
        return (i < rows && b * rows + i < total) ? b * rows + i : -1;
    }
    __device__ bool valid(i64) const { return true; }
};

// FP64 strided batched GEMM (dense.cu); dgemm_prepare sets its kernel
// attributes, outside any graph capture
void dgemm_strided(int M, int N, int K, const double* A, i64 asb, i64 ar, i64 ac, const double* B, i64 bsb, i64 br,
                   i64 bc, double* C, i64 csb, i64 cr, i64 cc, int batch, bool accumulate, cudaStream_t s);
void dgemm_prepare();

// host copy of an instance
struct NucHost {
    NucInst d;
};

// A: H[kz][(u v)] = sum_t Wz[kz][t] Phi[(u v)][t];  B: H2[ky][kz][u] = sum_v Wy[ky][v] H[kz][u][v];
// C: Vk[kx][(ky kz)] = sum_u Wx[kx][u] H2[(ky kz)][u]
static void nuc_contract_fp64(const NucInst& in, const double* W, const double* Phi, double* Vk, cudaStream_t s) {
    const int* U = in.U;
    const int* nk = in.nk;
    const i64 UxUy = (i64)U[0] * U[1], nzy = (i64)nk[2] * nk[1];
    const double* Wx = W + in.w_off[0];
    const double* Wy = W + in.w_off[1];
    const double* Wz = W + in.w_off[2];
    DevBuf<double> H((i64)nk[2] * UxUy, s), H2(nzy * U[0], s);
    dgemm_strided(nk[2], (int)UxUy, U[2], Wz, 0, U[2], 1, Phi + in.phi_off, 0, 1, U[2], H.p, 0, UxUy, 1, 1, false,
                  s);
    // H2 rows ordered (ky, kz): Vk comes out as [kx][ky][kz], kz innermost (the
    // scatter's fastest-varying key along a matrix row)
    dgemm_strided(nk[1], U[0], U[1], Wy, 0, U[1], 1, H.p, UxUy, 1, U[1], H2.p, U[0], (i64)nk[2] * U[0], 1, nk[2],
                  false, s);
    dgemm_strided(nk[0], (int)nzy, U[0], Wx, 0, U[0], 1, H2.p, 0, 1, U[0], Vk + in.vk_off, 0, nzy, 1, 1, false, s);
}

static void nuc_contract_mixed(const NucInst& in, const double* W, const double* Phi, double* Vk, int* err,
                               cudaStream_t s) {
    constexpr int S = MIXED_SLICES, BN = tile_n(MIXED_SLICES);
    const int* U = in.U;
    const int* nk = in.nk;
    const i64 UxUy = (i64)U[0] * U[1], nzy = (i64)nk[2] * nk[1];
    const double* Wx = W + in.w_off[0];
    const double* Wy = W + in.w_off[1];
    const double* Wz = W + in.w_off[2];
    DevBuf<double> H((i64)nk[2] * UxUy, s), H2(nzy * U[0], s);
    {   // A: rows (u v) of the field against the z keys
        TiledSlices As, Bs;
        const i64 mb = (UxUy + TC_BM - 1) / TC_BM, nbt = (nk[2] + BN - 1) / BN;
        As.alloc(mb, TC_BM, U[2], S, s);
        slice_tiled(DenseRows{Phi + in.phi_off, U[2]}, UxUy, U[2], As, s);
        Bs.alloc(nbt, BN, U[2], S, s);
        slice_tiled(DenseRows{Wz, U[2]}, nk[2], U[2], Bs, s);
        TileWork w;
        w.a_rows = (int)UxUy;
        w.a_blocks = (int)mb;
        w.n_total = nk[2];
        w.C = H.p;
        w.rs = 1;
        w.cs = UxUy;
        tc_gemm_tiled(As.view(), Bs.view(), w, (int)nbt, err, s);
    }
    {   // B: batch kz, rows u of H[kz] (K = v) against the y keys (shared by every batch)
        TiledSlices As, Bs;
        const int mb = (U[0] + TC_BM - 1) / TC_BM, nbt = (nk[1] + BN - 1) / BN;
        As.alloc((i64)nk[2] * mb, TC_BM, U[1], S, s);
        slice_tiled(BatchedRows{H.p, U[1], U[0], mb}, (i64)nk[2] * U[0], U[1], As, s);
        Bs.alloc(nbt, BN, U[1], S, s);
        slice_tiled(DenseRows{Wy, U[1]}, nk[1], U[1], Bs, s);
        const int ntiles = nk[2] * nbt;
        DevBuf<int> tiles(4 * (i64)ntiles, s);
        k_shared_b_tiles<<<(ntiles + 255) / 256, 256, 0, s>>>(nk[2], nbt, nk[1], BN, tiles.p, tiles.p + ntiles,
                                                              tiles.p + 2 * ntiles, tiles.p + 3 * ntiles);
        GLI_CHECK_LAUNCH();
        TileWork w;
        w.a_rows = U[0];
        w.a_blocks = mb;
        w.a_batched = 1;
        w.tile_batch = tiles.p;
        w.tile_col0 = tiles.p + ntiles;
        w.tile_ncols = tiles.p + 2 * ntiles;
        w.tile_bblock = tiles.p + 3 * ntiles;
        w.C = H2.p;
        w.rs = 1;
        w.cs = U[0];
        tc_gemm_tiled(As.view(), Bs.view(), w, ntiles, err, s);
    }
    {   // C: rows (kz ky) of H2 (K = u) against the x keys
        TiledSlices As, Bs;
        const i64 mb = (nzy + TC_BM - 1) / TC_BM, nbt = (nk[0] + BN - 1) / BN;
        As.alloc(mb, TC_BM, U[0], S, s);
        slice_tiled(DenseRows{H2.p, U[0]}, nzy, U[0], As, s);
        Bs.alloc(nbt, BN, U[0], S, s);
        slice_tiled(DenseRows{Wx, U[0]}, nk[0], U[0], Bs, s);
        TileWork w;
        w.a_rows = (int)nzy;
        w.a_blocks = (int)mb;
        w.n_total = nk[0];
        w.C = Vk + in.vk_off;
        w.rs = 1;
        w.cs = nzy;
        tc_gemm_tiled(As.view(), Bs.view(), w, (int)nbt, err, s);
    }
}

// streams of the per-instance contractions (per thread and device)
struct StreamRing {
    int device = -1;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    void ensure(int dev, int n) {
        if (device != dev) {
            streams.clear();
            events.clear();
            device = dev;
        }
        while ((int)streams.size() < n) {
            cudaStream_t st;
            cudaEvent_t ev;
            GLI_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            GLI_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            streams.push_back(st);
            events.push_back(ev);
        }
    }
};
static thread_local StreamRing t_ring;
static thread_local cudaEvent_t t_fork = nullptr;
static thread_local int t_fork_dev = -1;

// streams and the fork event exist before any capture starts
static void ensure_streams(int device, int n) {
    if (t_fork_dev != device) {
        GLI_CUDA(cudaEventCreateWithFlags(&t_fork, cudaEventDisableTiming));
        t_fork_dev = device;
    }
    t_ring.ensure(device, n);
}

// Queues one chunk of instances (descriptors already on the device): weights,
// field, per-instance contractions on `nstreams` forked streams (int8-sliced
// tensor-core products when `sliced`, else the FP64 tensor-core GEMM),
// scatter.  Makes no call that a stream capture forbids.
static void enqueue_chunk(const std::vector<NucHost>& hosts, const NucInst* d_inst, const double* F, int nf, int nb,
                          const int* coords, const double* npos, const double* ncharge, bool sliced, int nstreams,
                          int num_sms, int* err, cudaStream_t s) {
    const int ni = (int)hosts.size();
    i64 w_total = 0, phi_total = 0, vk_total = 0;
    int max_nk = 1, max_u = 1;
    i64 max_rows = 1;
    for (const NucHost& h : hosts) {
        for (int a = 0; a < 3; ++a) {
            w_total = std::max(w_total, h.d.w_off[a] + (i64)h.d.nk[a] * h.d.U[a]);
            max_nk = std::max(max_nk, h.d.nk[a]);
            max_u = std::max(max_u, h.d.U[a]);
        }
        const i64 cells = (i64)h.d.U[0] * h.d.U[1] * h.d.U[2];
        phi_total = std::max(phi_total, h.d.phi_off + cells);
        vk_total = std::max(vk_total, h.d.vk_off + (i64)h.d.nk[0] * h.d.nk[1] * h.d.nk[2]);
        max_rows = std::max(max_rows, (i64)h.d.U[0] * h.d.U[1]);
    }
    DevBuf<double> W(w_total, s), Phi(phi_total, s), Vk(vk_total, s);
    k_nuc_weights<<<dim3((unsigned)((max_u + 127) / 128), (unsigned)max_nk, (unsigned)(3 * ni)), 128, 0, s>>>(
        d_inst, F, nf, nb, coords, W.p);
    GLI_CHECK_LAUNCH();
    {
        const unsigned fb = (unsigned)std::min<i64>(max_rows, std::max<i64>(1, (i64)num_sms * 16));
        k_nuc_field<<<dim3(fb, (unsigned)ni), 128, 0, s>>>(d_inst, npos, ncharge, Phi.p);
        GLI_CHECK_LAUNCH();
    }
    // per-instance contractions, largest first, round-robin over the streams
    std::vector<int> order(ni);
    for (int k = 0; k < ni; ++k) order[k] = k;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return hosts[a].d.N > hosts[b].d.N; });
    GLI_CUDA(cudaEventRecord(t_fork, s));
    for (int k = 0; k < nstreams; ++k) GLI_CUDA(cudaStreamWaitEvent(t_ring.streams[k], t_fork, 0));
    for (int k = 0; k < ni; ++k) {
        cudaStream_t st = t_ring.streams[k % nstreams];
        const NucInst& in = hosts[order[k]].d;
        if (sliced)
            nuc_contract_mixed(in, W.p, Phi.p, Vk.p, err, st);
        else
            nuc_contract_fp64(in, W.p, Phi.p, Vk.p, st);
    }
    for (int k = 0; k < nstreams; ++k) {
        GLI_CUDA(cudaEventRecord(t_ring.events[k], t_ring.streams[k]));
        GLI_CUDA(cudaStreamWaitEvent(s, t_ring.events[k], 0));
    }
    // one block per x pair (ix, jx) of the largest instance
    i64 max_pairs = 1;
    for (const NucHost& h : hosts) max_pairs = std::max<i64>(max_pairs, (i64)h.d.n[0] * h.d.n[0]);
    k_nuc_scatter<<<dim3((unsigned)max_pairs, (unsigned)ni), 256, 0, s>>>(d_inst, Vk.p, sliced ? 0 : 1);
    GLI_CHECK_LAUNCH();
}

// Captures the chunk as one CUDA graph and launches it once
static void run_chunk_graph(const std::vector<NucHost>& hosts, const NucInst* d_inst, const double* F, int nf,
                            int nb, const int* coords, const double* npos, const double* ncharge, bool sliced,
                            int nstreams, int num_sms, int* err, cudaStream_t s) {
    tc_gemm_prepare();
    dgemm_prepare();
    GLI_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
        enqueue_chunk(hosts, d_inst, F, nf, nb, coords, npos, ncharge, sliced, nstreams, num_sms, err, s);
    } catch (...) {
        cudaStreamEndCapture(s, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
    }
    GLI_CUDA(cudaStreamEndCapture(s, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    GLI_CUDA(ie);
    const cudaError_t le = cudaGraphLaunch(exec, s);
    const cudaError_t se = le == cudaSuccess ? cudaStreamSynchronize(s) : le;
    cudaGraphExecDestroy(exec);
    GLI_CUDA(se);
}

static thread_local NuclearBatchStats t_nuc_stats;
const NuclearBatchStats& last_nuclear_stats() { return t_nuc_stats; }

void nuclear_batch_device(const double* h_coeffs, i64 nb, const std::vector<NuclearJob>& jobs, double tol, int form,
                          cudaStream_t s) {
    if (form != FORM_FP64 && form != FORM_MIXED)
        fail(GLI_ERR_ARGUMENT, "form %d is not a nuclear evaluation form (0 = FP64, 1 = mixed)", form);
    if (!(tol >= 0)) fail(GLI_ERR_ARGUMENT, "tol must be non-negative");
    if (jobs.empty()) return;
    NuclearBatchStats stats;
    // factor shifts needed: 0 .. max |i_a - j_a| over every instance
    int L = 1;
    i64 total_nuclei = 0, total_coords = 0;
    for (const NuclearJob& j : jobs) {
        if (j.nn <= 0 || !j.nuclei) fail(GLI_ERR_ARGUMENT, "every instance needs at least one nucleus");
        if (j.nn > 4096) fail(GLI_ERR_LIMIT, "at most 4096 nuclei per instance (got %d)", j.nn);
        if (!j.d_out) fail(GLI_ERR_ARGUMENT, "an instance has no output buffer");
        for (int a = 0; a < 3; ++a) {
            if (j.axes[a].empty() || j.axes[a].size() > 256)
                fail(GLI_ERR_LIMIT, "axis %d has %zu points (1..256)", a, j.axes[a].size());
            L = std::max(L, j.axes[a].back() - j.axes[a].front() + 1);
            total_coords += (i64)j.axes[a].size();
        }
        total_nuclei += j.nn;
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
    if (h_mmax < 0) {  // every factor below tol
        for (const NuclearJob& j : jobs) {
            const i64 N = (i64)j.axes[0].size() * j.axes[1].size() * j.axes[2].size();
            GLI_CUDA(cudaMemsetAsync(j.d_out, 0, N * N * sizeof(double), s));
        }
        t_nuc_stats = stats;
        return;
    }
    // host plan and one packed upload: descriptors, coordinates, nuclei
    const i64 ni = (i64)jobs.size();
    std::vector<NucHost> hosts(ni);
    std::vector<int> coords;
    coords.reserve(total_coords);
    std::vector<double> npos, nq;
    npos.reserve(3 * total_nuclei);
    nq.reserve(total_nuclei);
    for (i64 k = 0; k < ni; ++k) {
        const NuclearJob& j = jobs[k];
        NucInst& in = hosts[k].d;
        for (int a = 0; a < 3; ++a) {
            in.n[a] = (int)j.axes[a].size();
            in.coord_off[a] = (int)coords.size();
            coords.insert(coords.end(), j.axes[a].begin(), j.axes[a].end());
            in.u0[a] = 6 * j.axes[a].front() - h_mmax;
            in.U[a] = 6 * (j.axes[a].back() - j.axes[a].front()) + 2 * h_mmax + 1;
            in.nk[a] = in.n[a] * (in.n[a] + 1) / 2;
        }
        in.N = (i64)in.n[0] * in.n[1] * in.n[2];
        in.nuc0 = (int)nq.size();
        in.nnuc = j.nn;
        for (int q = 0; q < j.nn; ++q) {
            for (int a = 0; a < 3; ++a) npos.push_back(j.nuclei[q].pos[a]);
            nq.push_back((double)j.nuclei[q].charge);
        }
        in.out = j.d_out;
        if ((i64)in.nk[2] * in.nk[1] > ((i64)65535 * TC_BM))
            fail(GLI_ERR_LIMIT, "instance %lld: too many key pairs", (long long)k);
    }
    // chunks: instances whose packed buffers stay under a memory budget (and
    // the weights kernel's grid limit: 3 x instances <= 65535)
    const i64 budget = (i64)4 << 30;  // bytes of packed W, Phi, Vk per chunk
    std::vector<std::pair<i64, i64>> chunks;
    {
        i64 start = 0, bytes = 0;
        for (i64 k = 0; k < ni; ++k) {
            const NucInst& in = hosts[k].d;
            const i64 sz = 8 * ((i64)in.nk[0] * in.U[0] + (i64)in.nk[1] * in.U[1] + (i64)in.nk[2] * in.U[2] +
                                (i64)in.U[0] * in.U[1] * in.U[2] + (i64)in.nk[0] * in.nk[1] * in.nk[2]);
            if (k > start && (bytes + sz > budget || k - start >= 16384)) {
                chunks.push_back({start, k});
                start = k;
                bytes = 0;
            }
            bytes += sz;
        }
        chunks.push_back({start, ni});
    }
    DevBuf<int> d_coords((i64)coords.size(), s);
    DevBuf<double> d_npos((i64)npos.size(), s), d_nq((i64)nq.size(), s);
    GLI_CUDA(cudaMemcpyAsync(d_coords.p, coords.data(), coords.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(d_npos.p, npos.data(), npos.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(d_nq.p, nq.data(), nq.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    DevBuf<NucInst> d_inst(ni, s);
    DevBuf<int> err(1, s);
    err.zero();
    // per chunk: offsets within the chunk's packed buffers, then upload the descriptors
    for (auto& c : chunks) {
        i64 w = 0, phi = 0, vk = 0;
        for (i64 k = c.first; k < c.second; ++k) {
            NucInst& in = hosts[k].d;
            for (int a = 0; a < 3; ++a) {
                in.w_off[a] = w;
                w += (i64)in.nk[a] * in.U[a];
            }
            in.phi_off = phi;
            phi += (i64)in.U[0] * in.U[1] * in.U[2];
            in.vk_off = vk;
            vk += (i64)in.nk[0] * in.nk[1] * in.nk[2];
        }
    }
    std::vector<NucInst> hd(ni);
    for (i64 k = 0; k < ni; ++k) hd[k] = hosts[k].d;
    GLI_CUDA(cudaMemcpyAsync(d_inst.p, hd.data(), ni * sizeof(NucInst), cudaMemcpyHostToDevice, s));
    // the host staging vectors must outlive the copies
    GLI_CUDA(cudaStreamSynchronize(s));

    const Context& ctx = context();
    const bool graphs = getenv("GLI_B200_NO_GRAPHS") == nullptr;
    ensure_streams(ctx.device, 8);
    for (size_t c = 0; c < chunks.size(); ++c) {
        const std::vector<NucHost> part(hosts.begin() + chunks[c].first, hosts.begin() + chunks[c].second);
        const NucInst* dptr = d_inst.p + chunks[c].first;
        // streams for the per-instance contractions and, in the mixed form, the
        // contraction path: chosen by timing the first chunk of a batch of this
        // shape (cached per shape key).  Candidate c: c % 16 streams, c >= 16
        // the int8-sliced tensor-core contractions (mixed form only; they pay
        // only where the GEMMs are large enough to carry the slicing passes)
        char key[160];
        snprintf(key, sizeof(key), "nuclear form=%d dev=%d inst=%zu maxN=%lld", form, ctx.device, part.size(),
                 (long long)std::max_element(part.begin(), part.end(), [](const NucHost& a, const NucHost& b) {
                     return a.d.N < b.d.N;
                 })->d.N);
        auto run = [&](int cand) {
            const bool sliced = cand >= 16;
            const int nstreams = cand % 16;
            if (graphs)
                run_chunk_graph(part, dptr, F.p, nf, (int)nb, d_coords.p, d_npos.p, d_nq.p, sliced, nstreams,
                                ctx.num_sms, err.p, s);
            else
                enqueue_chunk(part, dptr, F.p, nf, (int)nb, d_coords.p, d_npos.p, d_nq.p, sliced, nstreams,
                              ctx.num_sms, err.p, s);
        };
        std::vector<int> cands = part.size() == 1 ? std::vector<int>{1} : std::vector<int>{1, 2, 4, 8};
        if (form == FORM_MIXED)
            for (size_t k = 0, n0 = cands.size(); k < n0; ++k) cands.push_back(16 + cands[k]);
        const int choice = autotune().choose(key, cands, [&](int cand) {
            cudaEvent_t e0, e1;
            GLI_CUDA(cudaEventCreate(&e0));
            GLI_CUDA(cudaEventCreate(&e1));
            GLI_CUDA(cudaEventRecord(e0, s));
            run(cand);
            GLI_CUDA(cudaEventRecord(e1, s));
            GLI_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return (double)ms;
        });
        stats.streams = choice % 16;
        run(choice);
        stats.chunks += 1;
    }
    int h_err = 0;
    GLI_CUDA(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    if (h_err) fail(GLI_ERR_INTERNAL, "tensor-core stage: an mbarrier wait expired (code %d)", h_err);
    stats.instances = ni;
    t_nuc_stats = stats;
}

void nuclear_matrix_device(const double* h_coeffs, i64 nb, const std::vector<int> axes[3],
                           const struct atomic_nucleus* nuclei, int nn, double tol, double* d_out, cudaStream_t s) {
    if (nn <= 0) fail(GLI_ERR_ARGUMENT, "at least one nucleus is required");
    std::vector<NuclearJob> jobs(1);
    for (int a = 0; a < 3; ++a) jobs[0].axes[a] = axes[a];
    jobs[0].nuclei = nuclei;
    jobs[0].nn = nn;
    jobs[0].d_out = d_out;
    nuclear_batch_device(h_coeffs, nb, jobs, tol, FORM_FP64, s);
}

}  // namespace gli
