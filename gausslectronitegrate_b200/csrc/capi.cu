// extern "C" entry points: the reference's C API (include/gli_b200.h part 1)
// and the extensions (part 2).  Every entry point clears the thread's status,
// runs its device work on the thread's stream and, on failure, prints one line
// to stderr, records the status and returns empty results.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>
#include <new>

#include "gli_internal.cuh"

using gli::DevBuf;
using gli::i64;

namespace {

void report() {
    if (!getenv("GLI_B200_QUIET")) fprintf(stderr, "gausslectronitegrate_b200: %s\n", gli::last_message());
}

template <class F>
bool guarded(F&& f) {
    gli::clear_error();
    try {
        f();
        return true;
    } catch (const gli::Failure&) {
    } catch (const std::bad_alloc&) {
        gli::set_error(GLI_ERR_ALLOC, "host allocation failed");
    }
    report();
    return false;
}

template <class T>
T* host_alloc(i64 count) {
    if (count <= 0) return nullptr;
    void* p = aligned_malloc((size_t)count * sizeof(T));
    if (!p) gli::fail(GLI_ERR_ALLOC, "aligned_malloc of %lld bytes failed", (long long)(count * sizeof(T)));
    return (T*)p;
}


// Large device -> host copies into pageable memory (dense kinetic and nuclear
// matrices, dense tensors: up to GBs) go through two page-locked staging
// buffers: the DMA of one chunk overlaps the host copy of the previous one,
// which is split over a few threads (one core's memcpy into freshly mapped
// pages runs far below the link's rate).  Synchronous; smaller copies are one
// asynchronous cudaMemcpyAsync on the stream.
struct StagedD2H {
    static constexpr size_t kChunk = (size_t)32 << 20;
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void ensure() {
        for (int k = 0; k < 2; ++k) {
            if (!pin[k]) GLI_CUDA(cudaHostAlloc(&pin[k], kChunk, cudaHostAllocDefault));
            if (!ev[k]) GLI_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
        }
    }
    ~StagedD2H() {
        for (int k = 0; k < 2; ++k) {
            if (pin[k]) cudaFreeHost(pin[k]);
            if (ev[k]) cudaEventDestroy(ev[k]);
        }
    }
};
static thread_local StagedD2H t_staged;

static void parallel_memcpy(void* dst, const void* src, size_t bytes) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::min<size_t>(std::min<size_t>(8, hw > 1 ? hw / 2 : 1), std::max<size_t>(1, bytes >> 22));
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

template <class T>
void to_host(T* h, const T* d, i64 n, cudaStream_t s) {
    const size_t bytes = (size_t)n * sizeof(T);
    if (bytes < 2 * StagedD2H::kChunk) {
        if (n) GLI_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
        return;
    }
    t_staged.ensure();
    const size_t chunks = (bytes + StagedD2H::kChunk - 1) / StagedD2H::kChunk;
    for (size_t c = 0; c <= chunks; ++c) {
        if (c < chunks) {
            const size_t off = c * StagedD2H::kChunk, len = std::min(StagedD2H::kChunk, bytes - off);
            GLI_CUDA(cudaMemcpyAsync(t_staged.pin[c & 1], (const char*)d + off, len, cudaMemcpyDeviceToHost, s));
            GLI_CUDA(cudaEventRecord(t_staged.ev[c & 1], s));
        }
        if (c > 0) {  // the previous chunk: wait for its DMA, copy it out of the staging buffer
            const size_t p = c - 1, off = p * StagedD2H::kChunk, len = std::min(StagedD2H::kChunk, bytes - off);
            GLI_CUDA(cudaEventSynchronize(t_staged.ev[p & 1]));
            parallel_memcpy((char*)h + off, t_staged.pin[p & 1], len);
        }
    }
}

static bool host_pinned(const void* p) {
    cudaPointerAttributes a = {};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host -> device copies of long arrays in pageable memory (class lists and
// values of the reference-facing calls: tens of MB) go through the same two
// page-locked staging buffers: the host copy of one chunk, split over a few
// threads, overlaps the DMA of the previous one.  Returns with the last DMAs
// queued on s (the buffers are not rewritten before their events complete).
template <class T>
void to_device(DevBuf<T>& d, const T* h, i64 n, cudaStream_t s) {
    d.alloc(n, s);
    const size_t bytes = (size_t)n * sizeof(T);
    constexpr size_t kChunk = (size_t)16 << 20;
    if (bytes < kChunk || host_pinned(h)) {
        if (n) GLI_CUDA(cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    t_staged.ensure();
    for (int k = 0; k < 2; ++k) GLI_CUDA(cudaEventSynchronize(t_staged.ev[k]));  // earlier uses of the buffers
    const size_t chunks = (bytes + kChunk - 1) / kChunk;
    for (size_t c = 0; c < chunks; ++c) {
        const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
        const int k = (int)(c & 1);
        if (c >= 2) GLI_CUDA(cudaEventSynchronize(t_staged.ev[k]));  // the buffer's previous DMA is done
        parallel_memcpy(t_staged.pin[k], (const char*)h + off, len);
        GLI_CUDA(cudaMemcpyAsync((char*)d.p + off, t_staged.pin[k], len, cudaMemcpyHostToDevice, s));
        GLI_CUDA(cudaEventRecord(t_staged.ev[k], s));
    }
}

void check_gdata(const struct gausslet_data* g) {
    if (!g || !g->coefficients || g->indices.num <= 0 || g->indices.num % 2 != 1)
        gli::fail(GLI_ERR_ARGUMENT, "gausslet data must hold an odd, positive number of coefficients");
    if (g->indices.istart != -(g->indices.num - 1) / 2)
        gli::fail(GLI_ERR_ARGUMENT, "gausslet coefficient indices must be centred (istart = -(num-1)/2)");
}

// smallest grid holding the given points (for the single-entry forms)
gli::GridDesc grid_around(const union cartesian_grid_point_3d* pts, int np) {
    gli::GridDesc g;
    for (int a = 0; a < 3; ++a) {
        i64 lo = pts[0].c[a], hi = pts[0].c[a];
        for (int k = 1; k < np; ++k) {
            lo = lmin(lo, pts[k].c[a]);
            hi = lmax(hi, pts[k].c[a]);
        }
        g.istart[a] = lo;
        g.num[a] = hi - lo + 1;
    }
    return g;
}

i64 lin_of(const gli::GridDesc& g, const union cartesian_grid_point_3d& p) {
    return ((p.x - g.istart[0]) * g.num[1] + (p.y - g.istart[1])) * g.num[2] + (p.z - g.istart[2]);
}

struct cartesian_grid_3d grid_struct(const gli::GridDesc& g) {
    struct cartesian_grid_3d r;
    for (int a = 0; a < 3; ++a) {
        r.coord_range[a].istart = g.istart[a];
        r.coord_range[a].num = g.num[a];
    }
    return r;
}

// one class on a grid spanning the points, evaluated by the staged contraction
double single_class(int kind, const struct gausslet_data* gdata, const union cartesian_grid_point_3d* pts, double tol) {
    check_gdata(gdata);
    const gli::GridDesc g = grid_around(pts, kind ? 4 : 2);
    const i64 N = g.points();
    i64 idx;
    if (kind == 0) {
        idx = lin_of(g, pts[0]) * N + lin_of(g, pts[1]);
    } else {
        if (N > 55000) gli::fail(GLI_ERR_LIMIT, "points span too many grid points for a four-index class");
        idx = ((lin_of(g, pts[0]) * N + lin_of(g, pts[1])) * N + lin_of(g, pts[2])) * N + lin_of(g, pts[3]);
    }
    gli::Context& ctx = gli::context();
    cudaStream_t s = ctx.stream;
    DevBuf<int64_t> d_idx(1, s);
    DevBuf<double> d_out(1, s);
    GLI_CUDA(cudaMemcpyAsync(d_idx.p, &idx, sizeof(idx), cudaMemcpyHostToDevice, s));
    gli::sparse_values_device(kind, gdata->coefficients, gdata->indices.num, g, d_idx.p, 1, tol, gli::FORM_FP64,
                              d_out.p, s, nullptr);
    double v = 0;
    to_host(&v, d_out.p, 1, s);
    GLI_CUDA(cudaStreamSynchronize(s));
    return v;
}

template <class Sparse, class IdxField>
void sparse_compute(int kind, const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid,
                    const glong* indices, glong num, double tol, int form, Sparse* out, IdxField idx_field) {
    out->grid = *grid;
    out->integral_values = nullptr;
    out->*idx_field = nullptr;
    out->num_entries = 0;
    guarded([&] {
        check_gdata(gdata);
        if (num < 0 || (num > 0 && !indices)) gli::fail(GLI_ERR_ARGUMENT, "invalid index list");
        const gli::GridDesc g = gli::grid_desc(grid);
        glong* h_idx = host_alloc<glong>(num);
        double* h_val = host_alloc<double>(num);
        if (num) memcpy(h_idx, indices, num * sizeof(glong));
        try {
            if (num) {
                gli::Context& ctx = gli::context();
                gli::sparse_values_host(kind, gdata->coefficients, gdata->indices.num, g, (const int64_t*)indices, num,
                                        tol, form, h_val, ctx.stream);
            }
        } catch (...) {
            aligned_free(h_idx);
            aligned_free(h_val);
            throw;
        }
        out->integral_values = h_val;
        out->*idx_field = h_idx;
        out->num_entries = num;
    });
}

template <class Indices, class IdxField>
void enumerate_host(int kind, const struct cartesian_grid_3d* grid, Indices* ret, IdxField field) {
    ret->grid = *grid;
    ret->*field = nullptr;
    ret->num = 0;
    guarded([&] {
        const gli::GridDesc g = gli::grid_desc(grid);
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        int64_t* d = nullptr;
        const i64 n = gli::enumerate_device(kind, g, &d, s);
        glong* h = nullptr;
        try {
            h = host_alloc<glong>(n);
            to_host((int64_t*)h, d, n, s);
            GLI_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaFreeAsync(d, s);
            aligned_free(h);
            throw;
        }
        cudaFreeAsync(d, s);
        ret->*field = h;
        ret->num = n;
    });
}

double sorted_lookup(const glong* idx, const double* val, glong m, glong key) {
    glong lo = 0, hi = m;
    while (lo < hi) {
        const glong mid = (lo + hi) / 2;
        if (key < idx[mid]) hi = mid;
        else if (key > idx[mid]) lo = mid + 1;
        else return val[mid];
    }
    return 0;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// status and device selection
int gli_b200_last_error(void) { return gli::last_error(); }
const char* gli_b200_last_error_message(void) { return gli::last_message(); }
const char* gli_b200_version(void) { return "0.1.0"; }

int gli_b200_device_count(void) {
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return c;
}

int gli_b200_set_device(int ordinal) {
    gli::clear_error();
    if (ordinal < 0) {
        gli::set_error(GLI_ERR_ARGUMENT, "negative device ordinal");
        return GLI_ERR_ARGUMENT;
    }
    return gli::set_device(ordinal);
}

long long gli_b200_launch_count(void) { return gli::launch_count(); }

int gli_b200_measure_fp64_peak(double* tflops) {
    *tflops = 0;
    guarded([&] { *tflops = gli::fp64_probe_tflops(); });
    return gli::last_error();
}

int gli_b200_set_timing(int enable) {
    gli::set_timing(enable != 0);
    return GLI_OK;
}

int gli_b200_last_stage_times(float ms[4], glong sizes[3]) {
    const gli::ContractStats& st = gli::last_stats();
    if (ms) {
        ms[0] = st.ms_tables;
        ms[1] = st.ms_a;
        ms[2] = st.ms_b;
        ms[3] = st.ms_c;
    }
    if (sizes) {
        sizes[0] = st.keys_a;
        sizes[1] = st.pairs;
        sizes[2] = st.U;
    }
    return GLI_OK;
}

int gli_b200_last_stage_c_times(float ms[2]) {
    const gli::ContractStats& st = gli::last_stats();
    ms[0] = st.ms_c_product;
    ms[1] = st.ms_c_class;
    return GLI_OK;
}

int gli_b200_last_plan(glong out[4]) {
    const gli::ContractStats& st = gli::last_stats();
    out[0] = st.keys_a;
    out[1] = st.pairs;
    out[2] = st.keys_used;
    out[3] = st.product ? std::max<i64>(1, st.products) : 0;
    return GLI_OK;
}

int gli_b200_last_paths(int out[3]) {
    const gli::ContractStats& st = gli::last_stats();
    out[0] = st.tc_a;
    out[1] = st.tc_b;
    out[2] = st.product ? (st.gather ? st.gather : 1) : 0;
    return GLI_OK;
}

int gli_b200_last_screening(double out[2]) {
    const gli::ContractStats& st = gli::last_stats();
    out[0] = st.screen_tol;
    out[1] = st.screen_bound;
    return GLI_OK;
}

int gli_b200_clear_caches(void) {
    gli::clear_error();
    try {
        gli::clear_eval_caches();
        gli::clear_table_cache();
    } catch (const gli::Failure&) {
    }
    return gli::last_error();
}

// ---------------------------------------------------------------------------
// kinetic (reference src/kinetic_integrals.c)
void compute_kinetic_gausslet_integrals(const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid,
                                        struct kinetic_gausslet_integrals* kgi) {
    kgi->grid = *grid;
    kgi->integral_values = nullptr;
    guarded([&] {
        check_gdata(gdata);
        const gli::GridDesc g = gli::grid_desc(grid);
        const i64 N = g.points();
        double* h = host_alloc<double>(N * N);
        try {
            gli::Context& ctx = gli::context();
            cudaStream_t s = ctx.stream;
            DevBuf<double> d(N * N, s);
            gli::kinetic_matrix_device(gdata->coefficients, gdata->indices.num, g, d.p, s);
            to_host(h, d.p, N * N, s);
            GLI_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            aligned_free(h);
            throw;
        }
        kgi->integral_values = h;
    });
}

void delete_kinetic_gausslet_integrals(struct kinetic_gausslet_integrals* kgi) {
    aligned_free(kgi->integral_values);
    kgi->integral_values = nullptr;
}

double compute_kinetic_gausslet_integral(const struct gausslet_data* gdata,
                                         const union cartesian_grid_point_3d points[2]) {
    double v = NAN;
    guarded([&] {
        check_gdata(gdata);
        const gli::GridDesc g = grid_around(points, 2);
        // a 1 x 1 x 1 grid per axis pair is enough: the entry only needs the
        // three axis distances, evaluated on the device as one matrix entry of
        // the per-axis grids below
        gli::GridDesc gx = g;
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        const i64 L = gx.max_range();
        DevBuf<double> k1(L, s);
        gli::kinetic_table_device(gdata->coefficients, gdata->indices.num, L, k1.p, s);
        std::vector<double> h(L);
        to_host(h.data(), k1.p, L, s);
        GLI_CUDA(cudaStreamSynchronize(s));
        const i64 dx = llabs(points[0].x - points[1].x), dy = llabs(points[0].y - points[1].y),
                  dz = llabs(points[0].z - points[1].z);
        v = h[dx] * (dy == 0) * (dz == 0) + (dx == 0) * h[dy] * (dz == 0) + (dx == 0) * (dy == 0) * h[dz];
    });
    return v;
}

// ---------------------------------------------------------------------------
// nuclear attraction (reference src/nuclear_integrals.c)
void compute_nuclear_gausslet_integrals(const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid,
                                        const struct atomic_nucleus* nuclei, const int num_nuclei, const double tol,
                                        struct nuclear_gausslet_integrals* ngi) {
    ngi->grid = *grid;
    ngi->integral_values = nullptr;
    ngi->nuclei = nullptr;
    ngi->num_nuclei = 0;
    guarded([&] {
        check_gdata(gdata);
        if (num_nuclei <= 0 || !nuclei) gli::fail(GLI_ERR_ARGUMENT, "at least one nucleus is required");
        const gli::GridDesc g = gli::grid_desc(grid);
        std::vector<int> axes[3];
        for (int a = 0; a < 3; ++a)
            for (i64 k = 0; k < g.num[a]; ++k) axes[a].push_back((int)(g.istart[a] + k));
        const i64 N = g.points();
        double* h = host_alloc<double>(N * N);
        struct atomic_nucleus* hn = nullptr;
        try {
            hn = host_alloc<struct atomic_nucleus>(num_nuclei);
            memcpy(hn, nuclei, num_nuclei * sizeof(*hn));
            gli::Context& ctx = gli::context();
            cudaStream_t s = ctx.stream;
            DevBuf<double> d(N * N, s);
            gli::nuclear_matrix_device(gdata->coefficients, gdata->indices.num, axes, nuclei, num_nuclei, tol, d.p, s);
            to_host(h, d.p, N * N, s);
            GLI_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            aligned_free(h);
            aligned_free(hn);
            throw;
        }
        ngi->integral_values = h;
        ngi->nuclei = hn;
        ngi->num_nuclei = num_nuclei;
    });
}

void delete_nuclear_gausslet_integrals(struct nuclear_gausslet_integrals* ngi) {
    aligned_free(ngi->integral_values);
    aligned_free(ngi->nuclei);
    ngi->integral_values = nullptr;
    ngi->nuclei = nullptr;
    ngi->num_nuclei = 0;
}

double compute_nuclear_gausslet_integral(const struct gausslet_data* gdata,
                                         const union cartesian_grid_point_3d points[2],
                                         const struct atomic_nucleus* nuclei, const int num_nuclei, const double tol) {
    double v = NAN;
    guarded([&] {
        check_gdata(gdata);
        if (num_nuclei <= 0 || !nuclei) gli::fail(GLI_ERR_ARGUMENT, "at least one nucleus is required");
        // per axis the (one or two) distinct coordinates of the two points
        std::vector<int> axes[3];
        int ia[3], ja[3];
        for (int a = 0; a < 3; ++a) {
            const int x = (int)points[0].c[a], y = (int)points[1].c[a];
            axes[a].push_back(std::min(x, y));
            if (x != y) axes[a].push_back(std::max(x, y));
            ia[a] = x <= y ? 0 : 1;
            ja[a] = (x == y) ? 0 : (y > x ? 1 : 0);
        }
        const int n[3] = {(int)axes[0].size(), (int)axes[1].size(), (int)axes[2].size()};
        const i64 N = (i64)n[0] * n[1] * n[2];
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        DevBuf<double> d(N * N, s);
        gli::nuclear_matrix_device(gdata->coefficients, gdata->indices.num, axes, nuclei, num_nuclei, tol, d.p, s);
        std::vector<double> h(N * N);
        to_host(h.data(), d.p, N * N, s);
        GLI_CUDA(cudaStreamSynchronize(s));
        const i64 i = ((i64)ia[0] * n[1] + ia[1]) * n[2] + ia[2];
        const i64 j = ((i64)ja[0] * n[1] + ja[1]) * n[2] + ja[2];
        v = h[i * N + j];
    });
    return v;
}

// ---------------------------------------------------------------------------
// ERIDA (reference src/erida_integrals.c)
void enumerate_symmetry_reduced_erida_indices(const struct cartesian_grid_3d* grid, struct sparse_erida_indices* ret) {
    enumerate_host(0, grid, ret, &sparse_erida_indices::two_indices);
}

void delete_sparse_erida_indices(struct sparse_erida_indices* indices) {
    aligned_free(indices->two_indices);
    indices->two_indices = nullptr;
    indices->num = 0;
}

void compute_sparse_erida_gausslet_integrals(const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid,
                                             const glong* two_indices, const glong num_indices, const double tol,
                                             struct sparse_erida_gausslet_integrals* erida) {
    sparse_compute(0, gdata, grid, two_indices, num_indices, tol, gli::FORM_FP64, erida,
                   &sparse_erida_gausslet_integrals::two_indices);
}

double compute_erida_gausslet_integral(const struct gausslet_data* gdata, const union cartesian_grid_point_3d points[2],
                                       const double tol) {
    double v = NAN;
    guarded([&] { v = single_class(0, gdata, points, tol); });
    return v;
}

double sparse_erida_gausslet_integrals_get_value(const struct sparse_erida_gausslet_integrals* erida,
                                                 const glong index) {
    return sorted_lookup(erida->two_indices, erida->integral_values, erida->num_entries, index);
}

glong minimum_octahedral_orbit_erida_tensor_index(const glong num_points, const glong* octahedral_perm[48],
                                                  const glong i, const glong j) {
    glong best = GLONG_MAX;
    for (int n = 0; n < 48; ++n) {
        const glong a = octahedral_perm[n][i], b = octahedral_perm[n][j];
        const glong v = a <= b ? a * num_points + b : b * num_points + a;
        best = lmin(best, v);
    }
    return best;
}

void fill_dense_erida_matrix(const struct sparse_erida_gausslet_integrals* erida,
                             const struct cartesian_grid_3d* grid_dense, double* erida_matrix) {
    guarded([&] {
        const gli::GridDesc gs = gli::grid_desc(&erida->grid), gd = gli::grid_desc(grid_dense);
        const i64 N = gd.points();
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        DevBuf<int64_t> di;
        DevBuf<double> dv, out(N * N, s);
        to_device(di, (const int64_t*)erida->two_indices, erida->num_entries, s);
        to_device(dv, (const double*)erida->integral_values, erida->num_entries, s);
        gli::fill_dense_device(0, gs, di.p, dv.p, erida->num_entries, gd, out.p, s);
        to_host(erida_matrix, out.p, N * N, s);
        GLI_CUDA(cudaStreamSynchronize(s));
    });
}

void project_sparse_erida_gausslet_integrals(const struct sparse_erida_gausslet_integrals* erida, const double* basis,
                                             const glong num_states, double* eri_proj) {
    guarded([&] {
        const gli::GridDesc g = gli::grid_desc(&erida->grid);
        const i64 N = g.points(), M = num_states;
        if (M <= 0) gli::fail(GLI_ERR_ARGUMENT, "number of basis states must be positive");
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        DevBuf<int64_t> di;
        DevBuf<double> dv, db, out(M * M * M * M, s);
        to_device(di, (const int64_t*)erida->two_indices, erida->num_entries, s);
        to_device(dv, (const double*)erida->integral_values, erida->num_entries, s);
        to_device(db, basis, N * M, s);
        gli::project_device(0, g, di.p, dv.p, erida->num_entries, db.p, M, out.p, s);
        to_host(eri_proj, out.p, M * M * M * M, s);
        GLI_CUDA(cudaStreamSynchronize(s));
    });
}

void delete_sparse_erida_gausslet_integrals(struct sparse_erida_gausslet_integrals* erida) {
    aligned_free(erida->two_indices);
    aligned_free(erida->integral_values);
    erida->two_indices = nullptr;
    erida->integral_values = nullptr;
    erida->num_entries = 0;
}

// ---------------------------------------------------------------------------
// ERI (reference src/eri_integrals.c)
void enumerate_symmetry_reduced_eri_indices(const struct cartesian_grid_3d* grid, struct sparse_eri_indices* ret) {
    enumerate_host(1, grid, ret, &sparse_eri_indices::four_indices);
}

void delete_sparse_eri_indices(struct sparse_eri_indices* indices) {
    aligned_free(indices->four_indices);
    indices->four_indices = nullptr;
    indices->num = 0;
}

void compute_sparse_eri_gausslet_integrals(const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid,
                                           const glong* four_indices, const glong num_indices, const double tol,
                                           struct sparse_eri_gausslet_integrals* eri) {
    sparse_compute(1, gdata, grid, four_indices, num_indices, tol, gli::FORM_FP64, eri,
                   &sparse_eri_gausslet_integrals::four_indices);
}

double compute_eri_gausslet_integral(const struct gausslet_data* gdata, const union cartesian_grid_point_3d points[4],
                                     const double tol) {
    double v = NAN;
    guarded([&] { v = single_class(1, gdata, points, tol); });
    return v;
}

double sparse_eri_gausslet_integrals_get_value(const struct sparse_eri_gausslet_integrals* eri, const glong index) {
    return sorted_lookup(eri->four_indices, eri->integral_values, eri->num_entries, index);
}

glong minimum_octahedral_orbit_eri_tensor_index(const glong num_points, const glong* octahedral_perm[48],
                                                const glong i, const glong j, const glong k, const glong l) {
    glong best = GLONG_MAX;
    for (int n = 0; n < 48; ++n) {
        glong a = octahedral_perm[n][i], b = octahedral_perm[n][j], c = octahedral_perm[n][k], d = octahedral_perm[n][l];
        glong ab = a <= b ? a * num_points + b : b * num_points + a;
        glong cd = c <= d ? c * num_points + d : d * num_points + c;
        if (ab > cd) {
            const glong t = ab;
            ab = cd;
            cd = t;
        }
        best = lmin(best, ab * (num_points * num_points) + cd);
    }
    return best;
}

void fill_dense_eri_tensor(const struct sparse_eri_gausslet_integrals* eri, const struct cartesian_grid_3d* grid_dense,
                           double* eri_tensor) {
    guarded([&] {
        const gli::GridDesc gs = gli::grid_desc(&eri->grid), gd = gli::grid_desc(grid_dense);
        const i64 N = gd.points();
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        DevBuf<int64_t> di;
        DevBuf<double> dv, out(N * N * N * N, s);
        to_device(di, (const int64_t*)eri->four_indices, eri->num_entries, s);
        to_device(dv, (const double*)eri->integral_values, eri->num_entries, s);
        gli::fill_dense_device(1, gs, di.p, dv.p, eri->num_entries, gd, out.p, s);
        to_host(eri_tensor, out.p, N * N * N * N, s);
        GLI_CUDA(cudaStreamSynchronize(s));
    });
}

void apply_sparse_eri_tensor(const struct sparse_eri_gausslet_integrals* eri, const double* states,
                             const glong num_states, double* ret) {
    guarded([&] {
        const gli::GridDesc g = gli::grid_desc(&eri->grid);
        const i64 N = g.points(), ns = num_states;
        if (ns <= 0) gli::fail(GLI_ERR_ARGUMENT, "number of states must be positive");
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        DevBuf<int64_t> di;
        DevBuf<double> dv, dst, out(N * N * ns, s);
        to_device(di, (const int64_t*)eri->four_indices, eri->num_entries, s);
        to_device(dv, (const double*)eri->integral_values, eri->num_entries, s);
        to_device(dst, states, N * N * ns, s);
        gli::apply_eri_device(g, di.p, dv.p, eri->num_entries, dst.p, ns, out.p, s);
        to_host(ret, out.p, N * N * ns, s);
        GLI_CUDA(cudaStreamSynchronize(s));
    });
}

void project_sparse_eri_gausslet_integrals(const struct sparse_eri_gausslet_integrals* eri, const double* basis,
                                           const glong num_states, double* eri_proj) {
    guarded([&] {
        const gli::GridDesc g = gli::grid_desc(&eri->grid);
        const i64 N = g.points(), M = num_states;
        if (M <= 0) gli::fail(GLI_ERR_ARGUMENT, "number of basis states must be positive");
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        DevBuf<int64_t> di;
        DevBuf<double> dv, db, out(M * M * M * M, s);
        to_device(di, (const int64_t*)eri->four_indices, eri->num_entries, s);
        to_device(dv, (const double*)eri->integral_values, eri->num_entries, s);
        to_device(db, basis, N * M, s);
        gli::project_device(1, g, di.p, dv.p, eri->num_entries, db.p, M, out.p, s);
        to_host(eri_proj, out.p, M * M * M * M, s);
        GLI_CUDA(cudaStreamSynchronize(s));
    });
}

void delete_sparse_eri_gausslet_integrals(struct sparse_eri_gausslet_integrals* eri) {
    aligned_free(eri->four_indices);
    aligned_free(eri->integral_values);
    eri->four_indices = nullptr;
    eri->integral_values = nullptr;
    eri->num_entries = 0;
}

// ---------------------------------------------------------------------------
// O_h grid permutations (reference src/symmetry.c:141-150)
void evaluate_octahedral_grid_permutations(const struct cartesian_grid_3d* grid, glong* perm[48]) {
    for (int g = 0; g < 48; ++g) perm[g] = nullptr;
    guarded([&] {
        const gli::GridDesc g = gli::grid_desc(grid);
        const i64 N = g.points();
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        DevBuf<int64_t> d(48 * N, s);
        gli::grid_perms_device(g, d.p, s);
        std::vector<glong*> h(48, nullptr);
        try {
            for (int k = 0; k < 48; ++k) {
                h[k] = host_alloc<glong>(N);
                to_host((int64_t*)h[k], d.p + k * N, N, s);
            }
            GLI_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            for (auto p : h) aligned_free(p);
            throw;
        }
        for (int k = 0; k < 48; ++k) perm[k] = h[k];
    });
}

// ---------------------------------------------------------------------------
// extensions
int gli_b200_sparse_values_dev(int kind, const double* coeffs, glong num_coeffs, const struct cartesian_grid_3d* grid,
                               const glong* d_indices, glong num, double tol, int form, double* d_values,
                               void* stream) {
    guarded([&] {
        if (kind != 0 && kind != 1) gli::fail(GLI_ERR_ARGUMENT, "kind must be 0 (ERIDA) or 1 (ERI)");
        if (!coeffs) gli::fail(GLI_ERR_ARGUMENT, "coefficients missing");
        const gli::GridDesc g = gli::grid_desc(grid);
        gli::Context& ctx = gli::context();
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx.stream;
        gli::sparse_values_device(kind, coeffs, num_coeffs, g, (const int64_t*)d_indices, num, tol, form, d_values, s,
                                  nullptr);
    });
    return gli::last_error();
}

// The same evaluation queued on the stream without a host wait (stream order:
// no synchronisation inside once the list's graph exists); the ticket is
// passed to gli_b200_sparse_values_wait, which reads the status.
int gli_b200_sparse_values_dev_async(int kind, const double* coeffs, glong num_coeffs,
                                     const struct cartesian_grid_3d* grid, const glong* d_indices, glong num,
                                     double tol, int form, double* d_values, void* stream, glong* ticket) {
    guarded([&] {
        if (kind != 0 && kind != 1) gli::fail(GLI_ERR_ARGUMENT, "kind must be 0 (ERIDA) or 1 (ERI)");
        if (!coeffs) gli::fail(GLI_ERR_ARGUMENT, "coefficients missing");
        if (!ticket) gli::fail(GLI_ERR_ARGUMENT, "ticket missing");
        if (num < 0) gli::fail(GLI_ERR_ARGUMENT, "num must be non-negative");
        const gli::GridDesc g = gli::grid_desc(grid);
        gli::Context& ctx = gli::context();
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx.stream;
        *ticket = gli::sparse_values_device_async(kind, coeffs, num_coeffs, g, (const int64_t*)d_indices, num, tol,
                                                  form, d_values, s);
    });
    return gli::last_error();
}

int gli_b200_sparse_values_wait(glong ticket) {
    guarded([&] { gli::sparse_values_wait(ticket); });
    return gli::last_error();
}

// Batched nuclear-attraction matrices: every instance its own grid and nuclei
// (same coefficients and tol), outputs in device memory.  Batches the matrix
// entry point compute_nuclear_gausslet_integrals (reference
// src/nuclear_integrals.c:133-266).
int gli_b200_nuclear_batch_dev(const struct gausslet_data* gdata, glong num_instances,
                               const struct cartesian_grid_3d* grids, const glong* nuclei_offsets,
                               const struct atomic_nucleus* nuclei, double tol, int form, double* const* d_out,
                               void* stream) {
    guarded([&] {
        check_gdata(gdata);
        if (num_instances < 0) gli::fail(GLI_ERR_ARGUMENT, "num_instances must be non-negative");
        if (num_instances == 0) return;
        if (!grids || !nuclei_offsets || !nuclei || !d_out) gli::fail(GLI_ERR_ARGUMENT, "batch arrays missing");
        std::vector<gli::NuclearJob> jobs((size_t)num_instances);
        for (glong k = 0; k < num_instances; ++k) {
            const gli::GridDesc g = gli::grid_desc(&grids[k]);
            for (int a = 0; a < 3; ++a)
                for (i64 c = 0; c < g.num[a]; ++c) jobs[k].axes[a].push_back((int)(g.istart[a] + c));
            const glong n0 = nuclei_offsets[k], n1 = nuclei_offsets[k + 1];
            if (n1 <= n0) gli::fail(GLI_ERR_ARGUMENT, "instance %lld has no nuclei", (long long)k);
            jobs[k].nuclei = nuclei + n0;
            jobs[k].nn = (int)(n1 - n0);
            jobs[k].d_out = d_out[k];
        }
        gli::Context& ctx = gli::context();
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx.stream;
        gli::nuclear_batch_device(gdata->coefficients, gdata->indices.num, jobs, tol, form, s);
    });
    return gli::last_error();
}

// The same batch with host outputs: h_out[k] receives instance k's N_k x N_k
// matrix (the device copies are made and released inside the call).
int gli_b200_nuclear_batch(const struct gausslet_data* gdata, glong num_instances,
                           const struct cartesian_grid_3d* grids, const glong* nuclei_offsets,
                           const struct atomic_nucleus* nuclei, double tol, int form, double* const* h_out) {
    guarded([&] {
        if (num_instances <= 0) return;
        if (!grids || !h_out) gli::fail(GLI_ERR_ARGUMENT, "batch arrays missing");
        gli::Context& ctx = gli::context();
        cudaStream_t s = ctx.stream;
        std::vector<DevBuf<double>> dev((size_t)num_instances);
        std::vector<double*> dptr((size_t)num_instances);
        std::vector<i64> n2((size_t)num_instances);
        for (glong k = 0; k < num_instances; ++k) {
            const gli::GridDesc g = gli::grid_desc(&grids[k]);
            n2[k] = g.points() * g.points();
            dev[k].alloc(n2[k], s);
            dptr[k] = dev[k].p;
        }
        if (gli_b200_nuclear_batch_dev(gdata, num_instances, grids, nuclei_offsets, nuclei, tol, form, dptr.data(),
                                       s) != GLI_OK)
            throw gli::Failure{gli::last_error()};
        for (glong k = 0; k < num_instances; ++k) to_host(h_out[k], dev[k].p, n2[k], s);
        GLI_CUDA(cudaStreamSynchronize(s));
    });
    return gli::last_error();
}

// instances, graph chunks and contraction streams of the last nuclear batch
void gli_b200_last_nuclear_batch(glong out[3]) {
    const gli::NuclearBatchStats& st = gli::last_nuclear_stats();
    out[0] = st.instances;
    out[1] = st.chunks;
    out[2] = st.streams;
}

int gli_b200_sparse_values(int kind, const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid,
                           const glong* indices, glong num, double tol, int form, double* values) {
    guarded([&] {
        if (kind != 0 && kind != 1) gli::fail(GLI_ERR_ARGUMENT, "kind must be 0 (ERIDA) or 1 (ERI)");
        check_gdata(gdata);
        const gli::GridDesc g = gli::grid_desc(grid);
        if (num <= 0) return;
        if (!indices || !values) gli::fail(GLI_ERR_ARGUMENT, "indices and values must not be NULL");
        gli::Context& ctx = gli::context();
        gli::sparse_values_host(kind, gdata->coefficients, gdata->indices.num, g, (const int64_t*)indices, num, tol,
                                form, values, ctx.stream);
    });
    return gli::last_error();
}

int gli_b200_enumerate_dev(int kind, const struct cartesian_grid_3d* grid, glong** d_indices, glong* num,
                           void* stream) {
    *d_indices = nullptr;
    *num = 0;
    guarded([&] {
        if (kind != 0 && kind != 1) gli::fail(GLI_ERR_ARGUMENT, "kind must be 0 (ERIDA) or 1 (ERI)");
        const gli::GridDesc g = gli::grid_desc(grid);
        gli::Context& ctx = gli::context();
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx.stream;
        int64_t* d = nullptr;
        *num = gli::enumerate_device(kind, g, &d, s);
        *d_indices = (glong*)d;
    });
    return gli::last_error();
}

int gli_b200_free_dev(void* d_ptr, void* stream) {
    guarded([&] {
        gli::Context& ctx = gli::context();
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx.stream;
        if (d_ptr) GLI_CUDA(cudaFreeAsync(d_ptr, s));
    });
    return gli::last_error();
}

}  // extern "C"
