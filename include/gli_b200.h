/*
 * gli_b200.h -- C ABI of libgli_b200, a B200 (sm_100a) implementation of the
 * gausslectronitegrate integral hot path.
 *
 * Part 1 declares the reference's own C interface with identical prototypes
 * and struct layouts, so that code written against the reference headers
 * (include/{eri,erida,nuclear,kinetic}_integrals.h, grid.h, range.h,
 * gausslet.h, symmetry.h, aligned_memory.h of the reference) links against
 * this library unchanged; the compatibility headers next to this file carry
 * the reference's header names and include this one.  Every bulk computation
 * runs in CUDA kernels on the GPU; there is no CPU fallback.  Results handed
 * back inside the reference structs are host memory from aligned_malloc(),
 * released by the matching delete_* call, exactly as in the reference.
 *
 * Part 2 declares extensions: error status, device-resident entry points
 * (class lists and values kept in HBM) and the precision form switch.
 *
 * Errors: the reference API returns void.  On failure (no CUDA device, a
 * CUDA error, an argument the reference would silently mis-handle such as a
 * non-symmetric grid for the symmetry-reduced paths) the call prints one line
 * to stderr, leaves the result empty (NULL arrays, zero counts) and records a
 * status readable with gli_b200_last_error() / gli_b200_last_error_message().
 */
#ifndef GLI_B200_H
#define GLI_B200_H

#include <assert.h>
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Part 1: types of the reference interface (same layout, own code)
 * ---------------------------------------------------------------------- */

/* universal integer, reference include/util.h:10 */
typedef int64_t glong;
#ifndef GLONG_MAX
#define GLONG_MAX INT64_MAX
#endif

/* reference include/range.h:10-14 */
struct range {
	glong istart;  /* first integer */
	glong num;     /* number of integers */
};

/* reference include/grid.h:10-17 */
union cartesian_grid_point_3d {
	struct {
		glong x, y, z;
	};
	glong c[3];
};

/* reference include/grid.h:23-26 */
struct cartesian_grid_3d {
	struct range coord_range[3];  /* x, y, z axes: first coordinate and count */
};

/* reference include/gausslet.h:10-14 */
struct gausslet_data {
	double* coefficients;  /* coefficients b_j of the elementary Gaussians */
	struct range indices;  /* j range, istart = -(num-1)/2 for the odd sets used */
};

/* reference include/nuclear_integrals.h:11-15 */
struct atomic_nucleus {
	double pos[3];  /* position in grid units */
	int charge;
};

/* reference include/kinetic_integrals.h:14-18 */
struct kinetic_gausslet_integrals {
	double* integral_values;  /* dense N x N, row-major */
	struct cartesian_grid_3d grid;
};

/* reference include/nuclear_integrals.h:31-37 */
struct nuclear_gausslet_integrals {
	double* integral_values;  /* dense N x N, row-major */
	struct cartesian_grid_3d grid;
	struct atomic_nucleus* nuclei;
	int num_nuclei;
};

/* reference include/eri_integrals.h:23-28 */
struct sparse_eri_indices {
	glong* four_indices;  /* ((i N + j) N + k) N + l, sorted ascending */
	glong num;
	struct cartesian_grid_3d grid;
};

/* reference include/eri_integrals.h:41-47 */
struct sparse_eri_gausslet_integrals {
	double* integral_values;
	glong* four_indices;
	glong num_entries;
	struct cartesian_grid_3d grid;
};

/* reference include/erida_integrals.h:21-26 */
struct sparse_erida_indices {
	glong* two_indices;  /* i N + j, sorted ascending */
	glong num;
	struct cartesian_grid_3d grid;
};

/* reference include/erida_integrals.h:39-45 */
struct sparse_erida_gausslet_integrals {
	double* integral_values;
	glong* two_indices;
	glong num_entries;
	struct cartesian_grid_3d grid;
};

/* ------------------------------------------------------------------------
 * Inline helpers the reference exposes from its headers (same behaviour).
 * ---------------------------------------------------------------------- */

/* reference include/util.h:43-62 */
static inline glong lmin(const glong a, const glong b) { return a <= b ? a : b; }
static inline glong lmax(const glong a, const glong b) { return a >= b ? a : b; }
static inline double square(const double x) { return x * x; }
static inline glong lsquare(const glong x) { return x * x; }

/* 64-byte aligned host allocations, reference include/aligned_memory.h:14-50 */
#define MEM_DATA_ALIGN 64
static inline void* aligned_malloc(size_t size)
{
	return aligned_alloc(MEM_DATA_ALIGN, (size + MEM_DATA_ALIGN - 1) & ~((size_t)MEM_DATA_ALIGN - 1));
}
static inline void* aligned_calloc(size_t size)
{
	void* p = aligned_malloc(size);
	if (p != NULL) memset(p, 0, size);
	return p;
}
static inline void aligned_free(void* p) { free(p); }

/* x-major linear indexing, reference include/grid.h:33-82 */
static inline glong cartesian_grid_3d_num_points(const struct cartesian_grid_3d* grid)
{
	return grid->coord_range[0].num * grid->coord_range[1].num * grid->coord_range[2].num;
}
static inline glong cartesian_grid_3d_cartesian_to_linear_index(const struct cartesian_grid_3d* grid,
	const glong ix, const glong iy, const glong iz)
{
	assert(0 <= ix && ix < grid->coord_range[0].num);
	assert(0 <= iy && iy < grid->coord_range[1].num);
	assert(0 <= iz && iz < grid->coord_range[2].num);
	return (ix * grid->coord_range[1].num + iy) * grid->coord_range[2].num + iz;
}
static inline glong cartesian_grid_point_3d_to_linear_index(const struct cartesian_grid_3d* grid,
	const union cartesian_grid_point_3d* pt)
{
	return cartesian_grid_3d_cartesian_to_linear_index(grid,
		pt->x - grid->coord_range[0].istart,
		pt->y - grid->coord_range[1].istart,
		pt->z - grid->coord_range[2].istart);
}
static inline void linear_index_to_cartesian_grid_point_3d(const struct cartesian_grid_3d* grid,
	const glong idx, union cartesian_grid_point_3d* pt)
{
	const glong nz = grid->coord_range[2].num, ny = grid->coord_range[1].num;
	pt->z = grid->coord_range[2].istart + idx % nz;
	pt->y = grid->coord_range[1].istart + (idx / nz) % ny;
	pt->x = grid->coord_range[0].istart + idx / (nz * ny);
}

/* ------------------------------------------------------------------------
 * Part 1: functions of the reference interface
 * ---------------------------------------------------------------------- */

/* kinetic: reference include/kinetic_integrals.h:7, :21, :24 */
double compute_kinetic_gausslet_integral(const struct gausslet_data* gdata, const union cartesian_grid_point_3d points[2]);
void compute_kinetic_gausslet_integrals(const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid, struct kinetic_gausslet_integrals* kgi);
void delete_kinetic_gausslet_integrals(struct kinetic_gausslet_integrals* kgi);

/* nuclear: reference include/nuclear_integrals.h:22-24, :40-43, :46 */
double compute_nuclear_gausslet_integral(
	const struct gausslet_data* gdata, const union cartesian_grid_point_3d points[2],
	const struct atomic_nucleus* nuclei, const int num_nuclei, const double tol);
void compute_nuclear_gausslet_integrals(
	const struct gausslet_data* gdata, const struct cartesian_grid_3d* grid,
	const struct atomic_nucleus* nuclei, const int num_nuclei,
	const double tol, struct nuclear_gausslet_integrals* ngi);
void delete_nuclear_gausslet_integrals(struct nuclear_gausslet_integrals* ngi);

/* ERI: reference include/eri_integrals.h:7, :14-16, :31, :34, :50-52, :55, :57, :59, :61, :64 */
double compute_eri_gausslet_integral(const struct gausslet_data* gdata, const union cartesian_grid_point_3d points[4], const double tol);
glong minimum_octahedral_orbit_eri_tensor_index(
	const glong num_points, const glong* octahedral_perm[48],
	const glong i, const glong j, const glong k, const glong l);
void enumerate_symmetry_reduced_eri_indices(const struct cartesian_grid_3d* grid, struct sparse_eri_indices* ret);
void delete_sparse_eri_indices(struct sparse_eri_indices* indices);
void compute_sparse_eri_gausslet_integrals(const struct gausslet_data* gdata,
	const struct cartesian_grid_3d* grid, const glong* four_indices, const glong num_indices,
	const double tol, struct sparse_eri_gausslet_integrals* eri);
double sparse_eri_gausslet_integrals_get_value(const struct sparse_eri_gausslet_integrals* eri, const glong index);
void project_sparse_eri_gausslet_integrals(const struct sparse_eri_gausslet_integrals* eri, const double* basis, const glong num_states, double* eri_proj);
void fill_dense_eri_tensor(const struct sparse_eri_gausslet_integrals* eri_sparse, const struct cartesian_grid_3d* grid_dense, double* eri_tensor);
void apply_sparse_eri_tensor(const struct sparse_eri_gausslet_integrals* eri, const double* states, const glong num_states, double* ret);
void delete_sparse_eri_gausslet_integrals(struct sparse_eri_gausslet_integrals* eri);

/* ERIDA: reference include/erida_integrals.h:7, :14, :29, :32, :48-50, :53, :55, :57, :60 */
double compute_erida_gausslet_integral(const struct gausslet_data* gdata, const union cartesian_grid_point_3d points[2], const double tol);
glong minimum_octahedral_orbit_erida_tensor_index(const glong num_points, const glong* octahedral_perm[48], const glong i, const glong j);
void enumerate_symmetry_reduced_erida_indices(const struct cartesian_grid_3d* grid, struct sparse_erida_indices* ret);
void delete_sparse_erida_indices(struct sparse_erida_indices* indices);
void compute_sparse_erida_gausslet_integrals(const struct gausslet_data* gdata,
	const struct cartesian_grid_3d* grid, const glong* two_indices, const glong num_indices,
	const double tol, struct sparse_erida_gausslet_integrals* erida);
double sparse_erida_gausslet_integrals_get_value(const struct sparse_erida_gausslet_integrals* erida, const glong index);
void project_sparse_erida_gausslet_integrals(const struct sparse_erida_gausslet_integrals* erida, const double* basis, const glong num_states, double* eri_proj);
void fill_dense_erida_matrix(const struct sparse_erida_gausslet_integrals* erida_sparse, const struct cartesian_grid_3d* grid_dense, double* erida_matrix);
void delete_sparse_erida_gausslet_integrals(struct sparse_erida_gausslet_integrals* erida);

/* O_h grid permutations: reference include/symmetry.h:24.  perm[g] receives a
 * 48-way table of aligned_malloc'ed arrays (caller frees each with aligned_free);
 * the grid must be rotationally symmetric. */
void evaluate_octahedral_grid_permutations(const struct cartesian_grid_3d* grid, glong* perm[48]);

/* ------------------------------------------------------------------------
 * Part 2: extensions (no reference counterpart unless noted)
 * ---------------------------------------------------------------------- */

enum gli_b200_status {
	GLI_OK = 0,
	GLI_ERR_CUDA = 1,        /* a CUDA runtime call failed */
	GLI_ERR_ARGUMENT = 2,    /* invalid argument (sizes, grid shape, form) */
	GLI_ERR_NO_DEVICE = 3,   /* no CUDA device visible */
	GLI_ERR_ALLOC = 4,       /* host allocation failed */
	GLI_ERR_LIMIT = 5,       /* a size exceeds a documented limit */
	GLI_ERR_INTERNAL = 6     /* an internal consistency check failed */
};

/* status and message of the last call made by this thread */
int gli_b200_last_error(void);
const char* gli_b200_last_error_message(void);

/* number of visible CUDA devices (0 without a GPU; never fails) */
int gli_b200_device_count(void);
/* CUDA device used by the calling thread's subsequent calls (default 0) */
int gli_b200_set_device(int ordinal);
/* library version string */
const char* gli_b200_version(void);

/* precision forms of the sparse ERI/ERIDA evaluation */
#define GLI_FORM_FP64 0   /* plain FP64 throughout: the drop-in form */
#define GLI_FORM_MIXED 1  /* the two bulk lattice stages as int8-sliced products on the
                             tensor cores (5 slices of 7 bits, row exponents, exact int32
                             accumulation), the last stage and all tables in FP64; about
                             1e-9 Ha max abs error on G10 integral values */

/* kinds of sparse class lists */
#define GLI_KIND_ERIDA 0
#define GLI_KIND_ERI 1

/* Sparse ERI (kind 1) / ERIDA (kind 0) values for a class list already in
 * device memory; d_values receives num doubles in device memory.  Same
 * semantics as compute_sparse_{eri,erida}_gausslet_integrals (reference
 * src/eri_integrals.c:544-678, src/erida_integrals.c:429-542).  stream is a
 * cudaStream_t (NULL = the library's per-thread stream); the call returns
 * when the values are complete (it reads the evaluation's status back).
 * Returns a gli_b200_status. */
int gli_b200_sparse_values_dev(int kind, const double* coeffs, glong num_coeffs,
	const struct cartesian_grid_3d* grid, const glong* d_indices, glong num,
	double tol, int form, double* d_values, void* stream);

/* The same evaluation in stream order: queued on stream without waiting for
 * it (the first call for a class list plans it exactly and waits once).  The
 * values in d_values are defined once gli_b200_sparse_values_wait(*ticket)
 * has returned 0; until then the class list and d_values must not be written
 * by other work.  Tickets belong to the calling thread. */
int gli_b200_sparse_values_dev_async(int kind, const double* coeffs, glong num_coeffs,
	const struct cartesian_grid_3d* grid, const glong* d_indices, glong num,
	double tol, int form, double* d_values, void* stream, glong* ticket);

/* Waits for the evaluation of `ticket` and every one queued before it on this
 * thread, in order, and reads their status.  An evaluation whose class list
 * no longer fits the plan its graph was sized for (the list was rewritten in
 * place) is evaluated again here.  Returns the first error met (the
 * evaluations after it stay pending). */
int gli_b200_sparse_values_wait(glong ticket);

/* Same evaluation with host buffers (copies inside): the reference call with a
 * form switch.  values receives num doubles. */
int gli_b200_sparse_values(int kind, const struct gausslet_data* gdata,
	const struct cartesian_grid_3d* grid, const glong* indices, glong num,
	double tol, int form, double* values);

/* Batched nuclear-attraction matrices on one device.  Instance k has grid
 * grids[k] (any box), nuclei nuclei[nuclei_offsets[k] .. nuclei_offsets[k+1])
 * and writes its N_k x N_k row-major matrix to the device buffer d_out[k];
 * all instances share the coefficients and tol.  form GLI_FORM_FP64 is the
 * reference's arithmetic; GLI_FORM_MIXED runs the three lattice contractions
 * as int8-sliced tensor-core products (about 1e-9 relative).  Each chunk of
 * instances is one CUDA graph launch; the number of concurrent instance
 * pipelines is chosen by the autotuner.  Batches the reference's
 * compute_nuclear_gausslet_integrals (include/nuclear_integrals.h:40-43,
 * src/nuclear_integrals.c:133-266). */
int gli_b200_nuclear_batch_dev(const struct gausslet_data* gdata, glong num_instances,
	const struct cartesian_grid_3d* grids, const glong* nuclei_offsets,
	const struct atomic_nucleus* nuclei, double tol, int form, double* const* d_out,
	void* stream);

/* The same batch with host outputs: h_out[k] (N_k x N_k doubles, caller
 * memory) receives instance k's matrix. */
int gli_b200_nuclear_batch(const struct gausslet_data* gdata, glong num_instances,
	const struct cartesian_grid_3d* grids, const glong* nuclei_offsets,
	const struct atomic_nucleus* nuclei, double tol, int form, double* const* h_out);

/* instances, graph chunks and concurrent instance pipelines of the calling
 * thread's last nuclear batch (no reference counterpart) */
void gli_b200_last_nuclear_batch(glong out[3]);

/* The autotuner's decisions as JSON (truncated to len bytes including the
 * terminating zero); returns the full length.  No reference counterpart. */
glong gli_b200_autotune_report(char* buf, glong len);

/* Checks the autotuner's selection logic on a synthetic cost model, without a
 * device; 0 on success.  No reference counterpart. */
int gli_b200_autotune_selftest(void);

/* ---- ERIDA far-field surrogate (no counterpart in the reference) ----------
 * A small MLP (features of the sorted displacement |dx| >= |dy| >= |dz| in
 * grid units: d/16, r/16, d/r; four tanh layers of width 64; FP32) trained on
 * this device on exact class values of the staged contraction.  It predicts
 * the residual of an ERIDA class value against the point-charge limit 1/r:
 *   r <= 6:          exact
 *   6 < r <= r_mlp:  1/r + s(r) MLP(d),  s(r) = exp(c0 + c1 r + c2 r^2)
 *   r > r_mlp:       1/r
 * (values in grid units; a grid of spacing h scales them by 1/h). */
typedef struct gli_b200_surrogate gli_b200_surrogate;

/* Train on the displacements 6 < r <= r_mlp (exact values on centred cubes of
 * 25..65 points, the same coefficients and tol as the evaluations it will
 * serve): `steps` full-batch Adam steps from learning rate lr with cosine
 * decay; holdout_fraction of the samples (seeded) is kept out of training for
 * the report.  *out is released with gli_b200_surrogate_free. */
int gli_b200_surrogate_train(const struct gausslet_data* gdata, double tol, double r_mlp, int steps,
	double lr, double holdout_fraction, unsigned long long seed, gli_b200_surrogate** out);
void gli_b200_surrogate_free(gli_b200_surrogate* s);
/* info: samples, hold-out samples, weighted loss, max |dz| train / hold-out,
 * max |residual error| train / hold-out (grid units), r_cut, r_mlp,
 * parameter count, c2, c0, c1 */
int gli_b200_surrogate_info(const gli_b200_surrogate* s, double info[13]);
/* copies min(n, count) parameters; returns the count */
glong gli_b200_surrogate_params(const gli_b200_surrogate* s, float* params, glong n);

/* ERIDA values of a class list (host arrays) from the surrogate with a seeded
 * audit: every class with r <= 6, every class whose displacement the network
 * missed by more than shell_tol at training (its error there is known), and
 * an audit sample of each radial shell (floor r; audit_fraction of its
 * classes, at least 4, those of smallest seeded hash of the class index; none
 * when audit_fraction is 0) are evaluated exactly;
 * a shell whose largest audit error exceeds shell_tol (grid units) is
 * evaluated exactly in full.  report (optional, max_shells x 4): per shell
 * classes, audited classes, max audit error, evaluated in full (1/0). */
int gli_b200_erida_surrogate_values(const gli_b200_surrogate* s, const struct gausslet_data* gdata,
	const struct cartesian_grid_3d* grid, const glong* indices, glong num, double tol,
	double audit_fraction, unsigned long long seed, double shell_tol, double* values,
	double* report, glong max_shells);

/* One forward and backward pass of the training kernels without an update:
 * weighted mean squared loss and its gradient for params (count from
 * gli_b200_mlp_param_count), n samples of 7 features X, targets T, weights W. */
int gli_b200_mlp_loss_grad(const float* params, const float* X, const float* T, const float* W, glong n,
	float* loss, float* grads);
int gli_b200_mlp_param_count(void);

/* Symmetry-reduced class list of kind 0/1 into device memory (reference
 * src/eri_integrals.c:382-526, src/erida_integrals.c:300-410).  *d_indices is
 * allocated with cudaMallocAsync on stream; release with gli_b200_free_dev. */
int gli_b200_enumerate_dev(int kind, const struct cartesian_grid_3d* grid,
	glong** d_indices, glong* num, void* stream);
int gli_b200_free_dev(void* d_ptr, void* stream);

/* Per-stage device times (ms) of the last staged evaluation on this thread:
 * [tables, stage A, stage B, stage C]; sizes = [keys, key pairs, lattice extent U].
 * Filled only when timing is enabled with gli_b200_set_timing(1). */
int gli_b200_set_timing(int enable);

/* Measured FP64 throughput of the current device (TFLOP/s): the faster of two
 * compute-only probes, scalar FMA chains and FP64 tensor-core MMAs (m8n8k4);
 * the denominator of the FP64 roofline. */
int gli_b200_measure_fp64_peak(double* tflops);

/* Number of kernels this library launched on the calling thread so far
 * (kernels inside a replayed CUDA graph count at every replay).  No reference
 * counterpart. */
long long gli_b200_launch_count(void);

/* C = A B^T for device matrices in FP64 (row-major; A: M x K with leading
 * dimension lda, B: N x K with ldb, C: M x N with ldc), evaluated on the
 * tcgen05 tensor cores by splitting every row into 7 int8 slices of 7 bits
 * under a per-row exponent and summing the exact int32 slice products of
 * order < 8: about 2^-50 of max|a_i| max|b_j| per product term.  K <= 8192.
 * No reference counterpart; the projections' contractions use it. */
int gli_b200_dgemm_sliced_dev(const double* d_A, glong lda, const double* d_B, glong ldb, double* d_C,
	glong ldc, glong M, glong N, glong K, void* stream);

/* Kinetic matrix (same values as compute_kinetic_gausslet_integrals) for
 * callers that must not allocate device memory -- code that reserved its whole
 * device-memory budget up front, code running while another framework captures
 * a CUDA graph or owns the allocator, or a latency-critical loop where
 * allocation is forbidden.  This entry point has no counterpart in the
 * reference and allocates nothing: d_coeffs (num_coeffs doubles) and d_matrix
 * (N x N doubles, N = grid points, row-major) are device memory supplied by the
 * caller; the only scratch, a per-axis table of at most 1024 doubles, lives in a
 * static device array inside the library, so the grid's largest axis may have
 * at most 1024 points (larger grids fail with GLI_ERR_LIMIT).  The array is
 * shared by every call on a device, so calls whose kernels overlap on the GPU
 * race; calls ordered on one stream do not.  Every call made outside a stream
 * capture looks the array's device address up in the current context; a call
 * made while its stream is being captured reuses the address of an earlier
 * call in the same context, so the first call in a context must come before
 * any capture.  Outside a capture both pointers are checked to be device (or
 * managed) memory, and host pointers fail with GLI_ERR_ARGUMENT.
 * stream is a cudaStream_t (NULL = the legacy default stream); the call returns
 * once the work is queued.  Returns a gli_b200_status. */
int gli_b200_kinetic_matrix_noalloc(const double* d_coeffs, glong num_coeffs,
	const struct cartesian_grid_3d* grid, double* d_matrix, void* stream);
int gli_b200_last_stage_times(float ms[4], glong sizes[3]);
/* Stage C of the same evaluation in two parts (ms, filled under
 * gli_b200_set_timing(1)): ms[0] the (pair, key) product GEMM (0 when stage C
 * ran per class), ms[1] the class-level kernel that followed it (the class
 * gather, or the per-class dot products).  No reference counterpart. */
int gli_b200_last_stage_c_times(float ms[2]);

/* Plan of the calling thread's last sparse evaluation: out[0] A keys, out[1]
 * (A, B) key pairs, out[2] distinct axis keys, out[3] the (pair, key) products
 * that stage C computed as the product GEMM (at least 1 when it ran so), 0 when
 * it ran per class. */
int gli_b200_last_plan(glong out[4]);

/* Arithmetic of the calling thread's last sparse evaluation, per stage:
 * out[0] stage A, out[1] stage B: 1 when the stage ran as int8-sliced products
 * on the tcgen05 tensor cores, 0 when it ran on the FP64 tensor-core GEMM;
 * out[2] stage C: 0 for the per-class FP64 dot products, else the (pair, key)
 * product GEMM plus a class gather: 1 through the classes' packed keys, 2
 * decoding and checking each class against a plan kept from an earlier
 * evaluation of the list.  No reference counterpart. */
int gli_b200_last_paths(int out[3]);

/* Screening of the calling thread's last sparse evaluation: out[0] the
 * threshold its Gaussian-pair products were masked at (the caller's tol for
 * the FP64 form; the mixed form raises it within its error budget), out[1] a
 * bound on how much that changes any class value against masking at the
 * caller's tol, in grid units (0 when the threshold is the caller's).  No
 * reference counterpart. */
int gli_b200_last_screening(double out[2]);

/* Drops the calling thread's captured evaluation graphs and every cached
 * lattice-table set, so that the next evaluation builds its tables and plans
 * from scratch (used to time cold evaluations).  No reference counterpart. */
int gli_b200_clear_caches(void);

#ifdef __cplusplus
}
#endif

#endif /* GLI_B200_H */
