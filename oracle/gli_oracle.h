/*
 * CPU oracle: a plain-C restatement of the reference algorithms for the
 * integral hot path.  TEST INFRASTRUCTURE ONLY -- the checker that the CUDA
 * library is compared against.  Nothing in the product links or calls it.
 *
 * Conventions (shared by every function below):
 *   coeffs/nb   gausslet coefficients b_j, odd count nb, j = -(nb-1)/2 .. (nb-1)/2
 *   grid[6]     {istart_x, num_x, istart_y, num_y, istart_z, num_z}
 *   linear grid index  (ix * num_y + iy) * num_z + iz  (0-based, x-major)
 *
 * Parity is pinned in tests/ against the reference's own golden fixtures
 * (test/data/*.hdf5 via the generators test/*_integrals.py) and notebook
 * known answers, and against the reference core compiled under oracle/_ref.
 */
#ifndef GLI_ORACLE_H
#define GLI_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* per-shift factor vector F_s[m], m = 2*jmin .. 2*jmax, trimmed at tol.
 * returns the trimmed length, *first = logical index of the first entry. */
int64_t oracle_factors(const double* coeffs, int64_t nb, int64_t shift, double tol,
                       double* out /* 2nb-1 */, int64_t* first);

/* ERIDA product vector P[s] (single, displacement independent), trimmed. */
int64_t oracle_erida_products(const double* coeffs, int64_t nb, double tol,
                              double* out /* 2nb-1 */, int64_t* first);

/* ERI product vector for the shift pair (s01, s23), trimmed. */
int64_t oracle_eri_products(const double* coeffs, int64_t nb, int64_t s01, int64_t s23,
                            double tol, double* out /* 4nb-3 */, int64_t* first);

double oracle_kinetic_single(const double* coeffs, int64_t nb, const int64_t p[6]);
void   oracle_kinetic_matrix(const double* coeffs, int64_t nb, const int64_t grid[6], double* out);

double oracle_nuclear_single(const double* coeffs, int64_t nb, const int64_t p[6],
                             const double* pos /* 3*nn */, const int* charges, int nn, double tol);
void   oracle_nuclear_matrix(const double* coeffs, int64_t nb, const int64_t grid[6],
                             const double* pos, const int* charges, int nn, double tol, double* out);
/* nuclear values for an explicit list of (i, j) linear index pairs */
void   oracle_nuclear_pairs(const double* coeffs, int64_t nb, const int64_t grid[6],
                            const double* pos, const int* charges, int nn, double tol,
                            const int64_t* pairs /* 2*np */, int64_t np, double* out);

double oracle_erida_single(const double* coeffs, int64_t nb, const int64_t p[6], double tol);
double oracle_eri_single(const double* coeffs, int64_t nb, const int64_t p[12], double tol);

void oracle_erida_values(const double* coeffs, int64_t nb, const int64_t grid[6],
                         const int64_t* idx, int64_t m, double tol, double* out);
void oracle_eri_values(const double* coeffs, int64_t nb, const int64_t grid[6],
                       const int64_t* idx, int64_t m, double tol, double* out);

/* canonical (symmetry-reduced) class lists, sorted ascending.
 * returns the count; writes at most cap entries (out may be NULL to count). */
int64_t oracle_enumerate_erida(const int64_t grid[6], int64_t* out, int64_t cap);
int64_t oracle_enumerate_eri(const int64_t grid[6], int64_t* out, int64_t cap);

/* canonical class index of an arbitrary tuple on a symmetric grid (-e, 2e+1)^3,
 * after moving the bounding-box centre to the origin */
int64_t oracle_canonical_erida(const int64_t grid[6], const int64_t p[6]);
int64_t oracle_canonical_eri(const int64_t grid[6], const int64_t p[12]);

/* sparse -> dense expansion (values missing from the sparse list read as 0) */
void oracle_fill_dense_erida(const int64_t grid_sparse[6], const int64_t* idx, const double* val,
                             int64_t m, const int64_t grid_dense[6], double* out);
void oracle_fill_dense_eri(const int64_t grid_sparse[6], const int64_t* idx, const double* val,
                           int64_t m, const int64_t grid_dense[6], double* out);

/* ret[(i*N+k)*ns + s] = sum_{j,l} V[i,j,k,l] * states[(j*N+l)*ns + s] */
void oracle_apply_eri(const int64_t grid[6], const int64_t* idx, const double* val, int64_t m,
                      const double* states, int64_t ns, double* ret);

/* T[n] = erf(sqrt(n) / (sqrt2 * w * den)) / (sqrt(n)/den) evaluated in long double */
void oracle_coulomb_table(int eri, int64_t len, double* out);

#ifdef __cplusplus
}
#endif
#endif
