/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain-C restatement of the reference algorithms for the integral hot path
 * of gausslectronitegrate.  Each function names the reference file:line it
 * restates.  Loop nests and accumulation orders follow the reference where they
 * define the floating-point result, so that this restatement can be pinned
 * bit-for-bit against the reference core built under oracle/_ref; the data
 * structures are this file's own (flat arrays, arithmetic O_h images instead
 * of permutation tables, a flat candidate sweep instead of a linked list).
 */
#include "gli_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

static inline i64 imin(i64 a, i64 b) { return a < b ? a : b; }
static inline i64 imax(i64 a, i64 b) { return a > b ? a : b; }
static inline i64 iabs64(i64 a) { return a < 0 ? -a : a; }
static inline double sq(double x) { return x * x; }

/* trim to the outermost entries with |v| > tol; returns length, *lo = first */
static i64 trim_window(const double* v, i64 n, double tol, i64* lo)
{
	i64 a = 0, b = n - 1;
	while (a < n && !(fabs(v[a]) > tol)) ++a;
	if (a == n) { *lo = 0; return 0; }
	while (!(fabs(v[b]) > tol)) --b;
	*lo = a;
	return b - a + 1;
}

/* ---------------------------------------------------------------------------
 * Gaussian-pair factors.  Restates src/gausslet_factors.c:12-81:
 *   F_s[i+j] += (sqrt(pi)/3) * b_i * b_j * exp(-(0.5*(3s + i - j))^2)
 * with index i+j counted from 2*jmin, then trimmed at tol. */
int64_t oracle_factors(const double* coeffs, int64_t nb, int64_t shift, double tol,
                       double* out, int64_t* first)
{
	const double prefac = 0.590817950301838675766;  /* sqrt(pi)/3 */
	const i64 nf = 2 * nb - 1;
	double* acc = calloc(nf, sizeof(double));
	for (i64 i = 0; i < nb; ++i)
		for (i64 j = 0; j < nb; ++j)
			acc[i + j] += prefac * coeffs[i] * coeffs[j] * exp(-sq(0.5 * (3 * shift + (i - j))));
	i64 lo;
	const i64 len = trim_window(acc, nf, tol, &lo);
	if (len > 0) memcpy(out, acc + lo, len * sizeof(double));
	*first = 2 * (-(nb - 1) / 2) + lo;
	free(acc);
	return len;
}

/* ERIDA product vector.  Restates src/erida_integrals.c:44-100:
 *   P[i-j] += (2 pi / 9) * b_i * b_j, index counted from -(nb-1), trimmed. */
int64_t oracle_erida_products(const double* coeffs, int64_t nb, double tol, double* out, int64_t* first)
{
	const double prefac = 0.69813170079773183077;  /* 2 pi / 9 */
	const i64 np = 2 * nb - 1;
	double* acc = calloc(np, sizeof(double));
	for (i64 i = 0; i < nb; ++i)
		for (i64 j = 0; j < nb; ++j)
			acc[i - j + (nb - 1)] += prefac * coeffs[i] * coeffs[j];
	i64 lo;
	const i64 len = trim_window(acc, np, tol, &lo);
	if (len > 0) memcpy(out, acc + lo, len * sizeof(double));
	*first = -(nb - 1) + lo;
	free(acc);
	return len;
}

/* ERI product vector for one shift pair.  Restates src/eri_integrals.c:46-110:
 * factors at tol 0 (exact zeros trimmed), correlation P[a-b] += F_k[a] F_l[b],
 * trimmed at tol. */
int64_t oracle_eri_products(const double* coeffs, int64_t nb, int64_t s01, int64_t s23,
                            double tol, double* out, int64_t* first)
{
	double* fk = malloc((2 * nb - 1) * sizeof(double));
	double* fl = malloc((2 * nb - 1) * sizeof(double));
	i64 ok, ol;
	const i64 nk = oracle_factors(coeffs, nb, s01, 0., fk, &ok);
	const i64 nl = oracle_factors(coeffs, nb, s23, 0., fl, &ol);
	const i64 base = ok - (ol + nl - 1);     /* smallest a - b */
	const i64 np = nk + nl - 1;
	double* acc = calloc(np > 0 ? np : 1, sizeof(double));
	for (i64 i = 0; i < nk; ++i)
		for (i64 j = 0; j < nl; ++j)
			acc[(ok + i) - (ol + j) - base] += fk[i] * fl[j];
	i64 lo = 0, len = 0;
	if (np > 0) len = trim_window(acc, np, tol, &lo);
	if (len > 0) memcpy(out, acc + lo, len * sizeof(double));
	*first = base + lo;
	free(acc); free(fk); free(fl);
	return len;
}

/* ---------------------------------------------------------------------------
 * Coulomb lookup tables.  Restates src/eri_integrals.c:18-27,569-574 (eri=1:
 * w = 1/3, dist = sqrt(n)/6) and src/erida_integrals.c:17-26,446-451 (eri=0:
 * w = sqrt(2)/3, dist = sqrt(n)/3), both in long double. */
void oracle_coulomb_table(int eri, int64_t len, double* out)
{
	const long double w = eri ? 1.L / 3 : 0.4714045207910316829338962414032327L;
	const long double den = eri ? 6 : 3;
	#pragma omp parallel for schedule(static)
	for (i64 n = 0; n < len; ++n) {
		const long double dist = sqrtl((long double)n) / den;
		long double v;
		if (dist > 0) v = erfl(dist / (sqrtl(2) * w)) / dist;
		else v = 0.7978845608028653558798921198687637L / w;
		out[n] = (double)v;
	}
}

/* ---------------------------------------------------------------------------
 * The per-class lattice sum shared by ERI and ERIDA.  Restates the loop body of
 * src/eri_integrals.c:624-669 (and src/erida_integrals.c:488-533): the 2-D
 * scatter of px*py into bins rho = (cx+x)^2 + (cy+y)^2, then one z pass per
 * non-empty bin, accumulated in bin order. */
static double lattice_sum(const double* p[3], const i64 first[3], const i64 len[3],
                          const i64 off[3], const double* table, double tol, double* bins)
{
	const i64 ax0 = off[0] + first[0], ax1 = off[0] + first[0] + len[0] - 1;
	const i64 ay0 = off[1] + first[1], ay1 = off[1] + first[1] + len[1] - 1;
	const i64 nbins = imax(ax0 * ax0, ax1 * ax1) + imax(ay0 * ay0, ay1 * ay1) + 1;
	memset(bins, 0, nbins * sizeof(double));
	for (i64 x = 0; x < len[0]; ++x) {
		if (fabs(p[0][x]) <= tol) continue;
		const i64 rx = (off[0] + first[0] + x) * (off[0] + first[0] + x);
		for (i64 y = 0; y < len[1]; ++y) {
			if (fabs(p[1][y]) <= tol) continue;
			const i64 ry = (off[1] + first[1] + y) * (off[1] + first[1] + y);
			bins[rx + ry] += p[0][x] * p[1][y];
		}
	}
	double val = 0;
	for (i64 r = 0; r < nbins; ++r) {
		if (bins[r] == 0) continue;
		double t = 0;
		for (i64 z = 0; z < len[2]; ++z) {
			if (fabs(p[2][z]) <= tol) continue;
			const i64 rz = (off[2] + first[2] + z) * (off[2] + first[2] + z);
			t += p[2][z] * table[r + rz];
		}
		t *= bins[r];
		val += t;
	}
	return val;
}

static i64 bins_bound(i64 maxc, i64 maxp) { return 2 * (maxc + maxp) * (maxc + maxp) + 1; }

static i64 grid_max_range(const int64_t g[6]) { return imax(imax(g[1], g[3]), g[5]); }

static void decode_point(const int64_t g[6], i64 idx, i64 p[3])
{
	const i64 z = idx % g[5]; idx /= g[5];
	const i64 y = idx % g[3];
	const i64 x = idx / g[3];
	p[0] = g[0] + x; p[1] = g[2] + y; p[2] = g[4] + z;
}

/* ERIDA values for an index list.  Restates src/erida_integrals.c:429-542. */
void oracle_erida_values(const double* coeffs, int64_t nb, const int64_t grid[6],
                         const int64_t* idx, int64_t m, double tol, double* out)
{
	double* P = malloc((2 * nb - 1) * sizeof(double));
	i64 pf;
	i64 pn = oracle_erida_products(coeffs, nb, tol, P, &pf);
	if (pn == 0) { pf = 0; }
	const i64 L = grid_max_range(grid);
	const i64 tlen = 3 * (3 * (L - 1) + (nb - 1)) * (3 * (L - 1) + (nb - 1)) + 1;
	double* table = malloc(tlen * sizeof(double));
	oracle_coulomb_table(0, tlen, table);
	const i64 N = grid[1] * grid[3] * grid[5];
	const i64 nbins = bins_bound(3 * (L - 1), nb);
	#pragma omp parallel
	{
		double* bins = malloc(nbins * sizeof(double));
		#pragma omp for schedule(dynamic, 4)
		for (i64 n = 0; n < m; ++n) {
			i64 pi[3], pj[3];
			decode_point(grid, idx[n] / N, pi);
			decode_point(grid, idx[n] % N, pj);
			const double* p[3] = { P, P, P };
			const i64 first[3] = { pf, pf, pf }, len[3] = { pn, pn, pn };
			const i64 off[3] = { 3 * (pi[0] - pj[0]), 3 * (pi[1] - pj[1]), 3 * (pi[2] - pj[2]) };
			out[n] = pn ? lattice_sum(p, first, len, off, table, tol, bins) : 0.0;
		}
		free(bins);
	}
	free(table); free(P);
}

/* ERI values for an index list.  Restates src/eri_integrals.c:544-678. */
void oracle_eri_values(const double* coeffs, int64_t nb, const int64_t grid[6],
                       const int64_t* idx, int64_t m, double tol, double* out)
{
	const i64 L = grid_max_range(grid);
	const i64 ns = 2 * L - 1;                 /* shifts -(L-1) .. L-1 */
	const i64 pmax = 4 * nb - 3;
	double* prod = malloc(ns * ns * pmax * sizeof(double));
	i64* pfirst = malloc(ns * ns * sizeof(i64));
	i64* plen = malloc(ns * ns * sizeof(i64));
	#pragma omp parallel for collapse(2) schedule(dynamic)
	for (i64 a = 0; a < ns; ++a)
		for (i64 b = 0; b < ns; ++b)
			plen[a * ns + b] = oracle_eri_products(coeffs, nb, a - (L - 1), b - (L - 1), tol,
			                                       prod + (a * ns + b) * pmax, &pfirst[a * ns + b]);
	const i64 tlen = 3 * (6 * (L - 1) + 2 * (nb - 1)) * (6 * (L - 1) + 2 * (nb - 1)) + 1;
	double* table = malloc(tlen * sizeof(double));
	oracle_coulomb_table(1, tlen, table);
	const i64 N = grid[1] * grid[3] * grid[5];
	const i64 nbins = bins_bound(6 * (L - 1), 2 * nb);
	#pragma omp parallel
	{
		double* bins = malloc(nbins * sizeof(double));
		#pragma omp for schedule(dynamic, 16)
		for (i64 n = 0; n < m; ++n) {
			i64 r = idx[n];
			const i64 il = r % N; r /= N;
			const i64 ik = r % N; r /= N;
			const i64 ij = r % N; r /= N;
			const i64 ii = r;
			i64 p0[3], p1[3], p2[3], p3[3];
			decode_point(grid, ii, p0); decode_point(grid, ij, p1);
			decode_point(grid, ik, p2); decode_point(grid, il, p3);
			const double* p[3];
			i64 first[3], len[3], off[3];
			int empty = 0;
			for (int a = 0; a < 3; ++a) {
				const i64 key = (p0[a] - p1[a] + L - 1) * ns + (p2[a] - p3[a] + L - 1);
				p[a] = prod + key * pmax;
				first[a] = pfirst[key];
				len[a] = plen[key];
				off[a] = 3 * ((p0[a] + p1[a]) - (p2[a] + p3[a]));
				if (len[a] == 0) empty = 1;
			}
			out[n] = empty ? 0.0 : lattice_sum(p, first, len, off, table, tol, bins);
		}
		free(bins);
	}
	free(table); free(prod); free(pfirst); free(plen);
}

/* single-entry forms: the same sums with tables sized for the entry alone.
 * Restate src/erida_integrals.c:119-201 and src/eri_integrals.c:133-232. */
double oracle_erida_single(const double* coeffs, int64_t nb, const int64_t p[6], double tol)
{
	const i64 L = imax(imax(iabs64(p[0] - p[3]), iabs64(p[1] - p[4])), iabs64(p[2] - p[5])) + 1;
	double* P = malloc((2 * nb - 1) * sizeof(double));
	i64 pf;
	const i64 pn = oracle_erida_products(coeffs, nb, tol, P, &pf);
	const i64 tlen = 3 * (3 * (L - 1) + (nb - 1)) * (3 * (L - 1) + (nb - 1)) + 1;
	double* table = malloc(tlen * sizeof(double));
	oracle_coulomb_table(0, tlen, table);
	double* bins = malloc(bins_bound(3 * (L - 1), nb) * sizeof(double));
	const double* pp[3] = { P, P, P };
	const i64 first[3] = { pf, pf, pf }, len[3] = { pn, pn, pn };
	const i64 off[3] = { 3 * (p[0] - p[3]), 3 * (p[1] - p[4]), 3 * (p[2] - p[5]) };
	const double v = pn ? lattice_sum(pp, first, len, off, table, tol, bins) : 0.0;
	free(bins); free(table); free(P);
	return v;
}

double oracle_eri_single(const double* coeffs, int64_t nb, const int64_t p[12], double tol)
{
	i64 L = 1;
	for (int a = 0; a < 3; ++a) {
		L = imax(L, iabs64(p[a] - p[3 + a]) + 1);
		L = imax(L, iabs64(p[6 + a] - p[9 + a]) + 1);
	}
	const i64 pmax = 4 * nb - 3;
	double* prod = malloc(3 * pmax * sizeof(double));
	const double* pp[3];
	i64 first[3], len[3], off[3];
	int empty = 0;
	for (int a = 0; a < 3; ++a) {
		len[a] = oracle_eri_products(coeffs, nb, p[a] - p[3 + a], p[6 + a] - p[9 + a], tol, prod + a * pmax, &first[a]);
		pp[a] = prod + a * pmax;
		off[a] = 3 * ((p[a] + p[3 + a]) - (p[6 + a] + p[9 + a]));
		if (len[a] == 0) empty = 1;
	}
	/* the reference sizes the table from the two pair shifts alone; the pair
	 * centres can lie further apart, so cover the offsets actually used */
	const i64 maxoff = imax(imax(iabs64(off[0]), iabs64(off[1])), iabs64(off[2]));
	const i64 span = imax(6 * (L - 1), maxoff) + 2 * (nb - 1);
	const i64 tlen = 3 * span * span + 1;
	double* table = malloc(tlen * sizeof(double));
	oracle_coulomb_table(1, tlen, table);
	double* bins = malloc(bins_bound(imax(6 * (L - 1), maxoff), 2 * nb) * sizeof(double));
	const double v = empty ? 0.0 : lattice_sum(pp, first, len, off, table, tol, bins);
	free(bins); free(table); free(prod);
	return v;
}

/* ---------------------------------------------------------------------------
 * Kinetic.  Restates src/kinetic_integrals.c:14-37 (1-D table) and :73-121. */
static double kinetic_1d(const double* c, i64 nb, i64 shift)
{
	double v = 0;
	for (i64 i = 0; i < nb; ++i)
		for (i64 j = 0; j < nb; ++j) {
			const i64 d = 3 * shift + (i - j);
			const double d2 = (double)(d * d);
			v += 0.5 * c[i] * c[j] * (1.5 * sqrt(M_PI) * (1 - 0.5 * d2) * exp(-0.25 * d2));
		}
	return v;
}

double oracle_kinetic_single(const double* coeffs, int64_t nb, const int64_t p[6])
{
	const i64 d[3] = { iabs64(p[0] - p[3]), iabs64(p[1] - p[4]), iabs64(p[2] - p[5]) };
	const double k[3] = { kinetic_1d(coeffs, nb, d[0]), kinetic_1d(coeffs, nb, d[1]), kinetic_1d(coeffs, nb, d[2]) };
	return k[0] * (d[1] == 0) * (d[2] == 0) + (d[0] == 0) * k[1] * (d[2] == 0) + (d[0] == 0) * (d[1] == 0) * k[2];
}

void oracle_kinetic_matrix(const double* coeffs, int64_t nb, const int64_t g[6], double* out)
{
	const i64 L = grid_max_range(g);
	double* k1 = malloc(L * sizeof(double));
	for (i64 s = 0; s < L; ++s) k1[s] = kinetic_1d(coeffs, nb, s);
	const i64 N = g[1] * g[3] * g[5];
	#pragma omp parallel for schedule(static)
	for (i64 a = 0; a < N; ++a) {
		const i64 az = a % g[5], ay = (a / g[5]) % g[3], ax = a / (g[5] * g[3]);
		for (i64 b = 0; b < N; ++b) {
			const i64 bz = b % g[5], by = (b / g[5]) % g[3], bx = b / (g[5] * g[3]);
			out[a * N + b] = k1[iabs64(ax - bx)] * (ay == by) * (az == bz)
			               + (ax == bx) * k1[iabs64(ay - by)] * (az == bz)
			               + (ax == bx) * (ay == by) * k1[iabs64(az - bz)];
		}
	}
	free(k1);
}

/* ---------------------------------------------------------------------------
 * Nuclear attraction.  Restates src/nuclear_integrals.c:16-24 (kernel),
 * :31-126 (single entry) and :133-266 (matrix, upper triangle then mirror).
 * The scaled norm restates include/util.h:69-117. */
static double scaled_norm(const double v[3])
{
	const double a = fabs(v[0]), b = fabs(v[1]), c = fabs(v[2]);
	double big, s0, s1;
	if (b <= c) {
		if (a <= c) { if (c == 0) return 0; big = c; s0 = a; s1 = b; }
		else { big = a; s0 = b; s1 = c; }
	} else {
		if (a <= b) { big = b; s0 = a; s1 = c; }
		else { big = a; s0 = b; s1 = c; }
	}
	const double d0 = s0 / big, d1 = s1 / big;
	return big * sqrt(1 + d0 * d0 + d1 * d1);
}

static double nuclear_kernel(double dist)
{
	const double w = 1. / 3;
	return dist > 0 ? erf(dist / w) / dist : 2 / (sqrt(M_PI) * w);
}

struct factor_set { double* v; i64* first; i64* len; i64 nb; i64 L; };

static void factor_set_build(struct factor_set* fs, const double* coeffs, i64 nb, i64 L, double tol)
{
	const i64 ns = 2 * L - 1;
	fs->nb = nb; fs->L = L;
	fs->v = malloc(ns * (2 * nb - 1) * sizeof(double));
	fs->first = malloc(ns * sizeof(i64));
	fs->len = malloc(ns * sizeof(i64));
	for (i64 s = 0; s < ns; ++s)
		fs->len[s] = oracle_factors(coeffs, nb, s - (L - 1), tol, fs->v + s * (2 * nb - 1), &fs->first[s]);
}

static void factor_set_free(struct factor_set* fs) { free(fs->v); free(fs->first); free(fs->len); }

static double nuclear_entry(const struct factor_set* fs, const i64 pi[3], const i64 pj[3],
                            const double* pos, const int* charges, int nn, double tol)
{
	const double* f[3];
	i64 first[3], len[3];
	double centre[3];
	for (int a = 0; a < 3; ++a) {
		const i64 s = pi[a] - pj[a] + (fs->L - 1);
		f[a] = fs->v + s * (2 * fs->nb - 1);
		first[a] = fs->first[s];
		len[a] = fs->len[s];
		centre[a] = 0.5 * (pi[a] + pj[a]);
	}
	double val = 0;
	for (i64 x = 0; x < len[0]; ++x) {
		if (fabs(f[0][x]) <= tol) continue;
		const double px = centre[0] + (first[0] + x) / 6.0;
		for (i64 y = 0; y < len[1]; ++y) {
			if (fabs(f[1][y]) <= tol) continue;
			const double py = centre[1] + (first[1] + y) / 6.0;
			for (i64 z = 0; z < len[2]; ++z) {
				if (fabs(f[2][z]) <= tol) continue;
				const double pz = centre[2] + (first[2] + z) / 6.0;
				const double w = f[0][x] * f[1][y] * f[2][z];
				for (int k = 0; k < nn; ++k) {
					const double d[3] = { px - pos[3 * k], py - pos[3 * k + 1], pz - pos[3 * k + 2] };
					val += charges[k] * w * nuclear_kernel(scaled_norm(d));
				}
			}
		}
	}
	return val;
}

double oracle_nuclear_single(const double* coeffs, int64_t nb, const int64_t p[6],
                             const double* pos, const int* charges, int nn, double tol)
{
	const i64 L = imax(imax(iabs64(p[0] - p[3]), iabs64(p[1] - p[4])), iabs64(p[2] - p[5])) + 1;
	struct factor_set fs;
	factor_set_build(&fs, coeffs, nb, L, tol);
	const i64 pi[3] = { p[0], p[1], p[2] }, pj[3] = { p[3], p[4], p[5] };
	const double v = nuclear_entry(&fs, pi, pj, pos, charges, nn, tol);
	factor_set_free(&fs);
	return v;
}

/* the matrix form computes centres as istart + 0.5*(i+j) from 0-based indices;
 * for integer coordinates this equals 0.5*(pi+pj) exactly. */
void oracle_nuclear_matrix(const double* coeffs, int64_t nb, const int64_t g[6],
                           const double* pos, const int* charges, int nn, double tol, double* out)
{
	struct factor_set fs;
	factor_set_build(&fs, coeffs, nb, grid_max_range(g), tol);
	const i64 N = g[1] * g[3] * g[5];
	#pragma omp parallel for schedule(dynamic)
	for (i64 a = 0; a < N; ++a) {
		i64 pa[3];
		decode_point(g, a, pa);
		for (i64 b = a; b < N; ++b) {
			i64 pb[3];
			decode_point(g, b, pb);
			out[a * N + b] = nuclear_entry(&fs, pa, pb, pos, charges, nn, tol);
		}
	}
	for (i64 a = 0; a < N; ++a)
		for (i64 b = 0; b < a; ++b)
			out[a * N + b] = out[b * N + a];
	factor_set_free(&fs);
}

void oracle_nuclear_pairs(const double* coeffs, int64_t nb, const int64_t g[6],
                          const double* pos, const int* charges, int nn, double tol,
                          const int64_t* pairs, int64_t np, double* out)
{
	struct factor_set fs;
	factor_set_build(&fs, coeffs, nb, grid_max_range(g), tol);
	#pragma omp parallel for schedule(dynamic)
	for (i64 n = 0; n < np; ++n) {
		i64 a = pairs[2 * n], b = pairs[2 * n + 1];
		if (a > b) { const i64 t = a; a = b; b = t; }   /* the matrix stores the upper triangle */
		i64 pa[3], pb[3];
		decode_point(g, a, pa);
		decode_point(g, b, pb);
		out[n] = nuclear_entry(&fs, pa, pb, pos, charges, nn, tol);
	}
	factor_set_free(&fs);
}

/* ---------------------------------------------------------------------------
 * Octahedral symmetry.  O_h is the group of the 48 signed 3x3 permutation
 * matrices (the reference tabulates the same set at src/symmetry.c:9-58); the
 * canonical class index is the minimum over the orbit, which does not depend on
 * the order in which the elements are visited.  Images are computed
 * arithmetically instead of through per-element permutation tables
 * (src/symmetry.c:120-150). */
static const int PERM3[6][3] = { {0,1,2}, {0,2,1}, {1,0,2}, {1,2,0}, {2,0,1}, {2,1,0} };

static inline i64 op_lin(int g, const i64 p[3], i64 e, i64 L)
{
	const int* pm = PERM3[g >> 3];
	i64 q[3];
	for (int a = 0; a < 3; ++a) {
		const i64 v = p[pm[a]];
		q[a] = ((g >> a) & 1) ? -v : v;
	}
	return ((q[0] + e) * L + (q[1] + e)) * L + (q[2] + e);
}

static inline i64 pair_key(i64 a, i64 b, i64 N) { return a <= b ? a * N + b : b * N + a; }

/* bounding-box centre normalisation of include/... the python module
 * (python/pymodule.c:~1437-1450 / ~711-728): per axis c = min + max,
 * trans = c / 2 (truncating), bias = c - 2 trans in {-1, 0, 1}. */
static void centre_shift(const i64* pts, int np, i64 trans[3], i64 bias[3])
{
	for (int a = 0; a < 3; ++a) {
		i64 lo = pts[a], hi = pts[a];
		for (int k = 1; k < np; ++k) { lo = imin(lo, pts[3 * k + a]); hi = imax(hi, pts[3 * k + a]); }
		const i64 c = lo + hi;
		trans[a] = c / 2;
		bias[a] = c - 2 * trans[a];
	}
}

/* minimum over bias shifts x O_h x index permutations; points in coordinates.
 * Restates minimum_octahedral_orbit_erida_tensor_index (src/erida_integrals.c:209-234)
 * combined with the bias-shift loop of the enumerator (:355-376). */
static i64 orbit_min_pair(const i64 p[6], const i64 bias[3], i64 e, i64 L, i64 stop_below)
{
	const i64 N = L * L * L;
	i64 best = INT64_MAX;
	for (i64 bx = 0; bx <= iabs64(bias[0]); ++bx)
	for (i64 by = 0; by <= iabs64(bias[1]); ++by)
	for (i64 bz = 0; bz <= iabs64(bias[2]); ++bz) {
		const i64 s[3] = { bx * bias[0], by * bias[1], bz * bias[2] };
		const i64 a[3] = { p[0] - s[0], p[1] - s[1], p[2] - s[2] };
		const i64 b[3] = { p[3] - s[0], p[4] - s[1], p[5] - s[2] };
		for (int g = 0; g < 48; ++g) {
			const i64 v = pair_key(op_lin(g, a, e, L), op_lin(g, b, e, L), N);
			if (v < best) { best = v; if (best < stop_below) return best; }
		}
	}
	return best;
}

/* Restates minimum_octahedral_orbit_eri_tensor_index (src/eri_integrals.c:240-291)
 * with the bias-shift loop of the enumerator (:464-487). */
static i64 orbit_min_quad(const i64 p[12], const i64 bias[3], i64 e, i64 L, i64 stop_below)
{
	const i64 N = L * L * L;
	i64 best = INT64_MAX;
	for (i64 bx = 0; bx <= iabs64(bias[0]); ++bx)
	for (i64 by = 0; by <= iabs64(bias[1]); ++by)
	for (i64 bz = 0; bz <= iabs64(bias[2]); ++bz) {
		const i64 s[3] = { bx * bias[0], by * bias[1], bz * bias[2] };
		i64 q[4][3];
		for (int k = 0; k < 4; ++k)
			for (int a = 0; a < 3; ++a) q[k][a] = p[3 * k + a] - s[a];
		for (int g = 0; g < 48; ++g) {
			i64 ab = pair_key(op_lin(g, q[0], e, L), op_lin(g, q[1], e, L), N);
			i64 cd = pair_key(op_lin(g, q[2], e, L), op_lin(g, q[3], e, L), N);
			if (ab > cd) { const i64 t = ab; ab = cd; cd = t; }
			const i64 v = ab * (N * N) + cd;
			if (v < best) { best = v; if (best < stop_below) return best; }
		}
	}
	return best;
}

static int symmetric_extent(const int64_t g[6], i64* e)
{
	*e = -g[0];
	for (int a = 0; a < 3; ++a)
		if (g[2 * a] != -*e || g[2 * a + 1] != 2 * *e + 1) return 0;
	return 1;
}

int64_t oracle_canonical_erida(const int64_t grid[6], const int64_t p[6])
{
	i64 e;
	if (!symmetric_extent(grid, &e)) return -1;
	i64 trans[3], bias[3];
	centre_shift(p, 2, trans, bias);
	i64 q[6];
	for (int k = 0; k < 2; ++k)
		for (int a = 0; a < 3; ++a) q[3 * k + a] = p[3 * k + a] - trans[a];
	return orbit_min_pair(q, bias, e, 2 * e + 1, INT64_MIN);
}

int64_t oracle_canonical_eri(const int64_t grid[6], const int64_t p[12])
{
	i64 e;
	if (!symmetric_extent(grid, &e)) return -1;
	i64 trans[3], bias[3];
	centre_shift(p, 4, trans, bias);
	i64 q[12];
	for (int k = 0; k < 4; ++k)
		for (int a = 0; a < 3; ++a) q[3 * k + a] = p[3 * k + a] - trans[a];
	return orbit_min_quad(q, bias, e, 2 * e + 1, INT64_MIN);
}

static int cmp_i64(const void* a, const void* b)
{
	const i64 x = *(const i64*)a, y = *(const i64*)b;
	return (x > y) - (x < y);
}

/* growable per-thread buffers merged at the end */
struct vec { i64* v; i64 n, cap; };
static void vec_push(struct vec* s, i64 x)
{
	if (s->n == s->cap) { s->cap = s->cap ? 2 * s->cap : 1024; s->v = realloc(s->v, s->cap * sizeof(i64)); }
	s->v[s->n++] = x;
}

static i64 merge_sorted_out(struct vec* parts, int nparts, int64_t* out, int64_t cap)
{
	i64 total = 0;
	for (int t = 0; t < nparts; ++t) total += parts[t].n;
	i64* all = malloc((total > 0 ? total : 1) * sizeof(i64));
	i64 k = 0;
	for (int t = 0; t < nparts; ++t) { memcpy(all + k, parts[t].v, parts[t].n * sizeof(i64)); k += parts[t].n; free(parts[t].v); }
	qsort(all, total, sizeof(i64), cmp_i64);
	if (out) memcpy(out, all, imin(total, cap) * sizeof(i64));
	free(all);
	return total;
}

/* ERIDA class list.  Restates src/erida_integrals.c:300-410: candidates with
 * ix <= jx and every axis' doubled box centre in {-1,0,1}; a candidate is kept
 * when no element of its orbit has a smaller index. */
int64_t oracle_enumerate_erida(const int64_t grid[6], int64_t* out, int64_t cap)
{
	i64 e;
	if (!symmetric_extent(grid, &e)) return -1;
	const i64 L = 2 * e + 1, N = L * L * L;
	int nthreads = 1;
#ifdef _OPENMP
	nthreads = omp_get_max_threads();
#endif
	struct vec* parts = calloc(nthreads, sizeof(struct vec));
	#pragma omp parallel for schedule(dynamic)
	for (i64 i = 0; i < N; ++i) {
		int t = 0;
#ifdef _OPENMP
		t = omp_get_thread_num();
#endif
		i64 pi[3];
		decode_point(grid, i, pi);
		for (i64 jx = -e; jx <= e; ++jx) {
			if (jx < pi[0]) continue;
			const i64 cx = pi[0] + jx;
			if (cx < -1 || cx > 1) continue;
			for (i64 jy = -e; jy <= e; ++jy) {
				const i64 cy = pi[1] + jy;
				if (cy < -1 || cy > 1) continue;
				for (i64 jz = -e; jz <= e; ++jz) {
					const i64 cz = pi[2] + jz;
					if (cz < -1 || cz > 1) continue;
					const i64 j = ((jx + e) * L + (jy + e)) * L + (jz + e);
					const i64 idx = i * N + j;
					const i64 p[6] = { pi[0], pi[1], pi[2], jx, jy, jz };
					const i64 bias[3] = { cx, cy, cz };
					if (orbit_min_pair(p, bias, e, L, idx) >= idx) vec_push(&parts[t], idx);
				}
			}
		}
	}
	const i64 n = merge_sorted_out(parts, nthreads, out, cap);
	free(parts);
	return n;
}

/* ERI class list.  Restates src/eri_integrals.c:382-526 (x-ordering i<=j,
 * k<=l, i<=k on the x coordinate; doubled box centres in {-1,0,1}; minimality
 * over the orbit with bias shifts). */
int64_t oracle_enumerate_eri(const int64_t grid[6], int64_t* out, int64_t cap)
{
	i64 e;
	if (!symmetric_extent(grid, &e)) return -1;
	const i64 L = 2 * e + 1, N = L * L * L;
	/* per-axis admissible coordinate quadruples */
	i64 nq = 0;
	i64* quads = malloc(L * L * L * L * 4 * sizeof(i64));
	for (i64 a = -e; a <= e; ++a) for (i64 b = -e; b <= e; ++b)
	for (i64 c = -e; c <= e; ++c) for (i64 d = -e; d <= e; ++d) {
		const i64 ctr = imin(imin(a, b), imin(c, d)) + imax(imax(a, b), imax(c, d));
		if (ctr < -1 || ctr > 1) continue;
		quads[4 * nq] = a; quads[4 * nq + 1] = b; quads[4 * nq + 2] = c; quads[4 * nq + 3] = d;
		++nq;
	}
	int nthreads = 1;
#ifdef _OPENMP
	nthreads = omp_get_max_threads();
#endif
	struct vec* parts = calloc(nthreads, sizeof(struct vec));
	#pragma omp parallel for schedule(dynamic) collapse(2)
	for (i64 qx = 0; qx < nq; ++qx)
	for (i64 qy = 0; qy < nq; ++qy) {
		const i64* X = quads + 4 * qx;
		if (X[0] > X[1] || X[2] > X[3] || X[0] > X[2]) continue;
		int t = 0;
#ifdef _OPENMP
		t = omp_get_thread_num();
#endif
		const i64* Y = quads + 4 * qy;
		for (i64 qz = 0; qz < nq; ++qz) {
			const i64* Z = quads + 4 * qz;
			i64 p[12], lin[4];
			for (int k = 0; k < 4; ++k) {
				p[3 * k] = X[k]; p[3 * k + 1] = Y[k]; p[3 * k + 2] = Z[k];
				lin[k] = ((X[k] + e) * L + (Y[k] + e)) * L + (Z[k] + e);
			}
			const i64 idx = ((lin[0] * N + lin[1]) * N + lin[2]) * N + lin[3];
			i64 bias[3];
			bias[0] = imin(imin(X[0], X[1]), imin(X[2], X[3])) + imax(imax(X[0], X[1]), imax(X[2], X[3]));
			bias[1] = imin(imin(Y[0], Y[1]), imin(Y[2], Y[3])) + imax(imax(Y[0], Y[1]), imax(Y[2], Y[3]));
			bias[2] = imin(imin(Z[0], Z[1]), imin(Z[2], Z[3])) + imax(imax(Z[0], Z[1]), imax(Z[2], Z[3]));
			if (orbit_min_quad(p, bias, e, L, idx) >= idx) vec_push(&parts[t], idx);
		}
	}
	free(quads);
	const i64 n = merge_sorted_out(parts, nthreads, out, cap);
	free(parts);
	return n;
}

/* ---------------------------------------------------------------------------
 * Sparse -> dense.  Restates src/erida_integrals.c:683-765 and
 * src/eri_integrals.c:850-967 (canonicalise in the sparse grid, then the
 * binary search of :685-707 / :549-571, 0 when absent). */
static double lookup(const int64_t* idx, const double* val, i64 m, i64 key)
{
	i64 lo = 0, hi = m;
	while (lo < hi) {
		const i64 mid = (lo + hi) / 2;
		if (key < idx[mid]) hi = mid;
		else if (key > idx[mid]) lo = mid + 1;
		else return val[mid];
	}
	return 0;
}

void oracle_fill_dense_erida(const int64_t gs[6], const int64_t* idx, const double* val,
                             int64_t m, const int64_t gd[6], double* out)
{
	const i64 N = gd[1] * gd[3] * gd[5];
	#pragma omp parallel for schedule(static)
	for (i64 a = 0; a < N; ++a) {
		i64 p[6];
		decode_point(gd, a, p);
		for (i64 b = 0; b < N; ++b) {
			decode_point(gd, b, p + 3);
			out[a * N + b] = lookup(idx, val, m, oracle_canonical_erida(gs, p));
		}
	}
}

void oracle_fill_dense_eri(const int64_t gs[6], const int64_t* idx, const double* val,
                           int64_t m, const int64_t gd[6], double* out)
{
	const i64 N = gd[1] * gd[3] * gd[5];
	#pragma omp parallel for collapse(2) schedule(static)
	for (i64 a = 0; a < N; ++a)
	for (i64 b = 0; b < N; ++b) {
		i64 p[12];
		decode_point(gd, a, p);
		decode_point(gd, b, p + 3);
		for (i64 c = 0; c < N; ++c) {
			decode_point(gd, c, p + 6);
			for (i64 d = 0; d < N; ++d) {
				decode_point(gd, d, p + 9);
				out[((a * N + b) * N + c) * N + d] = lookup(idx, val, m, oracle_canonical_eri(gs, p));
			}
		}
	}
}

/* Restates src/eri_integrals.c:974-1100 (physicist's grouping (i,k),(j,l)). */
void oracle_apply_eri(const int64_t g[6], const int64_t* idx, const double* val, int64_t m,
                      const double* states, int64_t ns, double* ret)
{
	const i64 N = g[1] * g[3] * g[5];
	memset(ret, 0, N * N * ns * sizeof(double));
	#pragma omp parallel for collapse(2) schedule(static)
	for (i64 i = 0; i < N; ++i)
	for (i64 k = 0; k < N; ++k) {
		i64 p[12];
		decode_point(g, i, p);
		decode_point(g, k, p + 6);
		double* r = ret + (i * N + k) * ns;
		for (i64 j = 0; j < N; ++j) {
			decode_point(g, j, p + 3);
			for (i64 l = 0; l < N; ++l) {
				decode_point(g, l, p + 9);
				const double v = lookup(idx, val, m, oracle_canonical_eri(g, p));
				const double* st = states + (j * N + l) * ns;
				for (i64 s = 0; s < ns; ++s) r[s] += v * st[s];
			}
		}
	}
}
