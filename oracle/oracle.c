/*
 * Oracle (TEST INFRASTRUCTURE ONLY; see oracle.h): CPU restatement of the reference algorithms.
 * Each function names the reference file:line it follows.  Written for this project from the
 * reference's behaviour; the demag tensor uses Newell, Williams & Dunlop, J. Geophys. Res. 98
 * (1993) 9551, evaluated in binary128 so that its 27-point differences are exact to double.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* constants: src/magneto/mmm/constants.h */
static const double MU0 = 4.0 * 3.14159265358979323846264338327950288L * 1e-7;
static const double ELECTRON_CHARGE = 1.602176487e-19;
static const double MU_BOHR = 9.2740154e-24;
static const double GYROMAGNETIC_RATIO = 2.211e5; /* magnum/micromagnetics/constants.py:33 */

/* ------------------------------------------------------------------------------------------ */
/* threads                                                                                     */
/* ------------------------------------------------------------------------------------------ */
static int g_threads = 1;
void or_set_threads(int n) { g_threads = n > 0 ? n : 1; }

typedef void (*range_fn)(void *ctx, size_t lo, size_t hi);
typedef struct { range_fn fn; void *ctx; size_t lo, hi; } job_t;
static void *job_run(void *p) { job_t *j = (job_t *)p; j->fn(j->ctx, j->lo, j->hi); return NULL; }

static void parallel_for(size_t n, range_fn fn, void *ctx)
{
	int T = g_threads;
	if (T <= 1 || n < 2) { fn(ctx, 0, n); return; }
	if ((size_t)T > n) T = (int)n;
	pthread_t th[256];
	job_t jobs[256];
	if (T > 256) T = 256;
	for (int t = 0; t < T; ++t) {
		jobs[t].fn = fn; jobs[t].ctx = ctx;
		jobs[t].lo = n * t / T; jobs[t].hi = n * (t + 1) / T;
		if (t > 0) pthread_create(&th[t], NULL, job_run, &jobs[t]);
	}
	job_run(&jobs[0]);
	for (int t = 1; t < T; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------------------------ */
/* field terms                                                                                 */
/* ------------------------------------------------------------------------------------------ */

/* mmm/exchange/exchange_cpu.cpp:60-235 (both variants): H_i = 2 A_i/(mu0 Ms_i) *
 * sum_nb w (M_nb/Ms_nb - M_i/Ms_i), neighbours with Ms == 0 skipped.  Returns the CPU path's
 * energy value, -mu0/2 dx dy dz sum_i (M_i/Ms_i).H_i (exchange_cpu.cpp:130-137). */
double or_exchange(int nx, int ny, int nz, double dx, double dy, double dz, int px, int py, int pz,
                   const double *Ms, const double *A, const double *M, double *H)
{
	const size_t n = (size_t)nx * ny * nz, nxy = (size_t)nx * ny;
	const double w[3] = {1.0 / (dx * dx), 1.0 / (dy * dy), 1.0 / (dz * dz)};
	double energy = 0.0;
	for (int z = 0; z < nz; ++z)
		for (int y = 0; y < ny; ++y)
			for (int x = 0; x < nx; ++x) {
				const size_t i = z * nxy + (size_t)y * nx + x;
				const double ms = Ms[i];
				if (ms == 0.0) { H[i] = H[i + n] = H[i + 2 * n] = 0.0; continue; }
				const double mi[3] = {M[i] / ms, M[i + n] / ms, M[i + 2 * n] / ms};
				double s[3] = {0, 0, 0};
				/* neighbour list: (exists, index, weight) */
				long nb[6]; int ok[6]; int dim[6];
				ok[0] = x > 0 || px;      nb[0] = x > 0 ? (long)i - 1 : (long)i + nx - 1;            dim[0] = 0;
				ok[1] = x < nx - 1 || px; nb[1] = x < nx - 1 ? (long)i + 1 : (long)i - (nx - 1);     dim[1] = 0;
				ok[2] = y > 0 || py;      nb[2] = y > 0 ? (long)i - nx : (long)(i + nxy - nx);       dim[2] = 1;
				ok[3] = y < ny - 1 || py; nb[3] = y < ny - 1 ? (long)(i + nx) : (long)(i - (nxy - nx)); dim[3] = 1;
				ok[4] = z > 0 || pz;      nb[4] = z > 0 ? (long)(i - nxy) : (long)(i + n - nxy);     dim[4] = 2;
				ok[5] = z < nz - 1 || pz; nb[5] = z < nz - 1 ? (long)(i + nxy) : (long)(i - (n - nxy)); dim[5] = 2;
				for (int q = 0; q < 6; ++q) {
					if (!ok[q]) continue;
					const size_t j = (size_t)nb[q];
					const double msj = Ms[j];
					if (msj == 0.0) continue;
					for (int c = 0; c < 3; ++c) s[c] += (M[j + c * n] / msj - mi[c]) * w[dim[q]];
				}
				const double pre = (2 / MU0) * A[i];
				for (int c = 0; c < 3; ++c) H[i + c * n] = pre * s[c] / ms;
				energy += mi[0] * H[i] + mi[1] * H[i + n] + mi[2] * H[i + 2 * n];
			}
	return energy * (-MU0 / 2.0 * dx * dy * dz);
}

/* mmm/anisotropy/anisotropy_cpu.cpp:29-73 (cross-product energy form). */
double or_uniaxial_anisotropy(size_t n, const double *axis, const double *k, const double *Ms,
                              const double *M, double *H)
{
	double e = 0.0;
	for (size_t i = 0; i < n; ++i) {
		const double ms = Ms[i], kk = k[i];
		if (ms == 0.0 || kk == 0.0) { H[i] = H[i + n] = H[i + 2 * n] = 0.0; continue; }
		const double a[3] = {axis[i], axis[i + n], axis[i + 2 * n]};
		const double s[3] = {M[i] / ms, M[i + n] / ms, M[i + 2 * n] / ms};
		const double d = s[0] * a[0] + s[1] * a[1] + s[2] * a[2];
		const double f = 2.0 * kk * d / ms / MU0;
		for (int c = 0; c < 3; ++c) H[i + c * n] = f * a[c];
		const double cx = a[1] * s[2] - a[2] * s[1], cy = a[2] * s[0] - a[0] * s[2], cz = a[0] * s[1] - a[1] * s[0];
		e += kk * (cx * cx + cy * cy + cz * cz);
	}
	return e;
}

/* anisotropy_cpu.cpp:75-119 */
double or_cubic_anisotropy(size_t n, const double *axis1, const double *axis2, const double *k,
                           const double *Ms, const double *M, double *H)
{
	double e = 0.0;
	for (size_t i = 0; i < n; ++i) {
		const double ms = Ms[i];
		if (ms == 0.0) { H[i] = H[i + n] = H[i + 2 * n] = 0.0; continue; }
		const double kk = k[i];
		double m[3] = {M[i], M[i + n], M[i + 2 * n]};
		const double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
		for (int c = 0; c < 3; ++c) m[c] = len > 0 ? m[c] / len : 0.0;
		const double u1[3] = {axis1[i], axis1[i + n], axis1[i + 2 * n]};
		const double u2[3] = {axis2[i], axis2[i + n], axis2[i + 2 * n]};
		const double u3[3] = {u1[1] * u2[2] - u1[2] * u2[1], u1[2] * u2[0] - u1[0] * u2[2], u1[0] * u2[1] - u1[1] * u2[0]};
		const double a1 = u1[0] * m[0] + u1[1] * m[1] + u1[2] * m[2];
		const double a2 = u2[0] * m[0] + u2[1] * m[1] + u2[2] * m[2];
		const double a3 = u3[0] * m[0] + u3[1] * m[1] + u3[2] * m[2];
		const double s1 = a1 * a1, s2 = a2 * a2, s3 = a3 * a3;
		const double f = (-2 / MU0) * kk / ms;
		for (int c = 0; c < 3; ++c)
			H[i + c * n] = f * ((s2 + s3) * a1 * u1[c] + (s1 + s3) * a2 * u2[c] + (s1 + s2) * a3 * u3[c]);
		e += kk * (s1 * s2 + s1 * s3 + s2 * s3);
	}
	return e;
}

/* mmm/llge/llge_cpu.cpp:25-45 */
void or_llge(size_t n, const double *f1, const double *f2, const double *M, const double *H, double *dM)
{
	for (size_t i = 0; i < n; ++i) {
		const double m[3] = {M[i], M[i + n], M[i + 2 * n]}, h[3] = {H[i], H[i + n], H[i + 2 * n]};
		const double a[3] = {m[1] * h[2] - m[2] * h[1], m[2] * h[0] - m[0] * h[2], m[0] * h[1] - m[1] * h[0]};
		const double b[3] = {m[1] * a[2] - m[2] * a[1], m[2] * a[0] - m[0] * a[2], m[0] * a[1] - m[1] * a[0]};
		for (int c = 0; c < 3; ++c) dM[i + c * n] = f1[i] * a[c] + f2[i] * b[c];
	}
}

/* mmm/spintorque/fdm_zhangli_cpu.cpp:57-200 */
void or_fdm_zhangli(int nx, int ny, int nz, double dx, double dy, double dz, int do_precess,
                    const double *P, const double *xi, const double *Ms, const double *alpha,
                    const double *j, const double *M, double *dM)
{
	const size_t n = (size_t)nx * ny * nz, nxy = (size_t)nx * ny;
	const int dims[3] = {nx, ny, nz};
	const size_t strides[3] = {1, (size_t)nx, nxy};
	const double del[3] = {dx, dy, dz};
	for (int z = 0; z < nz; ++z)
		for (int y = 0; y < ny; ++y)
			for (int x = 0; x < nx; ++x) {
				const size_t i = z * nxy + (size_t)y * nx + x;
				const double ms = Ms[i];
				if (ms == 0.0) { dM[i] = dM[i + n] = dM[i + 2 * n] = 0.0; continue; }
				const int pos[3] = {x, y, z};
				double g[3][3]; /* g[d][c] = dM_c/dx_d */
				for (int d = 0; d < 3; ++d) {
					for (int c = 0; c < 3; ++c) {
						if (dims[d] <= 1) { g[d][c] = 0.0; continue; }
						const double *Mc = M + c * n;
						if (pos[d] == 0) g[d][c] = (Mc[i + strides[d]] - Mc[i]) / del[d];
						else if (pos[d] == dims[d] - 1) g[d][c] = (Mc[i] - Mc[i - strides[d]]) / del[d];
						else g[d][c] = (Mc[i + strides[d]] - Mc[i - strides[d]]) / (2 * del[d]);
					}
				}
				const double jj[3] = {j[i], j[i + n], j[i + 2 * n]};
				double u[3];
				for (int c = 0; c < 3; ++c) u[c] = jj[0] * g[0][c] + jj[1] * g[1][c] + jj[2] * g[2][c];
				const double m[3] = {M[i], M[i + n], M[i + 2 * n]};
				const double B[3] = {m[1] * u[2] - m[2] * u[1], m[2] * u[0] - m[0] * u[2], m[0] * u[1] - m[1] * u[0]};
				const double A[3] = {m[1] * B[2] - m[2] * B[1], m[2] * B[0] - m[0] * B[2], m[0] * B[1] - m[1] * B[0]};
				const double p = P[i], x_i = xi[i], al = alpha[i];
				const double bj = p * MU_BOHR / (ELECTRON_CHARGE * ms * (1.0 + x_i * x_i));
				const double bjp = bj / (1.0 + al * al);
				double f1, f2;
				if (do_precess) { f1 = -bjp / (ms * ms) * (1.0 + al * x_i); f2 = -bjp / ms * (x_i - al); }
				else { f1 = -bjp / (ms * ms) * (al * x_i); f2 = -bjp / ms * (-al); }
				for (int c = 0; c < 3; ++c) dM[i + c * n] = f1 * A[c] + f2 * B[c];
			}
}

/* math/ScaledAbsMax.cpp:33-68: uniform scale -> absMax(M)/s, else max over s_i != 0. */
double or_scaled_abs_max(size_t n, const double *M, const double *s)
{
	int uniform = 1;
	for (size_t i = 1; i < n && uniform; ++i) uniform = (s[i] == s[0]);
	double best = 0.0;
	if (uniform) {
		for (size_t i = 0; i < n; ++i) {
			const double q = M[i] * M[i] + M[i + n] * M[i + n] + M[i + 2 * n] * M[i + 2 * n];
			if (q > best) best = q;
		}
		return sqrt(best) / s[0];
	}
	for (size_t i = 0; i < n; ++i) {
		if (s[i] == 0.0) continue;
		const double q = (M[i] * M[i] + M[i + n] * M[i + n] + M[i + 2 * n] * M[i + 2 * n]) / (s[i] * s[i]);
		if (q > best) best = q;
	}
	return sqrt(best);
}

/* VectorMatrix::normalize(Matrix) -> CPUDevice::normalize3 (matrix/device/cpu/CPUDevice.cpp:
 * 244-271): with float_norm the norm is formed as the CPU path does, from float-cast components
 * with float arithmetic (std::sqrt of a float argument is the float overload); cells with zero
 * norm are left unchanged. */
void or_normalize(size_t n, const double *Ms, double *M, int float_norm)
{
	for (size_t i = 0; i < n; ++i) {
		double norm;
		if (float_norm) {
			const float e0 = (float)M[i], e1 = (float)M[i + n], e2 = (float)M[i + 2 * n];
			norm = (double)sqrtf(e0 * e0 + e1 * e1 + e2 * e2);
		} else {
			norm = sqrt(M[i] * M[i] + M[i + n] * M[i + n] + M[i + 2 * n] * M[i + 2 * n]);
		}
		if (norm == 0.0) continue;
		const double sc = Ms[i] / norm;
		M[i] *= sc; M[i + n] *= sc; M[i + 2 * n] *= sc;
	}
}

/* ------------------------------------------------------------------------------------------ */
/* demag tensor                                                                                */
/* ------------------------------------------------------------------------------------------ */

/* mmm/demag/tensor_round.cpp:20-106 */
static int round4(int x) { return (x & 3) ? (x | 3) + 1 : x; }
static int round8(int x) { return (x & 7) ? (x | 7) + 1 : x; }
static int round2(int x) { return (x & 1) ? x + 1 : x; }
static int round_pot(int x) { int p = 1; while (p < x) p <<= 1; return p; }
static int max_prime_factor(int n)
{
	int best = 1;
	for (int p = 2; (long)p * p <= n; ++p)
		while (n % p == 0) { best = p; n /= p; }
	return n > 1 ? (n > best ? n : best) : best;
}
int or_round_tensor_dimension(int dim, int periodic, int padding)
{
	if (periodic) return dim;
	const int t = 2 * dim - 1;
	if (t == 1) return 1;
	switch (padding) {
	case 0: return t;
	case 1: return round2(t);
	case 2: return round4(t);
	case 3: return round8(t);
	case 4: return round_pot(t);
	case 5: { int x = t + 1; while (max_prime_factor(x) > 5) ++x; return x; }
	default: return -1;
	}
}

typedef __float128 q_t;

/* Newell f (JGR 1993 eq. 27); even in every argument. */
static q_t newell_f(q_t x, q_t y, q_t z)
{
	const q_t x2 = x * x, y2 = y * y, z2 = z * z, R2 = x2 + y2 + z2;
	if (R2 == 0) return 0;
	const q_t R = sqrtq(R2);
	q_t r = (2 * x2 - y2 - z2) * R / 6;
	if (x2 + z2 > 0 && y != 0) r += y / 2 * (z2 - x2) * asinhq(y / sqrtq(x2 + z2));
	if (x2 + y2 > 0 && z != 0) r += z / 2 * (y2 - x2) * asinhq(z / sqrtq(x2 + y2));
	if (x != 0 && y != 0 && z != 0) r -= x * y * z * atanq(y * z / (x * R));
	return r;
}

/* Newell g (JGR 1993 eq. 32); odd in x and y, even in z. */
static q_t newell_g(q_t x, q_t y, q_t z)
{
	const q_t x2 = x * x, y2 = y * y, z2 = z * z, R2 = x2 + y2 + z2;
	if (R2 == 0) return 0;
	const q_t R = sqrtq(R2);
	q_t r = -x * y * R / 3;
	if (x2 + y2 > 0 && x != 0 && y != 0 && z != 0) r += x * y * z * asinhq(z / sqrtq(x2 + y2));
	if (y2 + z2 > 0 && y != 0 && x != 0) r += y / 6 * (3 * z2 - y2) * asinhq(x / sqrtq(y2 + z2));
	if (x2 + z2 > 0 && x != 0 && y != 0) r += x / 6 * (3 * z2 - x2) * asinhq(y / sqrtq(x2 + z2));
	if (z != 0 && x != 0 && y != 0) r -= z * z2 / 6 * atanq(x * y / (z * R));
	if (y != 0 && x != 0 && z != 0) r -= z * y2 / 2 * atanq(x * z / (y * R));
	if (x != 0 && y != 0 && z != 0) r -= z * x2 / 2 * atanq(y * z / (x * R));
	return r;
}

typedef struct {
	int nx, ny, nz, gx, gy, gz;   /* grid of sample points (0..nx) x (0..ny) x (0..nz) */
	q_t dx, dy, dz;
	q_t *F[6];                    /* f_xx, f_yy, f_zz, g_xy, g_xz, g_yz on the point grid */
} tensor_ctx;

static void tensor_points(void *p, size_t lo, size_t hi)
{
	tensor_ctx *c = (tensor_ctx *)p;
	for (size_t q = lo; q < hi; ++q) {
		const int i = (int)(q % c->gx), j = (int)((q / c->gx) % c->gy), k = (int)(q / ((size_t)c->gx * c->gy));
		const q_t X = i * c->dx, Y = j * c->dy, Z = k * c->dz;
		c->F[0][q] = newell_f(X, Y, Z);
		c->F[1][q] = newell_f(Y, X, Z);
		c->F[2][q] = newell_f(Z, Y, X);
		c->F[3][q] = newell_g(X, Y, Z);
		c->F[4][q] = newell_g(X, Z, Y);
		c->F[5][q] = newell_g(Y, Z, X);
	}
}

typedef struct {
	tensor_ctx *t;
	int ex, ey, ez;
	double *out;
} scatter_ctx;

static void tensor_cells(void *p, size_t lo, size_t hi)
{
	scatter_ctx *s = (scatter_ctx *)p;
	tensor_ctx *c = s->t;
	const q_t V = c->dx * c->dy * c->dz;
	const q_t pref = 1 / (4 * M_PIq * V);
	for (size_t q = lo; q < hi; ++q) {
		const int i = (int)(q % c->nx), j = (int)((q / c->nx) % c->ny), k = (int)(q / ((size_t)c->nx * c->ny));
		q_t acc[6] = {0, 0, 0, 0, 0, 0};
		for (int cz = -1; cz <= 1; ++cz)
			for (int cy = -1; cy <= 1; ++cy)
				for (int cx = -1; cx <= 1; ++cx) {
					/* second-difference weights (-1, 2, -1) in each direction */
					const int w = (cx ? -1 : 2) * (cy ? -1 : 2) * (cz ? -1 : 2);
					const int X = i + cx, Y = j + cy, Z = k + cz;
					const int ax = X < 0 ? -X : X, ay = Y < 0 ? -Y : Y, az = Z < 0 ? -Z : Z;
					const int sx = X < 0 ? -1 : 1, sy = Y < 0 ? -1 : 1, sz = Z < 0 ? -1 : 1;
					const size_t g = ((size_t)az * c->gy + ay) * c->gx + ax;
					acc[0] += w * c->F[0][g];
					acc[1] += w * c->F[1][g];
					acc[2] += w * c->F[2][g];
					acc[3] += w * sx * sy * c->F[3][g];
					acc[4] += w * sx * sz * c->F[4][g];
					acc[5] += w * sy * sz * c->F[5][g];
				}
		/* with weights (-1, 2, -1) the sum is 4 pi V times the demag tensor N; the stored field is
		 * -N (H = (-N) * M, mmm/demag/demag_tensor.cpp:176-177). */
		const double v[6] = {(double)(-pref * acc[0]), (double)(-pref * acc[3]), (double)(-pref * acc[4]),
		                     (double)(-pref * acc[1]), (double)(-pref * acc[5]), (double)(-pref * acc[2])};
		/* scatter to the 8 octants with parity signs (mmm/demag/tensor.cpp:167-180); the
		 * multiplicity division there makes zero coordinates count once. */
		for (int o = -1; o <= 1; o += 2)
			for (int pp = -1; pp <= 1; pp += 2)
				for (int r = -1; r <= 1; r += 2) {
					if ((i == 0 && o < 0) || (j == 0 && pp < 0) || (k == 0 && r < 0)) continue;
					const int I = (o * i + s->ex) % s->ex, J = (pp * j + s->ey) % s->ey, K = (r * k + s->ez) % s->ez;
					double *d = s->out + 6 * (((size_t)K * s->ey + J) * s->ex + I);
					d[0] = v[0];
					d[1] = o * pp * v[1];
					d[2] = o * r * v[2];
					d[3] = v[3];
					d[4] = pp * r * v[4];
					d[5] = v[5];
				}
	}
}

void or_demag_tensor(int nx, int ny, int nz, double dx, double dy, double dz, int ex, int ey, int ez, double *out)
{
	tensor_ctx c;
	c.nx = nx; c.ny = ny; c.nz = nz;
	c.gx = nx + 1; c.gy = ny + 1; c.gz = nz + 1;
	c.dx = dx; c.dy = dy; c.dz = dz;
	const size_t np = (size_t)c.gx * c.gy * c.gz;
	for (int f = 0; f < 6; ++f) c.F[f] = (q_t *)malloc(sizeof(q_t) * np);
	parallel_for(np, tensor_points, &c);
	memset(out, 0, sizeof(double) * 6 * (size_t)ex * ey * ez);
	scatter_ctx s = {&c, ex, ey, ez, out};
	parallel_for((size_t)nx * ny * nz, tensor_cells, &s);
	for (int f = 0; f < 6; ++f) free(c.F[f]);
}

/* ------------------------------------------------------------------------------------------ */
/* convolution                                                                                 */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
	const double *N; int nx, ny, nz, ex, ey, ez; const double *M; double *H;
} conv_ctx;

/* math/conv/SymmetricMatrixVectorConvolution_Simple.cpp:36-80 */
static void conv_direct_range(void *p, size_t lo, size_t hi)
{
	conv_ctx *c = (conv_ctx *)p;
	const size_t n = (size_t)c->nx * c->ny * c->nz;
	for (size_t t = lo; t < hi; ++t) {
		const int x = (int)(t % c->nx), y = (int)((t / c->nx) % c->ny), z = (int)(t / ((size_t)c->nx * c->ny));
		long double h0 = 0, h1 = 0, h2 = 0;
		for (int o = 0; o < c->nz; ++o)
			for (int q = 0; q < c->ny; ++q)
				for (int m = 0; m < c->nx; ++m) {
					const int X = (x - m + c->ex) % c->ex, Y = (y - q + c->ey) % c->ey, Z = (z - o + c->ez) % c->ez;
					const double *Nv = c->N + 6 * (((size_t)Z * c->ey + Y) * c->ex + X);
					const size_t s = ((size_t)o * c->ny + q) * c->nx + m;
					const double mx = c->M[s], my = c->M[s + n], mz = c->M[s + 2 * n];
					h0 += (long double)Nv[0] * mx + (long double)Nv[1] * my + (long double)Nv[2] * mz;
					h1 += (long double)Nv[1] * mx + (long double)Nv[3] * my + (long double)Nv[4] * mz;
					h2 += (long double)Nv[2] * mx + (long double)Nv[4] * my + (long double)Nv[5] * mz;
				}
		c->H[t] = (double)h0; c->H[t + n] = (double)h1; c->H[t + 2 * n] = (double)h2;
	}
}

void or_conv_direct(const double *N, int nx, int ny, int nz, int ex, int ey, int ez, const double *M, double *H)
{
	conv_ctx c = {N, nx, ny, nz, ex, ey, ez, M, H};
	parallel_for((size_t)nx * ny * nz, conv_direct_range, &c);
}

/* ---- FFT: mixed-radix decimation-in-time, double; the reference delegates to FFTW
 * (math/conv/kernels/Transformer_CPU.cpp), whose results differ from any exact DFT only by
 * rounding. ---- */
typedef struct { double re, im; } cpx;

static void dft_rec(int n, const cpx *x, size_t xs, cpx *y, cpx *tmp, const cpx *tw, int twn, int sign)
{
	if (n == 1) { y[0] = x[0]; return; }
	int p = 2;
	while (n % p) ++p;
	const int m = n / p;
	for (int r = 0; r < p; ++r) dft_rec(m, x + r * xs, xs * p, y + (size_t)r * m, tmp, tw, twn, sign);
	/* Y[k + q m] = sum_r W_n^{r (k + q m)} y_r[k] */
	const int step = twn / n;
	for (int k = 0; k < m; ++k) {
		for (int q = 0; q < p; ++q) {
			double re = 0, im = 0;
			for (int r = 0; r < p; ++r) {
				const long e = ((long)r * (k + (long)q * m)) % n;
				cpx w = tw[e * step];
				if (sign > 0) w.im = -w.im;
				const cpx v = y[(size_t)r * m + k];
				re += v.re * w.re - v.im * w.im;
				im += v.re * w.im + v.im * w.re;
			}
			tmp[q] = (cpx){re, im};
		}
		for (int q = 0; q < p; ++q) y[k + (size_t)q * m] = tmp[q];
	}
}

static cpx *twiddles(int n)
{
	cpx *t = (cpx *)malloc(sizeof(cpx) * n);
	for (int k = 0; k < n; ++k) {
		const long double a = -2.0L * 3.14159265358979323846264338327950288L * k / n;
		t[k].re = (double)cosl(a);
		t[k].im = (double)sinl(a);
	}
	return t;
}

typedef struct {
	cpx *data; int len; size_t inner, outer; const cpx *tw; int sign;
} fft_axis_ctx;

static void fft_axis_range(void *p, size_t lo, size_t hi)
{
	fft_axis_ctx *c = (fft_axis_ctx *)p;
	cpx *a = (cpx *)malloc(sizeof(cpx) * c->len), *b = (cpx *)malloc(sizeof(cpx) * c->len);
	cpx *tmp = (cpx *)malloc(sizeof(cpx) * c->len);
	for (size_t l = lo; l < hi; ++l) {
		const size_t o = l / c->inner, i = l % c->inner;
		cpx *base = c->data + o * c->len * c->inner + i;
		for (int k = 0; k < c->len; ++k) a[k] = base[k * c->inner];
		dft_rec(c->len, a, 1, b, tmp, c->tw, c->len, c->sign);
		for (int k = 0; k < c->len; ++k) base[k * c->inner] = b[k];
	}
	free(a); free(b); free(tmp);
}

/* 3-D transform of a (len0, len1, len2) array, x fastest. */
static void fft3(cpx *d, const int L[3], int sign)
{
	size_t inner = 1;
	for (int ax = 0; ax < 3; ++ax) {
		size_t outer = 1;
		for (int b = ax + 1; b < 3; ++b) outer *= L[b];
		if (L[ax] > 1) {
			cpx *tw = twiddles(L[ax]);
			fft_axis_ctx c = {d, L[ax], inner, outer, tw, sign};
			parallel_for(inner * outer, fft_axis_range, &c);
			free(tw);
		}
		inner *= L[ax];
	}
}

/* TensorFieldSetup.cpp:35-74: transformed tensor components (full complex spectra). */
static cpx **conv_fft_prepare(const double *N, int ex, int ey, int ez)
{
	const size_t P = (size_t)ex * ey * ez;
	const int L[3] = {ex, ey, ez};
	cpx **Nh = (cpx **)malloc(6 * sizeof(cpx *));
	for (int c = 0; c < 6; ++c) {
		Nh[c] = (cpx *)malloc(sizeof(cpx) * P);
		for (size_t i = 0; i < P; ++i) Nh[c][i] = (cpx){N[6 * i + c], 0.0};
		fft3(Nh[c], L, -1);
	}
	return Nh;
}

static void conv_fft_free(cpx **Nh)
{
	if (!Nh) return;
	for (int c = 0; c < 6; ++c) free(Nh[c]);
	free(Nh);
}

/* math/conv/MatrixVectorConvolution_FFT.cpp:110-241 (CPU path): forward transforms of the padded
 * M, multiplication by the transformed tensor scaled by 1/(ex ey ez) (cpu_multiplication.cpp:
 * 56-91), inverse transform, crop. */
static void conv_fft_apply(cpx **Nh, int nx, int ny, int nz, int ex, int ey, int ez, const double *M, double *H)
{
	const size_t P = (size_t)ex * ey * ez, n = (size_t)nx * ny * nz;
	const int L[3] = {ex, ey, ez};
	cpx *Mh[3];
	for (int c = 0; c < 3; ++c) {
		Mh[c] = (cpx *)calloc(P, sizeof(cpx));
		for (int z = 0; z < nz; ++z)
			for (int y = 0; y < ny; ++y)
				for (int x = 0; x < nx; ++x)
					Mh[c][((size_t)z * ey + y) * ex + x].re = M[c * n + ((size_t)z * ny + y) * nx + x];
		fft3(Mh[c], L, -1);
	}
	const double scale = 1.0 / (double)P;
	for (size_t i = 0; i < P; ++i) {
		const cpx a = Mh[0][i], b = Mh[1][i], c = Mh[2][i];
		const cpx *t[6] = {&Nh[0][i], &Nh[1][i], &Nh[2][i], &Nh[3][i], &Nh[4][i], &Nh[5][i]};
#define CM(u, v) ((cpx){(u).re * (v)->re - (u).im * (v)->im, (u).re * (v)->im + (u).im * (v)->re})
		const cpx x0 = CM(a, t[0]), x1 = CM(b, t[1]), x2 = CM(c, t[2]);
		const cpx y0 = CM(a, t[1]), y1 = CM(b, t[3]), y2 = CM(c, t[4]);
		const cpx z0 = CM(a, t[2]), z1 = CM(b, t[4]), z2 = CM(c, t[5]);
#undef CM
		Mh[0][i] = (cpx){(x0.re + x1.re + x2.re) * scale, (x0.im + x1.im + x2.im) * scale};
		Mh[1][i] = (cpx){(y0.re + y1.re + y2.re) * scale, (y0.im + y1.im + y2.im) * scale};
		Mh[2][i] = (cpx){(z0.re + z1.re + z2.re) * scale, (z0.im + z1.im + z2.im) * scale};
	}
	for (int c = 0; c < 3; ++c) {
		fft3(Mh[c], L, +1);
		for (int z = 0; z < nz; ++z)
			for (int y = 0; y < ny; ++y)
				for (int x = 0; x < nx; ++x)
					H[c * n + ((size_t)z * ny + y) * nx + x] = Mh[c][((size_t)z * ey + y) * ex + x].re;
		free(Mh[c]);
	}
}

void or_conv_fft(const double *N, int nx, int ny, int nz, int ex, int ey, int ez, const double *M, double *H)
{
	cpx **Nh = conv_fft_prepare(N, ex, ey, ez);
	conv_fft_apply(Nh, nx, ny, nz, ex, ey, ez, M, H);
	conv_fft_free(Nh);
}

/* ------------------------------------------------------------------------------------------ */
/* Runge-Kutta solver                                                                          */
/* ------------------------------------------------------------------------------------------ */

/* magnum/evolver/tableaus.py:54-139 */
typedef struct { int s, order, fsal; double a[8], b[8][8], c[8], ec[8]; } tableau_t;

static void make_tableau(int which, tableau_t *t)
{
	memset(t, 0, sizeof(*t));
	if (which == 2) { /* dp54 */
		t->s = 7; t->order = 5; t->fsal = 1;
		const double a[7] = {0.0, 1.0 / 5.0, 3.0 / 10.0, 4.0 / 5.0, 8.0 / 9.0, 1.0, 1.0};
		const double b[7][6] = {{0},
		                        {1.0 / 5.0},
		                        {3.0 / 40.0, 9.0 / 40.0},
		                        {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0},
		                        {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0},
		                        {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0},
		                        {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
		const double c4[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0, -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};
		const double c5[7] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
		for (int i = 0; i < 7; ++i) {
			t->a[i] = a[i];
			for (int j = 0; j < 6; ++j) t->b[i][j] = b[i][j];
			t->c[i] = c5[i];
			t->ec[i] = c4[i] - c5[i];
		}
	} else if (which == 0) { /* rkf45 */
		t->s = 6; t->order = 4; t->fsal = 0;
		const double a[6] = {0.0, 1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0};
		const double b[6][5] = {{0},
		                        {1.0 / 4.0},
		                        {3.0 / 32.0, 9.0 / 32.0},
		                        {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0},
		                        {439.0 / 216.0, -8.0, 3680.0 / 513.0, -845.0 / 4104.0},
		                        {-8.0 / 27.0, 2.0, -3544.0 / 2565.0, 1859.0 / 4104.0, -11.0 / 40.0}};
		const double c4[6] = {25.0 / 216.0, 0.0, 1408.0 / 2565.0, 2197.0 / 4104.0, -1.0 / 5.0, 0.0};
		const double c5[6] = {16.0 / 135.0, 0.0, 6656.0 / 12825.0, 28561.0 / 56430.0, -9.0 / 50.0, 2.0 / 55.0};
		for (int i = 0; i < 6; ++i) {
			t->a[i] = a[i];
			for (int j = 0; j < 5; ++j) t->b[i][j] = b[i][j];
			t->c[i] = c4[i];
			t->ec[i] = c4[i] - c5[i];
		}
	} else if (which == 1) { /* cc45 */
		t->s = 6; t->order = 4; t->fsal = 0;
		const double a[6] = {0.0, 1.0 / 5.0, 3.0 / 10.0, 3.0 / 5.0, 1.0, 7.0 / 8.0};
		const double b[6][5] = {{0},
		                        {1.0 / 5.0},
		                        {3.0 / 40.0, 9.0 / 40.0},
		                        {3.0 / 10.0, -9.0 / 10.0, 6.0 / 5.0},
		                        {-11.0 / 54.0, 5.0 / 2.0, -70.0 / 27.0, 35.0 / 27.0},
		                        {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};
		const double c4[6] = {2825.0 / 27648.0, 0.0, 18575.0 / 48384.0, 13525.0 / 55296.0, 277.0 / 14336.0, 1.0 / 4.0};
		const double c5[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};
		for (int i = 0; i < 6; ++i) {
			t->a[i] = a[i];
			for (int j = 0; j < 5; ++j) t->b[i][j] = b[i][j];
			t->c[i] = c4[i];
			t->ec[i] = c4[i] - c5[i];
		}
	} else { /* rk23 */
		t->s = 4; t->order = 3; t->fsal = 1;
		const double a[4] = {0.0, 0.5, 3.0 / 4.0, 1.0};
		const double b[4][3] = {{0}, {1.0 / 2.0}, {0.0, 3.0 / 4.0}, {2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0}};
		const double c2[4] = {7.0 / 24.0, 1.0 / 4.0, 1.0 / 3.0, 1.0 / 8.0};
		const double c3[4] = {2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0, 0.0};
		for (int i = 0; i < 4; ++i) {
			t->a[i] = a[i];
			for (int j = 0; j < 3; ++j) t->b[i][j] = b[i][j];
			t->c[i] = c3[i];
			t->ec[i] = c2[i] - c3[i];
		}
	}
}

struct or_solver {
	or_solver_config cfg;
	size_t n;
	int ex, ey, ez;
	double *Ms, *A, *alpha, *kuni, *kcub, *ax1, *ax2, *P, *xi, *j, *N;
	double *f1, *f2;
	cpx **Nh;             /* tensor spectrum (FFT convolution) */
	double *y, *y0, *ytmp, *yerr, *k[8], *Htmp, *Hacc, *dtmp;
	int k0_is_fsal;       /* state.dydt_in available (held in k[0]) */
	tableau_t tab;
	double t, h, h_next; int have_next;
	long steps, attempts, rejected;
};

static double *dup(const double *src, size_t n)
{
	double *d = (double *)malloc(sizeof(double) * n);
	if (src) memcpy(d, src, sizeof(double) * n); else memset(d, 0, sizeof(double) * n);
	return d;
}

or_solver *or_solver_create(const or_solver_config *cfg, const double *Ms, const double *A,
                            const double *alpha, const double *k_uni, const double *k_cub,
                            const double *axis1, const double *axis2, const double *P,
                            const double *xi, const double *j, const double *tensor, int ex,
                            int ey, int ez)
{
	or_solver *s = (or_solver *)calloc(1, sizeof(or_solver));
	s->cfg = *cfg;
	const size_t n = (size_t)cfg->nx * cfg->ny * cfg->nz;
	s->n = n; s->ex = ex; s->ey = ey; s->ez = ez;
	s->Ms = dup(Ms, n); s->A = dup(A, n); s->alpha = dup(alpha, n);
	s->kuni = dup(k_uni, n); s->kcub = dup(k_cub, n);
	s->ax1 = dup(axis1, 3 * n); s->ax2 = dup(axis2, 3 * n);
	s->P = dup(P, n); s->xi = dup(xi, n); s->j = dup(j, 3 * n);
	s->N = tensor ? dup(tensor, 6 * (size_t)ex * ey * ez) : NULL;
	s->Nh = (tensor && cfg->use_fft) ? conv_fft_prepare(s->N, ex, ey, ez) : NULL;
	/* LandauLifshitzGilbert.__initFactors (landau_lifshitz_gilbert.py:133-158) */
	s->f1 = dup(NULL, n); s->f2 = dup(NULL, n);
	for (size_t i = 0; i < n; ++i) {
		if (s->Ms[i] != 0.0) {
			const double gp = GYROMAGNETIC_RATIO / (1.0 + s->alpha[i] * s->alpha[i]);
			s->f1[i] = cfg->do_precess ? -gp : 0.0;
			s->f2[i] = -s->alpha[i] * gp / s->Ms[i];
		}
	}
	s->y = dup(NULL, 3 * n); s->y0 = dup(NULL, 3 * n); s->ytmp = dup(NULL, 3 * n);
	s->yerr = dup(NULL, 3 * n); s->Htmp = dup(NULL, 3 * n); s->Hacc = dup(NULL, 3 * n);
	s->dtmp = dup(NULL, 3 * n);
	for (int q = 0; q < 8; ++q) s->k[q] = dup(NULL, 3 * n);
	make_tableau(cfg->tableau, &s->tab);
	s->h = cfg->h0;
	return s;
}

void or_solver_destroy(or_solver *s)
{
	if (!s) return;
	double *bufs[] = {s->Ms, s->A, s->alpha, s->kuni, s->kcub, s->ax1, s->ax2, s->P, s->xi, s->j, s->N,
	                  s->f1, s->f2, s->y, s->y0, s->ytmp, s->yerr, s->Htmp, s->Hacc, s->dtmp};
	for (size_t q = 0; q < sizeof(bufs) / sizeof(bufs[0]); ++q) free(bufs[q]);
	for (int q = 0; q < 8; ++q) free(s->k[q]);
	conv_fft_free(s->Nh);
	free(s);
}

/* LandauLifshitzGilbert.update("M") (landau_lifshitz_gilbert.py:84-88): assign + normalise. */
void or_solver_set_M(or_solver *s, const double *M)
{
	memcpy(s->y, M, sizeof(double) * 3 * s->n);
	or_normalize(s->n, s->Ms, s->y, s->cfg.float_norm);
	s->t = 0; s->h = s->cfg.h0; s->have_next = 0; s->k0_is_fsal = 0;
	s->steps = s->attempts = s->rejected = 0;
}

void or_solver_get_M(or_solver *s, double *M) { memcpy(M, s->y, sizeof(double) * 3 * s->n); }

static void add_to(double *acc, const double *v, size_t n3)
{
	for (size_t i = 0; i < n3; ++i) acc[i] += v[i];
}

/* calculate_H_tot + calculate_dMdt (landau_lifshitz_gilbert.py:92-125) at state M, time t. */
static void rhs(or_solver *s, const double *M, double t, double *dMdt, double *Heff, double *Hdemag)
{
	const or_solver_config *c = &s->cfg;
	const size_t n = s->n, n3 = 3 * n;
	double *H = Heff ? Heff : s->Hacc;
	memset(H, 0, sizeof(double) * n3);
	if (c->terms & 1) {
		if (c->use_fft) conv_fft_apply(s->Nh, c->nx, c->ny, c->nz, s->ex, s->ey, s->ez, M, s->Htmp);
		else or_conv_direct(s->N, c->nx, c->ny, c->nz, s->ex, s->ey, s->ez, M, s->Htmp);
		if (Hdemag) memcpy(Hdemag, s->Htmp, sizeof(double) * n3);
		add_to(H, s->Htmp, n3);
	}
	if (c->terms & 2) {
		or_exchange(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->pbc[0], c->pbc[1], c->pbc[2], s->Ms, s->A, M,
		            s->Htmp);
		add_to(H, s->Htmp, n3);
	}
	if (c->terms & 4) {
		or_uniaxial_anisotropy(n, s->ax1, s->kuni, s->Ms, M, s->Htmp);
		add_to(H, s->Htmp, n3);
	}
	if (c->terms & 8) {
		or_cubic_anisotropy(n, s->ax1, s->ax2, s->kcub, s->Ms, M, s->Htmp);
		add_to(H, s->Htmp, n3);
	}
	if (c->terms & 32) {
		/* uniform applied field with a linear rise (the H_ext_fn form of alternating_field.py:68-72) */
		double f = 1.0;
		if (c->pulse_rise > 0) f = t / c->pulse_rise < 1.0 ? t / c->pulse_rise : 1.0;
		for (int q = 0; q < 3; ++q) {
			const double hq = c->H_ext[q] + c->H_pulse[q] * f;
			for (size_t i = 0; i < n; ++i) H[q * n + i] += hq;
		}
	}
	if (dMdt) {
		or_llge(n, s->f1, s->f2, M, H, dMdt);
		if (c->terms & 16) {
			or_fdm_zhangli(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->zl_do_precess, s->P, s->xi, s->Ms,
			               s->alpha, s->j, M, s->dtmp);
			add_to(dMdt, s->dtmp, n3);
		}
	}
}

void or_solver_eval(or_solver *s, double *H_eff, double *dMdt, double *H_demag)
{
	double *d = dMdt ? dMdt : NULL;
	rhs(s, s->y, s->t, d, H_eff, H_demag);
}

/* RungeKutta.apply (magnum/evolver/runge_kutta.py:89-137); returns k[0] of this attempt.
 * With a first-same-as-last tableau, k[0] and k[last] swap buffers afterwards, so k[0] holds
 * state.dydt_in for the next attempt while the returned buffer stays intact until the next
 * attempt's last stage. */
static double *rk_apply(or_solver *s, double h)
{
	const tableau_t *tb = &s->tab;
	const size_t n3 = 3 * s->n;
	double **k = s->k;
	s->attempts++;
	if (!(tb->fsal && s->k0_is_fsal)) rhs(s, s->y, s->t, k[0], NULL, NULL);
	for (int st = 1; st < tb->s; ++st) {
		memcpy(s->ytmp, s->y, sizeof(double) * n3);
		for (int q = 0; q < st; ++q) {
			const double f = h * tb->b[st][q];
			for (size_t i = 0; i < n3; ++i) s->ytmp[i] += f * k[q][i];
		}
		rhs(s, s->ytmp, s->t + h * tb->a[st], k[st], NULL, NULL);
	}
	memset(s->yerr, 0, sizeof(double) * n3);
	for (int st = 0; st < tb->s; ++st) {
		const double fc = h * tb->c[st], fe = h * tb->ec[st];
		for (size_t i = 0; i < n3; ++i) {
			s->y[i] += fc * k[st][i];
			s->yerr[i] += fe * k[st][i];
		}
	}
	double *k0 = k[0];
	if (tb->fsal) {
		k[0] = k[tb->s - 1];
		k[tb->s - 1] = k0;
		s->k0_is_fsal = 1;
	}
	return k0;
}

/* MicroMagneticsStepSizeController.adjust_stepsize
 * (magnum/micromagnetics/micro_magnetics_stepsize_controller.py:35-73). */
static int controller(or_solver *s, double h, const double *dydt, double *h_new)
{
	const double max_y_err = or_scaled_abs_max(s->n, s->yerr, s->Ms);
	const double max_dydt = or_scaled_abs_max(s->n, dydt, s->Ms);
	const double e_abs = max_y_err;
	if (h * max_dydt == 0.0) { *h_new = 5e-14; return 1; }
	const double e_rel = e_abs / (h * max_dydt);
	int accept = (e_abs <= s->cfg.eps_abs) && (e_rel <= s->cfg.eps_rel);
	const int order = s->tab.order;
	/* e_abs == 0 raises ZeroDivisionError in the reference; here it means "grow by the maximum" */
	const double sa = e_abs > 0 ? 0.85 * pow(s->cfg.eps_abs / e_abs, 1.0 / (order + 1.0)) : 5.0;
	const double sr = e_rel > 0 ? 0.85 * pow(s->cfg.eps_rel / e_rel, 1.0 / order) : 5.0;
	double sc = sa < sr ? sa : sr;
	if (sc < 0.2) sc = 0.2;
	if (sc > 5.0) sc = 5.0;
	double hn = h * sc;
	if (hn < 1e-15) hn = 1e-15;
	if (hn > 1e-10) hn = 1e-10;
	if (hn == 1e-15) accept = 1;
	*h_new = hn;
	return accept;
}

/* RungeKutta.evolve (runge_kutta.py:47-87) + MicroMagneticsState.finish_step
 * (micro_magnetics.py:49-50). */
void or_solver_step(or_solver *s, double t_max)
{
	const size_t n3 = 3 * s->n;
	memcpy(s->y0, s->y, sizeof(double) * n3);
	double h_try = s->have_next ? s->h_next : s->h;
	double h_new = h_try;
	for (;;) {
		const double *dydt = rk_apply(s, h_try);
		const int accept = controller(s, h_try, dydt, &h_new);
		if (!accept) {
			s->rejected++;
			if (!s->cfg.fsal_reuse_after_reject) s->k0_is_fsal = 0;
			memcpy(s->y, s->y0, sizeof(double) * n3);
			h_try = h_new;
			continue;
		}
		break;
	}
	if (s->t + h_try > t_max) {
		h_try = t_max - s->t;
		memcpy(s->y, s->y0, sizeof(double) * n3);
		rk_apply(s, h_try);
	}
	s->t += h_try;
	s->h = h_try;
	s->h_next = h_new;
	s->have_next = 1;
	s->steps++;
	or_normalize(s->n, s->Ms, s->y, s->cfg.float_norm);
}

static void average_M(or_solver *s, double *out)
{
	const size_t n = s->n;
	for (int c = 0; c < 3; ++c) {
		double acc = 0;
		for (size_t i = 0; i < n; ++i) acc += s->y[c * n + i];
		out[c] = acc / (double)n;
	}
}

/* Solver.solve(condition.Time(t_end)) with an EveryNthSecond(sample_dt) step handler
 * (magnum/solver/solver.py:76-139, condition.py:121-157). */
int or_solver_run(or_solver *s, double t_end, double sample_dt, double *sample_t, double *samples, int max_samples)
{
	int count = 0;
	const int sampling = sample_dt > 0;
#define HANDLE()                                                                        \
	if (sampling) {                                                                     \
		const double r = fmod(s->t, sample_dt);                                         \
		if ((fabs(r) < 1e-16 || fabs(r - sample_dt) < 1e-16) && count < max_samples) {  \
			sample_t[count] = s->t;                                                     \
			average_M(s, samples + 3 * count);                                          \
			++count;                                                                    \
		}                                                                               \
	}
	HANDLE();
	while (!(s->t >= t_end)) {
		double t1 = 1e100;
		if (sampling) {
			const double toi = ((double)(long long)(s->t / sample_dt) + 1) * sample_dt;
			if (toi > s->t && toi < t1) t1 = toi;
		}
		or_solver_step(s, t1);
		HANDLE();
	}
#undef HANDLE
	return count;
}

void or_solver_stats(or_solver *s, double *o)
{
	o[0] = s->t; o[1] = s->h; o[2] = s->have_next ? s->h_next : s->h;
	o[3] = (double)s->steps; o[4] = (double)s->attempts; o[5] = (double)s->rejected;
}

/* Timing helper: one attempt from the current state; y, t and the counters of accepted steps
 * are restored afterwards (the first-same-as-last stage becomes this attempt's last stage). */
void or_solver_attempt(or_solver *s, double h)
{
	const size_t n3 = 3 * s->n;
	memcpy(s->y0, s->y, sizeof(double) * n3);
	rk_apply(s, h);
	memcpy(s->y, s->y0, sizeof(double) * n3);
}
