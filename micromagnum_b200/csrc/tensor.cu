// Demagnetisation tensor on the GPU in FP64.  Replaces GenerateDemagTensor / calculateDemagTensor
// (mmm/demag/demag_tensor.cpp:116-186, mmm/demag/tensor.cpp:35-191), non-periodic case.
//
// For a cell offset X = (i dx, j dy, k dz) the tensor of two uniformly magnetised boxes is
//   N_ab(X) = (1/V) * Int_{[-d,d]^3} prod_c (d_c - |u_c|) K_ab(X + u) du,
//   K_ab(r) = (delta_ab r^2 - 3 r_a r_b) / (4 pi |r|^5),
// the average of the point-dipole kernel over all pairs of points of the two cells (the tent
// weights are the overlap lengths).  The reference evaluates Newell's closed forms in long double
// near the origin and truncated asymptotic series further out (tensor_integrals.h:370-462).
// Here:
//  * offsets whose boxes touch (|i|,|j|,|k| <= 1) use Newell's closed forms f and g (Newell,
//    Williams & Dunlop, JGR 98 (1993) 9551) with the 27-point second difference in FP64 -- the
//    cancellation there is mild;
//  * every other offset uses tensor-product Gauss-Legendre quadrature on the two linear halves
//    of each tent, with n nodes per half chosen from the distance D between the box X+[-d,d]
//    and the singularity at 0: rho = r + sqrt(r^2+1), r = D/(d_c/2), n = ceil(20/ln rho) + 1.
//    This keeps the relative error near 1e-15 (checked against a binary128 Newell evaluation),
//    including the far field where the reference's series truncation is visible (~1e-8 in H).
// Output: the NEGATED tensor in the reference's Matrix(Shape(6, ex, ey, ez)) layout (component
// fastest), components (xx, xy, xz, yy, yz, zz), scattered into the eight octants with the
// parities of tensor.cpp:167-180.
#include "mm_common.cuh"

#include <cmath>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace mm {
namespace {

constexpr int GL_MAX = 40;

struct GLTable {
	double *x = nullptr;  // nodes on [-1, 1], table for n starts at n(n-1)/2
	double *w = nullptr;
};

// Gauss-Legendre nodes and weights by Newton iteration on P_n (long double).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w)
{
	x.resize(n);
	w.resize(n);
	for (int i = 0; i < n; ++i) {
		long double z = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L));
		long double dp = 0;
		for (int it = 0; it < 100; ++it) {
			long double p0 = 1, p1 = z;
			for (int k = 2; k <= n; ++k) {
				const long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
				p0 = p1;
				p1 = p2;
			}
			if (n == 1) { p1 = z; p0 = 1; }
			dp = n * (z * p1 - p0) / (z * z - 1);
			const long double dz = p1 / dp;
			z -= dz;
			if (fabsl(dz) < 1e-21L) break;
		}
		{
			long double p0 = 1, p1 = z;
			for (int k = 2; k <= n; ++k) {
				const long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
				p0 = p1;
				p1 = p2;
			}
			dp = n * (z * p1 - p0) / (z * z - 1);
		}
		x[i] = (double)z;
		w[i] = (double)(2.0L / ((1 - z * z) * dp * dp));
	}
}

// The node/weight table lives in device memory, so each device gets its own (built on first use).
mm_status gl_table(GLTable **out)
{
	static std::mutex mu;
	static std::vector<GLTable> tabs;
	int dev = 0;
	MM_CUDA(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(mu);
	if ((int)tabs.size() <= dev) tabs.resize(dev + 1);
	GLTable &tab = tabs[dev];
	if (!tab.x) {
		std::vector<double> hx, hw, x, w;
		for (int n = 1; n <= GL_MAX; ++n) {
			if (n == 1) { x = {0.0}; w = {2.0}; }
			else gauss_legendre(n, x, w);
			hx.insert(hx.end(), x.begin(), x.end());
			hw.insert(hw.end(), w.begin(), w.end());
		}
		MM_CUDA(cudaMalloc(&tab.x, hx.size() * sizeof(double)));
		MM_CUDA(cudaMalloc(&tab.w, hw.size() * sizeof(double)));
		MM_CUDA(cudaMemcpy(tab.x, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice));
		MM_CUDA(cudaMemcpy(tab.w, hw.data(), hw.size() * sizeof(double), cudaMemcpyHostToDevice));
	}
	*out = &tab;
	return MM_OK;
}

// Newell f (even in every argument).
__device__ double newell_f(double x, double y, double z)
{
	const double x2 = x * x, y2 = y * y, z2 = z * z, R2 = x2 + y2 + z2;
	if (R2 == 0.0) return 0.0;
	const double R = sqrt(R2);
	double r = (2 * x2 - y2 - z2) * R / 6;
	if (x2 + z2 > 0 && y != 0) r += y / 2 * (z2 - x2) * asinh(y / sqrt(x2 + z2));
	if (x2 + y2 > 0 && z != 0) r += z / 2 * (y2 - x2) * asinh(z / sqrt(x2 + y2));
	if (x != 0 && y != 0 && z != 0) r -= x * y * z * atan(y * z / (x * R));
	return r;
}

// Newell g (odd in x and y, even in z).
__device__ double newell_g(double x, double y, double z)
{
	const double x2 = x * x, y2 = y * y, z2 = z * z, R2 = x2 + y2 + z2;
	if (R2 == 0.0) return 0.0;
	const double R = sqrt(R2);
	double r = -x * y * R / 3;
	if (x != 0 && y != 0 && z != 0) r += x * y * z * asinh(z / sqrt(x2 + y2));
	if (x != 0 && y != 0) {
		if (y2 + z2 > 0) r += y / 6 * (3 * z2 - y2) * asinh(x / sqrt(y2 + z2));
		if (x2 + z2 > 0) r += x / 6 * (3 * z2 - x2) * asinh(y / sqrt(x2 + z2));
	}
	if (x != 0 && y != 0 && z != 0) {
		r -= z * z2 / 6 * atan(x * y / (z * R));
		r -= z * y2 / 2 * atan(x * z / (y * R));
		r -= z * x2 / 2 * atan(y * z / (x * R));
	}
	return r;
}

// Negated tensor (xx, xy, xz, yy, yz, zz) at offset (i, j, k) from Newell's formulas.
__device__ void tensor_newell(int i, int j, int k, double dx, double dy, double dz, double *v)
{
	double acc[6] = {0, 0, 0, 0, 0, 0};
	for (int cz = -1; cz <= 1; ++cz)
		for (int cy = -1; cy <= 1; ++cy)
			for (int cx = -1; cx <= 1; ++cx) {
				const double w = (cx ? -1.0 : 2.0) * (cy ? -1.0 : 2.0) * (cz ? -1.0 : 2.0);
				const double X = (i + cx) * dx, Y = (j + cy) * dy, Z = (k + cz) * dz;
				acc[0] += w * newell_f(X, Y, Z);
				acc[3] += w * newell_f(Y, X, Z);
				acc[5] += w * newell_f(Z, Y, X);
				acc[1] += w * newell_g(X, Y, Z);
				acc[2] += w * newell_g(X, Z, Y);
				acc[4] += w * newell_g(Y, Z, X);
			}
	const double pref = -1.0 / (4.0 * PI * dx * dy * dz);
	for (int c = 0; c < 6; ++c) v[c] = pref * acc[c];
}

__device__ int gl_order(double D, double halfwidth)
{
	const double r = D / halfwidth;
	const double rho = r + sqrt(r * r + 1.0);
	const double lr = log(rho);
	if (!(lr > 0.0)) return GL_MAX + 1;
	const double n = ceil(20.0 / lr) + 1.0;
	return n < 3.0 ? 3 : (n > GL_MAX ? GL_MAX + 1 : (int)n);
}

// Negated tensor at offset (i, j, k) by quadrature; returns false if the orders needed exceed
// the table (the caller then uses Newell's formulas).
__device__ bool tensor_quad(int i, int j, int k, double dx, double dy, double dz, const double *glx,
                            const double *glw, double *v)
{
	const double X[3] = {i * dx, j * dy, k * dz};
	const double a[3] = {dx, dy, dz};
	double g2 = 0;
	for (int c = 0; c < 3; ++c) {
		const double g = fmax(fabs(X[c]) - a[c], 0.0);
		g2 += g * g;
	}
	const double D = sqrt(g2);
	int n[3];
	for (int c = 0; c < 3; ++c) {
		n[c] = gl_order(D, 0.5 * a[c]);
		if (n[c] > GL_MAX) return false;
	}
	const double *xs[3], *ws[3];
	for (int c = 0; c < 3; ++c) {
		xs[c] = glx + n[c] * (n[c] - 1) / 2;
		ws[c] = glw + n[c] * (n[c] - 1) / 2;
	}
	double acc[6] = {0, 0, 0, 0, 0, 0};
	// u_c in [-a_c, 0] and [0, a_c]: u = (s - 1 + ... ) mapped per half, tent weight (a - |u|)
	for (int hz = 0; hz < 2; ++hz)
		for (int qz = 0; qz < n[2]; ++qz) {
			const double uz = (hz ? 0.5 : -0.5) * a[2] + 0.5 * a[2] * xs[2][qz];
			const double wz = 0.5 * a[2] * ws[2][qz] * (a[2] - fabs(uz));
			const double rz = X[2] + uz;
			for (int hy = 0; hy < 2; ++hy)
				for (int qy = 0; qy < n[1]; ++qy) {
					const double uy = (hy ? 0.5 : -0.5) * a[1] + 0.5 * a[1] * xs[1][qy];
					const double wyz = wz * 0.5 * a[1] * ws[1][qy] * (a[1] - fabs(uy));
					const double ry = X[1] + uy;
					const double ryz2 = ry * ry + rz * rz;
					double s_xx = 0, s_xy = 0, s_xz = 0, s_yy = 0, s_yz = 0, s_zz = 0;
					for (int hx = 0; hx < 2; ++hx)
						for (int qx = 0; qx < n[0]; ++qx) {
							const double ux = (hx ? 0.5 : -0.5) * a[0] + 0.5 * a[0] * xs[0][qx];
							const double wx = 0.5 * a[0] * ws[0][qx] * (a[0] - fabs(ux));
							const double rx = X[0] + ux;
							const double r2 = rx * rx + ryz2;
							const double ir = rsqrt(r2);
							const double ir3 = ir * ir * ir;
							const double w3 = wx * ir3;
							const double w5 = 3.0 * w3 / r2;
							s_xx += w3 - w5 * rx * rx;
							s_yy += w3 - w5 * ry * ry;
							s_zz += w3 - w5 * rz * rz;
							s_xy -= w5 * rx * ry;
							s_xz -= w5 * rx * rz;
							s_yz -= w5 * ry * rz;
						}
					acc[0] += wyz * s_xx;
					acc[1] += wyz * s_xy;
					acc[2] += wyz * s_xz;
					acc[3] += wyz * s_yy;
					acc[4] += wyz * s_yz;
					acc[5] += wyz * s_zz;
				}
		}
	const double pref = -1.0 / (4.0 * PI * dx * dy * dz);
	for (int c = 0; c < 6; ++c) v[c] = pref * acc[c];
	return true;
}

__global__ void __launch_bounds__(128) k_demag_tensor(int nx, int ny, int nz, double dx, double dy,
                                                      double dz, int ex, int ey, int ez,
                                                      const double *__restrict__ glx,
                                                      const double *__restrict__ glw,
                                                      double *__restrict__ out)
{
	const size_t cnt = (size_t)nx * ny * nz;
	for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
		const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((size_t)nx * ny));
		double v[6];
		const bool touching = i <= 1 && j <= 1 && k <= 1;
		if (touching || !tensor_quad(i, j, k, dx, dy, dz, glx, glw, v)) tensor_newell(i, j, k, dx, dy, dz, v);
		for (int o = -1; o <= 1; o += 2)
			for (int p = -1; p <= 1; p += 2)
				for (int r = -1; r <= 1; r += 2) {
					if ((i == 0 && o < 0) || (j == 0 && p < 0) || (k == 0 && r < 0)) continue;
					const int I = (o * i + ex) % ex, J = (p * j + ey) % ey, K = (r * k + ez) % ez;
					double *d = out + 6 * (((size_t)K * ey + J) * ex + I);
					d[0] = v[0];
					d[1] = o * p * v[1];
					d[2] = o * r * v[2];
					d[3] = v[3];
					d[4] = p * r * v[4];
					d[5] = v[5];
				}
	}
}

// ---- periodic boundaries (tensor.cpp:35-165 with demag_tensor.cpp:116-186) --------------------
// Along a periodic axis the tensor of offset i sums the images i + r n (r < R, the repetitions);
// the octant scatter adds the mirrored images -(i + r n), so an entry sums displacements from
// -R n to (R - 1) n around it.  Offsets that coincide with their mirror (i + r n == 0) count
// half on each side, as the reference divides by its "mcs" factor.  The images beyond the R-th
// (the reference's infinity correction, tensor.cpp:60-165) are far from the box: their sum is the
// point-dipole tensor (V / 4 pi) d_a d_b (1 / r), here summed explicitly over TAIL_M further images
// and integrated in closed form beyond (line integrals with the first Euler-Maclaurin correction for
// the images along one periodic axis, quadrant integrals for the far corner of two periodic axes,
// tensor.cpp:104-161), below 1e-9 of the tail sums.  The reference approximates the same sums
// by asymptotic expansions; no three-axis corner term exists there, nor here.
constexpr int TAIL_M = 32;

// (V / 4 pi) d_a d_b (1 / r) at r = P: the far-field negated tensor of one cell (xx xy xz yy yz zz)
__device__ void point_dipole(const double P[3], double V4, double *v)
{
	const double r2 = P[0] * P[0] + P[1] * P[1] + P[2] * P[2];
	const double ir = rsqrt(r2), ir3 = ir * ir * ir, ir5 = ir3 * ir * ir;
	v[0] += V4 * (3 * P[0] * P[0] * ir5 - ir3);
	v[1] += V4 * 3 * P[0] * P[1] * ir5;
	v[2] += V4 * 3 * P[0] * P[2] * ir5;
	v[3] += V4 * (3 * P[1] * P[1] * ir5 - ir3);
	v[4] += V4 * 3 * P[1] * P[2] * ir5;
	v[5] += V4 * (3 * P[2] * P[2] * ir5 - ir3);
}

__device__ __forceinline__ int sym_idx(int a, int b)
{
	const int lo = a < b ? a : b, hi = a < b ? b : a;
	return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

// Integral over s in [0, inf) of d_a d_b (1 / r) at r = P + s e_A (P_A > 0), added times f.
__device__ void line_integral(const double P[3], int A, double f, double *v)
{
	const int B = (A + 1) % 3, C = (A + 2) % 3;
	const double x0 = P[A], y = P[B], z = P[C];
	const double r0 = sqrt(x0 * x0 + y * y + z * z), w = x0 + r0, ir3 = 1.0 / (r0 * r0 * r0);
	const double q = (w + r0) * ir3 / (w * w);
	v[sym_idx(A, A)] += f * x0 * ir3;
	v[sym_idx(A, B)] += f * y * ir3;
	v[sym_idx(A, C)] += f * z * ir3;
	v[sym_idx(B, B)] += f * (y * y * q - 1.0 / (r0 * w));
	v[sym_idx(B, C)] += f * y * z * q;
	v[sym_idx(C, C)] += f * (z * z * q - 1.0 / (r0 * w));
}

// Integral over s, t in [0, inf) of d_a d_b (1 / r) at r = P + s e_A + t e_B (P_A, P_B > 0).
__device__ void quadrant_integral(const double P[3], int A, int B, double f, double *v)
{
	const int C = 3 - A - B;
	const double x0 = P[A], y0 = P[B], z = P[C];
	const double r0 = sqrt(x0 * x0 + y0 * y0 + z * z);
	const double a2 = x0 * x0 + z * z, b2 = y0 * y0 + z * z;
	const double xx = x0 / a2 * (1.0 - y0 / r0), yy = y0 / b2 * (1.0 - x0 / r0);
	v[sym_idx(A, A)] += f * xx;
	v[sym_idx(B, B)] += f * yy;
	v[sym_idx(C, C)] -= f * (xx + yy);
	v[sym_idx(A, B)] += f / r0;
	v[sym_idx(A, C)] += f * z / a2 * (1.0 - y0 / r0);
	v[sym_idx(B, C)] += f * z / b2 * (1.0 - x0 / r0);
}

// f d_A d_a d_b (1 / r) at r = P, added (the derivative along A of d_a d_b (1 / r)).
__device__ void line_derivative(const double P[3], int A, double f, double *v)
{
	const double r2 = P[0] * P[0] + P[1] * P[1] + P[2] * P[2];
	const double ir = rsqrt(r2), ir5 = ir * ir * ir * ir * ir, ir7 = ir5 * ir * ir;
	const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
	for (int c = 0; c < 6; ++c) {
		const int a = ab[c][0], b = ab[c][1];
		double t = -15.0 * P[a] * P[b] * P[A] * ir7;
		if (a == b) t += 3.0 * P[A] * ir5;
		if (a == A) t += 3.0 * P[b] * ir5;
		if (b == A) t += 3.0 * P[a] * ir5;
		v[c] += f * t;
	}
}

// The images P + r L e_A for r >= TAIL_M, in place of their sum: the midpoint rule with its first
// Euler-Maclaurin correction, L^-1 int_{s_M}^inf f + (L / 24) d_A f(s_M), s_M = P + (TAIL_M - 1/2) L e_A
// (the next term is below 1e-9 of the sum).
__device__ void line_continuum(double P[3], int A, double L, double V4, double *v)
{
	const double p0 = P[A];
	P[A] = p0 + (TAIL_M - 0.5) * L;
	line_integral(P, A, V4 / L, v);
	line_derivative(P, A, V4 * L / 24.0, v);
	P[A] = p0;
}

// Images P + r L e_A, r >= 0 (point dipoles of one cell).
__device__ void line_tail(double P[3], int A, double L, double V4, double *v)
{
	const double p0 = P[A];
	for (int r = 0; r < TAIL_M; ++r) {
		P[A] = p0 + r * L;
		point_dipole(P, V4, v);
	}
	P[A] = p0;
	line_continuum(P, A, L, V4, v);
}

// Images P + r L_A e_A + s L_B e_B, r, s >= 0.
__device__ void corner_tail(double P[3], int A, int B, double LA, double LB, double V4, double *v)
{
	const double pa = P[A], pb = P[B];
	for (int s = 0; s < TAIL_M; ++s) {
		P[B] = pb + s * LB;
		for (int r = 0; r < TAIL_M; ++r) {
			P[A] = pa + r * LA;
			point_dipole(P, V4, v);
		}
		P[A] = pa;
		line_continuum(P, A, LA, V4, v);
	}
	P[B] = pb;
	for (int r = 0; r < TAIL_M; ++r) {
		P[A] = pa + r * LA;
		line_continuum(P, B, LB, V4, v);
	}
	P[B] = pb + (TAIL_M - 0.5) * LB;
	P[A] = pa + (TAIL_M - 0.5) * LA;
	quadrant_integral(P, A, B, V4 / (LA * LB), v);
	P[A] = pa;
	P[B] = pb;
}

// Sum over images of the negated tensor of source offset (i, j, k), halved for each coordinate
// at zero displacement, plus the far images (tails); out[6] per source offset.
__global__ void __launch_bounds__(128) k_tensor_images(int nx, int ny, int nz, double dx, double dy, double dz,
                                                       int Rx, int Ry, int Rz, int tails,
                                                       const double *__restrict__ glx,
                                                       const double *__restrict__ glw, double *__restrict__ out)
{
	const size_t cnt = (size_t)nx * ny * nz;
	const int n3[3] = {nx, ny, nz}, R3[3] = {Rx, Ry, Rz};
	const double d3[3] = {dx, dy, dz};
	const double V4 = dx * dy * dz / (4.0 * PI);
	for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
		const int ijk[3] = {(int)(q % nx), (int)((q / nx) % ny), (int)(q / ((size_t)nx * ny))};
		double S[6] = {0, 0, 0, 0, 0, 0};
		for (int rz = 0; rz < Rz; ++rz)
			for (int ry = 0; ry < Ry; ++ry)
				for (int rx = 0; rx < Rx; ++rx) {
					const int I = ijk[0] + rx * nx, J = ijk[1] + ry * ny, K = ijk[2] + rz * nz;
					const double w = (I == 0 ? 0.5 : 1.0) * (J == 0 ? 0.5 : 1.0) * (K == 0 ? 0.5 : 1.0);
					double v[6];
					const bool touching = I <= 1 && J <= 1 && K <= 1;
					if (touching || !tensor_quad(I, J, K, dx, dy, dz, glx, glw, v)) tensor_newell(I, J, K, dx, dy, dz, v);
					for (int c = 0; c < 6; ++c) S[c] += w * v[c];
				}
		if (tails) {
			// one periodic axis beyond its repetitions, the others within theirs (tensor.cpp:60-104)
			for (int A = 0; A < 3; ++A) {
				if (R3[A] <= 1) continue;
				const int B = (A + 1) % 3, C = (A + 2) % 3;
				for (int rc = 0; rc < R3[C]; ++rc)
					for (int rb = 0; rb < R3[B]; ++rb) {
						const int IB = ijk[B] + rb * n3[B], IC = ijk[C] + rc * n3[C];
						const double w = (IB == 0 ? 0.5 : 1.0) * (IC == 0 ? 0.5 : 1.0);
						double P[3];
						P[A] = (ijk[A] + R3[A] * n3[A]) * d3[A];
						P[B] = IB * d3[B];
						P[C] = IC * d3[C];
						double v[6] = {0, 0, 0, 0, 0, 0};
						line_tail(P, A, n3[A] * d3[A], V4, v);
						for (int c = 0; c < 6; ++c) S[c] += w * v[c];
					}
			}
			// two periodic axes beyond their repetitions (tensor.cpp:105-161)
			for (int A = 0; A < 3; ++A)
				for (int B = A + 1; B < 3; ++B) {
					if (R3[A] <= 1 || R3[B] <= 1) continue;
					const int C = 3 - A - B;
					for (int rc = 0; rc < R3[C]; ++rc) {
						const int IC = ijk[C] + rc * n3[C];
						const double w = IC == 0 ? 0.5 : 1.0;
						double P[3];
						P[A] = (ijk[A] + R3[A] * n3[A]) * d3[A];
						P[B] = (ijk[B] + R3[B] * n3[B]) * d3[B];
						P[C] = IC * d3[C];
						double v[6] = {0, 0, 0, 0, 0, 0};
						corner_tail(P, A, B, n3[A] * d3[A], n3[B] * d3[B], V4, v);
						for (int c = 0; c < 6; ++c) S[c] += w * v[c];
					}
				}
		}
		for (int c = 0; c < 6; ++c) out[6 * q + c] = S[c];
	}
}

// Every entry (I, J, K) of the padded tensor gathers its sources of the eight octants: along an
// axis, octant o = +-1 reads source offset (o I + e) mod e when that is below n (tensor.cpp:166-180
// scatters the same sums), with the parity signs of the off-diagonal components.
__global__ void __launch_bounds__(128) k_tensor_gather(int nx, int ny, int nz, int ex, int ey, int ez,
                                                       const double *__restrict__ S, double *__restrict__ out)
{
	const size_t cnt = (size_t)ex * ey * ez;
	for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
		const int I = (int)(q % ex), J = (int)((q / ex) % ey), K = (int)(q / ((size_t)ex * ey));
		double acc[6] = {0, 0, 0, 0, 0, 0};
		for (int o = -1; o <= 1; o += 2) {
			const int i = (o * I + ex) % ex;
			if (i >= nx) continue;
			for (int p = -1; p <= 1; p += 2) {
				const int j = (p * J + ey) % ey;
				if (j >= ny) continue;
				for (int r = -1; r <= 1; r += 2) {
					const int k = (r * K + ez) % ez;
					if (k >= nz) continue;
					const double *s = S + 6 * (((size_t)k * ny + j) * nx + i);
					acc[0] += s[0];
					acc[1] += o * p * s[1];
					acc[2] += o * r * s[2];
					acc[3] += s[3];
					acc[4] += p * r * s[4];
					acc[5] += s[5];
				}
			}
		}
		for (int c = 0; c < 6; ++c) out[6 * q + c] = acc[c];
	}
}

} // namespace
} // namespace mm

using namespace mm;

extern "C" {

MM_API int mm_round_tensor_dimension(int dim, int periodic, int padding)
{
	// mmm/demag/tensor_round.cpp:90-106
	if (periodic) return dim;
	const int t = 2 * dim - 1;
	if (t == 1) return 1;
	auto round_to = [](int x, int m) { return (x % m) ? x + (m - x % m) : x; };
	switch (padding) {
	case MM_PADDING_DISABLE: return t;
	case MM_PADDING_ROUND_2: return round_to(t, 2);
	case MM_PADDING_ROUND_4: return round_to(t, 4);
	case MM_PADDING_ROUND_8: return round_to(t, 8);
	case MM_PADDING_ROUND_POT: { int p = 1; while (p < t) p <<= 1; return p; }
	case MM_PADDING_SMALL_PRIME_FACTORS: {
		int x = t + 1;
		for (;; ++x) {
			int m = x;
			for (int p : {2, 3, 5}) while (m % p == 0) m /= p;
			if (m == 1) return x;
		}
	}
	default: return -1;
	}
}

MM_API mm_status mm_demag_tensor(int nx, int ny, int nz, double dx, double dy, double dz, int ex,
                                 int ey, int ez, double *N_out, void *stream)
{
	if (nx <= 0 || ny <= 0 || nz <= 0 || !(dx > 0) || !(dy > 0) || !(dz > 0) || !N_out)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_demag_tensor: invalid argument");
	if (ex < 2 * nx - 1 || ey < 2 * ny - 1 || ez < 2 * nz - 1)
		return fail(MM_ERR_UNSUPPORTED,
		            "mm_demag_tensor: padded sizes below 2n-1 (periodic boundaries) are not supported");
	cudaStream_t st = as_stream(stream);
	GLTable *gl = nullptr;
	MM_TRY(gl_table(&gl));
	MM_CUDA(cudaMemsetAsync(N_out, 0, sizeof(double) * 6 * (size_t)ex * ey * ez, st));
	const size_t cnt = (size_t)nx * ny * nz;
	const size_t want = (cnt + 127) / 128;
	const int grid = (int)(want < 65535u * 16 ? want : 65535u * 16);
	k_demag_tensor<<<grid, 128, 0, st>>>(nx, ny, nz, dx, dy, dz, ex, ey, ez, gl->x, gl->w, N_out);
	return after_launch("k_demag_tensor");
}

MM_API mm_status mm_demag_tensor_periodic(int nx, int ny, int nz, double dx, double dy, double dz, int pbc_x,
                                          int pbc_y, int pbc_z, int repeat, int ex, int ey, int ez, double *N_out,
                                          void *stream)
{
	if (nx <= 0 || ny <= 0 || nz <= 0 || !(dx > 0) || !(dy > 0) || !(dz > 0) || !N_out || repeat < 1)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_demag_tensor_periodic: invalid argument");
	const int n3[3] = {nx, ny, nz}, e3[3] = {ex, ey, ez}, pb[3] = {pbc_x, pbc_y, pbc_z};
	for (int a = 0; a < 3; ++a)
		if (pb[a] ? e3[a] != n3[a] : e3[a] < 2 * n3[a] - 1)
			return fail(MM_ERR_INVALID_ARGUMENT, "mm_demag_tensor_periodic: a periodic axis needs e == n, the "
			                                     "others e >= 2n - 1 (round_tensor_dimension)");
	if (!pbc_x && !pbc_y && !pbc_z) return mm_demag_tensor(nx, ny, nz, dx, dy, dz, ex, ey, ez, N_out, stream);
	cudaStream_t st = as_stream(stream);
	GLTable *gl = nullptr;
	MM_TRY(gl_table(&gl));
	const size_t cnt = (size_t)nx * ny * nz;
	double *S = nullptr;
	MM_CUDA(cudaMallocAsync(&S, 6 * cnt * sizeof(double), st));
	const char *off = std::getenv("MAGNUM_DEMAG_NO_INFINITY_CORRECTION");  // tensor.cpp:45
	const int Rx = pbc_x ? repeat : 1, Ry = pbc_y ? repeat : 1, Rz = pbc_z ? repeat : 1;
	const size_t want = (cnt + 127) / 128;
	k_tensor_images<<<(int)(want < 65535u * 16 ? want : 65535u * 16), 128, 0, st>>>(
	    nx, ny, nz, dx, dy, dz, Rx, Ry, Rz, off ? 0 : 1, gl->x, gl->w, S);
	mm_status r = after_launch("k_tensor_images");
	if (r == MM_OK) {
		const size_t out = (size_t)ex * ey * ez, w2 = (out + 127) / 128;
		k_tensor_gather<<<(int)(w2 < 65535u * 16 ? w2 : 65535u * 16), 128, 0, st>>>(nx, ny, nz, ex, ey, ez, S, N_out);
		r = after_launch("k_tensor_gather");
	}
	cudaFreeAsync(S, st);
	return r;
}

} // extern "C"
