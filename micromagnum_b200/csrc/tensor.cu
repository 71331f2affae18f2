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

mm_status gl_table(GLTable **out)
{
	static GLTable tab;
	static bool ready = false;
	if (!ready) {
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
		ready = true;
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

} // extern "C"
