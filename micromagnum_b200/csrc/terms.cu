// Stand-alone field terms behind the reference's per-term magneto calls: exchange, uniaxial and
// cubic anisotropy, LLG, Zhang-Li torque, scaled_abs_max, normalisation and the Runge-Kutta
// stage helpers.  These serve the drop-in boundary (one call per term, like the reference);
// the fused solver in solver.cu computes the same physics in one pass per stage.
//
// All kernels are grid-stride loops over cells, one thread per cell, x fastest so that every
// warp reads 32 consecutive elements of each SoA array.
#include "mm_common.cuh"

#include <mutex>

namespace mm {
namespace {

constexpr int TPB = 256;

inline int grid_for(size_t n)
{
	const size_t want = (n + TPB - 1) / TPB;
	const size_t cap = (size_t)num_sms() * 8;
	return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

// ---- exchange (mmm/exchange/exchange_cpu.cpp:60-235) ------------------------------------------
template <typename T, bool PX, bool PY, bool PZ>
__global__ void __launch_bounds__(TPB) k_exchange(int nx, int ny, int nz, double wx, double wy,
                                                  double wz, const T *__restrict__ Ms,
                                                  const T *__restrict__ A, const T *__restrict__ M,
                                                  T *__restrict__ H, double *energy)
{
	const size_t n = (size_t)nx * ny * nz;
	const size_t nxy = (size_t)nx * ny;
	double e = 0.0;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
	     i += (size_t)gridDim.x * blockDim.x) {
		const int x = (int)(i % nx);
		const int y = (int)((i / nx) % ny);
		const int z = (int)(i / nxy);
		const T ms = Ms[i];
		if (ms == T(0)) {
			store3(H, i, n, v3<T>(0, 0, 0));
			continue;
		}
		const V3<T> Mi = load3(M, i, n);
		const V3<T> mi = scale_rn(T(1) / ms, Mi);
		V3<T> sum = v3<T>(0, 0, 0);
		auto add = [&](size_t j, T w) {
			const T msj = Ms[j];
			if (msj != T(0)) {
				const V3<T> mj = scale_rn(T(1) / msj, load3(M, j, n));
				sum = sum + w * (mj - mi);
			}
		};
		const T Wx = (T)wx, Wy = (T)wy, Wz = (T)wz;
		if (x > 0) add(i - 1, Wx); else if (PX) add(i + nx - 1, Wx);
		if (x < nx - 1) add(i + 1, Wx); else if (PX) add(i - (nx - 1), Wx);
		if (y > 0) add(i - nx, Wy); else if (PY) add(i + nxy - nx, Wy);
		if (y < ny - 1) add(i + nx, Wy); else if (PY) add(i - (nxy - nx), Wy);
		if (z > 0) add(i - nxy, Wz); else if (PZ) add(i + n - nxy, Wz);
		if (z < nz - 1) add(i + nxy, Wz); else if (PZ) add(i - (n - nxy), Wz);
		const T pre = (T)(2.0 / MU0) * A[i] / ms;
		const V3<T> Hi = pre * sum;
		store3(H, i, n, Hi);
		if (energy) e += (double)dot(Mi, Hi);
	}
	if (energy) block_sum_to(energy, e);
}

template <typename T>
mm_status run_exchange(int nx, int ny, int nz, double dx, double dy, double dz, bool px, bool py,
                       bool pz, const void *Ms, const void *A, const void *M, void *H,
                       double *energy_host, cudaStream_t st)
{
	const size_t n = (size_t)nx * ny * nz;
	double *acc = nullptr;
	ScalarScratch *sc = nullptr;
	if (energy_host) {
		MM_TRY(scalar_scratch(&sc));
		acc = sc->dev;
		MM_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
	}
	const double wx = 1.0 / (dx * dx), wy = 1.0 / (dy * dy), wz = 1.0 / (dz * dz);
	const T *ms = (const T *)Ms, *a = (const T *)A, *m = (const T *)M;
	T *h = (T *)H;
	const int g = grid_for(n);
#define MM_EXCH(X, Y, Z) \
	if (px == X && py == Y && pz == Z) k_exchange<T, X, Y, Z><<<g, TPB, 0, st>>>(nx, ny, nz, wx, wy, wz, ms, a, m, h, acc);
	MM_EXCH(false, false, false) MM_EXCH(false, false, true) MM_EXCH(false, true, false)
	MM_EXCH(false, true, true) MM_EXCH(true, false, false) MM_EXCH(true, false, true)
	MM_EXCH(true, true, false) MM_EXCH(true, true, true)
#undef MM_EXCH
	MM_TRY(after_launch("k_exchange"));
	if (energy_host) {
		MM_CUDA(cudaMemcpyAsync(sc->host, acc, sizeof(double), cudaMemcpyDeviceToHost, st));
		MM_CUDA(cudaStreamSynchronize(st));
		*energy_host = -MU0 / 2.0 * sc->host[0] * dx * dy * dz;
	}
	return MM_OK;
}

// ---- uniaxial anisotropy (mmm/anisotropy/anisotropy_cpu.cpp:29-73) ----------------------------
template <typename T>
__global__ void __launch_bounds__(TPB) k_uniaxial(size_t n, const T *__restrict__ axis,
                                                  const T *__restrict__ k, const T *__restrict__ Ms,
                                                  const T *__restrict__ M, T *__restrict__ H,
                                                  double *energy)
{
	double e = 0.0;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
	     i += (size_t)gridDim.x * blockDim.x) {
		const T ms = Ms[i], kk = k[i];
		if (ms == T(0) || kk == T(0)) {
			store3(H, i, n, v3<T>(0, 0, 0));
			continue;
		}
		const V3<T> a = load3(axis, i, n);
		const V3<T> s = (T(1) / ms) * load3(M, i, n);
		const T d = dot(s, a);
		store3(H, i, n, (T(2) * kk * d / ms / (T)MU0) * a);
		if (energy) {
			const V3<T> c = cross(a, s);
			e += (double)kk * (double)dot(c, c);
		}
	}
	if (energy) block_sum_to(energy, e);
}

// ---- cubic anisotropy (anisotropy_cpu.cpp:75-119) ---------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TPB) k_cubic(size_t n, const T *__restrict__ axis1,
                                               const T *__restrict__ axis2, const T *__restrict__ k,
                                               const T *__restrict__ Ms, const T *__restrict__ M,
                                               T *__restrict__ H, double *energy)
{
	double e = 0.0;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
	     i += (size_t)gridDim.x * blockDim.x) {
		const T ms = Ms[i];
		if (ms == T(0)) {
			store3(H, i, n, v3<T>(0, 0, 0));
			continue;
		}
		const T kk = k[i];
		const V3<T> Mi = load3(M, i, n);
		const T len = sqrt(dot(Mi, Mi));
		const V3<T> m = len > T(0) ? (T(1) / len) * Mi : v3<T>(0, 0, 0);
		const V3<T> u1 = load3(axis1, i, n), u2 = load3(axis2, i, n);
		const V3<T> u3 = cross(u1, u2);
		const T a1 = dot(u1, m), a2 = dot(u2, m), a3 = dot(u3, m);
		const T a1s = a1 * a1, a2s = a2 * a2, a3s = a3 * a3;
		const V3<T> h = ((a2s + a3s) * a1) * u1 + ((a1s + a3s) * a2) * u2 + ((a1s + a2s) * a3) * u3;
		store3(H, i, n, ((T)(-2.0 / MU0) * kk / ms) * h);
		if (energy) e += (double)kk * (double)(a1s * a2s + a1s * a3s + a2s * a3s);
	}
	if (energy) block_sum_to(energy, e);
}

// ---- LLG right-hand side (mmm/llge/llge_cpu.cpp:25-45) ----------------------------------------
template <typename T>
__global__ void __launch_bounds__(TPB) k_llge(size_t n, const T *__restrict__ f1,
                                              const T *__restrict__ f2, const T *__restrict__ M,
                                              const T *__restrict__ H, T *__restrict__ dM)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
	     i += (size_t)gridDim.x * blockDim.x) {
		const V3<T> m = load3(M, i, n), h = load3(H, i, n);
		const V3<T> mxh = cross(m, h);
		const V3<T> mxmxh = cross(m, mxh);
		store3(dM, i, n, f1[i] * mxh + f2[i] * mxmxh);
	}
}

// ---- Zhang-Li torque (mmm/spintorque/fdm_zhangli_cpu.cpp:57-200) ------------------------------
// For double the reference's order of operations is kept (f1 M x (M x u) + f2 M x u with
// u = (j.grad)M).  For float the same expression is evaluated on unit m:
//   dM = -b'(1+alpha xi) m x (m x u) - b'(xi-alpha) m x u,
// which is algebraically identical but keeps every intermediate inside the float range
// (M x (M x u) reaches ~1e38 A^3/m^4 at j = 1e12 A/m^2, 2 nm cells).
template <typename T>
__global__ void __launch_bounds__(TPB) k_zhangli(int nx, int ny, int nz, double dx, double dy,
                                                 double dz, int do_precess, const T *__restrict__ P,
                                                 const T *__restrict__ xi, const T *__restrict__ Ms,
                                                 const T *__restrict__ alpha, const T *__restrict__ J,
                                                 const T *__restrict__ M, T *__restrict__ dM)
{
	const size_t n = (size_t)nx * ny * nz;
	const size_t nxy = (size_t)nx * ny;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
	     i += (size_t)gridDim.x * blockDim.x) {
		const double ms = (double)Ms[i];
		if (ms == 0.0) {
			store3(dM, i, n, v3<T>(0, 0, 0));
			continue;
		}
		const int x = (int)(i % nx);
		const int y = (int)((i / nx) % ny);
		const int z = (int)(i / nxy);
		const V3<T> Mi = load3(M, i, n);
		auto grad = [&](int c, int dim, size_t stride, double d) -> V3<T> {
			if (dim <= 1) return v3<T>(0, 0, 0);
			if (c == 0) return (T)(1.0 / d) * (load3(M, i + stride, n) - Mi);
			if (c == dim - 1) return (T)(1.0 / d) * (Mi - load3(M, i - stride, n));
			return (T)(1.0 / (2 * d)) * (load3(M, i + stride, n) - load3(M, i - stride, n));
		};
		const V3<T> gx = grad(x, nx, 1, dx), gy = grad(y, ny, nx, dy), gz = grad(z, nz, nxy, dz);
		const V3<T> j = load3(J, i, n);
		const V3<T> u = v3<T>(j.x * gx.x + j.y * gy.x + j.z * gz.x, j.x * gx.y + j.y * gy.y + j.z * gz.y,
		                      j.x * gx.z + j.y * gy.z + j.z * gz.z);
		const double p = (double)P[i], x_i = (double)xi[i], al = (double)alpha[i];
		const double bj = p * MU_BOHR / (ELECTRON_CHARGE * ms * (1.0 + x_i * x_i));
		const double bjp = bj / (1.0 + al * al);
		// (fdm_zhangli_cpu.cpp:85-101) factors with and without the precession term
		const double c1 = do_precess ? (1.0 + al * x_i) : (al * x_i);
		const double c2 = do_precess ? (x_i - al) : (-al);
		if constexpr (sizeof(T) == 8) {
			const double f1 = -bjp / (ms * ms) * c1;
			const double f2 = -bjp / ms * c2;
			const V3<T> B = cross(Mi, u);
			const V3<T> Av = cross(Mi, B);
			store3(dM, i, n, (T)f1 * Av + (T)f2 * B);
		} else {
			const V3<T> m = (T)(1.0 / ms) * Mi;
			const V3<T> B = cross(m, u);
			const V3<T> Av = cross(m, B);
			store3(dM, i, n, (T)(-bjp * c1) * Av + (T)(-bjp * c2) * B);
		}
	}
}

// ---- scaled_abs_max (math/ScaledAbsMax.cpp:33-68) ---------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TPB) k_scaled_abs_max(size_t n, const T *__restrict__ M,
                                                        const T *__restrict__ s, double *out)
{
	double best = 0.0;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
	     i += (size_t)gridDim.x * blockDim.x) {
		const double si = (double)s[i];
		if (si == 0.0) continue;
		const double mx = M[i], my = M[i + n], mz = M[i + 2 * n];
		best = fmax(best, (mx * mx + my * my + mz * mz) / (si * si));
	}
	block_max_to(out, best);
}

// ---- normalisation (kernels_simple.cu:88-103, the GPU path's semantics) -----------------------
template <typename T>
__global__ void __launch_bounds__(TPB) k_normalize(size_t n, const T *__restrict__ Ms, T *__restrict__ M)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
	     i += (size_t)gridDim.x * blockDim.x) {
		const V3<T> v = load3(M, i, n);
		const T len = sqrt(dot(v, v));
		store3(M, i, n, len == T(0) ? v3<T>(0, 0, 0) : (Ms[i] / len) * v);
	}
}

// ---- Runge-Kutta helpers (evolver/runge_kutta_cpu.cpp:28-194) ---------------------------------
constexpr int MAXK = 8;
template <typename T>
struct KPtrs {
	const T *k[MAXK];
	double b[MAXK];
	double ec[MAXK];
};

template <typename T>
__global__ void __launch_bounds__(TPB) k_rk_prepare(size_t n3, int nk, double h, KPtrs<T> kp,
                                                    const T *__restrict__ y, T *__restrict__ ytmp)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3;
	     i += (size_t)gridDim.x * blockDim.x) {
		T acc = y[i];
		for (int j = 0; j < nk; ++j)
			if (kp.b[j] != 0.0) acc += (T)(h * kp.b[j]) * kp.k[j][i];
		ytmp[i] = acc;
	}
}

template <typename T>
__global__ void __launch_bounds__(TPB) k_rk_combine(size_t n3, int nk, double h, KPtrs<T> kp,
                                                    T *__restrict__ y, T *__restrict__ yerr)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3;
	     i += (size_t)gridDim.x * blockDim.x) {
		T acc = y[i], err = T(0);
		for (int j = 0; j < nk; ++j) {
			const T kj = kp.k[j][i];
			if (kp.b[j] != 0.0) acc += (T)(h * kp.b[j]) * kj;
			if (kp.ec[j] != 0.0) err += (T)(h * kp.ec[j]) * kj;
		}
		y[i] = acc;
		yerr[i] = err;
	}
}

// ---- scaled error norm of the NR step-size controller (evolver/runge_kutta_cpu.cpp:196-252, the
// Euclidean branch): sum over all 3N equations of (|err_i| / (eps_rel |y_i| + eps_abs))^2 ------------
template <typename T>
__global__ void __launch_bounds__(TPB) k_rk_error_norm2(size_t n3, double eps_abs, double eps_rel,
                                                        const T *__restrict__ y, const T *__restrict__ yerr,
                                                        double *out)
{
	double acc = 0.0;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3;
	     i += (size_t)gridDim.x * blockDim.x) {
		const double d0 = eps_rel * fabs((double)y[i]) + eps_abs;
		const double r = fabs((double)yerr[i]) / fabs(d0);
		acc += r * r;
	}
	block_sum_to(out, acc);
}

template <typename T>
mm_status finish_energy(double *acc, ScalarScratch *sc, double *energy_host, cudaStream_t st)
{
	MM_CUDA(cudaMemcpyAsync(sc->host, acc, sizeof(double), cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	*energy_host = sc->host[0];
	return MM_OK;
}

bool bad_prec(int prec) { return prec != MM_F64 && prec != MM_F32; }

} // namespace
} // namespace mm

using namespace mm;

extern "C" {

MM_API mm_status mm_exchange(int prec, int nx, int ny, int nz, double dx, double dy, double dz,
                             int pbc_x, int pbc_y, int pbc_z, const void *Ms, const void *A,
                             const void *M, void *H, double *energy_host, void *stream)
{
	if (bad_prec(prec) || nx <= 0 || ny <= 0 || nz <= 0 || !Ms || !A || !M || !H ||
	    !(dx > 0) || !(dy > 0) || !(dz > 0))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_exchange: invalid argument");
	if (prec == MM_F64)
		return run_exchange<double>(nx, ny, nz, dx, dy, dz, pbc_x, pbc_y, pbc_z, Ms, A, M, H,
		                            energy_host, as_stream(stream));
	return run_exchange<float>(nx, ny, nz, dx, dy, dz, pbc_x, pbc_y, pbc_z, Ms, A, M, H,
	                           energy_host, as_stream(stream));
}

MM_API mm_status mm_uniaxial_anisotropy(int prec, size_t n, const void *axis, const void *k,
                                        const void *Ms, const void *M, void *H,
                                        double *energy_host, void *stream)
{
	if (bad_prec(prec) || n == 0 || !axis || !k || !Ms || !M || !H)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_uniaxial_anisotropy: invalid argument");
	cudaStream_t st = as_stream(stream);
	double *acc = nullptr;
	ScalarScratch *sc = nullptr;
	if (energy_host) {
		MM_TRY(scalar_scratch(&sc));
		acc = sc->dev;
		MM_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
	}
	if (prec == MM_F64)
		k_uniaxial<double><<<grid_for(n), TPB, 0, st>>>(n, (const double *)axis, (const double *)k,
		                                                (const double *)Ms, (const double *)M,
		                                                (double *)H, acc);
	else
		k_uniaxial<float><<<grid_for(n), TPB, 0, st>>>(n, (const float *)axis, (const float *)k,
		                                               (const float *)Ms, (const float *)M,
		                                               (float *)H, acc);
	MM_TRY(after_launch("k_uniaxial"));
	if (energy_host) return finish_energy<double>(acc, sc, energy_host, st);
	return MM_OK;
}

MM_API mm_status mm_cubic_anisotropy(int prec, size_t n, const void *axis1, const void *axis2,
                                     const void *k, const void *Ms, const void *M, void *H,
                                     double *energy_host, void *stream)
{
	if (bad_prec(prec) || n == 0 || !axis1 || !axis2 || !k || !Ms || !M || !H)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_cubic_anisotropy: invalid argument");
	cudaStream_t st = as_stream(stream);
	double *acc = nullptr;
	ScalarScratch *sc = nullptr;
	if (energy_host) {
		MM_TRY(scalar_scratch(&sc));
		acc = sc->dev;
		MM_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
	}
	if (prec == MM_F64)
		k_cubic<double><<<grid_for(n), TPB, 0, st>>>(n, (const double *)axis1, (const double *)axis2,
		                                             (const double *)k, (const double *)Ms,
		                                             (const double *)M, (double *)H, acc);
	else
		k_cubic<float><<<grid_for(n), TPB, 0, st>>>(n, (const float *)axis1, (const float *)axis2,
		                                            (const float *)k, (const float *)Ms,
		                                            (const float *)M, (float *)H, acc);
	MM_TRY(after_launch("k_cubic"));
	if (energy_host) return finish_energy<double>(acc, sc, energy_host, st);
	return MM_OK;
}

MM_API mm_status mm_llge(int prec, size_t n, const void *f1, const void *f2, const void *M,
                         const void *H, void *dM, void *stream)
{
	if (bad_prec(prec) || n == 0 || !f1 || !f2 || !M || !H || !dM)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_llge: invalid argument");
	cudaStream_t st = as_stream(stream);
	if (prec == MM_F64)
		k_llge<double><<<grid_for(n), TPB, 0, st>>>(n, (const double *)f1, (const double *)f2,
		                                            (const double *)M, (const double *)H, (double *)dM);
	else
		k_llge<float><<<grid_for(n), TPB, 0, st>>>(n, (const float *)f1, (const float *)f2,
		                                           (const float *)M, (const float *)H, (float *)dM);
	return after_launch("k_llge");
}

MM_API mm_status mm_fdm_zhangli(int prec, int nx, int ny, int nz, double dx, double dy,
                                double dz, int do_precess, const void *P, const void *xi,
                                const void *Ms, const void *alpha, const void *j,
                                const void *M, void *dM, void *stream)
{
	if (bad_prec(prec) || nx <= 0 || ny <= 0 || nz <= 0 || !P || !xi || !Ms || !alpha || !j ||
	    !M || !dM || !(dx > 0) || !(dy > 0) || !(dz > 0))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_fdm_zhangli: invalid argument");
	cudaStream_t st = as_stream(stream);
	const size_t n = (size_t)nx * ny * nz;
	if (prec == MM_F64)
		k_zhangli<double><<<grid_for(n), TPB, 0, st>>>(
		    nx, ny, nz, dx, dy, dz, do_precess, (const double *)P, (const double *)xi,
		    (const double *)Ms, (const double *)alpha, (const double *)j, (const double *)M,
		    (double *)dM);
	else
		k_zhangli<float><<<grid_for(n), TPB, 0, st>>>(
		    nx, ny, nz, dx, dy, dz, do_precess, (const float *)P, (const float *)xi,
		    (const float *)Ms, (const float *)alpha, (const float *)j, (const float *)M,
		    (float *)dM);
	return after_launch("k_zhangli");
}

MM_API mm_status mm_scaled_abs_max(int prec, size_t n, const void *M, const void *scale,
                                   double *result_host, void *stream)
{
	if (bad_prec(prec) || n == 0 || !M || !scale || !result_host)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_scaled_abs_max: invalid argument");
	cudaStream_t st = as_stream(stream);
	ScalarScratch *sc = nullptr;
	MM_TRY(scalar_scratch(&sc));
	MM_CUDA(cudaMemsetAsync(sc->dev, 0, sizeof(double), st));
	if (prec == MM_F64)
		k_scaled_abs_max<double><<<grid_for(n), TPB, 0, st>>>(n, (const double *)M,
		                                                      (const double *)scale, sc->dev);
	else
		k_scaled_abs_max<float><<<grid_for(n), TPB, 0, st>>>(n, (const float *)M,
		                                                     (const float *)scale, sc->dev);
	MM_TRY(after_launch("k_scaled_abs_max"));
	MM_CUDA(cudaMemcpyAsync(sc->host, sc->dev, sizeof(double), cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	*result_host = sqrt(sc->host[0]);
	return MM_OK;
}

MM_API mm_status mm_rk_scaled_error_norm(int prec, size_t n, double eps_abs, double eps_rel, const void *y,
                                         const void *y_error, double *norm_host, void *stream)
{
	if (bad_prec(prec) || n == 0 || !y || !y_error || !norm_host)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_rk_scaled_error_norm: invalid argument");
	cudaStream_t st = as_stream(stream);
	ScalarScratch *sc = nullptr;
	MM_TRY(scalar_scratch(&sc));
	MM_CUDA(cudaMemsetAsync(sc->dev, 0, sizeof(double), st));
	const size_t n3 = 3 * n;
	if (prec == MM_F64)
		k_rk_error_norm2<double><<<grid_for(n3), TPB, 0, st>>>(n3, eps_abs, eps_rel, (const double *)y,
		                                                       (const double *)y_error, sc->dev);
	else
		k_rk_error_norm2<float><<<grid_for(n3), TPB, 0, st>>>(n3, eps_abs, eps_rel, (const float *)y,
		                                                      (const float *)y_error, sc->dev);
	MM_TRY(after_launch("k_rk_error_norm2"));
	MM_CUDA(cudaMemcpyAsync(sc->host, sc->dev, sizeof(double), cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	*norm_host = sqrt(sc->host[0] / (double)n3);
	return MM_OK;
}

MM_API mm_status mm_normalize(int prec, size_t n, const void *Ms, void *M, void *stream)
{
	if (bad_prec(prec) || n == 0 || !Ms || !M)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_normalize: invalid argument");
	cudaStream_t st = as_stream(stream);
	if (prec == MM_F64)
		k_normalize<double><<<grid_for(n), TPB, 0, st>>>(n, (const double *)Ms, (double *)M);
	else
		k_normalize<float><<<grid_for(n), TPB, 0, st>>>(n, (const float *)Ms, (float *)M);
	return after_launch("k_normalize");
}

MM_API mm_status mm_rk_prepare_step(int prec, size_t n, int step, double h, const double *b_host,
                                    const void *const *k_host, const void *y, void *ytmp,
                                    void *stream)
{
	if (bad_prec(prec) || n == 0 || step < 0 || step > MAXK || (step > 0 && (!b_host || !k_host)) ||
	    !y || !ytmp)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_rk_prepare_step: invalid argument");
	cudaStream_t st = as_stream(stream);
	const size_t n3 = 3 * n;
	if (prec == MM_F64) {
		KPtrs<double> kp{};
		for (int j = 0; j < step; ++j) {
			if (!k_host[j]) return fail(MM_ERR_INVALID_ARGUMENT, "mm_rk_prepare_step: null k");
			kp.k[j] = (const double *)k_host[j];
			kp.b[j] = b_host[j];
		}
		k_rk_prepare<double><<<grid_for(n3), TPB, 0, st>>>(n3, step, h, kp, (const double *)y, (double *)ytmp);
	} else {
		KPtrs<float> kp{};
		for (int j = 0; j < step; ++j) {
			if (!k_host[j]) return fail(MM_ERR_INVALID_ARGUMENT, "mm_rk_prepare_step: null k");
			kp.k[j] = (const float *)k_host[j];
			kp.b[j] = b_host[j];
		}
		k_rk_prepare<float><<<grid_for(n3), TPB, 0, st>>>(n3, step, h, kp, (const float *)y, (float *)ytmp);
	}
	return after_launch("k_rk_prepare");
}

MM_API mm_status mm_rk_combine_result(int prec, size_t n, int nk, double h, const double *c_host,
                                      const double *ec_host, const void *const *k_host, void *y,
                                      void *y_error, void *stream)
{
	if (bad_prec(prec) || n == 0 || nk <= 0 || nk > MAXK || !c_host || !ec_host || !k_host || !y ||
	    !y_error)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_rk_combine_result: invalid argument");
	cudaStream_t st = as_stream(stream);
	const size_t n3 = 3 * n;
	if (prec == MM_F64) {
		KPtrs<double> kp{};
		for (int j = 0; j < nk; ++j) {
			if (!k_host[j]) return fail(MM_ERR_INVALID_ARGUMENT, "mm_rk_combine_result: null k");
			kp.k[j] = (const double *)k_host[j]; kp.b[j] = c_host[j]; kp.ec[j] = ec_host[j];
		}
		k_rk_combine<double><<<grid_for(n3), TPB, 0, st>>>(n3, nk, h, kp, (double *)y, (double *)y_error);
	} else {
		KPtrs<float> kp{};
		for (int j = 0; j < nk; ++j) {
			if (!k_host[j]) return fail(MM_ERR_INVALID_ARGUMENT, "mm_rk_combine_result: null k");
			kp.k[j] = (const float *)k_host[j]; kp.b[j] = c_host[j]; kp.ec[j] = ec_host[j];
		}
		k_rk_combine<float><<<grid_for(n3), TPB, 0, st>>>(n3, nk, h, kp, (float *)y, (float *)y_error);
	}
	return after_launch("k_rk_combine");
}

} // extern "C"

// ---- scaled_abs_max without allocation ------------------------------------------------------------
// mm_scaled_abs_max_noalloc returns what mm_scaled_abs_max returns, for callers that must not
// allocate memory once their set-up is done.  mm_scaled_abs_max creates a device accumulator
// (cudaMalloc) and a pinned host word (cudaMallocHost) on its first call on each device; a caller
// whose device memory is already handed out to a pool (so that a late cudaMalloc fails), or whose
// step loop must not meet the device-wide synchronisation a cudaMalloc/cudaMallocHost can imply,
// cannot make that first call mid-run.  This variant takes its scratch from a fixed array in the
// static device memory of this module, which the CUDA runtime places when it loads the module,
// and copies its one result word to the caller's host double.
//
// Scratch: NA_MAX_PARTIALS block maxima followed by the result word.  Pass 1 gives each block
// NA_CHUNK consecutive cells and writes one partial maximum per block; pass 2 (one block) folds
// partials [0, blocks) into the result word.  Nothing in the scratch has to start at zero: every
// slot that is read was written earlier in the same call.  The limit is therefore
// NA_MAX_PARTIALS * NA_CHUNK cells; larger fields are rejected.  All calls on one device share the
// array, so calls whose work overlaps on the device (other streams, other host threads) race.
namespace mm {
namespace {
constexpr int NA_MAX_PARTIALS = 65536;  // 512 KiB of partials (+ the result word)
constexpr int NA_CHUNK = TPB * 16;      // cells per pass-1 block: limit 268,435,456 cells
constexpr int NA_FINAL_THREADS = 1024;
constexpr int NA_MAX_DEVICES = 64;
} // namespace
} // namespace mm

static __device__ __align__(256) double g_na_scratch[mm::NA_MAX_PARTIALS + 1];

namespace mm {
namespace {

// Block-wide max (NaN wins) of a non-negative value, returned to thread 0 of a 1-D block.
__device__ __forceinline__ double na_block_max(double v)
{
	__shared__ double red[32];
	v = warp_max(v);
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	if (lane == 0) red[wid] = v;
	__syncthreads();
	if (wid == 0) {
		const int nw = blockDim.x >> 5;
		v = warp_max(lane < nw ? red[lane] : 0.0);
	}
	return v;
}

template <typename T>
__global__ void __launch_bounds__(TPB) k_scaled_abs_max_partials(size_t n, const T *__restrict__ M,
                                                                 const T *__restrict__ s,
                                                                 double *__restrict__ partials)
{
	const size_t base = (size_t)blockIdx.x * NA_CHUNK;
	const size_t end = n - base < (size_t)NA_CHUNK ? n : base + NA_CHUNK;
	double best = 0.0;
	for (size_t i = base + threadIdx.x; i < end; i += TPB) {
		const double si = (double)s[i];
		if (si == 0.0) continue;
		const double mx = M[i], my = M[i + n], mz = M[i + 2 * n];
		best = fmax(best, (mx * mx + my * my + mz * mz) / (si * si));
	}
	best = na_block_max(best);
	if (threadIdx.x == 0) partials[blockIdx.x] = best;
}

__global__ void __launch_bounds__(NA_FINAL_THREADS) k_scaled_abs_max_final(int blocks, double *scratch)
{
	double best = 0.0;
	for (int i = threadIdx.x; i < blocks; i += NA_FINAL_THREADS) best = nan_max(best, scratch[i]);
	best = na_block_max(best);
	if (threadIdx.x == 0) scratch[NA_MAX_PARTIALS] = best;
}

// Device address of g_na_scratch on the current device, looked up once per device and kept for
// the life of the process (a cudaDeviceReset of that device would leave it stale).
mm_status na_scratch(double **out)
{
	static std::mutex mu;
	static double *addr[NA_MAX_DEVICES] = {};
	int dev = 0;
	MM_CUDA(cudaGetDevice(&dev));
	if (dev < 0 || dev >= NA_MAX_DEVICES)
		return fail(MM_ERR_UNSUPPORTED, "mm_scaled_abs_max_noalloc: device index " + std::to_string(dev) +
		                                    " beyond the " + std::to_string(NA_MAX_DEVICES) + " supported");
	std::lock_guard<std::mutex> lock(mu);
	if (!addr[dev]) {
		double *ptr = nullptr;
		const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_na_scratch);
		if (e != cudaSuccess || !ptr)
			return fail(MM_ERR_CUDA, std::string("mm_scaled_abs_max_noalloc: cudaGetSymbolAddress of the "
			                                     "static scratch failed: ") + cudaGetErrorString(e));
		addr[dev] = ptr;
	}
	*out = addr[dev];
	return MM_OK;
}

} // namespace
} // namespace mm

extern "C" {

MM_API mm_status mm_scaled_abs_max_noalloc(int prec, size_t n, const void *M, const void *scale,
                                           double *result_host, void *stream)
{
	if (bad_prec(prec) || n == 0 || !M || !scale || !result_host)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_scaled_abs_max_noalloc: invalid argument");
	const size_t blocks = (n + NA_CHUNK - 1) / NA_CHUNK;
	if (blocks > (size_t)NA_MAX_PARTIALS)
		return fail(MM_ERR_INVALID_ARGUMENT,
		            "mm_scaled_abs_max_noalloc: n = " + std::to_string(n) + " cells exceeds its limit of " +
		                std::to_string((size_t)NA_MAX_PARTIALS * NA_CHUNK) + " cells (static scratch of " +
		                std::to_string(NA_MAX_PARTIALS) + " partial maxima of " + std::to_string(NA_CHUNK) +
		                " cells each); use mm_scaled_abs_max");
	double *scr = nullptr;
	MM_TRY(na_scratch(&scr));
	cudaStream_t st = as_stream(stream);
	if (prec == MM_F64)
		k_scaled_abs_max_partials<double><<<(unsigned)blocks, TPB, 0, st>>>(n, (const double *)M,
		                                                                    (const double *)scale, scr);
	else
		k_scaled_abs_max_partials<float><<<(unsigned)blocks, TPB, 0, st>>>(n, (const float *)M,
		                                                                   (const float *)scale, scr);
	MM_TRY(after_launch("k_scaled_abs_max_partials"));
	k_scaled_abs_max_final<<<1, NA_FINAL_THREADS, 0, st>>>((int)blocks, scr);
	MM_TRY(after_launch("k_scaled_abs_max_final"));
	double r = 0.0;
	MM_CUDA(cudaMemcpyAsync(&r, scr + NA_MAX_PARTIALS, sizeof(double), cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	*result_host = sqrt(r);
	return MM_OK;
}

} // extern "C"
