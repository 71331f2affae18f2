// Demag convolution H = N * M, zero-padded to (px, py, pz), as shared-memory FFT passes over
// HBM-resident spectra.  Replaces the reference's MatrixVectorConvolution_FFT::execute
// (math/conv/MatrixVectorConvolution_FFT.cpp:110-375): pad, 3x R2C along x, transpose,
// 3x C2C along y, transpose, 3x C2C along z, tensor multiply, and the inverses.
//
// B200 design:
//  * no transposes: the y and z passes read tiles of TB consecutive x-frequencies per row, so
//    every global access is a contiguous run of TB complex numbers;
//  * zero padding is never stored: the x pass reads only the nx real samples of each row and
//    writes only the rows y < ny, z < nz; the y pass pads in shared memory; the z pass pads,
//    transforms, multiplies, inverse-transforms and writes back only z < nz;
//  * two real rows share one complex FFT in the x passes (z = a + i b);
//  * the tensor spectrum is real (Nxx, Nyy, Nzz even in every axis; Nxy, Nxz, Nyz odd in
//    exactly two), so only Re N^ on ky <= py/2, kz <= pz/2 is stored, with the parity signs
//    restored on the fly: 4x fewer tensor bytes than the reference's 12 complex matrices
//    (SymmetricMatrixVectorConvolution_FFT.cpp:60-64 notes but does not use this);
//  * for 2-D problems (nz == 1) the forward y FFT, the multiply and the inverse y FFT are one
//    kernel.
// Spectra layout: cplx<T> S[c][z][y][kx], c < 3, z < nz, y < py, kx < hx, rows lx >= hx apart
// (lx even in FP32, so that every row starts on a 16-byte boundary).
#include "conv.cuh"
#include "fft_reg.cuh"
#include "tma.cuh"

#include <cmath>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

namespace mm {

FftRadices fft_factor(int n)
{
	FftRadices f{};
	f.n = n;
	int m = n;
	auto push = [&](int r) { f.r[f.count++] = r; m /= r; };
	while (m % 8 == 0 && f.count < FFT_MAX_PASSES) push(8);
	while (m % 4 == 0 && f.count < FFT_MAX_PASSES) push(4);
	while (m % 2 == 0 && f.count < FFT_MAX_PASSES) push(2);
	for (int p : {3, 5, 7})
		while (m % p == 0 && f.count < FFT_MAX_PASSES) push(p);
	for (int p = 11; m > 1 && f.count < FFT_MAX_PASSES; p += 2)
		while (m % p == 0 && f.count < FFT_MAX_PASSES) push(p);
	if (m != 1) f.count = -1;  // too many factors (cannot happen for n < 2^24)
	return f;
}

namespace {

constexpr int NT = 256;                 // threads per CTA for all passes
constexpr size_t SMEM_TARGET = 100 * 1024;

template <typename T>
mm_status make_twiddles(int n, void **out)
{
	std::vector<cplx<T>> h(n);
	for (int k = 0; k < n; ++k) {
		const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
		h[k].x = (T)cosl(a);
		h[k].y = (T)sinl(a);
	}
	MM_CUDA(cudaMalloc(out, sizeof(cplx<T>) * n));
	MM_CUDA(cudaMemcpy(*out, h.data(), sizeof(cplx<T>) * n, cudaMemcpyHostToDevice));
	return MM_OK;
}

template <typename T>
__device__ __forceinline__ void load_twiddles(cplx<T> *tw_s, const cplx<T> *tw_g, int n)
{
	const int tid = threadIdx.x, nthr = blockDim.x;
	for (int k = tid; k < n; k += nthr) tw_s[k] = tw_g[k];
}

// ---- x forward: real rows -> half spectra ------------------------------------------------------
// Real row r = (c*nz + z)*ny + y is M[r*nx .. r*nx+nx); its spectrum goes to S row
// (c*nz + z)*py + y.  Rows 2q and 2q+1 share complex line q.
template <typename T, bool SCALE>
__global__ void __launch_bounds__(NT) k_x_fwd(const T *__restrict__ M, const uint8_t *__restrict__ reg,
                                             const T *__restrict__ ms_tab, cplx<T> *__restrict__ S,
                                             int nx, int ny, int nz, int py, int hx, int lx, FftRadices rad,
                                             const cplx<T> *__restrict__ tw_g, int LP)
{
	using C = cplx<T>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int px = rad.n;
	C *tw = reinterpret_cast<C *>(smem_raw);
	C *b0 = tw + px;
	C *b1 = b0 + (size_t)LP * px;
	load_twiddles<T>(tw, tw_g, px);
	const int rows = 3 * ny * nz;
	const int nyz = ny * nz;
	const int line0 = blockIdx.x * LP;
	for (int e = threadIdx.x; e < LP * px; e += blockDim.x) {
		const int b = e / px, x = e % px;
		const int ra = 2 * (line0 + b), rb = ra + 1;
		T a = 0, bb = 0;
		if (x < nx) {
			if (ra < rows) {
				a = M[(size_t)ra * nx + x];
				if (SCALE) a *= ms_tab[reg ? reg[(size_t)(ra % nyz) * nx + x] : 0];
			}
			if (rb < rows) {
				bb = M[(size_t)rb * nx + x];
				if (SCALE) bb *= ms_tab[reg ? reg[(size_t)(rb % nyz) * nx + x] : 0];
			}
		}
		b0[e] = C{a, bb};
	}
	__syncthreads();
	C *res = fft_lines<T, false>(b0, b1, px, 1, LP, rad, tw);
	for (int e = threadIdx.x; e < LP * hx; e += blockDim.x) {
		const int b = e / hx, k = e % hx;
		const int ra = 2 * (line0 + b), rb = ra + 1;
		const C zk = res[b * px + k];
		const C zn = res[b * px + (px - k) % px];
		const T h = T(0.5);
		if (ra < rows) {
			const int c = ra / nyz, rem = ra % nyz;
			const size_t srow = (size_t)(c * nz + rem / ny) * py + rem % ny;
			S[srow * lx + k] = C{h * (zk.x + zn.x), h * (zk.y - zn.y)};
		}
		if (rb < rows) {
			const int c = rb / nyz, rem = rb % nyz;
			const size_t srow = (size_t)(c * nz + rem / ny) * py + rem % ny;
			S[srow * lx + k] = C{h * (zk.y + zn.y), h * (zn.x - zk.x)};
		}
	}
}

// ---- x inverse: half spectra -> real rows ------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_x_inv(const cplx<T> *__restrict__ S, T *__restrict__ H,
                                             int nx, int ny, int nz, int py, int hx, int lx, FftRadices rad,
                                             const cplx<T> *__restrict__ tw_g, int LP)
{
	using C = cplx<T>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int px = rad.n;
	C *tw = reinterpret_cast<C *>(smem_raw);
	C *b0 = tw + px;
	C *b1 = b0 + (size_t)LP * px;
	load_twiddles<T>(tw, tw_g, px);
	const int rows = 3 * ny * nz;
	const int nyz = ny * nz;
	const int line0 = blockIdx.x * LP;
	const bool even = (px % 2) == 0;
	for (int e = threadIdx.x; e < LP * px; e += blockDim.x) {
		const int b = e / px, k = e % px;
		const int ra = 2 * (line0 + b), rb = ra + 1;
		const bool mirror = k >= hx;
		const int kk = mirror ? px - k : k;
		// the imaginary parts at kx = 0 and at the Nyquist frequency of a real row are zero
		const bool realonly = (kk == 0) || (even && kk == px / 2);
		C A = {0, 0}, B = {0, 0};
		if (ra < rows) {
			const int c = ra / nyz, rem = ra % nyz;
			A = S[((size_t)(c * nz + rem / ny) * py + rem % ny) * lx + kk];
		}
		if (rb < rows) {
			const int c = rb / nyz, rem = rb % nyz;
			B = S[((size_t)(c * nz + rem / ny) * py + rem % ny) * lx + kk];
		}
		if (realonly) { A.y = 0; B.y = 0; }
		if (mirror) { A.y = -A.y; B.y = -B.y; }
		b0[e] = C{A.x - B.y, A.y + B.x};
	}
	__syncthreads();
	C *res = fft_lines<T, true>(b0, b1, px, 1, LP, rad, tw);
	for (int e = threadIdx.x; e < LP * nx; e += blockDim.x) {
		const int b = e / nx, x = e % nx;
		const int ra = 2 * (line0 + b), rb = ra + 1;
		const C z = res[b * px + x];
		if (ra < rows) H[(size_t)ra * nx + x] = z.x;
		if (rb < rows) H[(size_t)rb * nx + x] = z.y;
	}
}

// ---- y pass (3-D): column tiles, forward pads ny -> py, inverse crops py -> ny -----------------
template <typename T, bool INV>
__global__ void __launch_bounds__(NT) k_y(cplx<T> *__restrict__ S, int n_in, int n_out, int nz,
                                         int py, int hx, int lx, FftRadices rad,
                                         const cplx<T> *__restrict__ tw_g, int TB)
{
	using C = cplx<T>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *tw = reinterpret_cast<C *>(smem_raw);
	C *b0 = tw + py;
	C *b1 = b0 + (size_t)TB * py;
	load_twiddles<T>(tw, tw_g, py);
	const int kx0 = blockIdx.x * TB;
	const int z = blockIdx.y, c = blockIdx.z;
	C *base = S + (size_t)(c * nz + z) * py * lx;
	for (int e = threadIdx.x; e < TB * py; e += blockDim.x) {
		const int y = e / TB, b = e % TB;
		b0[e] = (y < n_in && kx0 + b < hx) ? base[(size_t)y * lx + kx0 + b] : C{0, 0};
	}
	__syncthreads();
	C *res = fft_lines<T, INV>(b0, b1, 1, TB, TB, rad, tw);
	for (int e = threadIdx.x; e < TB * n_out; e += blockDim.x) {
		const int y = e / TB, b = e % TB;
		if (kx0 + b < hx) base[(size_t)y * lx + kx0 + b] = res[e];
	}
}

// Real tensor spectrum with parity signs restored.  t points at component 0 of
// (kz', ky', kx); cs = component stride.
template <typename T, typename C>
__device__ __forceinline__ void tensor_apply(const T *__restrict__ t, size_t cs, T sy, T sz, C &m0,
                                             C &m1, C &m2)
{
	const T nxx = t[0], nxy = sy * t[cs], nxz = sz * t[2 * cs];
	const T nyy = t[3 * cs], nyz = sy * sz * t[4 * cs], nzz = t[5 * cs];
	const C a = m0, b = m1, c = m2;
	m0 = C{nxx * a.x + nxy * b.x + nxz * c.x, nxx * a.y + nxy * b.y + nxz * c.y};
	m1 = C{nxy * a.x + nyy * b.x + nyz * c.x, nxy * a.y + nyy * b.y + nyz * c.y};
	m2 = C{nxz * a.x + nyz * b.x + nzz * c.x, nxz * a.y + nyz * b.y + nzz * c.y};
}

// ---- z pass (3-D): forward FFT along z, tensor multiply, inverse FFT, all three components ----
template <typename T>
__global__ void __launch_bounds__(NT) k_z_mul(cplx<T> *__restrict__ S, const T *__restrict__ Nt,
                                             int nz, int py, int hx, int lx, int qy, int qz, FftRadices rad,
                                             const cplx<T> *__restrict__ tw_g, int TB)
{
	using C = cplx<T>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int pz = rad.n;
	C *tw = reinterpret_cast<C *>(smem_raw);
	C *b0 = tw + pz;
	C *b1 = b0 + (size_t)3 * TB * pz;
	load_twiddles<T>(tw, tw_g, pz);
	const int kx0 = blockIdx.x * TB;
	const int ky = blockIdx.y;
	const int L = 3 * TB;
	const size_t cstride = (size_t)nz * py * lx;
	for (int e = threadIdx.x; e < L * pz; e += blockDim.x) {
		const int zz = e / L, l = e % L, c = l / TB, b = l % TB;
		b0[e] = (zz < nz && kx0 + b < hx) ? S[c * cstride + ((size_t)zz * py + ky) * lx + kx0 + b] : C{0, 0};
	}
	__syncthreads();
	C *res = fft_lines<T, false>(b0, b1, 1, L, L, rad, tw);
	C *other = (res == b0) ? b1 : b0;
	const bool fy = ky > py / 2;
	const int kyr = fy ? py - ky : ky;
	const T sy = fy ? T(-1) : T(1);
	const size_t cs = (size_t)qz * qy * hx;
	for (int e = threadIdx.x; e < pz * TB; e += blockDim.x) {
		const int kz = e / TB, b = e % TB;
		if (kx0 + b >= hx) continue;
		const bool fz = kz > pz / 2;
		const int kzr = fz ? pz - kz : kz;
		const T sz = fz ? T(-1) : T(1);
		const T *t = Nt + ((size_t)kzr * qy + kyr) * hx + kx0 + b;
		C &m0 = res[kz * L + b], &m1 = res[kz * L + TB + b], &m2 = res[kz * L + 2 * TB + b];
		tensor_apply<T, C>(t, cs, sy, sz, m0, m1, m2);
	}
	__syncthreads();
	C *out = fft_lines<T, true>(res, other, 1, L, L, rad, tw);
	for (int e = threadIdx.x; e < L * nz; e += blockDim.x) {
		const int zz = e / L, l = e % L, c = l / TB, b = l % TB;
		if (kx0 + b < hx) S[c * cstride + ((size_t)zz * py + ky) * lx + kx0 + b] = out[e];
	}
}

// ---- y pass with multiply (2-D problems): forward y FFT, tensor multiply, inverse y FFT -------
template <typename T>
__global__ void __launch_bounds__(NT) k_y_mul2d(cplx<T> *__restrict__ S, const T *__restrict__ Nt,
                                               int ny, int hx, int lx, int qy, FftRadices rad,
                                               const cplx<T> *__restrict__ tw_g, int TB)
{
	using C = cplx<T>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int py = rad.n;
	C *tw = reinterpret_cast<C *>(smem_raw);
	C *b0 = tw + py;
	C *b1 = b0 + (size_t)3 * TB * py;
	load_twiddles<T>(tw, tw_g, py);
	const int kx0 = blockIdx.x * TB;
	const int L = 3 * TB;
	const size_t cstride = (size_t)py * lx;
	for (int e = threadIdx.x; e < L * py; e += blockDim.x) {
		const int y = e / L, l = e % L, c = l / TB, b = l % TB;
		b0[e] = (y < ny && kx0 + b < hx) ? S[c * cstride + (size_t)y * lx + kx0 + b] : C{0, 0};
	}
	__syncthreads();
	C *res = fft_lines<T, false>(b0, b1, 1, L, L, rad, tw);
	C *other = (res == b0) ? b1 : b0;
	const size_t cs = (size_t)qy * hx;  // qz == 1
	for (int e = threadIdx.x; e < py * TB; e += blockDim.x) {
		const int ky = e / TB, b = e % TB;
		if (kx0 + b >= hx) continue;
		const bool fy = ky > py / 2;
		const int kyr = fy ? py - ky : ky;
		const T sy = fy ? T(-1) : T(1);
		const T *t = Nt + (size_t)kyr * hx + kx0 + b;
		C &m0 = res[ky * L + b], &m1 = res[ky * L + TB + b], &m2 = res[ky * L + 2 * TB + b];
		tensor_apply<T, C>(t, cs, sy, T(1), m0, m1, m2);
	}
	__syncthreads();
	C *out = fft_lines<T, true>(res, other, 1, L, L, rad, tw);
	for (int e = threadIdx.x; e < L * ny; e += blockDim.x) {
		const int y = e / L, l = e % L, c = l / TB, b = l % TB;
		if (kx0 + b < hx) S[c * cstride + (size_t)y * lx + kx0 + b] = out[e];
	}
}

// ---- set-up: generic strided complex FFT (FP64) for the tensor spectrum ------------------------
// The array is viewed as [outer][len][inner]; line (o, i) is data[o*len*inner + k*inner + i].
template <typename T, bool INV>
__global__ void __launch_bounds__(NT) k_fft_axis(cplx<T> *__restrict__ data, int inner, int outer,
                                                FftRadices rad, const cplx<T> *__restrict__ tw_g,
                                                int TB)
{
	using C = cplx<T>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int len = rad.n;
	C *tw = reinterpret_cast<C *>(smem_raw);
	C *b0 = tw + len;
	C *b1 = b0 + (size_t)TB * len;
	load_twiddles<T>(tw, tw_g, len);
	if (inner == 1) {
		const int r0 = blockIdx.x * TB;
		for (int e = threadIdx.x; e < TB * len; e += blockDim.x) {
			const int b = e / len, k = e % len;
			b0[e] = (r0 + b < outer) ? data[(size_t)(r0 + b) * len + k] : C{0, 0};
		}
		__syncthreads();
		C *res = fft_lines<T, INV>(b0, b1, len, 1, TB, rad, tw);
		for (int e = threadIdx.x; e < TB * len; e += blockDim.x) {
			const int b = e / len, k = e % len;
			if (r0 + b < outer) data[(size_t)(r0 + b) * len + k] = res[e];
		}
	} else {
		const int i0 = blockIdx.x * TB;
		const size_t o = blockIdx.y;
		C *base = data + o * len * (size_t)inner;
		for (int e = threadIdx.x; e < TB * len; e += blockDim.x) {
			const int k = e / TB, b = e % TB;
			b0[e] = (i0 + b < inner) ? base[(size_t)k * inner + i0 + b] : C{0, 0};
		}
		__syncthreads();
		C *res = fft_lines<T, INV>(b0, b1, 1, TB, TB, rad, tw);
		for (int e = threadIdx.x; e < TB * len; e += blockDim.x) {
			const int k = e / TB, b = e % TB;
			if (i0 + b < inner) base[(size_t)k * inner + i0 + b] = res[e];
		}
	}
}

__global__ void k_tensor_component(const double *__restrict__ N, double2 *__restrict__ X, size_t cnt, int comp)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x)
		X[i] = double2{N[i * 6 + comp], 0.0};
}

// Keeps Re of the spectrum on kx < hx, ky <= py/2, kz <= pz/2, scaled by 1/(px py pz), and
// records max |Re| and max |Im| over the kept region (bit patterns of non-negative doubles).
template <typename T>
__global__ void k_tensor_extract(const double2 *__restrict__ X, T *__restrict__ out, int px, int py,
                                 int hx, int qy, int qz, double scale, double *maxre, double *maxim)
{
	const size_t cnt = (size_t)qz * qy * hx;
	double mr = 0, mi = 0;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x) {
		const int kx = (int)(i % hx);
		const int ky = (int)((i / hx) % qy);
		const int kz = (int)(i / ((size_t)hx * qy));
		const double2 v = X[((size_t)kz * py + ky) * px + kx];
		out[i] = (T)(v.x * scale);
		mr = fmax(mr, fabs(v.x));
		mi = fmax(mi, fabs(v.y));
	}
	block_max_to(maxre, mr);
	block_max_to(maxim, mi);
}

int pick_tile(int len, int ncomp, size_t elem, int cap)
{
	int tb = cap;
	while (tb > 1 && (size_t)(2 * ncomp * tb + 1) * len * elem > SMEM_TARGET) tb >>= 1;
	return tb;
}

template <typename T>
mm_status set_smem(const void *fn, size_t bytes)
{
	if (bytes > 48 * 1024)
		MM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
	return MM_OK;
}

// ---- CTA-Stockham passes (cta_fft, radix 16 in registers, shared-memory passes) -----------------
__host__ __device__ constexpr int ct_radix(int n) { return n < 16 ? n : 16; }
__host__ __device__ constexpr int ct_radix8(int n) { return n < 8 ? n : 8; }
__host__ __device__ constexpr int ct_tb(int n, int csize)
{
	int tb = 32;
	while (tb > 1 && ((long)n * tb * csize > 65536 || tb * (n / ct_radix(n)) > 512)) tb >>= 1;
	return tb;
}
__host__ __device__ constexpr int ct_lpb(int n, int csize)
{
	int l = 256 / (n / ct_radix(n));
	if (l < 1) l = 1;
	while (l > 1 && (long)(l * n + (l * n >> 5) + 1) * csize > 65536) l >>= 1;
	return l;
}

// y pass (3-D): TB columns per CTA; forward pads rows n_in -> N, inverse crops N -> n_out.
// (bx: column tile, plane = c nz + z; shared by the single-grid and the grouped kernels)
template <typename T, int N, int TB, bool INV, int R = ct_radix(N)>
__device__ __forceinline__ void y_ct_body(cplx<T> *__restrict__ S, int n_in, int n_out, int hx, int lx,
                                          const cplx<T> *__restrict__ twN, int bx, int plane)
{
	using C = cplx<T>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *sm = reinterpret_cast<C *>(smem_raw);
	const int tid = threadIdx.x;
	const int line = tid & (TB - 1), j0 = tid / TB;  // N / R threads per column
	const int kx = bx * TB + line;
	const bool ok = kx < hx;
	C *base = S + (size_t)plane * N * lx + (ok ? kx : 0);
	auto ld = [&](int, int k) -> C { return (ok && k < n_in) ? base[(size_t)k * lx] : C{0, 0}; };
	auto st = [&](int, int k, C v) {
		if (ok && k < n_out) base[(size_t)k * lx] = v;
	};
	cta_fft<T, N, R, TB, INV, SmCols<N, TB>>(sm, twN, line, j0, ld, st);
}

template <typename T, int N, int TB, bool INV>
__global__ void __launch_bounds__(TB * (N / ct_radix(N)), 2) k_y_ct(cplx<T> *__restrict__ S, int n_in, int n_out, int nz,
                                                                 int hx, int lx, const cplx<T> *__restrict__ twN)
{
	y_ct_body<T, N, TB, INV>(S, n_in, n_out, hx, lx, twN, blockIdx.x, blockIdx.z * nz + blockIdx.y);
}

// x pass forward: LPB complex lines per CTA (line q packs real rows 2q, 2q+1).
template <typename T, int N, int LPB, bool SCALE, int R = ct_radix(N), bool H0 = false>
__device__ __forceinline__ void x_fwd_ct_body(const T *__restrict__ M, const uint8_t *__restrict__ reg,
                                              const T *__restrict__ ms_tab, cplx<T> *__restrict__ S, int nx, int ny,
                                              int nz, int py, int hx, int lx, const cplx<T> *__restrict__ twN, int blk)
{
	using C = cplx<T>;
	constexpr int TPL = N / R;
	using SI = SmRows<N, LPB>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *sm = reinterpret_cast<C *>(smem_raw);
	const int tid = threadIdx.x;
	const int line = tid / TPL, j0 = tid % TPL;
	const int rows = 3 * ny * nz, nyz = ny * nz;
	const int ra = 2 * (blk * LPB + line), rb = ra + 1;
	const bool va = ra < rows, vb = rb < rows;
	const int qa = va ? ra : 0, qb = vb ? rb : 0;
	const T *Ma = M + (size_t)qa * nx, *Mb = M + (size_t)qb * nx;
	const uint8_t *Ra = reg ? reg + (size_t)(qa % nyz) * nx : nullptr;
	const uint8_t *Rb = reg ? reg + (size_t)(qb % nyz) * nx : nullptr;
	auto ld = [&](int, int x) -> C {
		T a = 0, b = 0;
		if (x < nx) {
			if (va) { a = Ma[x]; if (SCALE) a *= ms_tab[Ra ? Ra[x] : 0]; }
			if (vb) { b = Mb[x]; if (SCALE) b *= ms_tab[Rb ? Rb[x] : 0]; }
		}
		return C{a, b};
	};
	auto st = [&](int l, int k, C v) { sm[SI::at(l, k)] = v; };
	if constexpr (H0) cta_fft_h0<T, N, R, LPB, SI>(sm, twN, line, j0, ld, st);
	else cta_fft<T, N, R, LPB, false, SI>(sm, twN, line, j0, ld, st);
	__syncthreads();
	C *Sa = S + ((size_t)(qa / nyz * nz + qa % nyz / ny) * py + qa % nyz % ny) * lx;
	C *Sb = S + ((size_t)(qb / nyz * nz + qb % nyz / ny) * py + qb % nyz % ny) * lx;
	const T h = T(0.5);
	for (int k = j0; k < hx; k += TPL) {
		const C zk = sm[SI::at(line, k)], zn = sm[SI::at(line, (N - k) & (N - 1))];
		if (va) Sa[k] = C{h * (zk.x + zn.x), h * (zk.y - zn.y)};
		if (vb) Sb[k] = C{h * (zk.y + zn.y), h * (zn.x - zk.x)};
	}
}

template <typename T, int N, int LPB, bool SCALE>
__global__ void __launch_bounds__(LPB * (N / ct_radix(N))) k_x_fwd_ct(const T *__restrict__ M,
                                                                     const uint8_t *__restrict__ reg,
                                                                     const T *__restrict__ ms_tab,
                                                                     cplx<T> *__restrict__ S, int nx, int ny, int nz,
                                                                     int py, int hx, int lx, const cplx<T> *__restrict__ twN)
{
	x_fwd_ct_body<T, N, LPB, SCALE>(M, reg, ms_tab, S, nx, ny, nz, py, hx, lx, twN, blockIdx.x);
}

// x pass inverse: half spectra of rows 2q, 2q+1 -> real rows.
template <typename T, int N, int LPB, int R = ct_radix(N)>
__device__ __forceinline__ void x_inv_ct_body(const cplx<T> *__restrict__ S, T *__restrict__ H, int nx, int ny,
                                              int nz, int py, int hx, int lx, const cplx<T> *__restrict__ twN, int blk)
{
	using C = cplx<T>;
	constexpr int TPL = N / R;
	using SI = SmRows<N, LPB>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *sm = reinterpret_cast<C *>(smem_raw);
	const int tid = threadIdx.x;
	const int line = tid / TPL, j0 = tid % TPL;
	const int rows = 3 * ny * nz, nyz = ny * nz;
	const int ra = 2 * (blk * LPB + line), rb = ra + 1;
	const bool va = ra < rows, vb = rb < rows;
	const int qa = va ? ra : 0, qb = vb ? rb : 0;
	const C *Sa = S + ((size_t)(qa / nyz * nz + qa % nyz / ny) * py + qa % nyz % ny) * lx;
	const C *Sb = S + ((size_t)(qb / nyz * nz + qb % nyz / ny) * py + qb % nyz % ny) * lx;
	T *Ha = H + (size_t)qa * nx, *Hb = H + (size_t)qb * nx;
	auto ld = [&](int, int f) -> C {
		const bool mirror = f >= hx;
		const int ff = mirror ? N - f : f;
		C A = va ? Sa[ff] : C{0, 0};
		C B = vb ? Sb[ff] : C{0, 0};
		if (ff == 0 || 2 * ff == N) { A.y = 0; B.y = 0; }
		if (mirror) { A.y = -A.y; B.y = -B.y; }
		return C{A.x - B.y, A.y + B.x};
	};
	auto st = [&](int, int x, C v) {
		if (x < nx) {
			if (va) Ha[x] = v.x;
			if (vb) Hb[x] = v.y;
		}
	};
	cta_fft<T, N, R, LPB, true, SI>(sm, twN, line, j0, ld, st);
}

template <typename T, int N, int LPB>
__global__ void __launch_bounds__(LPB * (N / ct_radix(N))) k_x_inv_ct(const cplx<T> *__restrict__ S, T *__restrict__ H,
                                                                     int nx, int ny, int nz, int py, int hx, int lx,
                                                                     const cplx<T> *__restrict__ twN)
{
	x_inv_ct_body<T, N, LPB>(S, H, nx, ny, nz, py, hx, lx, twN, blockIdx.x);
}

// z pass with the tensor multiply (CTA-Stockham form): lines (c, b) = c * TB + b hold the z
// column of component c at x-frequency kx0 + b; forward transform into shared memory, multiply by
// the real symmetric tensor (three components meet in shared memory), inverse transform to HBM.
template <typename T, int PZ, int TB>
__global__ void __launch_bounds__(3 * TB * (PZ / ct_radix8(PZ))) k_z_ct(cplx<T> *__restrict__ S,
                                                                        const T *__restrict__ Nt, int nz, int py,
                                                                        int hx, int lx, int qy, int qz,
                                                                        const cplx<T> *__restrict__ twN)
{
	using C = cplx<T>;
	constexpr int R = ct_radix8(PZ);
	constexpr int LANES = 3 * TB;
	using SI = SmCols<PZ, LANES>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *sm = reinterpret_cast<C *>(smem_raw);
	const int tid = threadIdx.x;
	const int line = tid % LANES, j0 = tid / LANES;
	const int c = line / TB, b = line % TB;
	const int ky = blockIdx.y;
	const size_t cstride = (size_t)nz * py * lx, zstride = (size_t)py * lx;
	{
		const int kx = blockIdx.x * TB + b;
		const bool ok = kx < hx;
		C *col = S + c * cstride + (size_t)ky * lx + (ok ? kx : 0);
		auto ld = [&](int, int z) -> C { return (ok && z < nz) ? col[z * zstride] : C{0, 0}; };
		auto st = [&](int l, int k, C v) { sm[SI::at(l, k)] = v; };
		cta_fft<T, PZ, R, LANES, false, SI>(sm, twN, line, j0, ld, st);
	}
	__syncthreads();
	const bool fy = ky > py / 2;
	const int kyr = fy ? py - ky : ky;
	const T sy = fy ? T(-1) : T(1);
	const size_t cs = (size_t)qz * qy * hx, kzs = (size_t)qy * hx;
	for (int idx = tid; idx < PZ * TB; idx += LANES * (PZ / R)) {
		const int kz = idx / TB, bb = idx % TB;
		const int kx = blockIdx.x * TB + bb;
		if (kx >= hx) continue;
		const bool fz = kz > PZ / 2;
		const int kzr = fz ? PZ - kz : kz;
		const T sz = fz ? T(-1) : T(1);
		const T *t = Nt + (size_t)kzr * kzs + (size_t)kyr * hx + kx;
		C &m0 = sm[SI::at(bb, kz)], &m1 = sm[SI::at(TB + bb, kz)], &m2 = sm[SI::at(2 * TB + bb, kz)];
		tensor_apply<T, C>(t, cs, sy, sz, m0, m1, m2);
	}
	{
		const int kx = blockIdx.x * TB + b;
		const bool ok = kx < hx;
		C *col = S + c * cstride + (size_t)ky * lx + (ok ? kx : 0);
		auto ld = [&](int l, int k) -> C { return sm[SI::at(l, k)]; };
		auto st = [&](int, int z, C v) {
			if (ok && z < nz) col[z * zstride] = v;
		};
		__syncthreads();
		cta_fft<T, PZ, R, LANES, true, SI, true>(sm, twN, line, j0, ld, st);
	}
}

// Asynchronous copy of one real value global -> shared (LDGSTS, 4 or 8 bytes).
template <typename T>
__device__ __forceinline__ void cp_async_t(T *dst, const T *src)
{
	const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
	if constexpr (sizeof(T) == 4)
		asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
	else
		asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all_t() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared memory of the register z pass: the spectrum of two rows (2 PZ kz x 3 components x 32 kx)
// and the block's tensor entries ((PZ/2 + 1) x 6 x 32).
template <typename T>
constexpr size_t zr_smem(int pz) { return (size_t)2 * pz * 96 * 2 * sizeof(T) + (size_t)(pz / 2 + 1) * 192 * sizeof(T); }

// ---- z pass in registers ------------------------------------------------------------------------
// One thread per (kx, component, ky) column holds the whole length-PZ column in registers: the
// forward DFT (upper half zero padding, nz <= PZ/2), the tensor multiply through shared memory,
// and the inverse DFT, of which only the outputs z < nz are formed and stored.  A block covers
// 32 consecutive kx (one warp per component and row: coalesced 256-byte loads and stores) and the
// ky pair {b, py - b}, b = blockIdx.y <= py/2, whose tensor entries agree up to parity signs: each
// tensor value is read once per block and applied to up to four (ky, kz) combinations.
constexpr int ZR_THREADS = 192;  // 32 kx x 3 components x 2 rows

template <typename T, int PZ>
__device__ __forceinline__ void z_reg_body(cplx<T> *__restrict__ S, const T *__restrict__ Nt, int nz, int py, int hx,
                                           int lx, int qy, int qz, int bx, int b)
{
	using C = cplx<T>;
	constexpr int H = PZ / 2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *sm = reinterpret_cast<C *>(smem_raw);  // [row][kz][component][32 kx]
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int c = w % 3, r = w / 3;
	const int b1 = py - b;
	const bool two = b > 0 && b1 != b;
	const int kx = bx * 32 + lane;
	const bool ok = (r == 0 || two) && kx < hx;
	const size_t zstride = (size_t)py * lx;
	C *col = S + ((size_t)c * nz * py + (size_t)(r == 0 ? b : b1)) * lx + kx;
	// the block's tensor entries (kz' <= pz/2, 6 components, 32 kx at ky' = b) come in by
	// asynchronous copies while the columns are loaded and transformed
	T *tens = reinterpret_cast<T *>(sm + 2 * PZ * 96);
	static_assert(ZR_THREADS == 192, "one thread per (tensor component, kx) of a kz plane");
	{
		// thread (warp w, lane) copies component w at kx for every kz' (one pointer step per plane)
		const size_t kzs = (size_t)qy * hx;
		const T *src = Nt + (size_t)w * qz * kzs + (size_t)b * hx + kx;
		if (kx < hx) {
#pragma unroll
			for (int kzr = 0; kzr <= H; ++kzr, src += kzs) cp_async_t(&tens[kzr * 192 + threadIdx.x], src);
		}
	}
	C v[PZ];
#pragma unroll
	for (int z = 0; z < H; ++z) v[z] = (ok && z < nz) ? col[z * zstride] : C{0, 0};
	dft_reg_halfzero<T, PZ>(v);
	C *mine = sm + (r * PZ * 3 + c) * 32 + lane;
#pragma unroll
	for (int k = 0; k < PZ; ++k) mine[brev<PZ>(k) * 96] = v[k];
	cp_async_wait_all_t();
	__syncthreads();
	if (kx < hx) {
		for (int kzr = w; kzr <= H; kzr += ZR_THREADS / 32) {
			const T *t = tens + kzr * 192 + lane;
			const T nxx = t[0], nxy = t[32], nxz = t[64], nyy = t[96], nyz = t[128], nzz = t[160];
			const int nk = (kzr == 0 || kzr == H) ? 1 : 2;
#pragma unroll
			for (int rr = 0; rr < 2; ++rr) {
				if (rr && !two) break;
#pragma unroll
				for (int q = 0; q < 2; ++q) {
					if (q && nk < 2) break;
					const int kz = q ? PZ - kzr : kzr;
					const T sy = rr ? T(-1) : T(1), sz = q ? T(-1) : T(1);
					C *e = sm + ((rr * PZ + kz) * 3) * 32 + lane;
					const C m0 = e[0], m1 = e[32], m2 = e[64];
					const T xy = sy * nxy, xz = sz * nxz, yz = sy * sz * nyz;
					e[0] = C{nxx * m0.x + xy * m1.x + xz * m2.x, nxx * m0.y + xy * m1.y + xz * m2.y};
					e[32] = C{xy * m0.x + nyy * m1.x + yz * m2.x, xy * m0.y + nyy * m1.y + yz * m2.y};
					e[64] = C{xz * m0.x + yz * m1.x + nzz * m2.x, xz * m0.y + yz * m1.y + nzz * m2.y};
				}
			}
		}
	}
	__syncthreads();
#pragma unroll
	for (int k = 0; k < PZ; ++k) v[k] = mine[k * 96];
	dft_reg<T, PZ, true>(v);
	if (ok) {
#pragma unroll
		for (int z = 0; z < H; ++z)
			if (z < nz) col[z * zstride] = v[brev<PZ>(z)];
	}
}

template <typename T, int PZ>
__global__ void __launch_bounds__(ZR_THREADS, 2) k_z_reg(cplx<T> *__restrict__ S, const T *__restrict__ Nt, int nz,
                                                        int py, int hx, int lx, int qy, int qz)
{
	z_reg_body<T, PZ>(S, Nt, nz, py, hx, lx, qy, qz, blockIdx.x, blockIdx.y);
}

template <typename T, int PZ>
void fs_z_reg(ConvPlan *p, cudaStream_t st)
{
	const dim3 grid((p->hx + 31) / 32, p->qy);
	k_z_reg<T, PZ><<<grid, ZR_THREADS, zr_smem<T>(PZ), st>>>(
	    (cplx<T> *)p->spec, (const T *)p->tensor, p->nz, p->py, p->hx, p->lx, p->qy, p->qz);
}

// ---- y pass through TMA-staged tiles -------------------------------------------------------------
// Persistent CTAs walk tiles (TB columns of one (component, z) plane).  Each tile's input rows
// (the ny < N/2 data rows padded to N/2 by the TMA unit's zero fill going forward, all N rows
// going back) arrive by cp.async.bulk.tensor in one of two stage buffers while the previous tile is
// transformed; pass 0 reads the stage buffer, the later passes work in a skewed shared-memory
// buffer, and the last pass stores straight to HBM.  Thread 0 issues the loads; a bounded wait that
// runs out sets *err and ends the kernel instead of hanging.
template <int N, int TB, bool INV, class C>
struct YTmaGeom {
	static constexpr int ROWS = INV ? N : N / 2;
	static constexpr int BR = ROWS < 256 ? ROWS : 256;
	static constexpr int NBOX = ROWS / BR;
	static constexpr int E = (int)(sizeof(C) / 8);
	static constexpr uint32_t TILE_BYTES = (uint32_t)(TB * ROWS * sizeof(C));
	static constexpr size_t WORK = ((size_t)SmCols<N, TB, 4>::SIZE * sizeof(C) + 15) / 16 * 16;
	static constexpr size_t SMEM = 2 * (size_t)TILE_BYTES + WORK + 16;
	// the single-instance pass keeps the twiddle table W_N^k in shared memory behind the barriers
	static constexpr size_t TW = SMEM;
	static constexpr size_t SMEM_TW = SMEM + (size_t)N * sizeof(C);
};

// Columns per CTA of the single-instance TMA y pass: 32-byte rows, at most 256 threads, so that
// two CTAs (and their barriers) interleave on an SM.
__host__ __device__ constexpr int y_tma_tb(int n, int csize)
{
	int tb = ct_tb(n, csize);
	while (tb * csize > 32 && tb * (n / ct_radix(n)) > 256) tb >>= 1;
	return tb;
}

template <typename T, int N, int TB, bool INV>
__global__ void __launch_bounds__(TB * (N / ct_radix(N)), 2)
    k_y_tma(const __grid_constant__ CUtensorMap tmap, cplx<T> *__restrict__ S, int n_out, int hx, int lx,
            int tiles_x, int ntiles, const cplx<T> *__restrict__ twN, int *err)
{
	using C = cplx<T>;
	using G = YTmaGeom<N, TB, INV, C>;
	constexpr int R = ct_radix(N);
	using SI = SmCols<N, TB, 4>;
	extern __shared__ __align__(128) unsigned char smem_tma[];
	C *stage0 = reinterpret_cast<C *>(smem_tma);
	C *stage1 = stage0 + TB * G::ROWS;
	C *work = reinterpret_cast<C *>(smem_tma + 2 * (size_t)G::TILE_BYTES);
	uint64_t *bar = reinterpret_cast<uint64_t *>(smem_tma + 2 * (size_t)G::TILE_BYTES + G::WORK);
	const int tid = threadIdx.x;
	const int line = tid & (TB - 1), j0 = tid / TB;
	C *tws = reinterpret_cast<C *>(smem_tma + G::TW);
	for (int q = tid; q < N; q += blockDim.x) tws[q] = twN[q];
	auto issue = [&](int t, int b) {
		const int tx = t % tiles_x, plane = t / tiles_x;
		C *dst = b ? stage1 : stage0;
		mbar_expect_tx(&bar[b], G::TILE_BYTES);
#pragma unroll
		for (int q = 0; q < G::NBOX; ++q)
			tma_load_3d(dst + q * G::BR * TB, &tmap, tx * TB * G::E, q * G::BR, plane, &bar[b]);
	};
	if (tid == 0) {
		mbar_init(&bar[0], 1);
		mbar_init(&bar[1], 1);
		fence_proxy_async();
	}
	__syncthreads();
	if (tid == 0) {
		if ((int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
		if ((int)(blockIdx.x + gridDim.x) < ntiles) issue(blockIdx.x + gridDim.x, 1);
	}
	uint32_t parity = 0;  // bit b: phase parity expected next on bar[b]
	int k = 0;
	for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
		const int b = k & 1;
		const bool late = !mbar_wait(&bar[b], (parity >> b) & 1u);
		if (__syncthreads_or(late)) {
			if (tid == 0) {
				atomicExch(err, 1);
				mbar_drain2(bar, parity, b, t + (int)gridDim.x < ntiles);
			}
			return;
		}
		parity ^= 1u << b;
		const int tx = t % tiles_x, plane = t / tiles_x;
		const int kx = tx * TB + line;
		const bool ok = kx < hx;
		C *base = S + (size_t)plane * N * lx + (ok ? kx : 0);
		const C *sb = b ? stage1 : stage0;
		auto ld = [&](int, int r) -> C { return r < G::ROWS ? sb[r * TB + line] : C{0, 0}; };
		auto st = [&](int, int r, C v) {
			if (ok && r < n_out) base[(size_t)r * lx] = v;
		};
		const int next = t + 2 * (int)gridDim.x;
		auto release = [&]() {
			__syncthreads();  // every thread has read stage buffer b
			if (tid == 0 && next < ntiles) {
				fence_proxy_async();
				issue(next, b);
			}
		};
		if constexpr (INV) cta_fft<T, N, R, TB, INV, SI>(work, tws, line, j0, ld, st, release);
		else cta_fft_h0<T, N, R, TB, SI>(work, tws, line, j0, ld, st, release);  // rows >= N/2 are zero
	}
}

// ---- x passes through TMA-staged tiles -----------------------------------------------------------
// Persistent CTAs walk tiles of LPB complex lines (2 LPB real rows).  A tile's rows arrive by
// cp.async.bulk.tensor in a ring of stage buffers (xbox_n boxes of xbox_w 8-byte elements per row,
// so the staged rows are dense: real rows of nx values going forward, spectrum rows of lx complex
// values going back); pass 0 reads the stage buffer and writes a separate skewed work buffer, after
// which the stage is refilled with the tile STG strides ahead, so that up to STG tiles are loading
// while one is transformed.  Two CTAs share an SM.
template <int N, class C>
struct XTmaGeom {
	static constexpr int R = ct_radix(N);
	static constexpr int LPB = ct_lpb(N, sizeof(C));
	static constexpr int THREADS = LPB * (N / R);
	static constexpr size_t WORK = (size_t)SmRows<N, LPB, 4>::SIZE * sizeof(C);
	static constexpr size_t BUF = (WORK + 127) / 128 * 128;
	static constexpr size_t PER_SM = 228 * 1024;  // shared memory per SM (1 KB of it reserved per CTA)
	// forward stage: 2 LPB real rows of at most N/2 values and their region bytes
	static constexpr size_t SB_F = ((size_t)LPB * N * (sizeof(C) / 2 + 1) + 127) / 128 * 128;
	// forward extras: barriers, the 256-entry Ms table, the twiddle table W_N^k
	static constexpr size_t EXTRA_F = 64 + 256 * (sizeof(C) / 2) + (size_t)N * sizeof(C);
	static constexpr int STG_F = 2 * (3 * SB_F + BUF + EXTRA_F + 1024) <= PER_SM ? 3 : 2;
	static constexpr size_t SMEM_F = STG_F * SB_F + BUF + EXTRA_F;
	static constexpr int MINB_F = 2 * (SMEM_F + 1024) <= PER_SM ? 2 : 1;
	// inverse stage: 2 LPB spectrum rows of lx complex values (lx * sizeof(C) * 2 LPB <= BUF,
	// checked at set-up); the inverse reads its twiddles from global memory
	static constexpr size_t SB_I = BUF;
	static constexpr int STG_I = 2 * (3 * SB_I + BUF + 64 + 1024) <= PER_SM ? 3 : 2;
	static constexpr size_t SMEM_I = STG_I * SB_I + BUF + 64;
	static constexpr int MINB_I = 2 * (SMEM_I + 1024) <= PER_SM ? 2 : 1;
};

// After a bounded wait gave up in a ring of STG stage buffers on the tile t of local index k:
// waits (bounded again) for every load still in flight (tiles t, t + G, ..., t + (STG - 1) G
// that exist), so that no copy lands in shared memory after the CTA has exited.
template <int STG>
__device__ __forceinline__ void mbar_drain_ring(uint64_t *bar, uint32_t parity, int k, int t, int G, int ntiles)
{
	for (int i = 0; i < STG; ++i) {
		const int s = (k + i) % STG;
		if (t + i * G < ntiles) mbar_wait(&bar[s], (parity >> s) & 1u);
	}
}

// Forward: with SCALE the tile's region bytes (rows r % (ny nz), contiguous within a tile) ride
// along in the same stage behind the real rows, and the 256-entry Ms table sits in shared memory,
// so that pass 0 reads nothing but shared memory.
template <typename T, int N, bool SCALE>
__global__ void __launch_bounds__(XTmaGeom<N, cplx<T>>::THREADS, XTmaGeom<N, cplx<T>>::MINB_F)
    k_x_fwd_tma(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap rmap,
                const T *__restrict__ ms_tab, cplx<T> *__restrict__ S, int nx, int ny, int nz, int py, int hx,
                int lx, int ntiles, const cplx<T> *__restrict__ twN, int *err)
{
	using C = cplx<T>;
	using G = XTmaGeom<N, C>;
	constexpr int LPB = G::LPB, TPL = N / G::R, STG = G::STG_F;
	using SI = SmRows<N, LPB, 4>;
	extern __shared__ __align__(128) unsigned char smem_tma[];
	C *work = reinterpret_cast<C *>(smem_tma + STG * G::SB_F);
	unsigned char *extra = smem_tma + STG * G::SB_F + G::BUF;
	uint64_t *bar = reinterpret_cast<uint64_t *>(extra);
	T *msr = reinterpret_cast<T *>(extra + 64);
	C *tws = reinterpret_cast<C *>(extra + 64 + 256 * sizeof(T));
	const int tid = threadIdx.x;
	const int line = tid / TPL, j0 = tid % TPL;
	const int rows = 3 * ny * nz, nyz = ny * nz;
	const int G_ = (int)gridDim.x;
	const uint32_t row_bytes = (uint32_t)(2 * LPB * (size_t)nx * sizeof(T));
	const uint32_t tile_bytes = row_bytes + (SCALE ? (uint32_t)(2 * LPB * nx) : 0u);
	auto issue = [&](int t, int s) {
		unsigned char *dst = smem_tma + s * G::SB_F;
		mbar_expect_tx(&bar[s], tile_bytes);
		tma_load_3d(dst, &tmap, 0, 0, t * 2 * LPB, &bar[s]);
		if (SCALE) tma_load_2d(dst + row_bytes, &rmap, 0, (t * 2 * LPB) % nyz, &bar[s]);
	};
	if (SCALE)
		for (int r = tid; r < 256; r += blockDim.x) msr[r] = ms_tab[r];
	for (int q = tid; q < N; q += blockDim.x) tws[q] = twN[q];
	if (tid == 0) {
		for (int s = 0; s < STG; ++s) mbar_init(&bar[s], 1);
		fence_proxy_async();
	}
	__syncthreads();
	if (tid == 0)
		for (int s = 0; s < STG; ++s)
			if ((int)blockIdx.x + s * G_ < ntiles) issue(blockIdx.x + s * G_, s);
	uint32_t parity = 0;  // bit s: phase parity expected next on bar[s]
	int k = 0, s = 0;
	for (int t = blockIdx.x; t < ntiles; t += G_, ++k, s = s + 1 == STG ? 0 : s + 1) {
		// (this barrier also orders the previous tile's reads of the work buffer before pass 0)
		const bool late = !mbar_wait(&bar[s], (parity >> s) & 1u);
		if (__syncthreads_or(late)) {
			if (tid == 0) {
				atomicExch(err, 1);
				mbar_drain_ring<STG>(bar, parity, k, t, G_, ntiles);
			}
			return;
		}
		parity ^= 1u << s;
		const unsigned char *stage = smem_tma + s * G::SB_F;
		const T *rowa = reinterpret_cast<const T *>(stage) + (size_t)(2 * line) * nx;
		const T *rowb = rowa + nx;
		const uint8_t *rga = stage + row_bytes + (size_t)(2 * line) * nx;
		const uint8_t *rgb = rga + nx;
		const int ra = 2 * (t * LPB + line), rb = ra + 1;
		const bool va = ra < rows, vb = rb < rows;
		const int qa = va ? ra : 0, qb = vb ? rb : 0;
		auto ld = [&](int, int x) -> C {
			T a = 0, bb = 0;
			if (x < nx) {
				if (va) { a = rowa[x]; if (SCALE) a *= msr[rga[x]]; }
				if (vb) { bb = rowb[x]; if (SCALE) bb *= msr[rgb[x]]; }
			}
			return C{a, bb};
		};
		auto st = [&](int l, int kk, C v) { work[SI::at(l, kk)] = v; };
		const int next = t + STG * G_;
		auto release = [&]() {
			__syncthreads();  // every thread has read stage s
			if (tid == 0 && next < ntiles) {
				fence_proxy_async();
				issue(next, s);
			}
		};
		cta_fft_h0<T, N, G::R, LPB, SI>(work, tws, line, j0, ld, st, release);  // x >= nx, N/2 <= x: zero
		__syncthreads();
		C *Sa = S + ((size_t)(qa / nyz * nz + qa % nyz / ny) * py + qa % nyz % ny) * lx;
		C *Sb = S + ((size_t)(qb / nyz * nz + qb % nyz / ny) * py + qb % nyz % ny) * lx;
		const T h = T(0.5);
		for (int kk = j0; kk < hx; kk += TPL) {
			const C zk = work[SI::at(line, kk)], zn = work[SI::at(line, (N - kk) & (N - 1))];
			if (va) Sa[kk] = C{h * (zk.x + zn.x), h * (zk.y - zn.y)};
			if (vb) Sb[kk] = C{h * (zk.y + zn.y), h * (zn.x - zk.x)};
		}
	}
}

// x inverse: the 2 LPB spectrum rows of a tile lie in one (component, z) plane (ny a multiple of
// 2 LPB); the 4-D tensor map addresses them as (box element, box, y, plane).
template <typename T, int N>
__global__ void __launch_bounds__(XTmaGeom<N, cplx<T>>::THREADS, XTmaGeom<N, cplx<T>>::MINB_I)
    k_x_inv_tma(const __grid_constant__ CUtensorMap tmap, T *__restrict__ H, int nx, int ny, int hx, int lx,
                int ntiles, const cplx<T> *__restrict__ twN, int *err)
{
	using C = cplx<T>;
	using G = XTmaGeom<N, C>;
	constexpr int LPB = G::LPB, TPL = N / G::R, STG = G::STG_I;
	using SI = SmRows<N, LPB, 4>;
	extern __shared__ __align__(128) unsigned char smem_tma[];
	C *work = reinterpret_cast<C *>(smem_tma + STG * G::SB_I);
	uint64_t *bar = reinterpret_cast<uint64_t *>(smem_tma + STG * G::SB_I + G::BUF);
	const int tid = threadIdx.x;
	const int line = tid / TPL, j0 = tid % TPL;
	const int G_ = (int)gridDim.x;
	const uint32_t tile_bytes = (uint32_t)(2 * LPB * (size_t)lx * sizeof(C));
	auto issue = [&](int t, int s) {
		const int row0 = t * 2 * LPB;
		mbar_expect_tx(&bar[s], tile_bytes);
		tma_load_4d(smem_tma + s * G::SB_I, &tmap, 0, 0, row0 % ny, row0 / ny, &bar[s]);
	};
	if (tid == 0) {
		for (int s = 0; s < STG; ++s) mbar_init(&bar[s], 1);
		fence_proxy_async();
	}
	__syncthreads();
	if (tid == 0)
		for (int s = 0; s < STG; ++s)
			if ((int)blockIdx.x + s * G_ < ntiles) issue(blockIdx.x + s * G_, s);
	uint32_t parity = 0;
	int k = 0, s = 0;
	for (int t = blockIdx.x; t < ntiles; t += G_, ++k, s = s + 1 == STG ? 0 : s + 1) {
		// (this barrier also orders the previous tile's last-pass reads of the work buffer before
		// this tile's pass 0 writes)
		const bool late = !mbar_wait(&bar[s], (parity >> s) & 1u);
		if (__syncthreads_or(late)) {
			if (tid == 0) {
				atomicExch(err, 1);
				mbar_drain_ring<STG>(bar, parity, k, t, G_, ntiles);
			}
			return;
		}
		parity ^= 1u << s;
		const C *Sa = reinterpret_cast<const C *>(smem_tma + s * G::SB_I) + (size_t)(2 * line) * lx;
		const C *Sb = Sa + lx;
		const size_t ra = 2 * ((size_t)t * LPB + line);
		T *Ha = H + ra * nx, *Hb = Ha + nx;
		auto ld = [&](int, int f) -> C {
			const bool mirror = f >= hx;
			const int ff = mirror ? N - f : f;
			C A = Sa[ff], B = Sb[ff];
			if (ff == 0 || 2 * ff == N) { A.y = 0; B.y = 0; }
			if (mirror) { A.y = -A.y; B.y = -B.y; }
			return C{A.x - B.y, A.y + B.x};
		};
		auto st = [&](int, int x, C v) {
			if (x < nx) {
				Ha[x] = v.x;
				Hb[x] = v.y;
			}
		};
		const int next = t + STG * G_;
		auto release = [&]() {
			__syncthreads();  // every thread has read stage s
			if (tid == 0 && next < ntiles) {
				fence_proxy_async();
				issue(next, s);
			}
		};
		cta_fft<T, N, G::R, LPB, true, SI>(work, twN, line, j0, ld, st, release);
	}
}

// ---- fast-path geometry and dispatch ---------------------------------------------------------------


template <typename T>
bool fs_len_ok(int n)
{
	if (n < 4 || (n & (n - 1))) return false;
	return sizeof(T) == 4 ? n <= 2048 : n <= 1024;
}

template <typename T, int N>
mm_status fs_setup_len()
{
	using C = cplx<T>;
	constexpr int TB = ct_tb(N, sizeof(C)), LPB = ct_lpb(N, sizeof(C));
	const size_t sx = (size_t)SmRows<N, LPB>::SIZE * sizeof(C), sy = (size_t)SmCols<N, TB>::SIZE * sizeof(C);
	MM_TRY(set_smem<T>((const void *)k_x_fwd_ct<T, N, LPB, false>, sx));
	MM_TRY(set_smem<T>((const void *)k_x_fwd_ct<T, N, LPB, true>, sx));
	MM_TRY(set_smem<T>((const void *)k_x_inv_ct<T, N, LPB>, sx));
	MM_TRY(set_smem<T>((const void *)k_y_ct<T, N, TB, false>, sy));
	MM_TRY(set_smem<T>((const void *)k_y_ct<T, N, TB, true>, sy));
	return MM_OK;
}

// TMA-staged y passes: tensor maps over the spectrum, shared-memory size, persistent grid size.
// Used when the inverse pass's stage buffers fit in shared memory and the forward input is at
// most half the padded length (ny <= py/2, the zero padding the first pass relies on).
template <typename T, int N>
mm_status fs_setup_y_tma(ConvPlan *p)
{
	using C = cplx<T>;
	constexpr int TB = y_tma_tb(N, sizeof(C)), THREADS = TB * (N / ct_radix(N));
	using GF = YTmaGeom<N, TB, false, C>;
	using GI = YTmaGeom<N, TB, true, C>;
	p->tma_y = false;
	if (GI::SMEM_TW > 227 * 1024 || 2 * p->ny > p->py || TB * sizeof(C) < 16) return MM_OK;
	constexpr int E = GF::E;
	const uint64_t d0 = (uint64_t)p->lx * E, rowb = (uint64_t)p->lx * sizeof(C), planeb = rowb * p->py;
	MM_TRY(tma_encode_3d(&p->tm_yf, p->spec, d0, (uint64_t)p->ny, 3ull * p->nz, rowb, planeb, TB * E, GF::BR, 1));
	MM_TRY(tma_encode_3d(&p->tm_yi, p->spec, d0, (uint64_t)p->py, 3ull * p->nz, rowb, planeb, TB * E, GI::BR, 1));
	MM_TRY(set_smem<T>((const void *)k_y_tma<T, N, TB, false>, GF::SMEM_TW));
	MM_TRY(set_smem<T>((const void *)k_y_tma<T, N, TB, true>, GI::SMEM_TW));
	int bf = 0, bi = 0;
	MM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_y_tma<T, N, TB, false>, THREADS, GF::SMEM_TW));
	MM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bi, k_y_tma<T, N, TB, true>, THREADS, GI::SMEM_TW));
	if (bf < 1 || bi < 1) return MM_OK;
	p->grid_yf = bf * num_sms();
	p->grid_yi = bi * num_sms();
	if (!p->err) {
		MM_CUDA(cudaMalloc(&p->err, sizeof(int)));
		MM_CUDA(cudaMemset(p->err, 0, sizeof(int)));
	}
	p->tma_y = true;
	return MM_OK;
}

template <typename T, int N, bool INV>
void fs_y_tma(ConvPlan *p, cudaStream_t st)
{
	using C = cplx<T>;
	constexpr int TB = y_tma_tb(N, sizeof(C)), THREADS = TB * (N / ct_radix(N));
	using G = YTmaGeom<N, TB, INV, C>;
	const int tiles_x = (p->hx + TB - 1) / TB, ntiles = tiles_x * 3 * p->nz;
	const int grid = std::min(ntiles, INV ? p->grid_yi : p->grid_yf);
	k_y_tma<T, N, TB, INV><<<grid, THREADS, G::SMEM_TW, st>>>(INV ? p->tm_yi : p->tm_yf, (C *)p->spec,
	                                                       INV ? p->ny : N, p->hx, p->lx, tiles_x, ntiles,
	                                                       (const C *)p->tw_y, p->err);
}

// TMA-staged x passes.  The inverse pass's tensor map (over the spectrum) is fixed; the forward
// pass reads the state the caller passes, so its map is encoded per input pointer (a small cache
// keeps the solver's few state buffers).
template <typename T, int N>
mm_status fs_setup_x_tma(ConvPlan *p)
{
	using C = cplx<T>;
	using G = XTmaGeom<N, C>;
	constexpr int LPB = G::LPB;
	p->tma_xf = p->tma_xi = false;
	// the forward pass's half-zero first butterflies need nx <= N/2 (non-periodic zero padding)
	if (G::SMEM_F > 227 * 1024 || G::SMEM_I > 227 * 1024 || N < 64 || 2 * p->nx > N) return MM_OK;
	int occ = 0;
	// forward: dense real rows split into boxes of even width
	const size_t wf = (size_t)p->nx * sizeof(T) / 8;
	const size_t nbf = (wf + 255) / 256;
	if ((p->nx * sizeof(T)) % 16 == 0 && wf % (2 * nbf) == 0 && 2 * LPB * p->nx * sizeof(T) <= G::SB_F) {
		// region bytes ride behind the rows when a tile's rows are contiguous in the region map
		p->tma_xf_scale = p->nx % 16 == 0 && (p->ny * p->nz) % (2 * LPB) == 0 && p->nx / 8 <= 256 &&
		                  2 * LPB * p->nx * (sizeof(T) + 1) <= G::SB_F;
		MM_TRY(set_smem<T>((const void *)k_x_fwd_tma<T, N, false>, G::SMEM_F));
		MM_TRY(set_smem<T>((const void *)k_x_fwd_tma<T, N, true>, G::SMEM_F));
		MM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_x_fwd_tma<T, N, true>, G::THREADS, G::SMEM_F));
		if (occ >= 1) {
			p->grid_xf = occ * num_sms();
			p->xf_box_n = (int)nbf;
			p->xf_box_w = (int)(wf / nbf);
			p->tma_xf = true;
		}
	}
	// inverse: spectrum rows of a tile within one plane
	if (p->ny % (2 * LPB) == 0 && (size_t)2 * LPB * p->lx * sizeof(C) <= G::SB_I) {
		const uint64_t rowb = (uint64_t)p->lx * sizeof(C);
		const uint64_t dims[4] = {(uint64_t)p->xbox_w, (uint64_t)p->xbox_n, (uint64_t)p->ny, 3ull * p->nz};
		const uint64_t strides[3] = {(uint64_t)p->xbox_w * 8, rowb, rowb * p->py};
		const uint32_t box[4] = {(uint32_t)p->xbox_w, (uint32_t)p->xbox_n, (uint32_t)(2 * LPB), 1};
		MM_TRY(tma_encode(&p->tm_xi, p->spec, 4, dims, strides, box));
		MM_TRY(set_smem<T>((const void *)k_x_inv_tma<T, N>, G::SMEM_I));
		MM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_x_inv_tma<T, N>, G::THREADS, G::SMEM_I));
		if (occ >= 1) {
			p->grid_xi = occ * num_sms();
			p->tma_xi = true;
		}
	}
	if ((p->tma_xf || p->tma_xi) && !p->err) {
		MM_CUDA(cudaMalloc(&p->err, sizeof(int)));
		MM_CUDA(cudaMemset(p->err, 0, sizeof(int)));
	}
	return MM_OK;
}

// Tensor map of the forward x pass over the real rows at M (NULL when M is not 16-byte aligned).
// Tensor map of the region bytes of the forward x pass (NULL when not usable for `reg`).
const CUtensorMap *x_reg_map(ConvPlan *p, const uint8_t *reg, int lpb)
{
	if (!p->tma_xf_scale || !reg || (reinterpret_cast<uintptr_t>(reg) & 15)) return nullptr;
	if (p->xr_ptr == reg) return &p->xr_map;
	const uint64_t dims[2] = {(uint64_t)p->nx / 8, (uint64_t)p->ny * p->nz};
	const uint64_t strides[1] = {(uint64_t)p->nx};
	const uint32_t box[2] = {(uint32_t)(p->nx / 8), (uint32_t)(2 * lpb)};
	if (tma_encode(&p->xr_map, reg, 2, dims, strides, box) != MM_OK) {
		clear_error();
		return nullptr;
	}
	p->xr_ptr = reg;
	return &p->xr_map;
}

template <typename T>
const CUtensorMap *x_fwd_map(ConvPlan *p, const T *M, int lpb)
{
	if (reinterpret_cast<uintptr_t>(M) & 15) return nullptr;
	for (int i = 0; i < ConvPlan::XF_CACHE; ++i)
		if (p->xf_ptr[i] == M) return &p->xf_map[i];
	const int slot = p->xf_next;
	const uint64_t rows = 3ull * p->ny * p->nz;
	const uint64_t dims[3] = {(uint64_t)p->xf_box_w, (uint64_t)p->xf_box_n, rows};
	const uint64_t strides[2] = {(uint64_t)p->xf_box_w * 8, (uint64_t)p->nx * sizeof(T)};
	const uint32_t box[3] = {(uint32_t)p->xf_box_w, (uint32_t)p->xf_box_n, (uint32_t)(2 * lpb)};
	if (tma_encode(&p->xf_map[slot], M, 3, dims, strides, box) != MM_OK) {
		clear_error();
		return nullptr;
	}
	p->xf_ptr[slot] = M;
	p->xf_next = (slot + 1) % ConvPlan::XF_CACHE;
	return &p->xf_map[slot];
}

template <typename T, int N>
bool fs_x_fwd_tma(ConvPlan *p, const T *M, const uint8_t *reg, const T *ms_tab, cudaStream_t st)
{
	using C = cplx<T>;
	using G = XTmaGeom<N, C>;
	const CUtensorMap *map = x_fwd_map<T>(p, M, G::LPB);
	if (!map) return false;
	const CUtensorMap *rmap = map;
	if (ms_tab) {
		// a missing region map means region 0 everywhere: the staged kernel needs real bytes
		rmap = reg ? x_reg_map(p, reg, G::LPB) : nullptr;
		if (!rmap) return false;
	}
	const int lines = (3 * p->ny * p->nz + 1) / 2;
	const int ntiles = (lines + G::LPB - 1) / G::LPB;
	const int grid = std::min(ntiles, p->grid_xf);
	if (ms_tab)
		k_x_fwd_tma<T, N, true><<<grid, G::THREADS, G::SMEM_F, st>>>(*map, *rmap, ms_tab, (C *)p->spec, p->nx, p->ny,
		                                                            p->nz, p->py, p->hx, p->lx, ntiles,
		                                                            (const C *)p->tw_x, p->err);
	else
		k_x_fwd_tma<T, N, false><<<grid, G::THREADS, G::SMEM_F, st>>>(*map, *rmap, ms_tab, (C *)p->spec, p->nx, p->ny,
		                                                             p->nz, p->py, p->hx, p->lx, ntiles,
		                                                             (const C *)p->tw_x, p->err);
	return true;
}

template <typename T, int N>
void fs_x_inv_tma(ConvPlan *p, T *H, cudaStream_t st)
{
	using C = cplx<T>;
	using G = XTmaGeom<N, C>;
	const int ntiles = 3 * p->ny * p->nz / (2 * G::LPB);
	const int grid = std::min(ntiles, p->grid_xi);
	k_x_inv_tma<T, N><<<grid, G::THREADS, G::SMEM_I, st>>>(p->tm_xi, H, p->nx, p->ny, p->hx, p->lx, ntiles,
	                                                     (const C *)p->tw_x, p->err);
}

template <typename T, int N>
void fs_x_fwd(ConvPlan *p, const T *M, const uint8_t *reg, const T *ms_tab, cudaStream_t st)
{
	using C = cplx<T>;
	constexpr int LPB = ct_lpb(N, sizeof(C)), TPL = N / ct_radix(N);
	const int lines = (3 * p->ny * p->nz + 1) / 2;
	const dim3 grid((lines + LPB - 1) / LPB), block(LPB * TPL);
	const size_t smem = (size_t)SmRows<N, LPB>::SIZE * sizeof(C);
	if (ms_tab)
		k_x_fwd_ct<T, N, LPB, true><<<grid, block, smem, st>>>(M, reg, ms_tab, (C *)p->spec, p->nx, p->ny, p->nz,
		                                                       p->py, p->hx, p->lx, (const C *)p->tw_x);
	else
		k_x_fwd_ct<T, N, LPB, false><<<grid, block, smem, st>>>(M, reg, ms_tab, (C *)p->spec, p->nx, p->ny, p->nz,
		                                                        p->py, p->hx, p->lx, (const C *)p->tw_x);
}

template <typename T, int N>
void fs_x_inv(ConvPlan *p, T *H, cudaStream_t st)
{
	using C = cplx<T>;
	constexpr int LPB = ct_lpb(N, sizeof(C)), TPL = N / ct_radix(N);
	const int lines = (3 * p->ny * p->nz + 1) / 2;
	const dim3 grid((lines + LPB - 1) / LPB), block(LPB * TPL);
	k_x_inv_ct<T, N, LPB><<<grid, block, (size_t)SmRows<N, LPB>::SIZE * sizeof(C), st>>>(
	    (const C *)p->spec, H, p->nx, p->ny, p->nz, p->py, p->hx, p->lx, (const C *)p->tw_x);
}

template <typename T, int N, bool INV>
void fs_y(ConvPlan *p, cudaStream_t st)
{
	using C = cplx<T>;
	constexpr int TB = ct_tb(N, sizeof(C)), TPL = N / ct_radix(N);
	const dim3 grid((p->hx + TB - 1) / TB, p->nz, 3), block(TB * TPL);
	k_y_ct<T, N, TB, INV><<<grid, block, (size_t)SmCols<N, TB>::SIZE * sizeof(C), st>>>(
	    (C *)p->spec, INV ? N : p->ny, INV ? p->ny : N, p->nz, p->hx, p->lx, (const C *)p->tw_y);
}

constexpr int CT_ZTB = 32;

template <typename T, int PZ>
void fs_z(ConvPlan *p, cudaStream_t st)
{
	using C = cplx<T>;
	const dim3 grid((p->hx + CT_ZTB - 1) / CT_ZTB, p->py), block(3 * CT_ZTB * (PZ / ct_radix8(PZ)));
	k_z_ct<T, PZ, CT_ZTB><<<grid, block, (size_t)SmCols<PZ, 3 * CT_ZTB>::SIZE * sizeof(C), st>>>(
	    (C *)p->spec, (const T *)p->tensor, p->nz, p->py, p->hx, p->lx, p->qy, p->qz, (const C *)p->tw_z);
}

#define MM_FS_SWITCH(n, CALL)                                                                    \
	switch (n) {                                                                                 \
	case 4: CALL(4); break;                                                                      \
	case 8: CALL(8); break;                                                                      \
	case 16: CALL(16); break;                                                                    \
	case 32: CALL(32); break;                                                                    \
	case 64: CALL(64); break;                                                                    \
	case 128: CALL(128); break;                                                                  \
	case 256: CALL(256); break;                                                                  \
	case 512: CALL(512); break;                                                                  \
	case 1024: CALL(1024); break;                                                                \
	case 2048: if constexpr (sizeof(T) == 4) { CALL(2048); } break;                               \
	default: break;                                                                              \
	}

template <typename T>
mm_status fs_setup(ConvPlan *p)
{
	MM_TRY(fft_reg_init());
	// the power-of-two passes skip the zero upper half of a forward transform, so an axis without
	// zero padding (a periodic one, padded length n) takes the generic mixed-radix passes
	p->fast_x = fs_len_ok<T>(p->px) && 2 * p->nx <= p->px;
	p->fast_y = !p->is2d && fs_len_ok<T>(p->py) && 2 * p->ny <= p->py;
	p->fast_z = !p->is2d && p->pz >= 2 && p->pz <= 64 && (p->pz & (p->pz - 1)) == 0 && 2 * p->nz <= p->pz;
	mm_status r = MM_OK;
#define MM_SETUP(N) r = fs_setup_len<T, N>()
	if (p->fast_x) { MM_FS_SWITCH(p->px, MM_SETUP); MM_TRY(r); }
	if (p->fast_y) { MM_FS_SWITCH(p->py, MM_SETUP); MM_TRY(r); }
#undef MM_SETUP
#define MM_XTSETUP(N) r = fs_setup_x_tma<T, N>(p)
	if (p->fast_x) { MM_FS_SWITCH(p->px, MM_XTSETUP); MM_TRY(r); }
#undef MM_XTSETUP
#define MM_YTSETUP(N) r = fs_setup_y_tma<T, N>(p)
	if (p->fast_y) { MM_FS_SWITCH(p->py, MM_YTSETUP); MM_TRY(r); }
#undef MM_YTSETUP
	p->reg_z = p->fast_z && 2 * p->nz <= p->pz && p->pz <= (sizeof(T) == 4 ? 32 : 16);
	if (p->reg_z) {
		const size_t sz = zr_smem<T>(p->pz);
		switch (p->pz) {
		case 2: MM_TRY(set_smem<T>((const void *)k_z_reg<T, 2>, sz)); break;
		case 4: MM_TRY(set_smem<T>((const void *)k_z_reg<T, 4>, sz)); break;
		case 8: MM_TRY(set_smem<T>((const void *)k_z_reg<T, 8>, sz)); break;
		case 16: MM_TRY(set_smem<T>((const void *)k_z_reg<T, 16>, sz)); break;
		case 32: if constexpr (sizeof(T) == 4) { MM_TRY(set_smem<T>((const void *)k_z_reg<T, 32>, sz)); } break;
		}
	} else if (p->fast_z) {
		const size_t sz = (size_t)(p->pz * 3 * CT_ZTB + (p->pz * 3 * CT_ZTB >> 5) + 1) * sizeof(cplx<T>);
		switch (p->pz) {
		case 2: MM_TRY(set_smem<T>((const void *)k_z_ct<T, 2, CT_ZTB>, sz)); break;
		case 4: MM_TRY(set_smem<T>((const void *)k_z_ct<T, 4, CT_ZTB>, sz)); break;
		case 8: MM_TRY(set_smem<T>((const void *)k_z_ct<T, 8, CT_ZTB>, sz)); break;
		case 16: MM_TRY(set_smem<T>((const void *)k_z_ct<T, 16, CT_ZTB>, sz)); break;
		case 32: MM_TRY(set_smem<T>((const void *)k_z_ct<T, 32, CT_ZTB>, sz)); break;
		case 64: MM_TRY(set_smem<T>((const void *)k_z_ct<T, 64, CT_ZTB>, sz)); break;
		}
	}
	return MM_OK;
}

template <typename T>
mm_status tensor_spectrum(ConvPlan *p, const double *N, cudaStream_t st)
{
	const int px = p->px, py = p->py, pz = p->pz;
	const size_t cnt = (size_t)px * py * pz;
	double2 *X = nullptr;
	MM_CUDA(cudaMalloc(&X, cnt * sizeof(double2)));
	void *twx = nullptr, *twy = nullptr, *twz = nullptr;
	mm_status st_ = make_twiddles<double>(px, &twx);
	if (st_ == MM_OK) st_ = make_twiddles<double>(py, &twy);
	if (st_ == MM_OK) st_ = make_twiddles<double>(pz, &twz);
	double *mx = nullptr;
	if (st_ == MM_OK) st_ = cuda_status(cudaMalloc(&mx, 2 * sizeof(double)), "cudaMalloc");
	if (st_ == MM_OK) st_ = cuda_status(cudaMemsetAsync(mx, 0, 2 * sizeof(double), st), "cudaMemsetAsync");
	const double scale = 1.0 / ((double)px * py * pz);
	const size_t per = (size_t)p->qz * p->qy * p->hx;
	const int gsz = num_sms() * 8;
	for (int comp = 0; comp < 6 && st_ == MM_OK; ++comp) {
		k_tensor_component<<<gsz, NT, 0, st>>>(N, X, cnt, comp);
		st_ = after_launch("k_tensor_component");
		const int dims[3] = {px, py, pz};
		const FftRadices rads[3] = {p->rx, p->ry, p->rz};
		void *tws[3] = {twx, twy, twz};
		size_t inner = 1, outer = (size_t)py * pz;
		for (int ax = 0; ax < 3 && st_ == MM_OK; ++ax) {
			const int len = dims[ax];
			if (len > 1) {
				const int TB = pick_tile(len, 1, sizeof(double2), inner == 1 ? 4 : 16);
				const size_t smem = (size_t)(2 * TB + 1) * len * sizeof(double2);
				st_ = set_smem<double>((const void *)k_fft_axis<double, false>, smem);
				if (st_ != MM_OK) break;
				dim3 grid;
				if (inner == 1) grid = dim3((unsigned)((outer + TB - 1) / TB), 1, 1);
				else grid = dim3((unsigned)((inner + TB - 1) / TB), (unsigned)outer, 1);
				k_fft_axis<double, false><<<grid, NT, smem, st>>>(X, (int)inner, (int)outer, rads[ax],
				                                                 (const double2 *)tws[ax], TB);
				st_ = after_launch("k_fft_axis");
			}
			inner *= len;
			outer = ax == 0 ? pz : 1;
		}
		if (st_ != MM_OK) break;
		k_tensor_extract<T><<<gsz, NT, 0, st>>>(X, (T *)p->tensor + comp * per, px, py, p->hx, p->qy,
		                                       p->qz, scale, mx, mx + 1);
		st_ = after_launch("k_tensor_extract");
	}
	double hm[2] = {0, 0};
	if (st_ == MM_OK) st_ = cuda_status(cudaMemcpyAsync(hm, mx, sizeof(hm), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
	if (st_ == MM_OK) st_ = cuda_status(cudaStreamSynchronize(st), "cudaStreamSynchronize");
	p->max_imag_rel = hm[0] > 0 ? hm[1] / hm[0] : 0.0;
	cudaFree(X);
	cudaFree(twx);
	cudaFree(twy);
	cudaFree(twz);
	cudaFree(mx);
	return st_;
}

template <typename T>
mm_status plan_setup(ConvPlan *p, const double *N, cudaStream_t st)
{
	using C = cplx<T>;
	MM_TRY(make_twiddles<T>(p->px, &p->tw_x));
	MM_TRY(make_twiddles<T>(p->py, &p->tw_y));
	MM_TRY(make_twiddles<T>(p->pz, &p->tw_z));
	MM_CUDA(cudaMalloc(&p->tensor, sizeof(T) * 6 * (size_t)p->qz * p->qy * p->hx));
	MM_CUDA(cudaMalloc(&p->spec, p->spec_bytes()));
	MM_CUDA(cudaMemsetAsync(p->spec, 0, p->spec_bytes(), st));
	// launch geometry
	{
		int lp = 8;
		while (lp > 1 && (size_t)(2 * lp + 1) * p->px * sizeof(C) > SMEM_TARGET) lp >>= 1;
		p->lp_x = lp;
		p->smem_x = (size_t)(2 * lp + 1) * p->px * sizeof(C);
	}
	if (p->is2d) {
		p->tb_y = pick_tile(p->py, 3, sizeof(C), 32);
		p->smem_y = (size_t)(6 * p->tb_y + 1) * p->py * sizeof(C);
	} else {
		p->tb_y = pick_tile(p->py, 1, sizeof(C), 32);
		p->smem_y = (size_t)(2 * p->tb_y + 1) * p->py * sizeof(C);
		p->tb_z = pick_tile(p->pz, 3, sizeof(C), 32);
		p->smem_z = (size_t)(6 * p->tb_z + 1) * p->pz * sizeof(C);
	}
	if (p->smem_x > 227 * 1024 || p->smem_y > 227 * 1024 || p->smem_z > 227 * 1024)
		return fail(MM_ERR_UNSUPPORTED, "conv: FFT length too large for one CTA");
	MM_TRY(set_smem<T>((const void *)k_x_fwd<T, false>, p->smem_x));
	MM_TRY(set_smem<T>((const void *)k_x_fwd<T, true>, p->smem_x));
	MM_TRY(set_smem<T>((const void *)k_x_inv<T>, p->smem_x));
	if (p->is2d) {
		MM_TRY(set_smem<T>((const void *)k_y_mul2d<T>, p->smem_y));
	} else {
		MM_TRY(set_smem<T>((const void *)k_y<T, false>, p->smem_y));
		MM_TRY(set_smem<T>((const void *)k_y<T, true>, p->smem_y));
		MM_TRY(set_smem<T>((const void *)k_z_mul<T>, p->smem_z));
	}
	MM_TRY(fs_setup<T>(p));
	return tensor_spectrum<T>(p, N, st);
}

template <typename T>
mm_status execute(ConvPlan *p, const T *M, const uint8_t *reg, const T *ms_tab, T *H, cudaStream_t st)
{
	using C = cplx<T>;
	C *S = (C *)p->spec;
	const int rows = 3 * p->ny * p->nz;
	const int lines = (rows + 1) / 2;
	const int gx = (lines + p->lp_x - 1) / p->lp_x;
	// algorithmic bytes of each pass (every array element crossing HBM once)
	const double n = (double)p->nx * p->ny * p->nz, s = sizeof(T), c = sizeof(C);
	const double half = 3.0 * p->hx * p->ny * p->nz * c;      // x-transformed rows y < ny, z < nz
	const double ypad = 3.0 * p->hx * p->py * p->nz * c;      // y-transformed, z < nz
	const double tens = 6.0 * p->hx * p->qy * p->qz * s;
	ProfToken tk = prof_begin(st);
	bool staged = false;
	if (p->tma_xf) {
#define MM_XTF(N) staged = fs_x_fwd_tma<T, N>(p, M, reg, ms_tab, st)
		MM_FS_SWITCH(p->px, MM_XTF);
#undef MM_XTF
	}
	if (staged) {
	} else if (p->fast_x) {
#define MM_XF(N) fs_x_fwd<T, N>(p, M, reg, ms_tab, st)
		MM_FS_SWITCH(p->px, MM_XF);
#undef MM_XF
	} else if (ms_tab)
		k_x_fwd<T, true><<<gx, NT, p->smem_x, st>>>(M, reg, ms_tab, S, p->nx, p->ny, p->nz, p->py, p->hx, p->lx,
		                                            p->rx, (const C *)p->tw_x, p->lp_x);
	else
		k_x_fwd<T, false><<<gx, NT, p->smem_x, st>>>(M, reg, ms_tab, S, p->nx, p->ny, p->nz, p->py, p->hx, p->lx,
		                                             p->rx, (const C *)p->tw_x, p->lp_x);
	const char *xf_name = staged ? "k_x_fwd_tma" : p->fast_x ? "k_x_fwd_ct" : "k_x_fwd";
	MM_TRY(after_launch(xf_name));
	prof_end(tk, xf_name, 3 * n * s + (reg ? n : 0.0) + half, st);
	if (p->is2d) {
		const int gy = (p->hx + p->tb_y - 1) / p->tb_y;
		tk = prof_begin(st);
		k_y_mul2d<T><<<gy, NT, p->smem_y, st>>>(S, (const T *)p->tensor, p->ny, p->hx, p->lx, p->qy, p->ry,
		                                        (const C *)p->tw_y, p->tb_y);
		MM_TRY(after_launch("k_y_mul2d"));
		prof_end(tk, "k_y_mul2d", 2 * half + tens, st);
	} else {
		dim3 gy((p->hx + p->tb_y - 1) / p->tb_y, p->nz, 3);
		tk = prof_begin(st);
		if (p->tma_y) {
#define MM_YTF(N) fs_y_tma<T, N, false>(p, st)
			MM_FS_SWITCH(p->py, MM_YTF);
#undef MM_YTF
		} else if (p->fast_y) {
#define MM_YF(N) fs_y<T, N, false>(p, st)
			MM_FS_SWITCH(p->py, MM_YF);
#undef MM_YF
		} else
			k_y<T, false><<<gy, NT, p->smem_y, st>>>(S, p->ny, p->py, p->nz, p->py, p->hx, p->lx, p->ry,
			                                         (const C *)p->tw_y, p->tb_y);
		const char *yf_name = p->tma_y ? "k_y_tma (forward)" : p->fast_y ? "k_y_ct (forward)" : "k_y (forward)";
		MM_TRY(after_launch(yf_name));
		prof_end(tk, yf_name, half + ypad, st);
		dim3 gz((p->hx + p->tb_z - 1) / p->tb_z, p->py, 1);
		tk = prof_begin(st);
		if (p->reg_z) {
			switch (p->pz) {
			case 2: fs_z_reg<T, 2>(p, st); break;
			case 4: fs_z_reg<T, 4>(p, st); break;
			case 8: fs_z_reg<T, 8>(p, st); break;
			case 16: fs_z_reg<T, 16>(p, st); break;
			case 32: if constexpr (sizeof(T) == 4) { fs_z_reg<T, 32>(p, st); } break;
			}
		} else if (p->fast_z) {
			switch (p->pz) {
			case 2: fs_z<T, 2>(p, st); break;
			case 4: fs_z<T, 4>(p, st); break;
			case 8: fs_z<T, 8>(p, st); break;
			case 16: fs_z<T, 16>(p, st); break;
			case 32: fs_z<T, 32>(p, st); break;
			case 64: fs_z<T, 64>(p, st); break;
			}
		} else
			k_z_mul<T><<<gz, NT, p->smem_z, st>>>(S, (const T *)p->tensor, p->nz, p->py, p->hx, p->lx, p->qy, p->qz,
			                                      p->rz, (const C *)p->tw_z, p->tb_z);
		const char *z_name = p->reg_z ? "k_z_reg" : p->fast_z ? "k_z_ct" : "k_z_mul";
		MM_TRY(after_launch(z_name));
		prof_end(tk, z_name, 2 * ypad + tens, st);
		tk = prof_begin(st);
		if (p->tma_y) {
#define MM_YTI(N) fs_y_tma<T, N, true>(p, st)
			MM_FS_SWITCH(p->py, MM_YTI);
#undef MM_YTI
		} else if (p->fast_y) {
#define MM_YI(N) fs_y<T, N, true>(p, st)
			MM_FS_SWITCH(p->py, MM_YI);
#undef MM_YI
		} else
			k_y<T, true><<<gy, NT, p->smem_y, st>>>(S, p->py, p->ny, p->nz, p->py, p->hx, p->lx, p->ry,
			                                        (const C *)p->tw_y, p->tb_y);
		const char *yi_name = p->tma_y ? "k_y_tma (inverse)" : p->fast_y ? "k_y_ct (inverse)" : "k_y (inverse)";
		MM_TRY(after_launch(yi_name));
		prof_end(tk, yi_name, half + ypad, st);
	}
	tk = prof_begin(st);
	if (p->tma_xi) {
#define MM_XTI(N) fs_x_inv_tma<T, N>(p, H, st)
		MM_FS_SWITCH(p->px, MM_XTI);
#undef MM_XTI
	} else if (p->fast_x) {
#define MM_XI(N) fs_x_inv<T, N>(p, H, st)
		MM_FS_SWITCH(p->px, MM_XI);
#undef MM_XI
	} else
		k_x_inv<T><<<gx, NT, p->smem_x, st>>>(S, H, p->nx, p->ny, p->nz, p->py, p->hx, p->lx, p->rx,
		                                      (const C *)p->tw_x, p->lp_x);
	const char *xi_name = p->tma_xi ? "k_x_inv_tma" : p->fast_x ? "k_x_inv_ct" : "k_x_inv";
	MM_TRY(after_launch(xi_name));
	prof_end(tk, xi_name, half + 3 * n * s, st);
	return MM_OK;
}

} // namespace

mm_status fft_reg_init()
{
	double2 d[64];
	float2 f[64];
	for (int k = 0; k < 64; ++k) {
		const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / 64.0L;
		d[k] = double2{(double)cosl(a), (double)sinl(a)};
		f[k] = float2{(float)cosl(a), (float)sinl(a)};
	}
	MM_CUDA(cudaMemcpyToSymbol(c_w64d, d, sizeof(d)));
	MM_CUDA(cudaMemcpyToSymbol(c_w64f, f, sizeof(f)));
	return MM_OK;
}

size_t ConvPlan::spec_bytes() const
{
	const size_t c = prec == MM_F64 ? sizeof(double2) : sizeof(float2);
	return c * 3 * (size_t)nz * py * lx;
}

mm_status tma_encode(CUtensorMap *map, const void *base, int rank, const uint64_t *dims, const uint64_t *strides,
                     const uint32_t *box)
{
	return tma_encode_as(map, base, rank, dims, strides, box, 8);
}

mm_status tma_encode_as(CUtensorMap *map, const void *base, int rank, const uint64_t *dims, const uint64_t *strides,
                        const uint32_t *box, int esize)
{
	using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
	                            const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
	                            CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
	static Encode encode = nullptr;
	if (!encode) {
		void *fn = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
		    q != cudaDriverEntryPointSuccess || !fn) {
			cudaGetLastError();
			return fail(MM_ERR_UNSUPPORTED, "conv: cuTensorMapEncodeTiled is not available from the driver");
		}
		encode = reinterpret_cast<Encode>(fn);
	}
	if (esize != 1 && esize != 4 && esize != 8) return fail(MM_ERR_INVALID_ARGUMENT, "tensor map element size");
	if (rank < 1 || rank > 5 || (reinterpret_cast<uintptr_t>(base) & 15) || ((box[0] * esize) & 15))
		return fail(MM_ERR_INVALID_ARGUMENT, "conv: tensor map not 16-byte aligned");
	cuuint64_t d[5], sb[4];
	cuuint32_t bx[5], estr[5];
	for (int i = 0; i < rank; ++i) {
		d[i] = dims[i];
		bx[i] = box[i];
		estr[i] = 1;
		if (box[i] < 1 || box[i] > 256) return fail(MM_ERR_INVALID_ARGUMENT, "conv: tensor map box beyond 256");
	}
	for (int i = 0; i + 1 < rank; ++i) {
		sb[i] = strides[i];
		if (strides[i] & 15) return fail(MM_ERR_INVALID_ARGUMENT, "conv: tensor map stride not 16-byte aligned");
	}
	const CUtensorMapDataType dt = esize == 1   ? CU_TENSOR_MAP_DATA_TYPE_UINT8
	                               : esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32
	                                            : CU_TENSOR_MAP_DATA_TYPE_UINT64;
	const CUresult r = encode(map, dt, (cuuint32_t)rank, const_cast<void *>(base), d, sb,
	                          bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
	                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS)
		return fail(MM_ERR_CUDA, "conv: cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
	return MM_OK;
}

mm_status tma_encode_3d(CUtensorMap *map, const void *base, uint64_t d0, uint64_t d1, uint64_t d2,
                        uint64_t stride1, uint64_t stride2, uint32_t b0, uint32_t b1, uint32_t b2)
{
	const uint64_t dims[3] = {d0, d1, d2}, strides[2] = {stride1, stride2};
	const uint32_t box[3] = {b0, b1, b2};
	return tma_encode(map, base, 3, dims, strides, box);
}

ConvPlan::~ConvPlan()
{
	cudaFree(tw_x);
	cudaFree(tw_y);
	cudaFree(tw_z);
	cudaFree(tensor);
	cudaFree(tensor_kx);
	cudaFree(spec);
	cudaFree(err);
}

int conv_launches(const ConvPlan *p) { return p->is2d ? 3 : 5; }

mm_status conv_plan_create(ConvPlan **out, int prec, int nx, int ny, int nz, int px, int py, int pz,
                           const double *N, cudaStream_t st)
{
	if (prec != MM_F64 && prec != MM_F32) return fail(MM_ERR_INVALID_ARGUMENT, "conv: bad precision");
	if (nx <= 0 || ny <= 0 || nz <= 0 || px < nx || py < ny || pz < nz || !N)
		return fail(MM_ERR_INVALID_ARGUMENT, "conv: invalid sizes or null tensor");
	ConvPlan *p = new ConvPlan();
	p->prec = prec;
	p->nx = nx; p->ny = ny; p->nz = nz;
	p->px = px; p->py = py; p->pz = pz;
	p->hx = px / 2 + 1;
	{
		// row stride: 8-byte elements per row a multiple of 2 * xbox_n, so that a row splits into
		// xbox_n TMA boxes of xbox_w (even, <= 256) elements with 16-byte aligned rows
		const int E = prec == MM_F32 ? 1 : 2;
		int w = p->hx * E;
		const int nb = (w + 255) / 256;
		w = (w + 2 * nb - 1) / (2 * nb) * (2 * nb);
		p->lx = w / E;
		p->xbox_n = nb;
		p->xbox_w = w / nb;
	}
	p->qy = py / 2 + 1;
	p->qz = pz / 2 + 1;
	p->is2d = (nz == 1 && pz == 1);
	p->rx = fft_factor(px);
	p->ry = fft_factor(py);
	p->rz = fft_factor(pz);
	if (p->rx.count < 0 || p->ry.count < 0 || p->rz.count < 0) {
		delete p;
		return fail(MM_ERR_UNSUPPORTED, "conv: FFT length has too many prime factors");
	}
	const mm_status s = prec == MM_F64 ? plan_setup<double>(p, N, st) : plan_setup<float>(p, N, st);
	if (s != MM_OK) {
		delete p;
		return s;
	}
	*out = p;
	return MM_OK;
}

mm_status conv_execute(ConvPlan *p, const void *M, const uint8_t *regions, const void *ms_table,
                       void *H, cudaStream_t st)
{
	if (p->prec == MM_F64)
		return execute<double>(p, (const double *)M, regions, (const double *)ms_table, (double *)H, st);
	return execute<float>(p, (const float *)M, regions, (const float *)ms_table, (float *)H, st);
}

// ---- grouped convolution: many plans, one launch per pass and transform length -------------------
// Every member plan uses the power-of-two passes (register z pass included).  The members' blocks
// of one pass and one length form a work list (member, block); a member whose run flag is 0
// skips its blocks, so finished instances drop out without rebuilding the lists.
namespace {

template <typename T>
struct GDesc {
	cplx<T> *spec;
	const T *tensor;
	const T *tensor_t;  // fused y+z members: the reduced tensor kx-major, [hx][qz][qy][6]
	const cplx<T> *tw_x, *tw_y;
	const T *M[4];
	T *H[2];
	const uint8_t *reg;
	const T *ms_tab;
	const int *flags;   // the member's run flags: [0] runs, [1] gated runs (NULL: always)
	int nx, ny, nz, py, hx, lx, qy, qz;
};

// Tile-shape variants the autotuner chooses from per pass and length: 0 the default (radix 16,
// the single-instance tile), 1 half the lines/columns per CTA, 2 radix-8 passes, 3 (y passes
// only) TMA-staged tiles on persistent CTAs.
constexpr int GRP_VARIANTS = 4;
__host__ __device__ constexpr int var_radix(int n, int v) { return v == 2 ? (n < 8 ? n : 8) : ct_radix(n); }
__host__ __device__ constexpr int var_tb(int n, int csize, int v)
{
	return v == 1 ? (ct_tb(n, csize) > 1 ? ct_tb(n, csize) / 2 : 1) : ct_tb(n, csize);
}
__host__ __device__ constexpr int var_lpb(int n, int csize, int v)
{
	return v == 1 ? (ct_lpb(n, csize) > 1 ? ct_lpb(n, csize) / 2 : 1) : ct_lpb(n, csize);
}

__device__ __forceinline__ bool member_skips(const int *flags, int gate)
{
	return flags && (!flags[0] || (gate && !flags[gate]));
}

template <typename T, int N, int LPB, int R>
__global__ void __launch_bounds__(LPB * (N / R)) k_x_fwd_grp(const GDesc<T> *__restrict__ d,
                                                                      const int2 *__restrict__ items, int input,
                                                                      int gate)
{
	const int2 it = items[blockIdx.x];
	if (member_skips(d[it.x].flags, gate)) return;
	const GDesc<T> g = d[it.x];
	x_fwd_ct_body<T, N, LPB, true, R, true>(g.M[input], g.reg, g.ms_tab, g.spec, g.nx, g.ny, g.nz, g.py, g.hx, g.lx,
	                                  g.tw_x, it.y);
}

template <typename T, int N, int LPB, int R>
__global__ void __launch_bounds__(LPB * (N / R)) k_x_inv_grp(const GDesc<T> *__restrict__ d,
                                                                      const int2 *__restrict__ items, int output,
                                                                      int gate)
{
	const int2 it = items[blockIdx.x];
	if (member_skips(d[it.x].flags, gate)) return;
	const GDesc<T> g = d[it.x];
	x_inv_ct_body<T, N, LPB, R>(g.spec, g.H[output], g.nx, g.ny, g.nz, g.py, g.hx, g.lx, g.tw_x, it.y);
}

template <typename T, int N, int TB, bool INV, int R>
__global__ void __launch_bounds__(TB * (N / R)) k_y_grp(const GDesc<T> *__restrict__ d,
                                                                    const int2 *__restrict__ items, int gate)
{
	const int2 it = items[blockIdx.x];
	if (member_skips(d[it.x].flags, gate)) return;
	const GDesc<T> g = d[it.x];
	const int tiles = (g.hx + TB - 1) / TB;
	y_ct_body<T, N, TB, INV, R>(g.spec, INV ? N : g.ny, INV ? g.ny : N, g.hx, g.lx, g.tw_y, it.y % tiles,
	                            it.y / tiles);
}

template <typename T, int PZ>
__global__ void __launch_bounds__(ZR_THREADS, 3) k_z_grp(const GDesc<T> *__restrict__ d, const int2 *__restrict__ items,
                                                        int gate)
{
	const int2 it = items[blockIdx.x];
	if (member_skips(d[it.x].flags, gate)) return;
	const GDesc<T> g = d[it.x];
	const int tiles = (g.hx + 31) / 32;
	z_reg_body<T, PZ>(g.spec, g.tensor, g.nz, g.py, g.hx, g.lx, g.qy, g.qz, it.y % tiles, it.y / tiles);
}

// Grouped y pass through TMA-staged tiles (the autotuner's variant 3): persistent CTAs walk the
// work list (member, column tile) of one length, skipping members whose run flags say so; each
// member has its own tensor maps (maps[2 member + INV], in global memory).  Pipeline as k_y_tma.
template <typename T, int N, bool INV>
__global__ void __launch_bounds__(ct_tb(N, sizeof(cplx<T>)) * (N / ct_radix(N)), 1)
    k_y_tma_grp(const GDesc<T> *__restrict__ d, const CUtensorMap *__restrict__ maps, const int2 *__restrict__ items,
                int n_items, int gate, int *err)
{
	using C = cplx<T>;
	constexpr int TB = ct_tb(N, sizeof(C));
	using G = YTmaGeom<N, TB, INV, C>;
	constexpr int R = ct_radix(N);
	using SI = SmCols<N, TB, 4>;
	extern __shared__ __align__(128) unsigned char smem_tma[];
	C *stage0 = reinterpret_cast<C *>(smem_tma);
	C *stage1 = stage0 + TB * G::ROWS;
	C *work = reinterpret_cast<C *>(smem_tma + 2 * (size_t)G::TILE_BYTES);
	uint64_t *bar = reinterpret_cast<uint64_t *>(smem_tma + 2 * (size_t)G::TILE_BYTES + G::WORK);
	const int tid = threadIdx.x;
	const int line = tid & (TB - 1), j0 = tid / TB;
	// this CTA's tiles: t = blockIdx.x + k gridDim.x, members that run only
	auto next_tile = [&](int t) {
		while (t < n_items && member_skips(d[items[t].x].flags, gate)) t += gridDim.x;
		return t;
	};
	auto issue = [&](int t, int b) {
		const int2 it = items[t];
		const int tiles_x = (d[it.x].hx + TB - 1) / TB;
		const int tx = it.y % tiles_x, plane = it.y / tiles_x;
		C *dst = b ? stage1 : stage0;
		const CUtensorMap *map = &maps[2 * it.x + (INV ? 1 : 0)];
		// the maps were written by a host copy before the launch: order those writes before the
		// tensor-map proxy reads them
		asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
		mbar_expect_tx(&bar[b], G::TILE_BYTES);
#pragma unroll
		for (int q = 0; q < G::NBOX; ++q)
			tma_load_3d(dst + q * G::BR * TB, map, tx * TB * G::E, q * G::BR, plane, &bar[b]);
	};
	if (tid == 0) {
		mbar_init(&bar[0], 1);
		mbar_init(&bar[1], 1);
		fence_proxy_async();
	}
	__syncthreads();
	int t = next_tile(blockIdx.x);
	int t1 = t < n_items ? next_tile(t + gridDim.x) : n_items;
	if (tid == 0) {
		if (t < n_items) issue(t, 0);
		if (t1 < n_items) issue(t1, 1);
	}
	uint32_t parity = 0;
	for (int k = 0; t < n_items; ++k) {
		const int b = k & 1;
		const bool late = !mbar_wait(&bar[b], (parity >> b) & 1u);
		if (__syncthreads_or(late)) {
			if (tid == 0) {
				atomicExch(err, 1);
				mbar_drain2(bar, parity, b, t1 < n_items);
			}
			return;
		}
		parity ^= 1u << b;
		const int2 it = items[t];
		const GDesc<T> &g = d[it.x];
		const int tiles_x = (g.hx + TB - 1) / TB;
		const int tx = it.y % tiles_x, plane = it.y / tiles_x;
		const int kx = tx * TB + line;
		const bool ok = kx < g.hx;
		const int lx = g.lx, n_out = INV ? g.ny : N;
		C *base = g.spec + (size_t)plane * N * lx + (ok ? kx : 0);
		const C *sb = b ? stage1 : stage0;
		auto ld = [&](int, int r) -> C { return r < G::ROWS ? sb[r * TB + line] : C{0, 0}; };
		auto st = [&](int, int r, C v) {
			if (ok && r < n_out) base[(size_t)r * lx] = v;
		};
		const int t2 = t1 < n_items ? next_tile(t1 + gridDim.x) : n_items;
		auto release = [&]() {
			__syncthreads();  // every thread has read stage buffer b
			if (tid == 0 && t2 < n_items) {
				fence_proxy_async();
				issue(t2, b);
			}
		};
		if constexpr (INV) cta_fft<T, N, R, TB, INV, SI>(work, g.tw_y, line, j0, ld, st, release);
		else cta_fft_h0<T, N, R, TB, SI>(work, g.tw_y, line, j0, ld, st, release);
		t = t1;
		t1 = t2;
	}
}

// Asynchronous copy of one complex value global -> shared (LDGSTS, 8 or 16 bytes).
template <class C>
__device__ __forceinline__ void cp_async_c(C *dst, const C *src)
{
	const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
	if constexpr (sizeof(C) == 8)
		asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
	else
		asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all_c() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit_c() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group_c() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Fused y and z passes for small members (the autotuner-free path of the grouped convolution):
// one CTA takes a tile of TB x-frequency columns of one member and keeps all of its y-z data in
// shared memory: the forward y transforms of the 3*NZ (component, z) lines of every column (ny
// data rows, zero padded to PY), the z transform, tensor multiply and inverse z transform of every
// (ky, column) in registers (3 components x PZ values per thread, the zero half of each z column
// skipped), and the inverse y transforms, whose rows y < ny go back to HBM.  The full y spectrum
// never reaches HBM: the pass reads and writes the x-transformed rows once and reads the tensor.
// Lines are split into G groups of LG lines so that a group's transform needs at most 512 threads
// (128 registers per thread for the z columns); tiles stay within ~104 KB of shared memory so
// that two CTAs share an SM.
// Reduced tensor [6][qz][qy][hx] -> kx-major [hx][qz][qy][6] (one thread per destination entry).
template <typename T>
__global__ void k_tensor_kx(const T *__restrict__ src, T *__restrict__ dst, int hx, int qy, int qz)
{
	const size_t ne = (size_t)6 * hx * qy * qz;
	for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ne; e += (size_t)gridDim.x * blockDim.x) {
		const int c = (int)(e % 6);
		size_t r = e / 6;
		const int ky = (int)(r % qy);
		r /= qy;
		const int kz = (int)(r % qz);
		const int kx = (int)(r / qz);
		dst[e] = src[(((size_t)c * qz + kz) * qy + ky) * hx + kx];
	}
}

// NARROW: one kx column per CTA (a small group, such as the tail of a batch, then spreads over more
// SMs); each line's transforms and each (ky, column)'s multiply are the same operations either
// way, so the results do not depend on the choice.
template <int PY, int PZ, class C, bool NARROW = false>
struct YZGeom {
	static constexpr int NZ = PZ / 2;  // planes a member of this group can have (nz <= pz/2)
	static constexpr int R = ct_radix(PY), TPL = PY / R;
	static constexpr size_t line_bytes = (size_t)PY * sizeof(C);
	static constexpr int tb_for(int tb)
	{
		return (tb > 1 && (size_t)3 * NZ * tb * line_bytes * 33 / 32 > 104 * 1024) ? tb_for(tb / 2) : tb;
	}
	static constexpr int TB = NARROW ? 1 : tb_for(8);
	static constexpr int L = 3 * NZ * TB;
	static constexpr int g_for(int g) { return ((L / g) * TPL > 512 && L % (2 * g) == 0) ? g_for(g * 2) : g; }
	static constexpr int G = g_for(1);
	static constexpr int LG = L / G;
	static constexpr int THREADS = LG * TPL;
	static constexpr size_t GROUP_ELEMS = SmCols<PY, LG, 4>::SIZE;
	static constexpr size_t DATA = ((size_t)G * GROUP_ELEMS * sizeof(C) + 15) / 16 * 16;
	// behind the y-z data: the tile's reduced tensor entries, kx-major [TB][PZ/2+1][PY/2+1][6],
	// copied in while the forward y transforms run
	static constexpr int QY = PY / 2 + 1, QZ = PZ / 2 + 1;
	static constexpr size_t TENS = (size_t)TB * QZ * QY * 6 * (sizeof(C) / 2);
	static constexpr size_t SMEM = DATA + TENS;
	static constexpr bool fits = SMEM <= 227 * 1024 && THREADS >= 32 && THREADS <= 1024 && L % G == 0;
};

template <typename T, int PY, int PZ, bool NARROW = false>
__global__ void __launch_bounds__(YZGeom<PY, PZ, cplx<T>, NARROW>::THREADS)
    k_yz_grp(const GDesc<T> *__restrict__ d, const int2 *__restrict__ items, int gate)
{
	using C = cplx<T>;
	using G = YZGeom<PY, PZ, C, NARROW>;
	constexpr int TB = G::TB, LG = G::LG, NZ = G::NZ, H = PZ / 2;
	using SI = SmCols<PY, LG, 4>;
	const int2 it = items[blockIdx.x];
	if (member_skips(d[it.x].flags, gate)) return;
	const GDesc<T> &g = d[it.x];
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *smem = reinterpret_cast<C *>(smem_raw);
	const int tid = threadIdx.x;
	const int nz = g.nz, ny = g.ny, hx = g.hx, lx = g.lx;
	const int kx0 = it.y * TB;
	// line l = (c * NZ + z) * TB + col of group l / LG
	auto elem = [&](int l, int k) -> C & { return smem[(size_t)(l / LG) * G::GROUP_ELEMS + SI::at(l % LG, k)]; };
	// the tile's x-transformed rows (y < ny) land in the groups' buffers by asynchronous copies
	// issued all at once; lines outside the member (z >= nz, kx >= hx) are never stored
	{
		// a thread keeps its column and walks the (component-plane, row) pairs, y fastest, with
		// the row position carried forward instead of divided out per element
		static_assert(G::THREADS % TB == 0, "a thread keeps its column");
		constexpr int STEP = G::THREADS / TB;
		const int col = tid % TB, kx = kx0 + col, rows = 3 * NZ * ny;
		int row = tid / TB, cz = row / ny, y = row - cz * ny;
		if (kx < hx) {
			while (row < rows) {
				const int c = cz / NZ, z = cz % NZ;
				if (z < nz) {
					const int l = cz * TB + col;
					cp_async_c(&smem[(size_t)(l / LG) * G::GROUP_ELEMS + SI::at(l % LG, y)],
					           g.spec + ((size_t)(c * nz + z) * g.py + y) * lx + kx);
				}
				row += STEP;
				if (row >= rows) break;
				y += STEP;
				while (y >= ny) {
					y -= ny;
					++cz;
				}
			}
		}
	}
	cp_async_commit_c();
	// the tile's tensor entries: one contiguous run of the kx-major tensor (columns kx < hx)
	using T2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
	T2 *tsm = reinterpret_cast<T2 *>(smem_raw + G::DATA);
	{
		const int cols = hx - kx0 < TB ? hx - kx0 : TB;
		const int pairs = cols * G::QZ * G::QY * 3;
		const C *src = reinterpret_cast<const C *>(g.tensor_t + (size_t)kx0 * G::QZ * G::QY * 6);
		for (int e = tid; e < pairs; e += G::THREADS) cp_async_c(reinterpret_cast<C *>(tsm) + e, src + e);
	}
	cp_async_commit_c();
	cp_async_wait_group_c<1>();  // the y-z data (the tensor may still be arriving)
	__syncthreads();
	// forward y transforms in place (rows ny.. are the zero padding)
	for (int grp = 0; grp < G::G; ++grp) {
		const int line = tid % LG, j0 = tid / LG;
		C *sm = smem + (size_t)grp * G::GROUP_ELEMS;
		auto ld = [&](int ll, int y) -> C { return y < ny ? sm[SI::at(ll, y)] : C{0, 0}; };
		auto st = [&](int ll, int k, C v) { sm[SI::at(ll, k)] = v; };
		cta_fft_h0<T, PY, G::R, LG, SI, true>(sm, g.tw_y, line, j0, ld, st);  // rows ny <= PY/2 .. are zero
	}
	cp_async_wait_group_c<0>();
	__syncthreads();
	// z transforms, tensor multiply, inverse z transforms: one thread per (ky, column)
	for (int item = tid; item < PY * TB; item += G::THREADS) {
		const int col = item % TB, ky = item / TB;
		const int kx = kx0 + col;
		if (kx >= hx) continue;
		C v[3][PZ];
#pragma unroll
		for (int c = 0; c < 3; ++c) {
#pragma unroll
			for (int z = 0; z < H; ++z) v[c][z] = z < nz ? elem((c * NZ + (z < NZ ? z : 0)) * TB + col, ky) : C{0, 0};
			dft_reg_halfzero<T, PZ>(v[c]);
		}
		const bool fy = ky > PY / 2;
		const int kyr = fy ? PY - ky : ky;
		const T sy = fy ? T(-1) : T(1);
		// kz and PZ - kz share the tensor entries (sign of the z-odd components flipped): each
		// reduced entry is read once
#pragma unroll
		for (int kzr = 0; kzr <= H; ++kzr) {
			// the six components of entry (kx, kzr, kyr), contiguous pairs in shared memory
			const T2 *t = tsm + ((col * G::QZ + kzr) * G::QY + kyr) * 3;
			const T2 t0 = t[0], t1 = t[1], t2 = t[2];
			const T nxx = t0.x, nxy = t0.y, nxz = t1.x, nyy = t1.y, nyz = t2.x, nzz = t2.y;
#pragma unroll
			for (int q = 0; q < ((kzr == 0 || kzr == H) ? 1 : 2); ++q) {
				const int p = brev<PZ>(q ? PZ - kzr : kzr);
				const T sz = q ? T(-1) : T(1);
				const T xy = sy * nxy, xz = sz * nxz, yz = sy * sz * nyz;
				const C m0 = v[0][p], m1 = v[1][p], m2 = v[2][p];
				v[0][p] = C{nxx * m0.x + xy * m1.x + xz * m2.x, nxx * m0.y + xy * m1.y + xz * m2.y};
				v[1][p] = C{xy * m0.x + nyy * m1.x + yz * m2.x, xy * m0.y + nyy * m1.y + yz * m2.y};
				v[2][p] = C{xz * m0.x + yz * m1.x + nzz * m2.x, xz * m0.y + yz * m1.y + nzz * m2.y};
			}
		}
#pragma unroll
		for (int c = 0; c < 3; ++c) {
			C w[PZ];
#pragma unroll
			for (int k = 0; k < PZ; ++k) w[k] = v[c][brev<PZ>(k)];  // natural order for the inverse
			dft_reg<T, PZ, true>(w);
#pragma unroll
			for (int z = 0; z < H; ++z)
				if (z < nz && z < NZ) elem((c * NZ + z) * TB + col, ky) = w[brev<PZ>(z)];
		}
	}
	__syncthreads();
	// inverse y transforms, rows y < ny to HBM
	for (int grp = 0; grp < G::G; ++grp) {
		const int line = tid % LG, j0 = tid / LG;
		const int l = grp * LG + line;
		const int col = l % TB, cz = l / TB, c = cz / NZ, z = cz % NZ;
		const int kx = kx0 + col;
		const bool ok = kx < hx && z < nz;
		C *dst = g.spec + ((size_t)(c * nz + (ok ? z : 0)) * g.py) * lx + (ok ? kx : 0);
		C *sm = smem + (size_t)grp * G::GROUP_ELEMS;
		auto ld = [&](int ll, int k) -> C { return sm[SI::at(ll, k)]; };
		auto st = [&](int, int y, C val) {
			if (ok && y < ny) dst[(size_t)y * lx] = val;
		};
		if (grp > 0) __syncthreads();
		cta_fft<T, PY, G::R, LG, true, SI, true>(sm, g.tw_y, line, j0, ld, st);
	}
}

} // namespace

struct ConvGroup {
	int prec = MM_F32;
	int count = 0;
	void *desc = nullptr;  // GDesc<T>[count]
	struct List {
		int pass;     // 0 x forward, 1 y forward, 2 z, 3 y inverse, 4 x inverse, 6 fused y+z (len = py*64+pz)
		int len;      // transform length of the pass
		int variant;  // tile shape chosen by the autotuner (GRP_VARIANTS)
		int2 *items;
		int n;
		int grid;     // persistent grid of variant 3
	};
	std::vector<List> lists;
	CUtensorMap *maps = nullptr;  // [2 member + inverse]: spectrum views of the y passes
	bool maps_ok = false;         // every member's maps exist (variant 3 possible)
	int *err = nullptr;           // set when a staged pass gave up waiting
	bool one_output = false;      // some member has no second output
	// the lists of one phase (independent members) run side by side on these streams
	static constexpr int POOL = 8;
	cudaStream_t pool[POOL] = {};
	cudaEvent_t fork = nullptr, join[POOL] = {};
	~ConvGroup()
	{
		cudaFree(desc);
		cudaFree(maps);
		cudaFree(err);
		for (auto &l : lists) cudaFree(l.items);
		for (auto &q : pool)
			if (q) cudaStreamDestroy(q);
		for (auto &e : join)
			if (e) cudaEventDestroy(e);
		if (fork) cudaEventDestroy(fork);
	}
};

namespace {

// Calls f(std::integral_constant<int, N>, std::integral_constant<int, V>) for a length and a
// variant; variants other than 0 exist for lengths 16..512.
template <typename T, class F>
void with_len_variant(int len, int v, F &&f)
{
	auto go = [&](auto nc) {
		constexpr int N = decltype(nc)::value;
		if constexpr (N >= 16 && N <= 512) {
			if (v == 1) { f(nc, std::integral_constant<int, 1>()); return; }
			if (v == 2) { f(nc, std::integral_constant<int, 2>()); return; }
		}
		f(nc, std::integral_constant<int, 0>());
	};
#define MM_WLV(N) go(std::integral_constant<int, N>())
	MM_FS_SWITCH(len, MM_WLV);
#undef MM_WLV
}

// Calls f(integral_constant PY, integral_constant PZ) for a fused y+z pass key (py * 64 + pz).
template <class F>
void with_yz(int key, F &&f)
{
	const int py = key / 64, pz = key % 64;
	auto by_pz = [&](auto pyc) {
		switch (pz) {
		case 2: f(pyc, std::integral_constant<int, 2>()); break;
		case 4: f(pyc, std::integral_constant<int, 4>()); break;
		case 8: f(pyc, std::integral_constant<int, 8>()); break;
		}
	};
	switch (py) {
	case 16: by_pz(std::integral_constant<int, 16>()); break;
	case 32: by_pz(std::integral_constant<int, 32>()); break;
	case 64: by_pz(std::integral_constant<int, 64>()); break;
	case 128: by_pz(std::integral_constant<int, 128>()); break;
	case 256: by_pz(std::integral_constant<int, 256>()); break;
	case 512: by_pz(std::integral_constant<int, 512>()); break;
	}
}

// Whether a member takes the fused y+z pass (and its columns per CTA).
template <typename T>
int yz_tb_dims(int py, int pz, int nz)
{
	int tb = 0;
	if (py < 16 || py > 512 || (pz != 2 && pz != 4 && pz != 8) || 2 * nz > pz) return 0;
	with_yz(py * 64 + pz, [&](auto pyc, auto pzc) {
		using G = YZGeom<decltype(pyc)::value, decltype(pzc)::value, cplx<T>>;
		if constexpr (G::fits) tb = G::TB;
	});
	return tb;
}
template <typename T>
int yz_tb(const ConvPlan *p)
{
	return yz_tb_dims<T>(p->py, p->pz, p->nz);
}

} // namespace

int conv_group_fused(int prec, int py, int pz, int nz)
{
	return prec == MM_F32 ? yz_tb_dims<float>(py, pz, nz) > 0 : yz_tb_dims<double>(py, pz, nz) > 0;
}

namespace {

// Threads of one CTA of a pass/length/variant (0 when the variant does not exist).
template <typename T>
int group_threads(int pass, int len, int v)
{
	using C = cplx<T>;
	if (pass == 2) return v == 0 ? ZR_THREADS : 0;
	if (pass == 6) {
		int t = 0;
		with_yz(len, [&](auto pyc, auto pzc) {
			constexpr int PY = decltype(pyc)::value, PZ = decltype(pzc)::value;
			using G0 = YZGeom<PY, PZ, C>;
			using G1 = YZGeom<PY, PZ, C, true>;
			if (v == 0 && G0::fits) t = G0::THREADS;
			if (v == 1 && G1::fits && G0::fits && G0::TB > 1) t = G1::THREADS;
		});
		return t;
	}
	if (v == 3) {
		if (pass != 1 && pass != 3) return 0;
		const int tb = ct_tb(len, (int)sizeof(C));
		if (tb * (int)sizeof(C) < 16 || tb * (int)(sizeof(C) / 8) > 256) return 0;
		return tb * (len / ct_radix(len));
	}
	if (v != 0 && (len < 16 || len > 512)) return 0;
	const int csz = (int)sizeof(C);
	const int lines = (pass == 0 || pass == 4) ? var_lpb(len, csz, v) : var_tb(len, csz, v);
	if (v == 1 && lines == ((pass == 0 || pass == 4) ? ct_lpb(len, csz) : ct_tb(len, csz))) return 0;
	const int t = lines * (len / var_radix(len, v));
	return (t >= 32 && t <= 1024 && (v != 2 || var_radix(len, v) != ct_radix(len))) ? t : 0;
}

// Blocks of one member for a pass/length/variant.
template <typename T>
int group_blocks(const ConvPlan *p, int pass, int len, int v)
{
	const int csz = (int)sizeof(cplx<T>);
	if (pass == 0 || pass == 4) {
		const int lpb = var_lpb(len, csz, v);
		return ((3 * p->ny * p->nz + 1) / 2 + lpb - 1) / lpb;
	}
	if (pass == 6) {
		const int tb = v == 1 ? 1 : yz_tb<T>(p);
		return (p->hx + tb - 1) / tb;
	}
	if (pass == 1 || pass == 3) {
		const int tb = var_tb(len, csz, v == 3 ? 0 : v);
		return (p->hx + tb - 1) / tb * 3 * p->nz;
	}
	return (p->hx + 31) / 32 * p->qy;
}

template <typename T>
size_t group_smem_bytes(int pass, int len, int v)
{
	using C = cplx<T>;
	size_t r = 0;
	if (pass == 2) return zr_smem<T>(len);
	if (pass == 6) {
		with_yz(len, [&](auto pyc, auto pzc) {
			constexpr int PY = decltype(pyc)::value, PZ = decltype(pzc)::value;
			r = v == 1 ? YZGeom<PY, PZ, C, true>::SMEM : YZGeom<PY, PZ, C>::SMEM;
		});
		return r;
	}
	if (v == 3) {
		auto y3 = [&](auto nc) {
			constexpr int N = decltype(nc)::value, TB = ct_tb(N, sizeof(C));
			r = pass == 1 ? YTmaGeom<N, TB, false, C>::SMEM : YTmaGeom<N, TB, true, C>::SMEM;
		};
#define MM_Y3(N) y3(std::integral_constant<int, N>())
		MM_FS_SWITCH(len, MM_Y3);
#undef MM_Y3
		return r;
	}
	with_len_variant<T>(len, v, [&](auto nc, auto vc) {
		constexpr int N = decltype(nc)::value, V = decltype(vc)::value;
		constexpr int LPB = var_lpb(N, sizeof(C), V), TB = var_tb(N, sizeof(C), V);
		r = (pass == 0 || pass == 4) ? (size_t)SmRows<N, LPB>::SIZE * sizeof(C) : (size_t)SmCols<N, TB>::SIZE * sizeof(C);
	});
	return r;
}

template <typename T>
mm_status group_smem(int pass, int len, int v)
{
	using C = cplx<T>;
	mm_status r = MM_OK;
	const size_t sm = group_smem_bytes<T>(pass, len, v);
	if (pass == 6) {
		with_yz(len, [&](auto pyc, auto pzc) {
			constexpr int PY = decltype(pyc)::value, PZ = decltype(pzc)::value;
			if (v == 1) {
				if constexpr (YZGeom<PY, PZ, C, true>::fits) r = set_smem<T>((const void *)k_yz_grp<T, PY, PZ, true>, sm);
			} else {
				if constexpr (YZGeom<PY, PZ, C>::fits) r = set_smem<T>((const void *)k_yz_grp<T, PY, PZ>, sm);
			}
		});
		return r;
	}
	if (pass == 2) {
		switch (len) {
		case 2: r = set_smem<T>((const void *)k_z_grp<T, 2>, sm); break;
		case 4: r = set_smem<T>((const void *)k_z_grp<T, 4>, sm); break;
		case 8: r = set_smem<T>((const void *)k_z_grp<T, 8>, sm); break;
		case 16: r = set_smem<T>((const void *)k_z_grp<T, 16>, sm); break;
		case 32: if constexpr (sizeof(T) == 4) { r = set_smem<T>((const void *)k_z_grp<T, 32>, sm); } break;
		}
		return r;
	}
	if (v == 3) {
		auto y3 = [&](auto nc) {
			constexpr int N = decltype(nc)::value;
			r = set_smem<T>(pass == 1 ? (const void *)k_y_tma_grp<T, N, false> : (const void *)k_y_tma_grp<T, N, true>, sm);
		};
#define MM_Y3(N) y3(std::integral_constant<int, N>())
		MM_FS_SWITCH(len, MM_Y3);
#undef MM_Y3
		return r;
	}
	with_len_variant<T>(len, v, [&](auto nc, auto vc) {
		constexpr int N = decltype(nc)::value, V = decltype(vc)::value;
		constexpr int LPB = var_lpb(N, sizeof(C), V), TB = var_tb(N, sizeof(C), V), R = var_radix(N, V);
		if (pass == 0) r = set_smem<T>((const void *)k_x_fwd_grp<T, N, LPB, R>, sm);
		if (pass == 4) r = set_smem<T>((const void *)k_x_inv_grp<T, N, LPB, R>, sm);
		if (pass == 1) r = set_smem<T>((const void *)k_y_grp<T, N, TB, false, R>, sm);
		if (pass == 3) r = set_smem<T>((const void *)k_y_grp<T, N, TB, true, R>, sm);
	});
	return r;
}

template <typename T>
void group_launch_v(const ConvGroup *g, int pass, int len, int v, const int2 *items, int n, int grid, int input,
                    int output, int gate, cudaStream_t st)
{
	using C = cplx<T>;
	const GDesc<T> *d = (const GDesc<T> *)g->desc;
	const size_t sm = group_smem_bytes<T>(pass, len, v);
	if (pass == 6) {
		with_yz(len, [&](auto pyc, auto pzc) {
			constexpr int PY = decltype(pyc)::value, PZ = decltype(pzc)::value;
			using G = YZGeom<PY, PZ, C>;
			using GN = YZGeom<PY, PZ, C, true>;
			if (v == 1) {
				if constexpr (GN::fits) k_yz_grp<T, PY, PZ, true><<<n, GN::THREADS, sm, st>>>(d, items, gate);
			} else {
				if constexpr (G::fits) k_yz_grp<T, PY, PZ><<<n, G::THREADS, sm, st>>>(d, items, gate);
			}
		});
		return;
	}
	if (v == 3) {
		auto y3 = [&](auto nc) {
			constexpr int N = decltype(nc)::value, TB = ct_tb(N, sizeof(C));
			const int threads = TB * (N / ct_radix(N));
			const int gr = grid < n ? grid : n;
			if (pass == 1) k_y_tma_grp<T, N, false><<<gr, threads, sm, st>>>(d, g->maps, items, n, gate, g->err);
			else k_y_tma_grp<T, N, true><<<gr, threads, sm, st>>>(d, g->maps, items, n, gate, g->err);
		};
#define MM_Y3(N) y3(std::integral_constant<int, N>())
		MM_FS_SWITCH(len, MM_Y3);
#undef MM_Y3
		return;
	}
	if (pass == 2) {
		switch (len) {
		case 2: k_z_grp<T, 2><<<n, ZR_THREADS, sm, st>>>(d, items, gate); break;
		case 4: k_z_grp<T, 4><<<n, ZR_THREADS, sm, st>>>(d, items, gate); break;
		case 8: k_z_grp<T, 8><<<n, ZR_THREADS, sm, st>>>(d, items, gate); break;
		case 16: k_z_grp<T, 16><<<n, ZR_THREADS, sm, st>>>(d, items, gate); break;
		case 32: if constexpr (sizeof(T) == 4) { k_z_grp<T, 32><<<n, ZR_THREADS, sm, st>>>(d, items, gate); } break;
		}
		return;
	}
	with_len_variant<T>(len, v, [&](auto nc, auto vc) {
		constexpr int N = decltype(nc)::value, V = decltype(vc)::value;
		constexpr int LPB = var_lpb(N, sizeof(C), V), TB = var_tb(N, sizeof(C), V), R = var_radix(N, V);
		constexpr int TPL = N / R;
		if (pass == 0) k_x_fwd_grp<T, N, LPB, R><<<n, LPB * TPL, sm, st>>>(d, items, input, gate);
		if (pass == 4) k_x_inv_grp<T, N, LPB, R><<<n, LPB * TPL, sm, st>>>(d, items, output, gate);
		if (pass == 1) k_y_grp<T, N, TB, false, R><<<n, TB * TPL, sm, st>>>(d, items, gate);
		if (pass == 3) k_y_grp<T, N, TB, true, R><<<n, TB * TPL, sm, st>>>(d, items, gate);
	});
}

template <typename T>
void group_launch(const ConvGroup *g, const ConvGroup::List &l, int input, int output, int gate, cudaStream_t st)
{
	group_launch_v<T>(g, l.pass, l.len, l.variant, l.items, l.n, l.grid, input, output, gate, st);
}

// Persistent grid of the TMA-staged grouped y pass (resident CTAs on the whole device).
template <typename T>
int group_grid(int pass, int len)
{
	using C = cplx<T>;
	int occ = 0;
	auto y3 = [&](auto nc) {
		constexpr int N = decltype(nc)::value, TB = ct_tb(N, sizeof(C));
		const int threads = TB * (N / ct_radix(N));
		const size_t sm = group_smem_bytes<T>(pass, N, 3);
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pass == 1 ? (const void *)k_y_tma_grp<T, N, false>
		                                                                  : (const void *)k_y_tma_grp<T, N, true>,
		                                                  threads, sm) != cudaSuccess)
			cudaGetLastError();
	};
#define MM_Y3(N) y3(std::integral_constant<int, N>())
	MM_FS_SWITCH(len, MM_Y3);
#undef MM_Y3
	return (occ > 0 ? occ : 1) * num_sms();
}

// The autotuner's choices, per precision, pass and length, for the process (tuned once, on the
// first group that uses a pass and length, by timing every variant on that group's members).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tuned;

template <typename T>
std::vector<int2> group_items(const ConvGroupMember *m, const std::vector<int> &mem, int pass, int len, int v)
{
	std::vector<int2> items;
	for (int i : mem) {
		const int nb = group_blocks<T>(m[i].plan, pass, len, v);
		for (int b = 0; b < nb; ++b) items.push_back(make_int2(i, b));
	}
	return items;
}

// Times every variant of one pass and length on the group's members (run flags ignored) and
// returns the fastest.
template <typename T>
mm_status group_tune(const ConvGroup *g, const ConvGroupMember *m, const std::vector<int> &mem, int pass, int len,
                     cudaStream_t st, int *best)
{
	*best = 0;
	float best_ms = 0.f;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	MM_CUDA(cudaEventCreate(&e0));
	MM_CUDA(cudaEventCreate(&e1));
	mm_status r = MM_OK;
	for (int v = 0; v < GRP_VARIANTS && r == MM_OK; ++v) {
		if (!group_threads<T>(pass, len, v) || group_smem_bytes<T>(pass, len, v) > 227 * 1024) continue;
		if (v == 3 && !g->maps_ok) continue;
		const int grid = v == 3 ? group_grid<T>(pass, len) : 0;
		const std::vector<int2> items = group_items<T>(m, mem, pass, len, v);
		int2 *di = nullptr;
		r = cuda_status(cudaMalloc(&di, sizeof(int2) * items.size()), "cudaMalloc");
		if (r == MM_OK) r = cuda_status(cudaMemcpyAsync(di, items.data(), sizeof(int2) * items.size(),
		                                                cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
		if (r == MM_OK) r = group_smem<T>(pass, len, v);
		if (r == MM_OK) {
			group_launch_v<T>(g, pass, len, v, di, (int)items.size(), grid, 0, 0, 0, st);  // warm-up
			cudaEventRecord(e0, st);
			for (int k = 0; k < 3; ++k) group_launch_v<T>(g, pass, len, v, di, (int)items.size(), grid, 0, 0, 0, st);
			cudaEventRecord(e1, st);
			r = cuda_status(cudaEventSynchronize(e1), "autotune launch");
		}
		float ms = 0.f;
		if (r == MM_OK) r = cuda_status(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
		if (r == MM_OK && (v == 0 || ms < best_ms)) {
			best_ms = ms;
			*best = v;
		}
		cudaFree(di);
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	return r;
}

template <typename T>
mm_status group_create(ConvGroup *g, const ConvGroupMember *m, int count, cudaStream_t st)
{
	std::vector<GDesc<T>> h(count);
	std::map<std::pair<int, int>, std::vector<int>> lists;  // (pass, length) -> members
	for (int i = 0; i < count; ++i) {
		ConvPlan *p = m[i].plan;
		if (!p || p->prec != g->prec || p->is2d || !p->fast_x || !p->fast_y || !p->reg_z)
			return fail(MM_ERR_UNSUPPORTED, "conv group: every member needs power-of-two 3-D padding with a register z pass");
		if (2 * p->nx > p->px || 2 * p->ny > p->py || 2 * p->nz > p->pz)
			return fail(MM_ERR_UNSUPPORTED, "conv group: every member needs zero padding to at least twice its size");
		GDesc<T> &d = h[i];
		d.spec = (cplx<T> *)p->spec;
		d.tensor = (const T *)p->tensor;
		d.tw_x = (const cplx<T> *)p->tw_x;
		d.tw_y = (const cplx<T> *)p->tw_y;
		for (int k = 0; k < 4; ++k) d.M[k] = (const T *)m[i].M[k];
		for (int k = 0; k < 2; ++k) d.H[k] = (T *)m[i].H[k];
		if (!d.H[1]) g->one_output = true;
		d.reg = m[i].reg;
		d.ms_tab = (const T *)m[i].ms_tab;
		d.flags = nullptr;  // the autotuner runs every member; the real flags are set below
		if (!d.reg || !d.ms_tab || !d.H[0]) return fail(MM_ERR_INVALID_ARGUMENT, "conv group: member without regions or output");
		d.nx = p->nx; d.ny = p->ny; d.nz = p->nz; d.py = p->py; d.hx = p->hx; d.lx = p->lx; d.qy = p->qy; d.qz = p->qz;
		d.tensor_t = nullptr;
		lists[{0, p->px}].push_back(i);
		if (yz_tb<T>(p) > 0) {
			lists[{6, p->py * 64 + p->pz}].push_back(i);  // y, z and the multiply in one pass
			// the fused pass reads the tensor by (kx, kz, ky) with its six components together;
			// the plan keeps that copy, so regrouping (members joining or leaving) allocates nothing
			if (!p->tensor_kx) {
				const size_t ne = (size_t)6 * p->hx * p->qy * p->qz;
				MM_CUDA(cudaMalloc(&p->tensor_kx, ne * sizeof(T)));
				k_tensor_kx<T><<<(unsigned)((ne + 255) / 256), 256, 0, st>>>((const T *)p->tensor, (T *)p->tensor_kx,
				                                                               p->hx, p->qy, p->qz);
				MM_CUDA(cudaGetLastError());
			}
			d.tensor_t = (const T *)p->tensor_kx;
		} else {
			lists[{1, p->py}].push_back(i);
			lists[{2, p->pz}].push_back(i);
			lists[{3, p->py}].push_back(i);
		}
		lists[{4, p->px}].push_back(i);
	}
	MM_CUDA(cudaMalloc(&g->desc, sizeof(GDesc<T>) * count));
	MM_CUDA(cudaMemcpyAsync(g->desc, h.data(), sizeof(GDesc<T>) * count, cudaMemcpyHostToDevice, st));
	// tensor maps of the TMA-staged y passes (variant 3): every member's spectrum, forward view of
	// its ny data rows (zero fill to N/2), inverse view of all py rows
	{
		std::vector<CUtensorMap> maps(2 * (size_t)count);
		bool ok = true;
		for (int i = 0; i < count && ok; ++i) {
			const ConvPlan *p = m[i].plan;
			const int E = (int)(sizeof(cplx<T>) / 8), tb = ct_tb(p->py, (int)sizeof(cplx<T>));
			if (2 * p->ny > p->py || tb * (int)sizeof(cplx<T>) < 16 || tb * E > 256) { ok = false; break; }
			const int rows_f = p->py / 2, rows_i = p->py;
			const uint64_t d0 = (uint64_t)p->lx * E, rowb = (uint64_t)p->lx * sizeof(cplx<T>), planeb = rowb * p->py;
			ok = tma_encode_3d(&maps[2 * i], p->spec, d0, (uint64_t)p->ny, 3ull * p->nz, rowb, planeb, tb * E,
			                   rows_f < 256 ? rows_f : 256, 1) == MM_OK &&
			     tma_encode_3d(&maps[2 * i + 1], p->spec, d0, (uint64_t)p->py, 3ull * p->nz, rowb, planeb, tb * E,
			                   rows_i < 256 ? rows_i : 256, 1) == MM_OK;
		}
		if (ok) {
			MM_CUDA(cudaMalloc(&g->maps, sizeof(CUtensorMap) * maps.size()));
			MM_CUDA(cudaMemcpyAsync(g->maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice, st));
			MM_CUDA(cudaMalloc(&g->err, sizeof(int)));
			MM_CUDA(cudaMemsetAsync(g->err, 0, sizeof(int), st));
			g->maps_ok = true;
		} else {
			clear_error();
		}
	}
	for (const auto &kv : lists) {
		const int pass = kv.first.first, len = kv.first.second;
		int v = 0;
		bool known = false;
		{
			std::lock_guard<std::mutex> lock(g_tune_mu);
			auto it = g_tuned.find(std::make_tuple(g->prec, pass, len));
			if (it != g_tuned.end()) { v = it->second; known = true; }
		}
		// MMB200_GROUP_VARIANT=0|1|2 fixes the variant (where it exists) instead of timing them
		if (const char *fv = std::getenv("MMB200_GROUP_VARIANT")) {
			const int f = std::atoi(fv);
			v = (f >= 0 && f < GRP_VARIANTS && group_threads<T>(pass, len, f)) ? f : 0;
			known = true;
		}
		if (pass == 6) {
			// the narrow tiles when the default ones would not fill the device twice over
			int blocks = 0;
			for (int i : kv.second) blocks += group_blocks<T>(m[i].plan, 6, len, 0);
			known = true;
			v = blocks < 2 * num_sms() && group_threads<T>(6, len, 1) > 0 ? 1 : 0;
		}
		if (!known) {
			MM_TRY(group_tune<T>(g, m, kv.second, pass, len, st, &v));
			std::lock_guard<std::mutex> lock(g_tune_mu);
			g_tuned[std::make_tuple(g->prec, pass, len)] = v;
		}
		const std::vector<int2> items = group_items<T>(m, kv.second, pass, len, v);
		if (v == 3 && !g->maps_ok) v = 0;
		ConvGroup::List l{pass, len, v, nullptr, (int)items.size(), v == 3 ? group_grid<T>(pass, len) : 0};
		MM_CUDA(cudaMalloc(&l.items, sizeof(int2) * l.n));
		MM_CUDA(cudaMemcpyAsync(l.items, items.data(), sizeof(int2) * l.n, cudaMemcpyHostToDevice, st));
		MM_TRY(group_smem<T>(pass, len, v));
		g->lists.push_back(l);
	}
	// lists in pass order (x forward, y forward, z, y inverse, x inverse)
	auto rank = [](int pass) { return pass == 6 ? 1 : (pass >= 1 ? pass + 1 : pass); };
	std::stable_sort(g->lists.begin(), g->lists.end(),
	                 [&](const ConvGroup::List &a, const ConvGroup::List &b) { return rank(a.pass) < rank(b.pass); });
	for (int i = 0; i < count; ++i) h[i].flags = m[i].flags;
	MM_CUDA(cudaMemcpyAsync(g->desc, h.data(), sizeof(GDesc<T>) * count, cudaMemcpyHostToDevice, st));
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

} // namespace

mm_status conv_group_create(ConvGroup **out, const ConvGroupMember *members, int count, cudaStream_t st)
{
	if (!out || !members || count < 1) return fail(MM_ERR_INVALID_ARGUMENT, "conv group: no members");
	ConvGroup *g = new ConvGroup();
	g->prec = members[0].plan ? members[0].plan->prec : MM_F32;
	g->count = count;
	mm_status rs = cuda_status(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming), "cudaEventCreate");
	for (int q = 0; q < ConvGroup::POOL && rs == MM_OK; ++q) {
		rs = cuda_status(cudaStreamCreateWithFlags(&g->pool[q], cudaStreamNonBlocking), "cudaStreamCreate");
		if (rs == MM_OK) rs = cuda_status(cudaEventCreateWithFlags(&g->join[q], cudaEventDisableTiming), "cudaEventCreate");
	}
	if (rs != MM_OK) {
		delete g;
		return rs;
	}
	const mm_status r = g->prec == MM_F64 ? group_create<double>(g, members, count, st)
	                                       : group_create<float>(g, members, count, st);
	if (r != MM_OK) {
		delete g;
		return r;
	}
	*out = g;
	return MM_OK;
}

// The lists of one phase (x forward; y forward and fused y+z; z; y inverse; x inverse) touch
// disjoint members, so each phase forks onto the group's stream pool and joins back on `st`
// (inside a stream capture this becomes parallel graph branches).
mm_status conv_group_execute(ConvGroup *g, int input, int gate, cudaStream_t st, int output)
{
	if (!g || input < 0 || input > 3) return fail(MM_ERR_INVALID_ARGUMENT, "conv group: bad input selector");
	if (output < 0 || output > 1 || (output == 1 && g->one_output))
		return fail(MM_ERR_INVALID_ARGUMENT, "conv group: bad output selector");
	auto rank = [](int pass) { return pass == 6 ? 1 : pass; };
	size_t i = 0;
	while (i < g->lists.size()) {
		size_t j = i;
		while (j < g->lists.size() && rank(g->lists[j].pass) == rank(g->lists[i].pass)) ++j;
		const int n = (int)(j - i);
		if (n == 1) {
			if (g->prec == MM_F64) group_launch<double>(g, g->lists[i], input, output, gate, st);
			else group_launch<float>(g, g->lists[i], input, output, gate, st);
			MM_TRY(after_launch("k_conv_grp"));
		} else {
			MM_CUDA(cudaEventRecord(g->fork, st));
			const int used = n < ConvGroup::POOL ? n : ConvGroup::POOL;
			for (int q = 0; q < used; ++q) MM_CUDA(cudaStreamWaitEvent(g->pool[q], g->fork, 0));
			for (size_t k = i; k < j; ++k) {
				cudaStream_t sq = g->pool[(k - i) % ConvGroup::POOL];
				if (g->prec == MM_F64) group_launch<double>(g, g->lists[k], input, output, gate, sq);
				else group_launch<float>(g, g->lists[k], input, output, gate, sq);
				MM_TRY(after_launch("k_conv_grp"));
			}
			for (int q = 0; q < used; ++q) {
				MM_CUDA(cudaEventRecord(g->join[q], g->pool[q]));
				MM_CUDA(cudaStreamWaitEvent(st, g->join[q], 0));
			}
		}
		i = j;
	}
	return MM_OK;
}

int conv_group_launches(const ConvGroup *g) { return g ? (int)g->lists.size() : 0; }

void conv_group_destroy(ConvGroup *g) { delete g; }

} // namespace mm

struct mm_conv {
	mm::ConvPlan *plan;
};

using namespace mm;

extern "C" {

MM_API mm_status mm_conv_create(mm_conv **out, int prec, int nx, int ny, int nz, int ex, int ey,
                                int ez, const double *N_device, void *stream)
{
	if (!out) return fail(MM_ERR_INVALID_ARGUMENT, "mm_conv_create: null out");
	ConvPlan *p = nullptr;
	MM_TRY(conv_plan_create(&p, prec, nx, ny, nz, ex, ey, ez, N_device, as_stream(stream)));
	*out = new mm_conv{p};
	return MM_OK;
}

MM_API mm_status mm_conv_execute(mm_conv *conv, const void *M, void *H, void *stream)
{
	if (!conv || !conv->plan || !M || !H) return fail(MM_ERR_INVALID_ARGUMENT, "mm_conv_execute: null argument");
	return conv_execute(conv->plan, M, nullptr, nullptr, H, as_stream(stream));
}

MM_API mm_status mm_conv_destroy(mm_conv *conv)
{
	if (conv) {
		delete conv->plan;
		delete conv;
	}
	return MM_OK;
}

} // extern "C"
