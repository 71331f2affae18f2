// Shared-memory batched 1-D FFT for the demag convolution (project-written; no cuFFT).
//
// Algorithm: Stockham auto-sort FFT (Stockham 1966; formulation of Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC'08), mixed radix
// 2/3/4/5/7/8 plus a direct O(p^2) pass for any other prime factor p.  A CTA transforms a set of
// lines that live in shared memory; element (line b, index k) sits at base[b*sb + k*sk].  Each
// pass reads one buffer and writes the other (ping-pong), so a transform of s passes ends in
// buf[s & 1].
//
// Twiddles come from a table tw[k] = exp(-2 pi i k / n), k < n, computed on the host in long
// double and rounded once; the inverse transform uses the conjugates.  Transforms are
// unnormalised in both directions (the 1/(px*py*pz) factor lives in the tensor spectrum, as in
// the reference's TensorFieldSetup.cpp:58-74).
#pragma once

#include <cuda_runtime.h>
#include <type_traits>

namespace mm {

template <typename T>
using cplx = typename std::conditional<sizeof(T) == 8, double2, float2>::type;

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return {a.x + b.x, a.y + b.y}; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return {a.x - b.x, a.y - b.y}; }
template <typename C>
__device__ __forceinline__ C conjc(C a) { return {a.x, -a.y}; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C>
__device__ __forceinline__ C mul_mi(C a)
{
	if (INV) return {-a.y, a.x};
	return {a.y, -a.x};
}

constexpr int FFT_MAX_PASSES = 24;

// Factorisation of one transform length: radices applied in order.
struct FftRadices {
	int n;
	int count;
	int r[FFT_MAX_PASSES];
};

// In-register DFT of size R for R in {2, 4, 8}; w8 = exp(-2 pi i / 8) from the table.
template <int R, bool INV, typename C>
__device__ __forceinline__ void dft_pow2(C *v, C w8)
{
	if constexpr (R == 2) {
		const C a = v[0], b = v[1];
		v[0] = cadd(a, b);
		v[1] = csub(a, b);
	} else if constexpr (R == 4) {
		const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
		const C t2 = cadd(v[1], v[3]), t3 = mul_mi<INV>(csub(v[1], v[3]));
		v[0] = cadd(t0, t2);
		v[2] = csub(t0, t2);
		v[1] = cadd(t1, t3);
		v[3] = csub(t1, t3);
	} else {  // R == 8: two radix-4 DFTs on even/odd samples, then a radix-2 combination
		C e[4] = {v[0], v[2], v[4], v[6]};
		C o[4] = {v[1], v[3], v[5], v[7]};
		dft_pow2<4, INV>(e, w8);
		dft_pow2<4, INV>(o, w8);
		const C w1 = INV ? conjc(w8) : w8;             // exp(-+2 pi i / 8)
		const C w3 = {-w1.x, w1.y};                    // exp(-+2 pi i 3/8)
		o[1] = cmul(o[1], w1);
		o[2] = mul_mi<INV>(o[2]);
		o[3] = cmul(o[3], w3);
#pragma unroll
		for (int k = 0; k < 4; ++k) {
			v[k] = cadd(e[k], o[k]);
			v[k + 4] = csub(e[k], o[k]);
		}
	}
}

// One Stockham pass of radix R (R in {2,3,4,5,7,8}).
template <typename T, int R, bool INV>
__device__ __forceinline__ void fft_pass(const cplx<T> *__restrict__ src, cplx<T> *__restrict__ dst,
                                         int sb, int sk, int nlines, int n, int Ns,
                                         const cplx<T> *__restrict__ tw, int tid, int nthr)
{
	using C = cplx<T>;
	const int m = n / R;
	const int total = m * nlines;
	const int tstride = n / (Ns * R);
	const bool kfast = (sk == 1);
	for (int it = tid; it < total; it += nthr) {
		int b, j;
		if (kfast) { j = it % m; b = it / m; }
		else { b = it % nlines; j = it / nlines; }
		const C *s = src + b * sb;
		C v[R];
#pragma unroll
		for (int r = 0; r < R; ++r) v[r] = s[(j + r * m) * sk];
		const int jm = j % Ns;
		if (jm != 0) {
			const int t = jm * tstride;
#pragma unroll
			for (int r = 1; r < R; ++r) {
				C w = tw[r * t];
				if (INV) w = conjc(w);
				v[r] = cmul(v[r], w);
			}
		}
		if constexpr (R == 2 || R == 4 || R == 8) {
			dft_pow2<R, INV>(v, tw[n / 8 > 0 && (n % 8) == 0 ? n / 8 : 0]);
		} else {
			// small odd prime: X_k = sum_r v_r W_R^{rk}, W_R^q = tw[q n/R]
			C x[R];
			const int step = n / R;
#pragma unroll
			for (int k = 0; k < R; ++k) {
				C acc = v[0];
#pragma unroll
				for (int r = 1; r < R; ++r) {
					C w = tw[((r * k) % R) * step];
					if (INV) w = conjc(w);
					acc = cadd(acc, cmul(v[r], w));
				}
				x[k] = acc;
			}
#pragma unroll
			for (int k = 0; k < R; ++k) v[k] = x[k];
		}
		const int base = (j / Ns) * Ns * R + jm;
		C *d = dst + b * sb;
#pragma unroll
		for (int r = 0; r < R; ++r) d[(base + r * Ns) * sk] = v[r];
	}
}

// Direct pass for a prime factor p not covered above (O(p^2) per butterfly group).
template <typename T, bool INV>
__device__ void fft_pass_generic(const cplx<T> *__restrict__ src, cplx<T> *__restrict__ dst,
                                 int sb, int sk, int nlines, int n, int Ns, int p,
                                 const cplx<T> *__restrict__ tw, int tid, int nthr)
{
	using C = cplx<T>;
	const int m = n / p;
	const int total = m * nlines;
	const int tstride = n / (Ns * p);
	const bool kfast = (sk == 1);
	for (int it = tid; it < total; it += nthr) {
		int b, j;
		if (kfast) { j = it % m; b = it / m; }
		else { b = it % nlines; j = it / nlines; }
		const C *s = src + b * sb;
		const int jm = j % Ns;
		const int base = (j / Ns) * Ns * p + jm;
		C *d = dst + b * sb;
		for (int k = 0; k < p; ++k) {
			C acc = {0, 0};
			for (int r = 0; r < p; ++r) {
				C v = s[(j + r * m) * sk];
				C w1 = tw[r * jm * tstride];
				C w2 = tw[((r * k) % p) * m];
				if (INV) { w1 = conjc(w1); w2 = conjc(w2); }
				acc = cadd(acc, cmul(cmul(v, w1), w2));
			}
			d[(base + k * Ns) * sk] = acc;
		}
	}
}

// Full transform of `nlines` lines of length rad.n held in buf0.  Returns the buffer that holds
// the result.  Must be called by all threads of the CTA (contains __syncthreads).
template <typename T, bool INV>
__device__ cplx<T> *fft_lines(cplx<T> *buf0, cplx<T> *buf1, int sb, int sk, int nlines,
                              const FftRadices &rad, const cplx<T> *tw)
{
	const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
	const int nthr = blockDim.x * blockDim.y * blockDim.z;
	cplx<T> *src = buf0, *dst = buf1;
	int Ns = 1;
	for (int p = 0; p < rad.count; ++p) {
		const int R = rad.r[p];
		switch (R) {
		case 2: fft_pass<T, 2, INV>(src, dst, sb, sk, nlines, rad.n, Ns, tw, tid, nthr); break;
		case 3: fft_pass<T, 3, INV>(src, dst, sb, sk, nlines, rad.n, Ns, tw, tid, nthr); break;
		case 4: fft_pass<T, 4, INV>(src, dst, sb, sk, nlines, rad.n, Ns, tw, tid, nthr); break;
		case 5: fft_pass<T, 5, INV>(src, dst, sb, sk, nlines, rad.n, Ns, tw, tid, nthr); break;
		case 7: fft_pass<T, 7, INV>(src, dst, sb, sk, nlines, rad.n, Ns, tw, tid, nthr); break;
		case 8: fft_pass<T, 8, INV>(src, dst, sb, sk, nlines, rad.n, Ns, tw, tid, nthr); break;
		default: fft_pass_generic<T, INV>(src, dst, sb, sk, nlines, rad.n, Ns, R, tw, tid, nthr); break;
		}
		__syncthreads();
		Ns *= R;
		cplx<T> *t = src; src = dst; dst = t;
	}
	return src;
}

} // namespace mm
