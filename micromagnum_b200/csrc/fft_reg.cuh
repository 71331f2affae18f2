// Register-resident FFT building blocks for power-of-two lengths (included by conv.cu only).
//
// dft_reg<T, N, INV>: an N-point DFT (N = 1..64) held entirely in one thread's registers,
// radix-2 decimation in frequency, fully unrolled, output in bit-reversed order (read it with
// brev<N>(k)).  Its twiddles W_64^q = exp(-2 pi i q / 64) live in a __constant__ table that every
// lane reads at the same compile-time index (a broadcast).
//
// Longer transforms (N = N1 * N2 <= 4096) use the four-step decomposition within a CTA:
//   X[f1 + N1 f2] = sum_t W_N2^(t f2) W_N^(t f1) sum_k x[t + N2 k] W_N1^(k f1)
// i.e. N2 threads each do an N1-point register DFT, multiply by W_N^(t f1), exchange through
// shared memory once, and finish with N2-point register DFTs.  No index arithmetic depends on
// runtime values except the tile offsets, so the inner work is straight-line code.
#pragma once

#include "fft.cuh"

namespace mm {

static __constant__ double2 c_w64d[64];
static __constant__ float2 c_w64f[64];

template <typename T>
__device__ __forceinline__ cplx<T> w64(int q);
template <>
__device__ __forceinline__ double2 w64<double>(int q) { return c_w64d[q]; }
template <>
__device__ __forceinline__ float2 w64<float>(int q) { return c_w64f[q]; }

// Uploads the W_64 table to the current device (idempotent).
mm_status fft_reg_init();

__host__ __device__ constexpr int brev_c(int k, int n)
{
	int r = 0;
	for (int m = n >> 1; m > 0; m >>= 1, k >>= 1) r = (r << 1) | (k & 1);
	return r;
}

template <int N>
__device__ __forceinline__ int brev(int k) { return brev_c(k, N); }

template <typename T, int N, bool INV>
__device__ __forceinline__ void dft_reg(cplx<T> (&v)[N])
{
	using C = cplx<T>;
#pragma unroll
	for (int span = N / 2; span >= 1; span >>= 1) {
#pragma unroll
		for (int b = 0; b < N; b += 2 * span) {
#pragma unroll
			for (int j = 0; j < span; ++j) {
				const C a = v[b + j], c = v[b + j + span];
				v[b + j] = cadd(a, c);
				C d = csub(a, c);
				const int q = j * (64 / (2 * span));  // W_{2 span}^j = W_64^q
				if (q == 16) {
					d = mul_mi<INV>(d);
				} else if (q != 0) {
					C w = w64<T>(q);
					if (INV) w = conjc(w);
					d = cmul(d, w);
				}
				v[b + j + span] = d;
			}
		}
	}
}

} // namespace mm
