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

// Radix-2 DIF stages of span SPAN0, SPAN0/2, ..., 1 over v[0..N) (the full DFT has SPAN0 = N/2).
template <typename T, int N, bool INV, int SPAN0>
__device__ __forceinline__ void dif_stages(cplx<T> (&v)[N])
{
	using C = cplx<T>;
#pragma unroll
	for (int span = SPAN0; span >= 1; span >>= 1) {
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

template <typename T, int N, bool INV>
__device__ __forceinline__ void dft_reg(cplx<T> (&v)[N])
{
	dif_stages<T, N, INV, N / 2>(v);
}

// Forward DFT of a column whose upper half v[N/2..N) is zero padding: the first DIF stage reduces
// to v[j + N/2] = v[j] W_N^j.  Output in bit-reversed order, like dft_reg.
template <typename T, int N>
__device__ __forceinline__ void dft_reg_halfzero(cplx<T> (&v)[N])
{
	if constexpr (N >= 2) {
#pragma unroll
		for (int j = 0; j < N / 2; ++j) {
			const int q = j * (64 / N);
			if (q == 0) v[j + N / 2] = v[j];
			else if (q == 16) v[j + N / 2] = mul_mi<false>(v[j]);
			else v[j + N / 2] = cmul(v[j], w64<T>(q));
		}
		dif_stages<T, N, false, N / 4>(v);
	}
}

} // namespace mm

namespace mm {

// ---- CTA-wide Stockham FFT with compile-time length and radix -----------------------------------
// LANES independent lines of length N live in shared memory; each of the N/R threads of a line
// performs R/Rp radix-Rp butterflies per pass (Rp = R except possibly a smaller last pass).  Pass 0
// reads its inputs through `ld(line, k)` (global memory, with zero padding), the last pass hands
// its outputs to `st(line, k, value)`; intermediate passes go through shared memory at
// `SmIdx::at(line, k)`.  All strides are compile-time powers of two.
__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }
__host__ __device__ constexpr int fft_npasses(int N, int R) { return (ilog2c(N) + ilog2c(R) - 1) / ilog2c(R); }
__host__ __device__ constexpr int fft_radix(int N, int R, int p)
{
	return ilog2c(N) - p * ilog2c(R) >= ilog2c(R) ? R : (1 << (ilog2c(N) - p * ilog2c(R)));
}

// Shared-memory layouts.  One padding slot per 2^SH elements skews the Stockham pass-0 writes
// (stride R) and the column tiles across the banks.  SH = 4 makes the radix-16 pass-0 writes of
// 8-byte elements conflict-free (consecutive butterflies 17 elements = 34 words apart, so a
// half-warp's 16 stores cover all 32 banks once); SH = 5 halves the padding.
template <int SH = 5>
__host__ __device__ constexpr int sm_pad(int raw) { return raw + (raw >> SH); }
template <int N, int LANES, int SH = 5>
struct SmCols {  // element (line, k) at k * LANES + line: lines are adjacent columns
	static constexpr int SIZE = N * LANES + (N * LANES >> SH) + 1;
	__device__ __forceinline__ static int at(int line, int k) { return sm_pad<SH>(k * LANES + line); }
};
template <int N, int LANES, int SH = 5>
struct SmRows {  // element (line, k) at line * N + k
	static constexpr int SIZE = N * LANES + (N * LANES >> SH) + 1;
	__device__ __forceinline__ static int at(int line, int k) { return sm_pad<SH>(line * N + k); }
};

// Hook run by every thread after pass 0 has stored its outputs (a no-op unless a kernel stages
// its inputs and can release their buffer once pass 0 has read them).
struct NoHook {
	__device__ __forceinline__ void operator()() const {}
};

// H0: the inputs at k >= N/2 are zero (a forward transform of zero-padded data), so pass 0 loads
// only the lower half of each butterfly's inputs and runs the half-zero register DFT.
template <typename T, int N, int R, int LANES, bool INV, class SmIdx, bool LD_SM, int p, bool H0, class LD,
          class ST, class HK = NoHook>
__device__ __forceinline__ void cta_fft_pass(cplx<T> *sm, const cplx<T> *__restrict__ twN, int line, int j0,
                                             LD &ld, ST &st, HK hk = HK())
{
	using C = cplx<T>;
	constexpr int P = fft_npasses(N, R);
	constexpr int Rp = fft_radix(N, R, p);
	constexpr int Ns = 1 << (p * ilog2c(R));  // product of the radices of earlier passes
	constexpr int TPL = N / R;
	constexpr int BPT = R / Rp;
	constexpr int M = N / Rp;                  // butterflies per line, input stride
	constexpr bool HALF = H0 && p == 0;
	static_assert(!HALF || (!INV && BPT == 1 && Rp >= 2), "half-zero pass 0: forward, one butterfly per thread");
	C v[BPT][Rp];
	if constexpr (p > 0) __syncthreads();
#pragma unroll
	for (int u = 0; u < BPT; ++u) {
		const int j = j0 + u * TPL;
#pragma unroll
		for (int q = 0; q < (HALF ? Rp / 2 : Rp); ++q) {
			if constexpr (p == 0) v[u][q] = ld(line, j + q * M);
			else v[u][q] = sm[SmIdx::at(line, j + q * M)];
		}
	}
	if constexpr (p > 0 || LD_SM) __syncthreads();  // all inputs read before any output lands
#pragma unroll
	for (int u = 0; u < BPT; ++u) {
		const int j = j0 + u * TPL;
		const int jm = j & (Ns - 1);
		if constexpr (Ns > 1) {
			if (jm != 0) {
#pragma unroll
				for (int q = 1; q < Rp; ++q) {
					C w = twN[q * jm * (N / (Ns * Rp))];
					if (INV) w = conjc(w);
					v[u][q] = cmul(v[u][q], w);
				}
			}
		}
		if constexpr (HALF) dft_reg_halfzero<T, Rp>(v[u]);
		else dft_reg<T, Rp, INV>(v[u]);
		const int base = (j / Ns) * Ns * Rp + jm;
#pragma unroll
		for (int k = 0; k < Rp; ++k) {
			const C val = v[u][brev<Rp>(k)];
			if constexpr (p == P - 1) st(line, base + k * Ns, val);
			else sm[SmIdx::at(line, base + k * Ns)] = val;
		}
	}
	if constexpr (p == 0) hk();
	if constexpr (p + 1 < P)
		cta_fft_pass<T, N, R, LANES, INV, SmIdx, LD_SM, p + 1, false>(sm, twN, line, j0, ld, st, hk);
}

// LD_SM: the loader reads the same shared memory the passes write (adds a barrier after pass 0's
// reads).
template <typename T, int N, int R, int LANES, bool INV, class SmIdx, bool LD_SM = false, class LD, class ST,
          class HK = NoHook>
__device__ __forceinline__ void cta_fft(cplx<T> *sm, const cplx<T> *__restrict__ twN, int line, int j0, LD &ld,
                                        ST &st, HK hk = HK())
{
	cta_fft_pass<T, N, R, LANES, INV, SmIdx, LD_SM, 0, false>(sm, twN, line, j0, ld, st, hk);
}

// Forward transform whose inputs at k >= N/2 are zero (ld is not called for them).
template <typename T, int N, int R, int LANES, class SmIdx, bool LD_SM = false, class LD, class ST,
          class HK = NoHook>
__device__ __forceinline__ void cta_fft_h0(cplx<T> *sm, const cplx<T> *__restrict__ twN, int line, int j0, LD &ld,
                                           ST &st, HK hk = HK())
{
	cta_fft_pass<T, N, R, LANES, false, SmIdx, LD_SM, 0, true>(sm, twN, line, j0, ld, st, hk);
}

} // namespace mm
