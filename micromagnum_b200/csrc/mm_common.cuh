// Shared helpers for the mmb200 CUDA library: status/error plumbing, physical constants,
// small vector algebra, launch accounting.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <atomic>
#include <mutex>

#include "../../include/mmb200.h"

namespace mm {

// ---- physical constants: the reference's values (src/magneto/mmm/constants.h) ----------------
constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double MU0 = 4.0 * PI * 1e-7;
constexpr double ELECTRON_CHARGE = 1.602176487e-19;
constexpr double MU_BOHR = 9.2740154e-24;
constexpr double GYROMAGNETIC_RATIO = 2.211e5;

// ---- errors --------------------------------------------------------------------------------------
void set_error(const std::string &msg);
void clear_error();
std::atomic<uint64_t> &launch_counter();

inline mm_status fail(mm_status st, const std::string &msg)
{
	set_error(msg);
	return st;
}

inline mm_status cuda_status(cudaError_t err, const char *what)
{
	if (err == cudaSuccess) return MM_OK;
	set_error(std::string(what) + ": " + cudaGetErrorString(err));
	return err == cudaErrorMemoryAllocation ? MM_ERR_OUT_OF_MEMORY : MM_ERR_CUDA;
}

// Checks the launch that was just issued and counts it.
inline mm_status after_launch(const char *what)
{
	launch_counter().fetch_add(1, std::memory_order_relaxed);
	return cuda_status(cudaGetLastError(), what);
}

#define MM_TRY(expr)                                                                           \
	do {                                                                                     \
		mm_status _st = (expr);                                                              \
		if (_st != MM_OK) return _st;                                                        \
	} while (0)

#define MM_CUDA(expr) MM_TRY(::mm::cuda_status((expr), #expr))

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- optional per-kernel timing (mm_profile_*): CUDA events around solver/convolution launches --
struct ProfToken {
	cudaEvent_t start = nullptr;
};
bool profiling_on();
ProfToken prof_begin(cudaStream_t st);
void prof_end(ProfToken tok, const char *name, double bytes, cudaStream_t st);

// ---- number of SMs of the current device (grid sizing) -------------------------------------------
int num_sms();

// ---- 3-vectors --------------------------------------------------------------------------------
template <typename T>
struct V3 {
	T x, y, z;
};

template <typename T>
__host__ __device__ __forceinline__ V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T>
__host__ __device__ __forceinline__ T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
__host__ __device__ __forceinline__ V3<T> cross(V3<T> a, V3<T> b)
{
	return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Products that are never fused into an FMA with a following add/sub: keeps differences such as
// M_j/Ms_j - M_i/Ms_i exactly zero for equal operands (the reference's CPU arithmetic does not
// contract either).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
template <typename T>
__device__ __forceinline__ V3<T> scale_rn(T s, V3<T> a) { return {mul_rn(s, a.x), mul_rn(s, a.y), mul_rn(s, a.z)}; }

template <typename T>
__device__ __forceinline__ V3<T> load3(const T *p, size_t i, size_t n)
{
	return {p[i], p[i + n], p[i + 2 * n]};
}
template <typename T>
__device__ __forceinline__ void store3(T *p, size_t i, size_t n, V3<T> v)
{
	p[i] = v.x;
	p[i + n] = v.y;
	p[i + 2 * n] = v.z;
}

// Order-preserving encodings of non-negative floating point numbers for atomicMax.
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v)
{
	atomicMax(reinterpret_cast<unsigned long long *>(addr),
	          static_cast<unsigned long long>(__double_as_longlong(v)));
}

// max that propagates NaN (fmax would drop it and hide a diverged state from the controller)
template <typename T>
__device__ __forceinline__ T nan_max(T a, T b)
{
	return (a > b || a != a) ? a : b;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

__device__ __forceinline__ int block_tid()
{
	return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ int block_threads() { return blockDim.x * blockDim.y * blockDim.z; }

// Block-wide max of a non-negative value (NaN wins), folded atomically into *out (double).
// Works for 1-D to 3-D blocks whose thread count is a multiple of 32 (at most 1024).
template <typename T>
__device__ __forceinline__ void block_max_to(double *out, T v)
{
	__shared__ T red[32];
	__syncthreads();  // red[] may still be read by a previous reduction in this block
	v = warp_max(v);
	const int tid = block_tid(), lane = tid & 31, wid = tid >> 5;
	if (lane == 0) red[wid] = v;
	__syncthreads();
	if (wid == 0) {
		const int nw = block_threads() >> 5;
		T w = lane < nw ? red[lane] : T(0);
		w = warp_max(w);
		if (lane == 0) atomic_max_nonneg(out, (double)w);
	}
}

// Block-wide sum (double), atomically added into *out.
__device__ __forceinline__ void block_sum_to(double *out, double v)
{
	__shared__ double red[32];
	__syncthreads();
	v = warp_sum(v);
	const int tid = block_tid(), lane = tid & 31, wid = tid >> 5;
	if (lane == 0) red[wid] = v;
	__syncthreads();
	if (wid == 0) {
		const int nw = block_threads() >> 5;
		double w = lane < nw ? red[lane] : 0.0;
		w = warp_sum(w);
		if (lane == 0) atomicAdd(out, w);
	}
}

// Serialises, across host threads, stream captures of the batch rounds against calls that can
// synchronise the whole device or allocate (instance set-up and tear-down): a device-wide
// synchronisation while another thread captures would invalidate that capture.
std::mutex &capture_mutex();

// A small pinned host scalar buffer + device scratch for reductions returned to the host.
struct ScalarScratch {
	double *dev = nullptr;
	double *host = nullptr;
};
mm_status scalar_scratch(ScalarScratch **out);

} // namespace mm
