// Tensor-memory-accelerator (TMA) staging helpers for the FFT passes: tensor-map encoding on the
// host (through the runtime's driver entry point, so the library does not link libcuda), and the
// mbarrier / cp.async.bulk.tensor primitives in inline PTX.  Loads only, never with cluster
// multicast: every copy lands in the issuing CTA's own shared memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "mm_common.cuh"

namespace mm {

// 3-D tiled tensor map over an array of 8-byte elements: dims[0] fastest, strides in bytes of
// dims 1 and 2 (multiples of 16), box[] elements per dimension (box[0] * 8 a multiple of 16).
// Out-of-range elements of a box read as zero.
mm_status tma_encode_3d(CUtensorMap *map, const void *base, uint64_t d0, uint64_t d1, uint64_t d2,
                        uint64_t stride1, uint64_t stride2, uint32_t b0, uint32_t b1, uint32_t b2);
// Same for rank 1..5: dims[0] fastest, strides[] in bytes of dims 1..rank-1.
mm_status tma_encode(CUtensorMap *map, const void *base, int rank, const uint64_t *dims, const uint64_t *strides,
                     const uint32_t *box);
// Same with elements of esize bytes (1, 4 or 8; copied as unsigned integers of that size).
mm_status tma_encode_as(CUtensorMap *map, const void *base, int rank, const uint64_t *dims, const uint64_t *strides,
                        const uint32_t *box, int esize);

// Spin limit of a bounded mbarrier wait (each try_wait already blocks for a while in hardware);
// a wait that exceeds it reports a timeout instead of hanging the GPU.
constexpr uint32_t TMA_WAIT_LIMIT = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation and earlier generic-proxy shared-memory accesses visible to the
// async proxy (the TMA unit).
__device__ __forceinline__ void fence_proxy_async()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
	             : "memory");
}

// Plain arrival (no transaction bytes).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the phase with the given parity to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
	const uint32_t a = smem_u32(bar);
	for (uint32_t it = 0; it < TMA_WAIT_LIMIT; ++it) {
		uint32_t done = 0;
		asm volatile(
		    "{\n\t.reg .pred p;\n\t"
		    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		    "selp.u32 %0, 1, 0, p;\n\t}"
		    : "=r"(done)
		    : "r"(a), "r"(parity)
		    : "memory");
		if (done) return true;
	}
	return false;
}

// After a bounded wait gave up in a two-buffer pipeline: waits (bounded again) for the loads
// still in flight, the one that timed out on buffer b and, when one was issued, the next one on
// the other buffer, so that no copy lands in shared memory after the CTA has exited.
__device__ __forceinline__ void mbar_drain2(uint64_t *bar, uint32_t parity, int b, bool other_issued)
{
	mbar_wait(&bar[b], (parity >> b) & 1u);
	if (other_issued) mbar_wait(&bar[b ^ 1], (parity >> (b ^ 1)) & 1u);
}

// 2-D, 3-D and 4-D tiled loads of one box into shared memory, completing on `bar` (transaction
// bytes).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar)
{
	asm volatile(
	    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
	    "[%4];" ::"r"(smem_u32(dst)),
	    "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
	    : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
	asm volatile(
	    "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
	    "%5}], [%6];" ::"r"(smem_u32(dst)),
	    "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
	    : "memory");
}

// Untiled bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global
// into this CTA's shared memory, completing on `bar` (transaction bytes).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
	                 smem_u32(dst)),
	             "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
	             : "memory");
}

// 3-D tiled load of one box into shared memory, completing on `bar` (transaction bytes).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar)
{
	asm volatile(
	    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
	    "[%5];" ::"r"(smem_u32(dst)),
	    "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
	    : "memory");
}

} // namespace mm
