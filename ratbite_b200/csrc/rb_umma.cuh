// Blackwell (sm_100a) tensor-core building blocks for the radiance cache's
// MLP: tcgen05.mma with operands in shared memory and the accumulator in
// tensor memory (TMEM), one CTA (cta_group::1), no clusters.
//
// Operand layout: a K-major tile of R rows x 64 bf16 (128 bytes per row)
// with the 128-byte swizzle: the 16-byte chunk c of row r is stored at
// r * 128 + ((c ^ (r & 7)) * 16); tiles start on 1024-byte boundaries, so
// every 8-row group is one swizzle atom. The matrix descriptor of such a
// tile (PTX ISA, tcgen05 shared-memory descriptor): start address >> 4,
// leading byte offset 16 (unused by a swizzled K-major tile whose K fits one
// atom), stride byte offset 1024 (between 8-row groups), version 1,
// layout type 2 (128-byte swizzle). A K step of 16 elements moves the start
// address by 32 bytes (the swizzle is applied to the absolute address).
//
// Instruction descriptor of kind::f16 (bf16 x bf16 -> f32, both K-major):
// bits 4-5 D format (1 = f32), 7-9 A format (1 = bf16), 10-12 B format
// (1 = bf16), 17-22 N >> 3, 24-28 M >> 4.
//
// Accumulator: for M = 128, row i of D is TMEM lane i and column j is TMEM
// column base + j (f32). Warp w of the CTA reads lanes 32 (w % 4) ..
// 32 (w % 4) + 31 with tcgen05.ld.32x32b (thread l gets lane 32 (w % 4) + l).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rb
{
namespace umma
{
__device__ __forceinline__ uint32_t smemAddr(const void* p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) (k in 0..63) in a swizzled K-major tile.
__device__ __forceinline__ uint32_t swzOffset(uint32_t r, uint32_t k)
{
	return r * 128u + ((((k >> 3) ^ r) & 7u) << 4) + ((k & 7u) << 1);
}

// Stores row r (64 bf16 packed as 32 words) of a swizzled K-major tile.
__device__ __forceinline__ void storeRow(unsigned char* tile, uint32_t r, const uint32_t (&w)[32])
{
#pragma unroll
	for (uint32_t c = 0; c < 8; ++c)
		*reinterpret_cast<uint4*>(tile + r * 128u + (((c ^ r) & 7u) << 4)) =
			make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
}
// Loads row r of a swizzled K-major tile as 32 packed words.
__device__ __forceinline__ void loadRow(const unsigned char* tile, uint32_t r, uint32_t (&w)[32])
{
#pragma unroll
	for (uint32_t c = 0; c < 8; ++c)
	{
		const uint4 v = *reinterpret_cast<const uint4*>(tile + r * 128u + (((c ^ r) & 7u) << 4));
		w[4 * c] = v.x; w[4 * c + 1] = v.y; w[4 * c + 2] = v.z; w[4 * c + 3] = v.w;
	}
}

// Matrix descriptor of a swizzled K-major tile at `tile` (1024-byte aligned),
// advanced by `kStep` K steps of 16 elements.
__device__ __forceinline__ uint64_t descK(const void* tile, uint32_t kStep)
{
	const uint64_t start = (smemAddr(tile) + 32u * kStep) >> 4;
	return (start & 0x3FFFull) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

constexpr uint32_t idescBf16(uint32_t m, uint32_t n)
{
	return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

// D (TMEM) = A B^T (+ D when accumulate): one instruction, issued by one thread.
__device__ __forceinline__ void mma(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, bool accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
		:: "r"(dTmem), "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate ? 1u : 0u) : "memory");
}
// Arrives on the mbarrier once every MMA this thread issued before has completed.
__device__ __forceinline__ void commit(uint64_t* bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
		:: "r"(smemAddr(bar)) : "memory");
}

__device__ __forceinline__ void barrierInit(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smemAddr(bar)), "r"(count) : "memory");
}
// Arrives once on the mbarrier (release at CTA scope).
__device__ __forceinline__ void barrierArrive(uint64_t* bar)
{
	asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" :: "r"(smemAddr(bar)) : "memory");
}
// Waits for the phase with the given parity to complete, at most `limit`
// polls; false when it gave up.
#ifndef RB_UMMA_SPIN_WAIT
#define RB_UMMA_SPIN_WAIT 0
#endif
__device__ __forceinline__ bool barrierWait(uint64_t* bar, uint32_t parity, uint32_t limit)
{
	const uint32_t a = smemAddr(bar);
	for (uint32_t i = 0; i < limit; ++i)
	{
		uint32_t done = 0;
#if RB_UMMA_SPIN_WAIT
		asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, p;\n\t}\n"
			: "=r"(done) : "r"(a), "r"(parity) : "memory");
#else
		asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, p;\n\t}\n"
			: "=r"(done) : "r"(a), "r"(parity) : "memory");
#endif
		if (done) return true;
	}
	return false;
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's shared-memory writes visible to the tensor cores.
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one whole warp: `cols` columns (a power of two >= 32);
// the base address is written to *slot (shared memory).
__device__ __forceinline__ void tmemAlloc(uint32_t* slot, uint32_t cols)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		:: "r"(smemAddr(slot)), "r"(cols) : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmemFree(uint32_t base, uint32_t cols)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(base), "r"(cols) : "memory");
}

// 16 consecutive f32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, uint32_t (&r)[16])
{
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 "
		"{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(taddr) : "memory");
}
__device__ __forceinline__ void tmemWaitLoad() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// TMEM address of this warp's lane quarter, column `col`.
__device__ __forceinline__ uint32_t laneAddr(uint32_t base, uint32_t col)
{
	return base + (((threadIdx.x >> 5) & 3u) * 32u << 16) + col;
}
} // namespace umma
} // namespace rb
