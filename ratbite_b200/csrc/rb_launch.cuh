// Grid helpers shared by the kernel translation units.
#pragma once

#include <cstdint>

#include "ratbite_b200.h"
#include "rb_math.cuh"

namespace rb
{
constexpr int kThreads = 128;

RB_D uint32_t gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
RB_D uint32_t gstride() { return gridDim.x * blockDim.x; }

// Warp-aggregated append: one atomic per warp for the lanes that push. Every
// lane active at the call must append to the same counter (call it inside
// the branch that selects the counter).
RB_D uint32_t appendIndex(uint32_t* counter)
{
	const uint32_t active = __activemask();
	const int leader = __ffs(active) - 1;
	const uint32_t lane = threadIdx.x & 31u;
	uint32_t base = 0;
	if (lane == static_cast<uint32_t>(leader)) base = atomicAdd(counter, __popc(active));
	base = __shfl_sync(active, base, leader);
	return base + __popc(active & ((1u << lane) - 1u));
}

// Queue slot of one entry, or kNoSlot when the queue already holds `cap`
// entries: the entry is dropped and RB_DEV_QUEUE_OVERFLOW set in *status.
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
RB_D uint32_t appendSlot(uint32_t* counter, uint32_t cap, uint32_t* status)
{
	const uint32_t i = appendIndex(counter);
	if (i < cap) return i;
	atomicOr(status, RB_DEV_QUEUE_OVERFLOW);
	return kNoSlot;
}

// Record of a surface in one of two regions of the record arrays, `sky`
// choosing the region: the tree region grows from 0 up (low word of
// *counter), the other from cap - 1 down (high word). One 64-bit atomic per
// warp for both. A record is kept only while the two regions together hold
// at most `cap`, so they never overlap; beyond it the entry is dropped with
// RB_DEV_QUEUE_OVERFLOW and kNoSlot returned. `order` gets the record's
// position in the order of arrival over both regions (0 .. total - 1).
RB_D uint32_t appendRegion(unsigned long long* counter, bool sky, uint32_t cap, uint32_t* status, uint32_t& order)
{
	const uint32_t active = __activemask();
	const uint32_t skyMask = __ballot_sync(active, sky), treeMask = active & ~skyMask;
	const int leader = __ffs(active) - 1;
	const uint32_t lane = threadIdx.x & 31u, below = (1u << lane) - 1u;
	unsigned long long base = 0;
	if (lane == static_cast<uint32_t>(leader))
		base = atomicAdd(counter, static_cast<unsigned long long>(__popc(treeMask))
			| (static_cast<unsigned long long>(__popc(skyMask)) << 32));
	base = __shfl_sync(active, base, leader);
	const uint32_t treeBase = static_cast<uint32_t>(base), skyBase = static_cast<uint32_t>(base >> 32);
	// records of both regions up to and including this one
	const uint64_t total = static_cast<uint64_t>(treeBase) + skyBase + __popc(active & below) + 1u;
	if (total > cap)
	{
		atomicOr(status, RB_DEV_QUEUE_OVERFLOW);
		return kNoSlot;
	}
	order = static_cast<uint32_t>(total - 1u);
	return sky ? cap - 1u - (skyBase + __popc(skyMask & below)) : treeBase + __popc(treeMask & below);
}
// The two region counts of a bounce (kRegionCounts), each at most cap and
// together at most cap.
RB_D uint2 regionCounts(const uint32_t* counts2, uint32_t cap)
{
	const uint32_t t = min(counts2[0], cap);
	return make_uint2(t, min(counts2[1], cap - t));
}

// Adds per-thread counts to a 64-bit counter with one atomic per warp.
RB_D void warpAdd(unsigned long long* dst, uint32_t v)
{
	unsigned long long s = v;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
	if ((threadIdx.x & 31u) == 0 && s) atomicAdd(dst, s);
}

// 32-bit integer hash (the "lowbias32" finaliser: xorshift-multiply rounds).
RB_HD uint32_t mix32(uint32_t x)
{
	x ^= x >> 16;
	x *= 0x7feb352du;
	x ^= x >> 15;
	x *= 0x846ca68bu;
	x ^= x >> 16;
	return x;
}

// A persistent grid of `blocks`, capped at the blocks of `threads` that
// `items` work items need (items 0: no cap): small waves then launch small
// grids.
inline int capBlocks(int blocks, uint32_t items, int threads)
{
	if (items == 0) return blocks;
	const uint32_t need = (items + static_cast<uint32_t>(threads) - 1) / static_cast<uint32_t>(threads);
	return need < static_cast<uint32_t>(blocks) ? static_cast<int>(need < 1 ? 1 : need) : blocks;
}

// Grid for a one-thread-per-item batch kernel (grid-stride loops cover the rest).
inline int gridFor(uint32_t n)
{
	const uint32_t b = (n + kThreads - 1) / kThreads;
	return static_cast<int>(b < 1 ? 1 : (b > 65535u * 4 ? 65535u * 4 : b));
}
} // namespace rb
