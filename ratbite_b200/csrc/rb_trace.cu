// Ray-traversal kernels: the extend (closest hit) and shadow (any hit)
// stages of the wavefront loop, and the batched trace / occlusion entry
// points. This translation unit keeps the compiler's default multiply-add
// contraction: the box tests are conservative by construction (outward
// rounding and padding of the quantized boxes), and the triangle test, which
// decides the reported hit, is written with explicitly rounded operations.

#include <cfloat>
#include <type_traits>

#include "rb_bvh.cuh"
#include "rb_launch.cuh"
#include "rb_wavefront.h"

namespace rb
{
namespace
{
// Node / leaf visits per step of the persistent loop, and the number of idle
// lanes at which the warp fetches new rays (all lanes idle always fetches).
// On B200, at-scale frame (extension ms): 16 / 1 (the default) 442; 2 / 8
// 433 (but shadow 75 -> 86); 1 / 8 448; 4 / 8 709; 8 / 8 1185. Measured
// with an instrumented build: a refill (warp atomic, queue slot and ray
// loads) takes about 4.8k of the 80k cycles of a 16-visit step, and 75 % of
// the lane-visit slots of a step do work. Staging each lane's next ray in
// shared memory with cp.async while it traces the current one (indices
// claimed 64 per atomic) was slower: extension 397 -> 483 ms.
#ifndef RB_STEP_BUDGET
#define RB_STEP_BUDGET 16
#endif
#ifndef RB_REFILL_LANES
#define RB_REFILL_LANES 1
#endif
// Resident blocks of 128 per SM the traversal kernels are compiled for
// (register cap 65536 / (128 x blocks)).
#ifndef RB_TRACE_MIN_BLOCKS
#define RB_TRACE_MIN_BLOCKS 8
#endif
// Traversal stack entries kept in shared memory per thread (the rest in
// local memory; 0: all local, the default). On B200, at-scale frame
// (extension / shadow ms per frame): all local 393 / 70; 8 entries in
// shared memory 407 / 84, 16: 404 / 83, 24: 404 / 83. Local memory is
// cached in L1, and the shared-memory carve-out costs L1 capacity that the
// BVH nodes and triangles use.
#ifndef RB_TRAV_SMEM_STACK
#define RB_TRAV_SMEM_STACK 0
#endif
constexpr int kStepBudget = RB_STEP_BUDGET;
constexpr int kRefillLanes = RB_REFILL_LANES;

// Persistent traversal warps with dynamic ray fetch: lanes whose rays have
// ended take the next ones from the stage's work counter (one atomic per warp
// for all idle lanes) once kRefillLanes of them are idle, between steps of
// kStepBudget visits, so lanes do not idle until the warp's longest ray ends.
// The loop exits are warp-uniform, so the full-mask warp votes are safe.
template<typename Traversal, typename Begin, typename Step>
RB_D void persistentTraversal(uint32_t n, uint32_t* workCounter, Begin&& begin, Step&& step)
{
	const uint32_t lane = threadIdx.x & 31u;
	bool active = false, exhausted = false;
	for (;;)
	{
		const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !active);
		if (!exhausted && idle && (idle == 0xFFFFFFFFu || __popc(idle) >= kRefillLanes))
		{
			const int leader = __ffs(idle) - 1;
			uint32_t base = 0;
			if (lane == static_cast<uint32_t>(leader)) base = atomicAdd(workCounter, __popc(idle));
			base = __shfl_sync(0xFFFFFFFFu, base, leader);
			if (base + __popc(idle) >= n) exhausted = true;
			if (!active)
			{
				const uint32_t idx = base + __popc(idle & ((1u << lane) - 1u));
				if (idx < n)
				{
					begin(idx);
					active = true;
				}
			}
		}
		if (__all_sync(0xFFFFFFFFu, !active)) break;
		if (active && step()) active = false;
	}
}

// The hit record's second word: the distance (flat), or the position of the
// hit's instance (two-level; the distance is not read downstream).
RB_D float hitWord(const ClosestTraversal& tr) { return tr.best.t; }
RB_D float hitWord(const ClosestTraversal2& tr) { return __uint_as_float(tr.bestInst); }

// counters (COUNT only): [0] rays, [1] nodes, [2] triangles. JOBS: a shared
// wavefront, each ray traced in its job's geometry. TWO: the two-level
// structure (RB_ACCEL_INSTANCED).
template<bool COUNT, bool JOBS, bool TWO = false>
__global__ void __launch_bounds__(kThreads, RB_TRACE_MIN_BLOCKS) kExtend(const __grid_constant__ DevScene sc, PathSoA s,
	int bounce, unsigned long long* counters)
{
	const uint32_t n = min(s.counts[bounce], s.queueCap);
	const uint32_t* q = s.queue[bounce & 1];
	uint32_t rays = 0, nodes = 0, tris = 0;
	uint32_t p = 0;
	const DevScene* js = &sc;
	typename std::conditional<TWO, ClosestTraversal2, ClosestTraversal>::type tr;
#if RB_TRAV_SMEM_STACK
	__shared__ uint2 smStack[RB_TRAV_SMEM_STACK * kThreads];
	HybridStack<uint2, RB_TRAV_SMEM_STACK, kThreads> stack{ smStack + threadIdx.x };
#else
	uint2 stack[kTraversalStack];
#endif
	auto step = [&]() {
		const DevGeometry& g = JOBS ? js->geo : sc.geo;
		if (!tr.template run<COUNT>(g, kStepBudget, JOBS ? js->status : sc.status, nodes, tris, stack)) return false;
		s.hit[p] = make_float4(__int_as_float(tr.best.tri), hitWord(tr), tr.best.b1, tr.best.b2);
		return true;
	};
	persistentTraversal<ClosestTraversal>(n, s.counts + kExtendFetch + bounce,
		[&](uint32_t idx) {
			p = q[idx];
			if (JOBS) js = &s.jobs[s.job[p]].scene;
			const float4 o = s.rayO[p], d = s.rayD[p];
			tr.init(JOBS ? js->geo : sc.geo, f3_of(o), f3_of(d), 0.0f, FLT_MAX);
			++rays;
		}, step);
	if (COUNT)
	{
		warpAdd(counters + 0, rays);
		warpAdd(counters + 1, nodes);
		warpAdd(counters + 2, tris);
	}
}

template<bool COUNT, bool JOBS, bool TWO = false>
__global__ void __launch_bounds__(kThreads, RB_TRACE_MIN_BLOCKS) kShadow(const __grid_constant__ DevScene sc, PathSoA s,
	int bounce, unsigned long long* counters)
{
	const uint32_t n = min(s.counts[kShadowCounts + bounce], s.queueCap);
	uint32_t rays = 0, nodes = 0, tris = 0;
	uint32_t r = 0;             // the shadow ray's surface record (queue position)
	const DevScene* js = &sc;
	typename std::conditional<TWO, AnyTraversal2, AnyTraversal>::type tr;
#if RB_TRAV_SMEM_STACK
	__shared__ uint32_t smStack[RB_TRAV_SMEM_STACK * kThreads];
	HybridStack<uint32_t, RB_TRAV_SMEM_STACK, kThreads> stack{ smStack + threadIdx.x };
#else
	uint32_t stack[kTraversalStack];
#endif
	auto step = [&]() {
		const DevGeometry& g = JOBS ? js->geo : sc.geo;
		if (!tr.template run<COUNT>(g, kStepBudget, JOBS ? js->status : sc.status, nodes, tris, stack)) return false;
		if (!tr.hit)
		{
			const uint32_t p = s.surfQueue[r];
			S4 L = s4(s.L[p]);
			L += s4(s.shC[r]);
			s.L[p] = f4(L);
		}
		return true;
	};
	persistentTraversal<AnyTraversal>(n, s.counts + kShadowFetch + bounce,
		[&](uint32_t idx) {
			r = s.shadowQueue[idx];
			if (JOBS) js = &s.jobs[s.job[s.surfQueue[r]]].scene;
			const float4 o = s.shO[r], d = s.shD[r];
			tr.init(JOBS ? js->geo : sc.geo, f3_of(o), f3_of(d), 0.0f, o.w);
			++rays;
		}, step);
	if (COUNT)
	{
		warpAdd(counters + 3, rays);
		warpAdd(counters + 4, nodes);
		warpAdd(counters + 5, tris);
	}
}

// Closest hit returned in the reference's 24-word payload layout.
__global__ void kTrace(DevScene sc, uint32_t n, const float* rays, uint32_t* payload, float* tOut, int32_t* triOut)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const f3 o = mk(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
		const f3 d = mk(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
		Hit h;
		uint32_t pos = 0;
		if (sc.geo.instanced)
		{
			ClosestTraversal2 tr;
			uint2 stack[kTraversalStack];
			uint32_t nn = 0, nt = 0;
			tr.init(sc.geo, o, d, 0.0f, FLT_MAX);
			while (!tr.run<false>(sc.geo, 1 << 30, sc.status, nn, nt, stack)) {}
			h = tr.best;
			pos = tr.bestInst;
		}
		else h = traceClosest(sc.geo, o, d, 0.0f, FLT_MAX, sc.status);
		uint32_t* pl = payload + 24 * static_cast<size_t>(i);
		for (int k = 0; k < 24; ++k) pl[k] = 0u;
		if (h.tri < 0)
		{
			pl[8] = kLightTypeSky << 30;
			tOut[i] = INFINITY;
			triOut[i] = -1;
			continue;
		}
		float4 a, b, c;
		uint2 aux;
		if (sc.geo.instanced) instancedTriangle(sc.geo, static_cast<uint32_t>(h.tri), pos, a, b, c, aux);
		else
		{
			a = sc.geo.triVerts[3 * h.tri]; b = sc.geo.triVerts[3 * h.tri + 1]; c = sc.geo.triVerts[3 * h.tri + 2];
			aux = sc.geo.triAux[h.tri];
		}
		const uint32_t sbt = __float_as_uint(c.w);
		uint32_t prim = aux.y, mat = sbt, lptr = kLightTypeNone << 30;
		if (sbt == 0xFFFFFFFFu)
		{
			lptr = (kLightTypeTriangle << 30) | (aux.y & ((1u << 30) - 1u));
			prim = sc.lights.triangles[aux.y].prim;
			mat = sc.lights.triangles[aux.y].material;
		}
		pl[0] = __float_as_uint(a.x); pl[1] = __float_as_uint(a.y); pl[2] = __float_as_uint(a.z);
		pl[3] = aux.x; pl[4] = prim; pl[5] = __float_as_uint(h.b1); pl[6] = __float_as_uint(h.b2);
		pl[7] = mat; pl[8] = lptr;
		const float* M = sc.geo.normalMatrix + 9u * __float_as_uint(b.w);
		for (int k = 0; k < 9; ++k) pl[9 + k] = __float_as_uint(M[k]);
		pl[18] = __float_as_uint(b.x); pl[19] = __float_as_uint(b.y); pl[20] = __float_as_uint(b.z);
		pl[21] = __float_as_uint(c.x); pl[22] = __float_as_uint(c.y); pl[23] = __float_as_uint(c.z);
		tOut[i] = h.t;
		triOut[i] = static_cast<int32_t>(__float_as_uint(a.w));
	}
}
__global__ void kOccluded(DevScene sc, uint32_t n, const float* rays, const float* tmax, uint32_t* out)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const f3 o = mk(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
		const f3 d = mk(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
		if (sc.geo.instanced)
		{
			AnyTraversal2 tr;
			uint32_t stack[kTraversalStack];
			uint32_t nn = 0, nt = 0;
			tr.init(sc.geo, o, d, 0.0f, tmax[i]);
			while (!tr.run<false>(sc.geo, 1 << 30, sc.status, nn, nt, stack)) {}
			out[i] = tr.hit ? 1u : 0u;
		}
		else out[i] = traceAny(sc.geo, o, d, 0.0f, tmax[i], sc.status) ? 1u : 0u;
	}
}
} // namespace

void queryTraceShape(LaunchShape& ls)
{
	auto occ = [&](const void* fn) {
		int b = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kThreads, 0);
		return (b < 1 ? 1 : b) * ls.smCount;
	};
	ls.blocksExtend = occ(reinterpret_cast<const void*>(kExtend<false, false>));
	ls.blocksShadow = occ(reinterpret_cast<const void*>(kShadow<false, false>));
}

void launchExtend(const DevScene& sc, const PathSoA& s, int bounce, const LaunchShape& ls, cudaStream_t st,
	unsigned long long* counters)
{
	const int g = capBlocks(ls.blocksExtend, ls.items, kThreads);
	if (s.jobs)
	{
		if (counters) kExtend<true, true><<<g, kThreads, 0, st>>>(sc, s, bounce, counters);
		else kExtend<false, true><<<g, kThreads, 0, st>>>(sc, s, bounce, nullptr);
	}
	else if (sc.geo.instanced)
	{
		if (counters) kExtend<true, false, true><<<g, kThreads, 0, st>>>(sc, s, bounce, counters);
		else kExtend<false, false, true><<<g, kThreads, 0, st>>>(sc, s, bounce, nullptr);
	}
	else if (counters) kExtend<true, false><<<g, kThreads, 0, st>>>(sc, s, bounce, counters);
	else kExtend<false, false><<<g, kThreads, 0, st>>>(sc, s, bounce, nullptr);
}
void launchShadow(const DevScene& sc, const PathSoA& s, int bounce, const LaunchShape& ls, cudaStream_t st,
	unsigned long long* counters)
{
	const int g = capBlocks(ls.blocksShadow, ls.items, kThreads);
	if (s.jobs)
	{
		if (counters) kShadow<true, true><<<g, kThreads, 0, st>>>(sc, s, bounce, counters);
		else kShadow<false, true><<<g, kThreads, 0, st>>>(sc, s, bounce, nullptr);
	}
	else if (sc.geo.instanced)
	{
		if (counters) kShadow<true, false, true><<<g, kThreads, 0, st>>>(sc, s, bounce, counters);
		else kShadow<false, false, true><<<g, kThreads, 0, st>>>(sc, s, bounce, nullptr);
	}
	else if (counters) kShadow<true, false><<<g, kThreads, 0, st>>>(sc, s, bounce, counters);
	else kShadow<false, false><<<g, kThreads, 0, st>>>(sc, s, bounce, nullptr);
}
void launchTrace(const DevScene& sc, uint32_t n, const float* rays, uint32_t* payload, float* t, int32_t* tri, cudaStream_t st)
{
	kTrace<<<gridFor(n), kThreads, 0, st>>>(sc, n, rays, payload, t, tri);
}
void launchOccluded(const DevScene& sc, uint32_t n, const float* rays, const float* tmax, uint32_t* out, cudaStream_t st)
{
	kOccluded<<<gridFor(n), kThreads, 0, st>>>(sc, n, rays, tmax, out);
}
} // namespace rb
