// Ray traversal of the 8-wide BVH (replaces OptiX's RT-core traversal behind
// optixTrace / optixTraverse, src/kernels/pathtrace.cu:1162, 1708).
//
// One thread per ray. Nodes are 96 B with 8-bit quantized child boxes
// (rb_scene.h); children that the ray enters are ordered near-to-far with a
// sorting network held in registers, the nearest is descended directly and the
// rest go on a short per-thread stack. Triangles use the watertight test of
// Woop, Benthin and Wald (JCGT 2013) evaluated with explicitly rounded
// operations (no FMA contraction) so distances and barycentrics are bitwise
// reproducible on the CPU; closest-hit ties on t go to the smaller canonical
// triangle id, which makes the result independent of traversal order.
#pragma once

#include "rb_instance.cuh"
#include "rb_math.cuh"
#include "rb_scene.h"

namespace rb
{
constexpr int kTraversalStack = kTraversalStackEntries;

// Traversal stack with its first S entries in shared memory and the rest in
// local memory. Entry k of thread t is word k * kStride + t of the block's
// shared array, so the lanes of a warp at one depth touch consecutive words.
// In shared memory the entries no longer compete with the BVH nodes and
// triangles for L1 (local memory is cached there). The traversal takes any
// stack type with operator[] (a plain local array, or this).
template<typename T, int S, int kStride>
struct HybridStack
{
	T* sm;                                   // the block's array + threadIdx.x
	T local[kTraversalStack - S];
	RB_D T& operator[](int k) { return k < S ? sm[k * kStride] : local[k - S]; }
};

// Traversal variants (compile-time): RB_TRAV_SORT orders the entered
// children near-to-far with a sorting network (1, the default; 0: descend
// the nearest, push the rest unordered; 2: direction-octant order, the
// builder placing children in slots by octant after Ylitie, Karras and Laine
// 2017, no sort); RB_TRAV_WHILE_WHILE runs interior nodes until a leaf
// before each leaf (0: one node or leaf per step); RB_TRAV_POSTPONE keeps a
// reached leaf aside and goes on with interior nodes, the warp testing the
// postponed leaves one triangle per lane once half of its lanes hold one or
// a lane has no node left (Aila and Laine 2009). On B200, at-scale frame
// (2.03M triangles, 1920x1080x256, extension ms per frame; nodes and
// triangles visited per ray): sorted 397 (13.3, 3.30); octant order 415
// (14.3, 3.79); sorted + postponed leaves 416 (13.6, 3.64); octant +
// postponed 440 (14.6, 4.15); octant order with one stack entry per node
// group (node, remaining-child mask) 526 (14.8, 3.80); earlier: nearest-only
// 509 against 493 sorted, while-while 559. Octant order saves the sort but
// visits more nodes and triangles than it saves; postponing adds visits
// (culling sees the postponed hits later) and the traversal is bound by
// instruction issue and L1/L2 latency, not by the node-versus-leaf
// divergence it removes. Triangle loads cached in L2 only (ld.global.cg,
// leaving L1 to the nodes and stacks) changed nothing (392.9 against 392.3
// ms), nor did register caps of 48 and 40 (10 and 12 resident blocks of 128:
// 391.4 and 402.3 ms) or step budgets of 32 (398.4 ms) and 4 refill lanes
// (390.5 ms).
#ifndef RB_TRAV_SORT
#define RB_TRAV_SORT 1
#endif
#ifndef RB_TRAV_POSTPONE
#define RB_TRAV_POSTPONE 0
#endif
#ifndef RB_TRAV_WHILE_WHILE
#define RB_TRAV_WHILE_WHILE 0
#endif

struct TraceRay
{
	f3 o, d;
	float ix, iy, iz;         // safe reciprocal direction for box tests
	int kx, ky, kz;
	float sx, sy, sz;
	uint32_t oct;             // direction octant: bit 0 x < 0, bit 1 y < 0, bit 2 z < 0
};

RB_D float safeRcp(float d) { return 1.0f / (fabsf(d) < 1e-20f ? copysignf(1e-20f, d) : d); }

RB_D float comp(f3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

RB_D TraceRay makeTraceRay(f3 o, f3 d)
{
	TraceRay r;
	r.o = o; r.d = d;
	r.ix = safeRcp(d.x); r.iy = safeRcp(d.y); r.iz = safeRcp(d.z);
	const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
	r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
	r.kx = r.kz == 2 ? 0 : r.kz + 1;
	r.ky = r.kx == 2 ? 0 : r.kx + 1;
	if (comp(d, r.kz) < 0.0f) { const int t = r.kx; r.kx = r.ky; r.ky = t; }
	const float dz = comp(d, r.kz);
	r.sx = __fdiv_rn(comp(d, r.kx), dz);
	r.sy = __fdiv_rn(comp(d, r.ky), dz);
	r.sz = __fdiv_rn(1.0f, dz);
	r.oct = (signbit(r.ix) ? 1u : 0u) | (signbit(r.iy) ? 2u : 0u) | (signbit(r.iz) ? 4u : 0u);
	return r;
}

// The part of a TraceRay the box tests read (origin, direction, safe
// reciprocal direction, octant): the two-level traversal's object-space
// rays, whose triangles are intersected with the world ray instead.
RB_D TraceRay makeBoxRay(f3 o, f3 d)
{
	TraceRay r;
	r.o = o; r.d = d;
	r.ix = safeRcp(d.x); r.iy = safeRcp(d.y); r.iz = safeRcp(d.z);
	r.kx = 0; r.ky = 1; r.kz = 2;
	r.sx = r.sy = r.sz = 0.0f;
	r.oct = (signbit(r.ix) ? 1u : 0u) | (signbit(r.iy) ? 2u : 0u) | (signbit(r.iz) ? 4u : 0u);
	return r;
}

// Watertight ray/triangle test. Returns true for a hit with tmin < t < tmax
// (t <= tmax when `inclusive`), writing t and the barycentrics of v1, v2.
RB_D bool intersectTriangle(const TraceRay& r, f3 v0, f3 v1, f3 v2, float tmin, float tmax, bool inclusive,
	float& t, float& b1, float& b2)
{
	const f3 A = mk(__fsub_rn(v0.x, r.o.x), __fsub_rn(v0.y, r.o.y), __fsub_rn(v0.z, r.o.z));
	const f3 B = mk(__fsub_rn(v1.x, r.o.x), __fsub_rn(v1.y, r.o.y), __fsub_rn(v1.z, r.o.z));
	const f3 C = mk(__fsub_rn(v2.x, r.o.x), __fsub_rn(v2.y, r.o.y), __fsub_rn(v2.z, r.o.z));
	const float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
	const float Ax = __fsub_rn(comp(A, r.kx), __fmul_rn(r.sx, Akz));
	const float Ay = __fsub_rn(comp(A, r.ky), __fmul_rn(r.sy, Akz));
	const float Bx = __fsub_rn(comp(B, r.kx), __fmul_rn(r.sx, Bkz));
	const float By = __fsub_rn(comp(B, r.ky), __fmul_rn(r.sy, Bkz));
	const float Cx = __fsub_rn(comp(C, r.kx), __fmul_rn(r.sx, Ckz));
	const float Cy = __fsub_rn(comp(C, r.ky), __fmul_rn(r.sy, Ckz));
	float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
	float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
	float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
	if (U == 0.0f || V == 0.0f || W == 0.0f)
	{
		U = __double2float_rn(__dsub_rn(__dmul_rn(Cx, By), __dmul_rn(Cy, Bx)));
		V = __double2float_rn(__dsub_rn(__dmul_rn(Ax, Cy), __dmul_rn(Ay, Cx)));
		W = __double2float_rn(__dsub_rn(__dmul_rn(Bx, Ay), __dmul_rn(By, Ax)));
	}
	if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
	const float det = __fadd_rn(__fadd_rn(U, V), W);
	if (det == 0.0f) return false;
	const float Az = __fmul_rn(r.sz, Akz), Bz = __fmul_rn(r.sz, Bkz), Cz = __fmul_rn(r.sz, Ckz);
	const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
	const float rcp = __fdiv_rn(1.0f, det);
	const float tt = __fmul_rn(T, rcp);
	if (!(tt > tmin && (inclusive ? tt <= tmax : tt < tmax))) return false;
	t = tt;
	b1 = __fmul_rn(V, rcp);
	b2 = __fmul_rn(W, rcp);
	return true;
}

struct NodeView
{
	float4 q[6];
};
RB_D NodeView loadNode(const BvhNode* nodes, uint32_t i)
{
	NodeView v;
	const float4* p = reinterpret_cast<const float4*>(nodes + i);
#pragma unroll
	for (int k = 0; k < 6; ++k) v.q[k] = __ldg(p + k);
	return v;
}
RB_D uint32_t nodeChild(const NodeView& v, int c)
{
	const float4& a = v.q[1 + c / 4];
	const float w = (c & 3) == 0 ? a.x : ((c & 3) == 1 ? a.y : ((c & 3) == 2 ? a.z : a.w));
	return __float_as_uint(w);
}
// Byte c (0..7) of a child plane row held in two words, as a float: the
// byte is placed in the mantissa of 2^23 with one byte permute and 2^23
// subtracted (exact), which keeps the conversion off the slower conversion
// pipe.
RB_D float planeQ(uint32_t w0, uint32_t w1, int c)
{
	const uint32_t word = c < 4 ? w0 : w1;
	const uint32_t bits = __byte_perm(word, 0x4B000000u, static_cast<uint32_t>(c & 3) | 0x7540u);
	return __fsub_rn(__uint_as_float(bits), 8388608.0f);
}
// Word w (0..11) of the 48-byte plane block: rows of 8 bytes, lo x,y,z then hi x,y,z.
RB_D uint32_t planeWord(const NodeView& v, int w)
{
	const float4& a = v.q[3 + w / 4];
	return __float_as_uint((w & 3) == 0 ? a.x : ((w & 3) == 1 ? a.y : ((w & 3) == 2 ? a.z : a.w)));
}

// Intersects the ray with the 8 child boxes; hitMask bit c set when child c
// is entered within [tmin, tmax]; tnear[c] is its entry distance. Empty
// slots carry inverted boxes, which rays miss except where rounding flattens
// the box (a ray far from a tiny node): the traversal skips empty references
// (kEmptyChild) wherever it takes a child. Per axis the
// near and far plane rows are chosen once from the sign of the reciprocal
// direction, which gives the same distances as taking the min and max of the
// two planes per child (the rounding is monotonic).
RB_D uint32_t childBoxes(const TraceRay& r, const NodeView& v, float tmin, float tmax, float tnear[8])
{
	const float ox = v.q[0].x, oy = v.q[0].y, oz = v.q[0].z;
	const uint32_t meta = __float_as_uint(v.q[0].w);
	const float scx = __uint_as_float(((meta >> 0) & 0xFFu) << 23);
	const float scy = __uint_as_float(((meta >> 8) & 0xFFu) << 23);
	const float scz = __uint_as_float(((meta >> 16) & 0xFFu) << 23);
	// rows: lo x = words 0,1; lo y = 2,3; lo z = 4,5; hi x = 6,7; hi y = 8,9; hi z = 10,11
	const bool nx = signbit(r.ix), ny = signbit(r.iy), nz = signbit(r.iz);
	const uint32_t lo0 = planeWord(v, 0), lo1 = planeWord(v, 1), lo2 = planeWord(v, 2), lo3 = planeWord(v, 3);
	const uint32_t lo4 = planeWord(v, 4), lo5 = planeWord(v, 5), hi0 = planeWord(v, 6), hi1 = planeWord(v, 7);
	const uint32_t hi2 = planeWord(v, 8), hi3 = planeWord(v, 9), hi4 = planeWord(v, 10), hi5 = planeWord(v, 11);
	const uint32_t nx0 = nx ? hi0 : lo0, nx1 = nx ? hi1 : lo1, fx0 = nx ? lo0 : hi0, fx1 = nx ? lo1 : hi1;
	const uint32_t ny0 = ny ? hi2 : lo2, ny1 = ny ? hi3 : lo3, fy0 = ny ? lo2 : hi2, fy1 = ny ? lo3 : hi3;
	const uint32_t nz0 = nz ? hi4 : lo4, nz1 = nz ? hi5 : lo5, fz0 = nz ? lo4 : hi4, fz1 = nz ? lo5 : hi5;
	// Plane distance t = (q 2^e + origin - o) / d as one FMA per plane,
	// fma(q, 2^e / d, (origin - o) / d): 2^e / d is exact (power of two), so
	// the error is the rounding of (origin - o) / d, a world-space error of
	// about |origin - o| 2^-24; the quantizer pads every box by one step
	// (at least 1/256 of the node's extent), far more than that for rays
	// inside the scene, so the test stays conservative.
	const float ax = scx * r.ix, ay = scy * r.iy, az = scz * r.iz;
	const float bx = (ox - r.o.x) * r.ix, by = (oy - r.o.y) * r.iy, bz = (oz - r.o.z) * r.iz;
	uint32_t mask = 0;
#pragma unroll
	for (int c = 0; c < 8; ++c)
	{
		const float tnx = __fmaf_rn(planeQ(nx0, nx1, c), ax, bx);
		const float tfx = __fmaf_rn(planeQ(fx0, fx1, c), ax, bx);
		const float tny = __fmaf_rn(planeQ(ny0, ny1, c), ay, by);
		const float tfy = __fmaf_rn(planeQ(fy0, fy1, c), ay, by);
		const float tnz = __fmaf_rn(planeQ(nz0, nz1, c), az, bz);
		const float tfz = __fmaf_rn(planeQ(fz0, fz1, c), az, bz);
		const float n = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
		const float f = fminf(fminf(tfx, tfy), fminf(tfz, tmax)) * 1.0000004f;
		tnear[c] = n;
		if (n <= f) mask |= 1u << c;
	}
	return mask;
}

// Integer-key form for the near-to-far order: key = entry distance bits
// with the low 3 mantissa bits replaced by the child slot (entry distances
// are >= 0, so their bit patterns order like the values), 0xFFFFFFF8 | slot
// for a child that is not entered. One min and one max per comparator.
RB_D void cswapU(uint32_t& a, uint32_t& b)
{
	const uint32_t lo = min(a, b), hi = max(a, b);
	a = lo;
	b = hi;
}
RB_D void sort8u(uint32_t k[8])
{
	cswapU(k[0], k[2]); cswapU(k[1], k[3]); cswapU(k[4], k[6]); cswapU(k[5], k[7]);
	cswapU(k[0], k[4]); cswapU(k[1], k[5]); cswapU(k[2], k[6]); cswapU(k[3], k[7]);
	cswapU(k[0], k[1]); cswapU(k[2], k[3]); cswapU(k[4], k[5]); cswapU(k[6], k[7]);
	cswapU(k[2], k[4]); cswapU(k[3], k[5]);
	cswapU(k[1], k[4]); cswapU(k[3], k[6]);
	cswapU(k[1], k[2]); cswapU(k[3], k[4]); cswapU(k[5], k[6]);
}
// Child reference of slot s (0..7) chosen at run time.
RB_D uint32_t nodeChildAt(const NodeView& v, uint32_t s)
{
	const float4 a = s < 4u ? v.q[1] : v.q[2];
	const uint32_t k = s & 3u;
	return __float_as_uint(k == 0u ? a.x : (k == 1u ? a.y : (k == 2u ? a.z : a.w)));
}

// Visit-order mask of a hit mask: bit v of the result is slot (v ^ oct).
RB_D uint32_t visitOrder(uint32_t m, uint32_t oct)
{
	if (oct & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
	if (oct & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
	if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu);
	return m;
}

struct Hit
{
	int32_t tri;       // BVH-order triangle index, -1 on a miss
	float t, b1, b2;
};

// Closest-hit traversal on (tmin, tmax) as a resumable state: run() visits
// at most `budget` nodes or leaves and returns true once the traversal has
// ended, so a persistent warp can hand an idle lane a new ray between calls.
// Sets RB_DEV_STACK_OVERFLOW in *status and keeps the best hit so far if the
// stack runs out. With COUNT, nNodes and nTris count the wide nodes loaded and
// triangles tested.
struct ClosestTraversal
{
	TraceRay r;
	float tmin;
	Hit best;
	uint32_t bestId;
	uint32_t cur;
	uint32_t leaf;         // postponed leaf (RB_TRAV_POSTPONE): its untested triangles, 0 for none
	int sp;
	bool done;

	RB_D void init(const DevGeometry& g, f3 o, f3 d, float tmin_, float tmax)
	{
		leaf = 0u;
		best = Hit{ -1, tmax, 0.0f, 0.0f };
		bestId = 0xFFFFFFFFu;
		tmin = tmin_;
		sp = 0;
		done = g.triCount == 0;
		r = makeTraceRay(o, d);
		cur = g.rootIsLeaf ? (kLeafBit | (static_cast<uint32_t>(g.triCount - 1) << 28)) : 0u;
	}

	// Intersects the triangles of the leaf `cur`.
	template<bool COUNT>
	RB_D void leafStep(const DevGeometry& g, uint32_t& nTris)
	{
		const uint32_t first = cur & 0x0FFFFFFFu;
		const uint32_t count = ((cur >> 28) & 0x7u) + 1u;
		if (COUNT) nTris += count;
		for (uint32_t i = first; i < first + count; ++i)
		{
			const float4 a = __ldg(g.triVerts + 3 * i);
			const float4 b = __ldg(g.triVerts + 3 * i + 1);
			const float4 c = __ldg(g.triVerts + 3 * i + 2);
			float t, u, v;
			if (intersectTriangle(r, f3_of(a), f3_of(b), f3_of(c), tmin, best.t, best.tri >= 0, t, u, v))
			{
				const uint32_t id = __float_as_uint(a.w);
				if (best.tri < 0 || t < best.t || id < bestId)
				{
					best = Hit{ static_cast<int32_t>(i), t, u, v };
					bestId = id;
				}
			}
		}
	}

	// Tests the children of the interior node `cur`; descends into the
	// nearest one entered (returns true) after pushing the others, farthest
	// first. Returns false when no child is entered.
	// Stack entries: (child reference, entry-distance bits, truncated down:
	// popping compares a value <= the true distance, so culling stays
	// conservative).
	template<bool COUNT, class Stack>
	RB_D bool nodeStep(const DevGeometry& g, uint32_t* status, uint32_t& nNodes, Stack& stack)
	{
		if (COUNT) ++nNodes;
		const NodeView nv = loadNode(g.nodes, cur);
		float tn[8];
		const uint32_t mask = childBoxes(r, nv, tmin, best.t, tn);
		if (!mask) return false;
#if RB_TRAV_SORT == 2
		// visit index of slot c is c ^ oct; the children after the first are
		// pushed so that the stack top holds the next one to visit
		const uint32_t om = visitOrder(mask, r.oct);
		const uint32_t firstV = static_cast<uint32_t>(__ffs(static_cast<int>(om)) - 1);
		const uint32_t rest = om & (om - 1u);
		const int nPush = __popc(rest);
		if (sp + nPush <= static_cast<int>(g.stackLimit))
		{
#pragma unroll
			for (int c = 0; c < 8; ++c)
			{
				const uint32_t v = static_cast<uint32_t>(c) ^ r.oct;
				if ((rest >> v) & 1u)
					stack[sp + __popc(rest >> (v + 1u))] = make_uint2(nodeChild(nv, c), __float_as_uint(tn[c]));
			}
			sp += nPush;
		}
		else if (nPush) atomicOr(status, RB_DEV_STACK_OVERFLOW);
		cur = nodeChildAt(nv, firstV ^ r.oct);
		if (cur == kEmptyChild) return false;
#elif RB_TRAV_SORT
		uint32_t key[8];
#pragma unroll
		for (int c = 0; c < 8; ++c)
			key[c] = ((mask >> c) & 1u) ? ((__float_as_uint(tn[c]) & 0x7FFFFFF8u) | static_cast<uint32_t>(c))
				: (0xFFFFFFF8u | static_cast<uint32_t>(c));
		sort8u(key);
		const int n = __popc(mask);
#pragma unroll
		for (int c = 7; c >= 1; --c)
		{
			if (c < n)
			{
				if (sp < static_cast<int>(g.stackLimit)) { stack[sp] = make_uint2(nodeChildAt(nv, key[c] & 7u), key[c] & ~7u); ++sp; }
				else atomicOr(status, RB_DEV_STACK_OVERFLOW);
			}
		}
		cur = nodeChildAt(nv, key[0] & 7u);
		if (cur == kEmptyChild) return false;
#else
		int nearest = 0;
		float nk = INFINITY;
#pragma unroll
		for (int c = 0; c < 8; ++c)
			if (((mask >> c) & 1u) && tn[c] < nk) { nk = tn[c]; nearest = c; }
#pragma unroll
		for (int c = 7; c >= 0; --c)
		{
			if (((mask >> c) & 1u) && c != nearest)
			{
				if (sp < static_cast<int>(g.stackLimit)) { stack[sp] = make_uint2(nodeChild(nv, c), __float_as_uint(tn[c])); ++sp; }
				else atomicOr(status, RB_DEV_STACK_OVERFLOW);
			}
		}
		cur = nodeChild(nv, nearest);
		if (cur == kEmptyChild) return false;
#endif
		return true;
	}

	// Pops the next entry that may still hold a closer hit; false when none is left.
	template<class Stack>
	RB_D bool pop(Stack& stack)
	{
		while (sp > 0)
		{
			--sp;
			const uint2 e = stack[sp];
			if (__uint_as_float(e.y) <= best.t && e.x != kEmptyChild) { cur = e.x; return true; }
		}
		return false;
	}

	// The stack lives outside the state (separate local arrays) so that the
	// scalar state can stay in registers.
	template<bool COUNT, class Stack>
	RB_D bool run(const DevGeometry& g, int budget, uint32_t* status, uint32_t& nNodes, uint32_t& nTris, Stack& stack)
	{
#if RB_TRAV_WHILE_WHILE
		// interior nodes until a leaf, then the leaf: lanes of a warp meet at
		// the leaf code instead of alternating node and leaf steps
		int it = 0;
		while (it < budget && !done)
		{
			while (!(cur & kLeafBit) && it < budget)
			{
				++it;
				if (!nodeStep<COUNT>(g, status, nNodes, stack) && !pop(stack))
				{
					done = true;
					break;
				}
			}
			if (done || it >= budget) break;
			++it;
			leafStep<COUNT>(g, nTris);
			if (!pop(stack)) done = true;
		}
#elif RB_TRAV_POSTPONE
		// cur: an interior node, a leaf, or kEmptyChild when no node is left
		for (int it = 0; it < budget && !done; ++it)
		{
			if ((cur & kLeafBit) && cur != kEmptyChild && leaf == 0u)
			{
				leaf = cur;                              // keep the leaf aside
				if (!pop(stack)) cur = kEmptyChild;
			}
			const bool noNode = (cur & kLeafBit) != 0u;  // nothing, or a second leaf
			if (noNode && leaf == 0u)
			{
				done = true;
				break;
			}
			const unsigned am = __activemask();
			const unsigned holding = __ballot_sync(am, leaf != 0u);
			const unsigned stuck = __ballot_sync(am, noNode);
			if (stuck || 2 * __popc(holding) >= __popc(am))
			{
				if (leaf) triangleStep<COUNT>(g, nTris);
			}
			else if (!nodeStep<COUNT>(g, status, nNodes, stack) && !pop(stack))
			{
				cur = kEmptyChild;
			}
		}
#else
		for (int it = 0; it < budget && !done; ++it)
		{
			if (cur & kLeafBit)
			{
				leafStep<COUNT>(g, nTris);
				if (!pop(stack)) done = true;
			}
			else if (!nodeStep<COUNT>(g, status, nNodes, stack) && !pop(stack))
			{
				done = true;
			}
		}
#endif
		return done;
	}

	// Tests the first untested triangle of the postponed leaf and advances it.
	template<bool COUNT>
	RB_D void triangleStep(const DevGeometry& g, uint32_t& nTris)
	{
		const uint32_t i = leaf & 0x0FFFFFFFu;
		const uint32_t left = (leaf >> 28) & 0x7u;       // triangles after this one
		if (COUNT) ++nTris;
		const float4 a = __ldg(g.triVerts + 3 * i);
		const float4 b = __ldg(g.triVerts + 3 * i + 1);
		const float4 c = __ldg(g.triVerts + 3 * i + 2);
		float t, u, v;
		if (intersectTriangle(r, f3_of(a), f3_of(b), f3_of(c), tmin, best.t, best.tri >= 0, t, u, v))
		{
			const uint32_t id = __float_as_uint(a.w);
			if (best.tri < 0 || t < best.t || id < bestId)
			{
				best = Hit{ static_cast<int32_t>(i), t, u, v };
				bestId = id;
			}
		}
		leaf = left ? (kLeafBit | ((left - 1u) << 28) | (i + 1u)) : 0u;
	}
};

// Any-hit traversal on (tmin, tmax), resumable like ClosestTraversal:
// occlusion test of a shadow ray.
struct AnyTraversal
{
	TraceRay r;
	float tmin, tmax;
	uint32_t cur;
	int sp;
	bool done, hit;

	RB_D void init(const DevGeometry& g, f3 o, f3 d, float tmin_, float tmax_)
	{
		tmin = tmin_;
		tmax = tmax_;
		sp = 0;
		hit = false;
		done = g.triCount == 0;
		r = makeTraceRay(o, d);
		cur = g.rootIsLeaf ? (kLeafBit | (static_cast<uint32_t>(g.triCount - 1) << 28)) : 0u;
	}

	template<bool COUNT, class Stack>
	RB_D bool run(const DevGeometry& g, int budget, uint32_t* status, uint32_t& nNodes, uint32_t& nTris, Stack& stack)
	{
		for (int it = 0; it < budget && !done; ++it)
		{
			if (cur == kEmptyChild)
			{
				// an empty slot entered through a flattened box: nothing to test
			}
			else if (cur & kLeafBit)
			{
				const uint32_t first = cur & 0x0FFFFFFFu;
				const uint32_t count = ((cur >> 28) & 0x7u) + 1u;
				for (uint32_t i = first; i < first + count; ++i)
				{
					if (COUNT) ++nTris;
					const float4 a = __ldg(g.triVerts + 3 * i);
					const float4 b = __ldg(g.triVerts + 3 * i + 1);
					const float4 c = __ldg(g.triVerts + 3 * i + 2);
					float t, u, v;
					if (intersectTriangle(r, f3_of(a), f3_of(b), f3_of(c), tmin, tmax, false, t, u, v))
					{
						hit = true;
						done = true;
						break;
					}
				}
				if (done) break;
			}
			else
			{
				if (COUNT) ++nNodes;
				const NodeView nv = loadNode(g.nodes, cur);
				float tn[8];
				const uint32_t mask = childBoxes(r, nv, tmin, tmax, tn);
#pragma unroll
				for (int c = 0; c < 8; ++c)
				{
					if ((mask >> c) & 1u)
					{
						if (sp < static_cast<int>(g.stackLimit)) stack[sp++] = nodeChild(nv, c);
						else atomicOr(status, RB_DEV_STACK_OVERFLOW);
					}
				}
			}
			if (sp == 0) { done = true; break; }
			cur = stack[--sp];
		}
		return done;
	}
};

// ---------------------------------------------------------------------------
// Two-level traversal (RB_ACCEL_INSTANCED). The top level's leaves hold
// instances; entering one pushes a return marker, takes the ray into the
// instance's object space for the box tests of its unit's BVH, and popping
// the marker brings the world ray back. Triangles are intersected in world
// space, each transformed with the flat upload's arithmetic
// (instancedTriangle), so hits equal the flat structure's bit for bit. The
// other instances of a top-level leaf wait on the stack as instance entries.
constexpr uint32_t kInstanceEntry = 0x40000000u;   // | position; node indices stay below 2^24
constexpr uint32_t kReturnEntry = 0x7FFFFFFFu;
constexpr uint32_t kNoInstance = 0xFFFFFFFFu;

RB_D bool isInstanceEntry(uint32_t e) { return (e >> 30) == 1u; }

struct ClosestTraversal2 : ClosestTraversal
{
	TraceRay rw;               // the world ray
	uint32_t inst;             // position of the instance being traversed, kNoInstance at the top level
	uint32_t bestInst;

	RB_D void init(const DevGeometry& g, f3 o, f3 d, float tmin_, float tmax)
	{
		leaf = 0u;
		best = Hit{ -1, tmax, 0.0f, 0.0f };
		bestId = 0xFFFFFFFFu;
		bestInst = 0u;
		tmin = tmin_;
		sp = 0;
		done = g.instanceCount == 0;
		rw = makeTraceRay(o, d);
		r = rw;
		inst = kNoInstance;
		cur = g.topRoot;
	}

	// Takes the ray into instance `pos`; false when the stack has no room
	// for the return marker.
	template<class Stack>
	RB_D bool enter(const DevGeometry& g, uint32_t* status, uint32_t pos, Stack& stack)
	{
		if (sp >= static_cast<int>(g.stackLimit)) { atomicOr(status, RB_DEV_STACK_OVERFLOW); return false; }
		stack[sp++] = make_uint2(kReturnEntry, 0u);
		const DevInstance& in = g.instances[pos];
		const float4 o = make_float4(rw.o.x, rw.o.y, rw.o.z, 0.0f);
		r = makeBoxRay(xfPoint(in.wi, o), xfDir(in.wi, rw.d));
		inst = pos;
		cur = __ldg(&in.root);
		return true;
	}

	// A top-level leaf: its first instance is entered, the others wait.
	template<class Stack>
	RB_D bool instanceLeaf(const DevGeometry& g, uint32_t* status, Stack& stack)
	{
		const uint32_t first = cur & 0x0FFFFFFFu;
		const uint32_t count = ((cur >> 28) & 0x7u) + 1u;
		for (uint32_t k = count - 1; k >= 1; --k)
		{
			if (sp < static_cast<int>(g.stackLimit)) stack[sp++] = make_uint2(kInstanceEntry | (first + k), 0u);
			else atomicOr(status, RB_DEV_STACK_OVERFLOW);
		}
		return enter(g, status, first, stack);
	}

	template<bool COUNT>
	RB_D void leafStep(const DevGeometry& g, uint32_t& nTris)
	{
		const uint32_t first = cur & 0x0FFFFFFFu;
		const uint32_t count = ((cur >> 28) & 0x7u) + 1u;
		if (COUNT) nTris += count;
		for (uint32_t i = first; i < first + count; ++i)
		{
			float4 a, b, c;
			instancedVerts(g, i, inst, a, b, c);
			float t, u, v;
			if (intersectTriangle(rw, f3_of(a), f3_of(b), f3_of(c), tmin, best.t, best.tri >= 0, t, u, v))
			{
				const uint32_t id = __float_as_uint(a.w);
				if (best.tri < 0 || t < best.t || id < bestId)
				{
					best = Hit{ static_cast<int32_t>(i), t, u, v };
					bestId = id;
					bestInst = inst;
				}
			}
		}
	}

	template<class Stack>
	RB_D bool pop(const DevGeometry& g, uint32_t* status, Stack& stack)
	{
		while (sp > 0)
		{
			--sp;
			const uint2 e = stack[sp];
			if (e.x == kReturnEntry) { r = rw; inst = kNoInstance; continue; }
			if (isInstanceEntry(e.x))
			{
				if (enter(g, status, e.x & 0x00FFFFFFu, stack)) return true;
				continue;
			}
			if (__uint_as_float(e.y) <= best.t && e.x != kEmptyChild) { cur = e.x; return true; }
		}
		return false;
	}

	template<bool COUNT, class Stack>
	RB_D bool run(const DevGeometry& g, int budget, uint32_t* status, uint32_t& nNodes, uint32_t& nTris, Stack& stack)
	{
		for (int it = 0; it < budget && !done; ++it)
		{
			if (cur == kEmptyChild)
			{
				if (!pop(g, status, stack)) done = true;
			}
			else if (cur & kLeafBit)
			{
				if (inst == kNoInstance)
				{
					if (!instanceLeaf(g, status, stack) && !pop(g, status, stack)) done = true;
				}
				else
				{
					leafStep<COUNT>(g, nTris);
					if (!pop(g, status, stack)) done = true;
				}
			}
			else if (!nodeStep<COUNT>(g, status, nNodes, stack) && !pop(g, status, stack))
			{
				done = true;
			}
		}
		return done;
	}
};

struct AnyTraversal2 : AnyTraversal
{
	TraceRay rw;
	uint32_t inst;

	RB_D void init(const DevGeometry& g, f3 o, f3 d, float tmin_, float tmax_)
	{
		tmin = tmin_;
		tmax = tmax_;
		sp = 0;
		hit = false;
		done = g.instanceCount == 0;
		rw = makeTraceRay(o, d);
		r = rw;
		inst = kNoInstance;
		cur = g.topRoot;
	}

	template<class Stack>
	RB_D bool enter(const DevGeometry& g, uint32_t* status, uint32_t pos, Stack& stack)
	{
		if (sp >= static_cast<int>(g.stackLimit)) { atomicOr(status, RB_DEV_STACK_OVERFLOW); return false; }
		stack[sp++] = kReturnEntry;
		const DevInstance& in = g.instances[pos];
		const float4 o = make_float4(rw.o.x, rw.o.y, rw.o.z, 0.0f);
		r = makeBoxRay(xfPoint(in.wi, o), xfDir(in.wi, rw.d));
		inst = pos;
		cur = __ldg(&in.root);
		return true;
	}

	template<bool COUNT, class Stack>
	RB_D bool run(const DevGeometry& g, int budget, uint32_t* status, uint32_t& nNodes, uint32_t& nTris, Stack& stack)
	{
		for (int it = 0; it < budget && !done; ++it)
		{
			bool next = true;        // take the next entry from the stack after this step
			if (cur == kEmptyChild)
			{
			}
			else if ((cur & kLeafBit) && inst == kNoInstance)
			{
				const uint32_t first = cur & 0x0FFFFFFFu;
				const uint32_t count = ((cur >> 28) & 0x7u) + 1u;
				for (uint32_t k = count - 1; k >= 1; --k)
				{
					if (sp < static_cast<int>(g.stackLimit)) stack[sp++] = kInstanceEntry | (first + k);
					else atomicOr(status, RB_DEV_STACK_OVERFLOW);
				}
				next = !enter(g, status, first, stack);
			}
			else if (cur & kLeafBit)
			{
				const uint32_t first = cur & 0x0FFFFFFFu;
				const uint32_t count = ((cur >> 28) & 0x7u) + 1u;
				for (uint32_t i = first; i < first + count; ++i)
				{
					if (COUNT) ++nTris;
					float4 a, b, c;
					instancedVerts(g, i, inst, a, b, c);
					float t, u, v;
					if (intersectTriangle(rw, f3_of(a), f3_of(b), f3_of(c), tmin, tmax, false, t, u, v))
					{
						hit = true;
						done = true;
						break;
					}
				}
				if (done) break;
			}
			else
			{
				if (COUNT) ++nNodes;
				const NodeView nv = loadNode(g.nodes, cur);
				float tn[8];
				const uint32_t mask = childBoxes(r, nv, tmin, tmax, tn);
#pragma unroll
				for (int c = 0; c < 8; ++c)
				{
					if ((mask >> c) & 1u)
					{
						if (sp < static_cast<int>(g.stackLimit)) stack[sp++] = nodeChild(nv, c);
						else atomicOr(status, RB_DEV_STACK_OVERFLOW);
					}
				}
			}
			if (!next) continue;
			bool found = false;
			while (sp > 0 && !found)
			{
				const uint32_t e = stack[--sp];
				if (e == kReturnEntry) { r = rw; inst = kNoInstance; }
				else if (isInstanceEntry(e)) found = enter(g, status, e & 0x00FFFFFFu, stack);
				else { cur = e; found = true; }
			}
			if (!found) { done = true; break; }
		}
		return done;
	}
};

template<bool COUNT>
RB_D Hit traceClosestT(const DevGeometry& g, f3 o, f3 d, float tmin, float tmax, uint32_t* status,
	uint32_t& nNodes, uint32_t& nTris)
{
	ClosestTraversal tr;
	uint2 stack[kTraversalStack];
	tr.init(g, o, d, tmin, tmax);
	while (!tr.run<COUNT>(g, 1 << 30, status, nNodes, nTris, stack)) {}
	return tr.best;
}

template<bool COUNT>
RB_D bool traceAnyT(const DevGeometry& g, f3 o, f3 d, float tmin, float tmax, uint32_t* status,
	uint32_t& nNodes, uint32_t& nTris)
{
	AnyTraversal tr;
	uint32_t stack[kTraversalStack];
	tr.init(g, o, d, tmin, tmax);
	while (!tr.run<COUNT>(g, 1 << 30, status, nNodes, nTris, stack)) {}
	return tr.hit;
}
RB_D Hit traceClosest(const DevGeometry& g, f3 o, f3 d, float tmin, float tmax, uint32_t* status)
{
	uint32_t a = 0, b = 0;
	return traceClosestT<false>(g, o, d, tmin, tmax, status, a, b);
}
RB_D bool traceAny(const DevGeometry& g, f3 o, f3 d, float tmin, float tmax, uint32_t* status)
{
	uint32_t a = 0, b = 0;
	return traceAnyT<false>(g, o, d, tmin, tmax, status, a, b);
}
} // namespace rb
