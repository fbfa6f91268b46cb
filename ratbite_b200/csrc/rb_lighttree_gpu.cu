// Light-tree construction on the device (no reference counterpart as code:
// the reference builds on the host, LightTree::Builder,
// src/core/light_tree.cpp:47-418, and rb_lighttree.cpp restates that). The
// output has the reference's layouts (PackedNode in depth-first order with
// the right child's index in `core`, LightPointer, 64-bit path masks,
// EmissiveTriangleLightData), so the sampling code cannot tell the two
// builders apart; the tree is a valid binned-SAOH tree, not a byte copy of
// the host one (the host builder's nth_element order is not reproduced).
//
// One block of 1024 threads builds the whole tree, level by level:
//  1. per light: bounds (a flat axis widened by one float epsilon, as the
//     host does), bounds centre, emission direction (normalised edge cross
//     product) and flux;
//  2. per level, one warp per segment of more than 8 lights: for each axis,
//     32 bins over the segment's centre bounds with their bounds, count,
//     flux and direction sums (fixed-point 64-bit integer sums, so results
//     do not depend on the order of the atomics), each bin's orientation
//     cone (the angle to its farthest light), then a sweep over the 31 split
//     planes costing both sides with the SAOH of Conty Estevez and Kulla
//     (2018): flux x box area x orientation measure, the axis cost scaled by
//     the ratio of the largest extent to the axis extent (as the host does);
//     the segment is partitioned stably at the cheapest plane, or halved when
//     no plane separates its lights;
//  3. children are numbered by a block-wide scan in level order, so the
//     build is deterministic;
//  4. subtree sizes bottom-up, depth-first indices top-down, then node
//     attributes bottom-up (NodeAttributes::add, src/core/light_tree_types.h
//     :65-100; leaf attributes as the host's generateLightNodeAttributes and
//     read back through the packed direction, as fillBranchNodeAttributes
//     does), pointers and masks.
// Segments deeper than 36 levels are halved rather than split by cost, so
// even 2^27 lights end within 60 levels and the 64-bit masks suffice.

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "ratbite_b200_kernels.h"
#include "rb_light.cuh"
#include "rb_scene.h"

namespace rb
{
namespace ltg
{
constexpr uint32_t kThreads = 1024;
constexpr uint32_t kWarps = kThreads / 32;
constexpr uint32_t kBins = 32;
constexpr uint32_t kMaxLeaf = 8;
constexpr uint32_t kHalveDepth = 36;
constexpr float kPiF = 3.14159265358979323846f;

// Scratch carved from one caller buffer (rb_k_build_light_tree_scratch_bytes).
struct Scratch
{
	float* lo;          // 3n: bounds
	float* hi;          // 3n
	float* cen;         // 3n: bounds centre
	float* dir;         // 3n: emission direction
	float* flux;        // n
	uint32_t* idx;      // n: light order
	uint32_t* tmp;      // n
	// nodes (at most 2n - 1)
	uint32_t* begin;
	uint32_t* end;
	uint32_t* left;     // child node ids (0: leaf)
	uint32_t* size;     // subtree node count
	uint32_t* pre;      // depth-first index
	uint32_t* split;    // per node of the current level: 1 when split
	uint64_t* mask;
	float* attr;        // 9 per node: mean[3], variance, flux, dir[3], sharpness
	uint32_t* levelStart; // 65 + 1 entries
	uint32_t* counters; // [0] node count, [1] levels
};
__host__ __device__ inline size_t alignUp(size_t v) { return (v + 255) / 256 * 256; }
__host__ __device__ inline size_t scratchBytes(uint32_t n)
{
	const size_t nn = n ? 2 * static_cast<size_t>(n) : 1;
	return alignUp(sizeof(float) * 13 * n) + 2 * alignUp(sizeof(uint32_t) * n) + 6 * alignUp(sizeof(uint32_t) * nn)
		+ alignUp(sizeof(uint64_t) * nn) + alignUp(sizeof(float) * 9 * nn) + alignUp(sizeof(uint32_t) * 72);
}
__host__ __device__ inline Scratch carve(void* p, uint32_t n)
{
	char* c = static_cast<char*>(p);
	const size_t nn = n ? 2 * static_cast<size_t>(n) : 1;
	Scratch s;
	float* f = reinterpret_cast<float*>(c);
	s.lo = f; s.hi = f + 3 * n; s.cen = f + 6 * n; s.dir = f + 9 * n; s.flux = f + 12 * n;
	c += alignUp(sizeof(float) * 13 * n);
	s.idx = reinterpret_cast<uint32_t*>(c); c += alignUp(sizeof(uint32_t) * n);
	s.tmp = reinterpret_cast<uint32_t*>(c); c += alignUp(sizeof(uint32_t) * n);
	uint32_t** arrays[6] = { &s.begin, &s.end, &s.left, &s.size, &s.pre, &s.split };
	for (uint32_t** a : arrays) { *a = reinterpret_cast<uint32_t*>(c); c += alignUp(sizeof(uint32_t) * nn); }
	s.mask = reinterpret_cast<uint64_t*>(c); c += alignUp(sizeof(uint64_t) * nn);
	s.attr = reinterpret_cast<float*>(c); c += alignUp(sizeof(float) * 9 * nn);
	s.levelStart = reinterpret_cast<uint32_t*>(c);
	s.counters = s.levelStart + 68;
	return s;
}

// ---- ordered keys for float min / max with integer atomics
__device__ __forceinline__ uint32_t okey(float f)
{
	const uint32_t b = __float_as_uint(f);
	return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ofloat(uint32_t k)
{
	return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// ---- the host builder's attribute arithmetic (rb_lighttree.cpp)
struct Attr
{
	float mean[3], variance, flux, dir[3], sharpness;
};
__device__ float axisLengthToSharpness(float l) { return l * (3.0f - l * l) / (1.0f - l * l); }
__device__ float sharpnessToAxisLength(float s)
{
	const float a = s / 3.0f;
	const float b = a * a * a;
	const float c = sqrtf(1.0f + 3.0f * (a * a) * (1.0f + a * a));
	const float theta = atan2f(c, b) / 3.0f;
	const float sqrt3 = 1.7320508075688772935274463415059f;
	const float d = sinf(theta) * sqrt3 - cosf(theta);
	return (s > 0x1.0p25f) ? 1.0f : sqrtf(1.0f + a * a) * d + a;
}
__device__ Attr add(const Attr& A, const Attr& B)
{
	Attr r;
	const float wa = A.flux / (A.flux + B.flux);
	const float wb = B.flux / (A.flux + B.flux);
	const float la = sharpnessToAxisLength(A.sharpness);
	const float lb = sharpnessToAxisLength(B.sharpness);
	float d[3] = { wa * la * A.dir[0] + wb * lb * B.dir[0], wa * la * A.dir[1] + wb * lb * B.dir[1],
	               wa * la * A.dir[2] + wb * lb * B.dir[2] };
	const float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
	for (int k = 0; k < 3; ++k) d[k] = len > 0.0001f ? d[k] / len : 0.0f;
	const float dm[3] = { B.mean[0] - A.mean[0], B.mean[1] - A.mean[1], B.mean[2] - A.mean[2] };
	const float dm2 = dm[0] * dm[0] + dm[1] * dm[1] + dm[2] * dm[2];
	for (int k = 0; k < 3; ++k) r.mean[k] = wa * A.mean[k] + wb * B.mean[k];
	r.variance = wa * A.variance + wb * B.variance + wa * wb * dm2;
	for (int k = 0; k < 3; ++k) r.dir[k] = d[k];
	r.flux = A.flux + B.flux;
	r.sharpness = axisLengthToSharpness(len);
	return r;
}
__device__ void normalizedCross(const float a[3], const float b[3], float out[3])
{
	const float c[3] = { a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1] };
	const float inv = 1.0f / sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
	for (int k = 0; k < 3; ++k) out[k] = c[k] * inv;
}
__device__ Attr leafAttr(const float* v, float flux)
{
	const float e1[3] = { v[3] - v[0], v[4] - v[1], v[5] - v[2] };
	const float e2[3] = { v[6] - v[0], v[7] - v[1], v[8] - v[2] };
	Attr a;
	normalizedCross(e1, e2, a.dir);
	for (int k = 0; k < 3; ++k) a.mean[k] = (v[k] + v[3 + k] + v[6 + k]) / 3.0f;
	a.variance = ((e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]) + (e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2])
		- (e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2])) / 18.0f;
	a.sharpness = axisLengthToSharpness(0.5f);
	a.flux = flux;
	return a;
}
__device__ void storeAttr(float* dst, const Attr& a)
{
	dst[0] = a.mean[0]; dst[1] = a.mean[1]; dst[2] = a.mean[2]; dst[3] = a.variance; dst[4] = a.flux;
	dst[5] = a.dir[0]; dst[6] = a.dir[1]; dst[7] = a.dir[2]; dst[8] = a.sharpness;
}
__device__ Attr loadAttr(const float* s)
{
	Attr a;
	a.mean[0] = s[0]; a.mean[1] = s[1]; a.mean[2] = s[2]; a.variance = s[3]; a.flux = s[4];
	a.dir[0] = s[5]; a.dir[1] = s[6]; a.dir[2] = s[7]; a.sharpness = s[8];
	return a;
}

// SAOH of a side (Conty Estevez and Kulla 2018): flux x area x orientation
// measure of the cone (theta_o = acos(cosTheta), theta_e = pi / 2).
__device__ float saoh(const float lo[3], const float hi[3], float flux, float cosTheta)
{
	float area = 0.0f;
	if (lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2])
	{
		const float d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
		area = 2.0f * (d0 * d1 + d0 * d2 + d1 * d2);
	}
	const float thetaO = acosf(fmaxf(fminf(cosTheta, 1.0f), -1.0f));
	const float thetaW = fminf(thetaO + kPiF / 2.0f, kPiF);
	const float so = sinf(thetaO), co = cosf(thetaO);
	const float orient = 2.0f * kPiF * (1.0f - co)
		+ kPiF / 2.0f * (2.0f * thetaW * so - cosf(thetaO - 2.0f * thetaW) - 2.0f * thetaO * so + co);
	return flux * area * orient;
}

// Per-warp bins of one axis in shared memory.
struct WarpBins
{
	uint32_t lo[3][kBins], hi[3][kBins];   // ordered keys
	uint32_t count[kBins];
	unsigned long long flux[kBins];        // fixed point
	unsigned long long cone[3][kBins];     // fixed point (two's complement)
	uint32_t cosMin[kBins];                // ordered key of the smallest cosine to the bin direction
};
constexpr double kConeScale = 4294967296.0;     // 2^32: sums of up to 2^27 unit components fit

// Cheapest split of segment [b, e) of idx (one warp). Returns the axis and
// the number of lights left of the plane (0 when no plane separates them);
// *bin receives the last bin of the left side.
__device__ uint32_t findSplit(const Scratch& S, uint32_t b, uint32_t e, WarpBins& W, uint32_t& axisOut, uint32_t& binOut)
{
	const uint32_t lane = threadIdx.x & 31u;
	// centre bounds, light bounds and the largest flux of the segment
	float cmin[3] = { INFINITY, INFINITY, INFINITY }, cmax[3] = { -INFINITY, -INFINITY, -INFINITY };
	float bmin[3] = { INFINITY, INFINITY, INFINITY }, bmax[3] = { -INFINITY, -INFINITY, -INFINITY };
	float fmax_ = 0.0f;
	for (uint32_t i = b + lane; i < e; i += 32)
	{
		const uint32_t l = S.idx[i];
		for (int k = 0; k < 3; ++k)
		{
			cmin[k] = fminf(cmin[k], S.cen[3 * l + k]); cmax[k] = fmaxf(cmax[k], S.cen[3 * l + k]);
			bmin[k] = fminf(bmin[k], S.lo[3 * l + k]); bmax[k] = fmaxf(bmax[k], S.hi[3 * l + k]);
		}
		fmax_ = fmaxf(fmax_, S.flux[l]);
	}
	for (int o = 16; o; o >>= 1)
	{
		for (int k = 0; k < 3; ++k)
		{
			cmin[k] = fminf(cmin[k], __shfl_xor_sync(0xFFFFFFFFu, cmin[k], o));
			cmax[k] = fmaxf(cmax[k], __shfl_xor_sync(0xFFFFFFFFu, cmax[k], o));
			bmin[k] = fminf(bmin[k], __shfl_xor_sync(0xFFFFFFFFu, bmin[k], o));
			bmax[k] = fmaxf(bmax[k], __shfl_xor_sync(0xFFFFFFFFu, bmax[k], o));
		}
		fmax_ = fmaxf(fmax_, __shfl_xor_sync(0xFFFFFFFFu, fmax_, o));
	}
	const float dims[3] = { bmax[0] - bmin[0], bmax[1] - bmin[1], bmax[2] - bmin[2] };
	const uint32_t largest = dims[0] > dims[1] && dims[0] > dims[2] ? 0u : (dims[1] > dims[2] ? 1u : 2u);
	const double fluxScale = fmax_ > 0.0f ? 1099511627776.0 / static_cast<double>(fmax_) / static_cast<double>(e - b) : 0.0;
	float bestCost = FLT_MAX;
	uint32_t bestAxis = 0, bestBin = 0, bestLeft = 0;
	for (uint32_t axis = 0; axis < 3; ++axis)
	{
		const float w = cmax[axis] - cmin[axis];
		if (!(w > 0.0f) || !(dims[axis] > 0.0f)) continue;
		const float scale = static_cast<float>(kBins) / w;
		auto binOf = [&](uint32_t l) {
			const float c = S.cen[3 * l + axis];
			return min(static_cast<uint32_t>(fmaxf((c - cmin[axis]) * scale, 0.0f)), kBins - 1u);
		};
		// clear this warp's bins (lane = bin)
		for (int k = 0; k < 3; ++k)
		{
			W.lo[k][lane] = 0xFFFFFFFFu; W.hi[k][lane] = 0u; W.cone[k][lane] = 0ull;
		}
		W.count[lane] = 0u; W.flux[lane] = 0ull; W.cosMin[lane] = 0xFFFFFFFFu;
		__syncwarp();
		for (uint32_t i = b + lane; i < e; i += 32)
		{
			const uint32_t l = S.idx[i], bin = binOf(l);
			for (int k = 0; k < 3; ++k)
			{
				atomicMin(&W.lo[k][bin], okey(S.lo[3 * l + k]));
				atomicMax(&W.hi[k][bin], okey(S.hi[3 * l + k]));
				atomicAdd(&W.cone[k][bin], static_cast<unsigned long long>(
					static_cast<long long>(llrint(static_cast<double>(S.dir[3 * l + k]) * kConeScale))));
			}
			atomicAdd(&W.count[bin], 1u);
			atomicAdd(&W.flux[bin], static_cast<unsigned long long>(llrint(static_cast<double>(S.flux[l]) * fluxScale)));
		}
		__syncwarp();
		// bin direction, then its cone: the smallest cosine to a light of the bin
		float bd[3];
		{
			double c[3];
			for (int k = 0; k < 3; ++k) c[k] = static_cast<double>(static_cast<long long>(W.cone[k][lane]));
			const double len = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
			for (int k = 0; k < 3; ++k) bd[k] = len > 0.0 ? static_cast<float>(c[k] / len) : 0.0f;
		}
		for (uint32_t i = b + lane; i < e; i += 32)
		{
			const uint32_t l = S.idx[i], bin = binOf(l);
			// direction of bin `bin` from shared memory
			double c[3];
			for (int k = 0; k < 3; ++k) c[k] = static_cast<double>(static_cast<long long>(W.cone[k][bin]));
			const double len = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
			float cosv = -1.0f;
			if (len > 0.0)
				cosv = static_cast<float>((c[0] * S.dir[3 * l] + c[1] * S.dir[3 * l + 1] + c[2] * S.dir[3 * l + 2]) / len);
			atomicMin(&W.cosMin[bin], okey(fminf(fmaxf(cosv, -1.0f), 1.0f)));
		}
		__syncwarp();
		// this lane's bin
		const uint32_t cnt = W.count[lane];
		const double fl = static_cast<double>(W.flux[lane]);
		float lo[3], hi[3];
		for (int k = 0; k < 3; ++k)
		{
			lo[k] = cnt ? ofloat(W.lo[k][lane]) : INFINITY;
			hi[k] = cnt ? ofloat(W.hi[k][lane]) : -INFINITY;
		}
		const float binTheta = cnt ? acosf(fmaxf(fminf(ofloat(W.cosMin[lane]), 1.0f), -1.0f)) : 0.0f;
		double cs[3];
		for (int k = 0; k < 3; ++k) cs[k] = static_cast<double>(static_cast<long long>(W.cone[k][lane]));
		// inclusive prefix (left sides) and suffix (right sides) by shuffles
		float pl[3], ph[3], sl[3], sh[3];
		double pf = fl, sf = fl, pc[3], sc[3];
		uint32_t pn = cnt, sn = cnt;
		for (int k = 0; k < 3; ++k) { pl[k] = sl[k] = lo[k]; ph[k] = sh[k] = hi[k]; pc[k] = sc[k] = cs[k]; }
		for (int o = 1; o < 32; o <<= 1)
		{
			float tl[3], th[3];
			double tc[3];
			for (int k = 0; k < 3; ++k)
			{
				tl[k] = __shfl_up_sync(0xFFFFFFFFu, pl[k], o); th[k] = __shfl_up_sync(0xFFFFFFFFu, ph[k], o);
				tc[k] = __shfl_up_sync(0xFFFFFFFFu, pc[k], o);
			}
			const double tf = __shfl_up_sync(0xFFFFFFFFu, pf, o);
			const uint32_t tn = __shfl_up_sync(0xFFFFFFFFu, pn, o);
			if (lane >= static_cast<uint32_t>(o))
			{
				for (int k = 0; k < 3; ++k) { pl[k] = fminf(pl[k], tl[k]); ph[k] = fmaxf(ph[k], th[k]); pc[k] += tc[k]; }
				pf += tf;
				pn += tn;
			}
			for (int k = 0; k < 3; ++k)
			{
				tl[k] = __shfl_down_sync(0xFFFFFFFFu, sl[k], o); th[k] = __shfl_down_sync(0xFFFFFFFFu, sh[k], o);
				tc[k] = __shfl_down_sync(0xFFFFFFFFu, sc[k], o);
			}
			const double uf = __shfl_down_sync(0xFFFFFFFFu, sf, o);
			const uint32_t un = __shfl_down_sync(0xFFFFFFFFu, sn, o);
			if (lane + static_cast<uint32_t>(o) < 32u)
			{
				for (int k = 0; k < 3; ++k) { sl[k] = fminf(sl[k], tl[k]); sh[k] = fmaxf(sh[k], th[k]); sc[k] += tc[k]; }
				sf += uf;
				sn += un;
			}
		}
		// cones of both sides: the side's mean direction and the largest
		// angle to it over its bins (bin angle plus the bin's own cone)
		auto sideCos = [&](const double c[3], uint32_t j0, uint32_t j1) {
			const double len = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
			float worst = 0.0f;
			for (uint32_t j = 0; j < 32; ++j)
			{
				const uint32_t nj = __shfl_sync(0xFFFFFFFFu, cnt, j);
				const float bj0 = __shfl_sync(0xFFFFFFFFu, bd[0], j), bj1 = __shfl_sync(0xFFFFFFFFu, bd[1], j);
				const float bj2 = __shfl_sync(0xFFFFFFFFu, bd[2], j), tj = __shfl_sync(0xFFFFFFFFu, binTheta, j);
				if (j < j0 || j > j1 || nj == 0 || !(len > 0.0)) continue;
				const float cj = static_cast<float>((c[0] * bj0 + c[1] * bj1 + c[2] * bj2) / len);
				worst = fmaxf(worst, acosf(fmaxf(fminf(cj, 1.0f), -1.0f)) + tj);
			}
			return len > 0.0 && worst < kPiF ? cosf(worst) : -1.0f;
		};
		const float cosL = sideCos(pc, 0, lane);
		const float cosR = sideCos(sc, lane, 31);
		// cost of the plane after bin `lane`: left = prefix(lane), right = suffix(lane + 1)
		float rl[3], rh[3];
		for (int k = 0; k < 3; ++k) { rl[k] = __shfl_down_sync(0xFFFFFFFFu, sl[k], 1); rh[k] = __shfl_down_sync(0xFFFFFFFFu, sh[k], 1); }
		const double rf = __shfl_down_sync(0xFFFFFFFFu, sf, 1);
		const uint32_t rn = __shfl_down_sync(0xFFFFFFFFu, sn, 1);
		const float rcos = __shfl_down_sync(0xFFFFFFFFu, cosR, 1);
		float cost = FLT_MAX;
		if (lane < 31u && pn > 0u && rn > 0u)
			cost = (saoh(pl, ph, static_cast<float>(pf / fluxScale), cosL)
				+ saoh(rl, rh, static_cast<float>(rf / fluxScale), rcos)) * (dims[largest] / dims[axis]);
		// cheapest plane of the axis (lowest bin on ties)
		float c = cost;
		uint32_t at = lane;
		for (int o = 16; o; o >>= 1)
		{
			const float oc = __shfl_xor_sync(0xFFFFFFFFu, c, o);
			const uint32_t oa = __shfl_xor_sync(0xFFFFFFFFu, at, o);
			if (oc < c || (oc == c && oa < at)) { c = oc; at = oa; }
		}
		const uint32_t leftCount = __shfl_sync(0xFFFFFFFFu, pn, at);
		if (c < bestCost)
		{
			bestCost = c;
			bestAxis = axis;
			bestBin = at;
			bestLeft = leftCount;
		}
		__syncwarp();
	}
	axisOut = bestAxis;
	binOut = bestBin;
	return bestCost < FLT_MAX ? bestLeft : 0u;
}

__global__ void __launch_bounds__(kThreads, 1) kBuildLightTree(uint32_t n, const float* __restrict__ world,
	const float* __restrict__ fluxIn, const uint32_t* __restrict__ material, const uint32_t* __restrict__ prim,
	const float* __restrict__ uvs, float camX, float camY, float camZ, double camXd, double camYd, double camZd, void* scratch,
	EmissiveTri* __restrict__ tris, PackedNode* __restrict__ nodes, uint32_t* __restrict__ pointers,
	uint64_t* __restrict__ masks, uint32_t* __restrict__ nodeCount)
{
	extern __shared__ __align__(16) unsigned char smraw[];
	WarpBins* bins = reinterpret_cast<WarpBins*>(smraw);
	__shared__ uint32_t scan[kThreads];
	__shared__ uint32_t sLevel, sLevelBegin, sLevelEnd, sNodes, sCarry;
	const Scratch S = carve(scratch, n);
	const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
	const double cam[3] = { camXd, camYd, camZd };
	(void)camX; (void)camY; (void)camZ;

	// 1. per-light data (camera-relative, as the host builder computes it)
	for (uint32_t k = t; k < n; k += kThreads)
	{
		const float* v = world + 9 * static_cast<size_t>(k);
		float q[3][3];
		for (int j = 0; j < 3; ++j)
			for (int a = 0; a < 3; ++a) q[j][a] = static_cast<float>(static_cast<double>(v[3 * j + a]) - cam[a]);
		const float e1[3] = { q[1][0] - q[0][0], q[1][1] - q[0][1], q[1][2] - q[0][2] };
		const float e2[3] = { q[2][0] - q[0][0], q[2][1] - q[0][1], q[2][2] - q[0][2] };
		float d[3];
		normalizedCross(e1, e2, d);
		for (int a = 0; a < 3; ++a)
		{
			float lo = fminf(q[0][a], fminf(q[1][a], q[2][a])), hi = fmaxf(q[0][a], fmaxf(q[1][a], q[2][a]));
			if (hi <= lo) { lo = hi - FLT_EPSILON; hi = hi + FLT_EPSILON; }
			S.lo[3 * k + a] = lo;
			S.hi[3 * k + a] = hi;
			S.cen[3 * k + a] = lo + (hi - lo) * 0.5f;
			S.dir[3 * k + a] = d[a];
		}
		S.flux[k] = fluxIn[k];
		S.idx[k] = k;
		EmissiveTri& et = tris[k];
		for (int j = 0; j < 9; ++j) et.v[j] = static_cast<float>(static_cast<double>(v[j]) - cam[j % 3]);
		for (int j = 0; j < 6; ++j) et.uv[j] = uvs ? uvs[6 * static_cast<size_t>(k) + j] : 0.0f;
		et.material = material[k];
		et.prim = prim[k];
	}
	if (t == 0)
	{
		S.begin[0] = 0; S.end[0] = n; S.left[0] = 0; S.mask[0] = 0ull;
		S.levelStart[0] = 0; S.levelStart[1] = 1;
		sLevel = 0; sLevelBegin = 0; sLevelEnd = 1; sNodes = 1;
	}
	__syncthreads();

	// 2-3. levels
	for (;;)
	{
		const uint32_t lb = sLevelBegin, le = sLevelEnd, depth = sLevel;
		if (lb >= le) break;
		for (uint32_t s = lb + warp; s < le; s += kWarps)
		{
			const uint32_t b = S.begin[s], e = S.end[s], cnt = e - b;
			uint32_t nLeft = 0;
			if (cnt > kMaxLeaf)
			{
				uint32_t axis = 0, bin = 0;
				nLeft = depth < kHalveDepth ? findSplit(S, b, e, bins[warp], axis, bin) : 0u;
				if (nLeft > 0 && nLeft < cnt)
				{
					// stable partition through tmp: left lights first
					float cmin = INFINITY, cmax = -INFINITY;
					for (uint32_t i = b + lane; i < e; i += 32)
					{
						const float c = S.cen[3 * S.idx[i] + axis];
						cmin = fminf(cmin, c); cmax = fmaxf(cmax, c);
					}
					for (int o = 16; o; o >>= 1)
					{
						cmin = fminf(cmin, __shfl_xor_sync(0xFFFFFFFFu, cmin, o));
						cmax = fmaxf(cmax, __shfl_xor_sync(0xFFFFFFFFu, cmax, o));
					}
					const float scale = static_cast<float>(kBins) / (cmax - cmin);
					auto goesLeft = [&](uint32_t i, uint32_t& l) {
						l = S.idx[i];
						return min(static_cast<uint32_t>(fmaxf((S.cen[3 * l + axis] - cmin) * scale, 0.0f)), kBins - 1u) <= bin;
					};
					// count first (the binning above decided on the same bins), then place
					uint32_t nl = 0;
					for (uint32_t i0 = b; i0 < e; i0 += 32)
					{
						uint32_t l = 0;
						const bool gl = i0 + lane < e && goesLeft(i0 + lane, l);
						nl += __popc(__ballot_sync(0xFFFFFFFFu, gl));
					}
					if (nl == 0 || nl == cnt) nLeft = cnt / 2;
					else
					{
						nLeft = nl;
						uint32_t lpos = b, rpos = b + nl;
						for (uint32_t i0 = b; i0 < e; i0 += 32)
						{
							const uint32_t i = i0 + lane;
							const bool in = i < e;
							uint32_t l = 0;
							const bool gl = in && goesLeft(i, l);
							const uint32_t ml = __ballot_sync(0xFFFFFFFFu, gl), mr = __ballot_sync(0xFFFFFFFFu, in && !gl);
							const uint32_t below = (1u << lane) - 1u;
							if (gl) S.tmp[lpos + __popc(ml & below)] = l;
							else if (in) S.tmp[rpos + __popc(mr & below)] = l;
							lpos += __popc(ml);
							rpos += __popc(mr);
						}
						__syncwarp();
						for (uint32_t i = b + lane; i < e; i += 32) S.idx[i] = S.tmp[i];
					}
					__syncwarp();
				}
				else nLeft = cnt / 2;                   // no plane separates the lights: halve the range
			}
			if (lane == 0)
			{
				S.split[s] = cnt > kMaxLeaf ? 1u : 0u;
				S.size[s] = nLeft;                      // left count, until the sizes pass
			}
		}
		__syncthreads();
		// number the children in level order: block scan of 2 x split
		if (t == 0) sCarry = 0;
		__syncthreads();
		for (uint32_t c0 = lb; c0 < le; c0 += kThreads)
		{
			const uint32_t s = c0 + t;
			scan[t] = s < le ? 2u * S.split[s] : 0u;
			__syncthreads();
			for (uint32_t o = 1; o < kThreads; o <<= 1)
			{
				const uint32_t v = t >= o ? scan[t - o] : 0u;
				__syncthreads();
				scan[t] += v;
				__syncthreads();
			}
			if (s < le && S.split[s])
			{
				const uint32_t c = sNodes + sCarry + scan[t] - 2u;
				const uint32_t b = S.begin[s], e = S.end[s], nl = S.size[s];
				S.left[s] = c;
				S.begin[c] = b; S.end[c] = b + nl; S.left[c] = 0; S.mask[c] = S.mask[s];
				S.begin[c + 1] = b + nl; S.end[c + 1] = e; S.left[c + 1] = 0;
				S.mask[c + 1] = S.mask[s] | (1ull << depth);
			}
			else if (s < le) S.left[s] = 0;
			__syncthreads();
			if (t == kThreads - 1) sCarry += scan[t];
			__syncthreads();
		}
		if (t == 0)
		{
			sNodes += sCarry;
			sLevelBegin = le;
			sLevelEnd = sNodes;
			sLevel = depth + 1;
			S.levelStart[depth + 2] = sNodes;
		}
		__syncthreads();
	}
	const uint32_t total = sNodes, levels = sLevel;

	// 4. subtree sizes (bottom-up), depth-first indices (top-down)
	for (int d = static_cast<int>(levels) - 1; d >= 0; --d)
	{
		for (uint32_t s = S.levelStart[d] + t; s < S.levelStart[d + 1]; s += kThreads)
			S.size[s] = S.left[s] ? 1u + S.size[S.left[s]] + S.size[S.left[s] + 1] : 1u;
		__syncthreads();
	}
	if (t == 0) S.pre[0] = 0;
	__syncthreads();
	for (uint32_t d = 0; d < levels; ++d)
	{
		for (uint32_t s = S.levelStart[d] + t; s < S.levelStart[d + 1]; s += kThreads)
			if (S.left[s])
			{
				S.pre[S.left[s]] = S.pre[s] + 1u;
				S.pre[S.left[s] + 1] = S.pre[s] + 1u + S.size[S.left[s]];
			}
		__syncthreads();
	}
	// leaves: attributes (world space), pointers, masks; branches: core
	for (uint32_t s = t; s < total; s += kThreads)
	{
		PackedNode& p = nodes[S.pre[s]];
		if (S.left[s])
		{
			p.core = ((1u << 31) - 1u) & S.pre[S.left[s] + 1];
			continue;
		}
		const uint32_t b = S.begin[s], e = S.end[s];
		Attr a = leafAttr(world + 9 * static_cast<size_t>(S.idx[b]), S.flux[S.idx[b]]);
		for (uint32_t i = b + 1; i < e; ++i) a = add(a, leafAttr(world + 9 * static_cast<size_t>(S.idx[i]), S.flux[S.idx[i]]));
		for (int k = 0; k < 3; ++k) p.mean[k] = a.mean[k];
		p.variance = a.variance;
		p.direction = octEncodeU32(mk(a.dir[0], a.dir[1], a.dir[2]));
		p.sharpness = a.sharpness;
		p.flux = a.flux;
		p.core = (1u << 31) | (((e - b) & 0xFu) << 27) | (b & ((1u << 27) - 1u));
		// the branches merge the leaf as read back through its packed form
		const f3 dd = octDecode(static_cast<float>(p.direction & 0xFFFFu) / 65535.0f,
			static_cast<float>(p.direction >> 16) / 65535.0f);
		a.dir[0] = dd.x; a.dir[1] = dd.y; a.dir[2] = dd.z;
		storeAttr(S.attr + 9 * static_cast<size_t>(s), a);
		for (uint32_t i = b; i < e; ++i)
		{
			pointers[i] = (kLightTypeTriangle << 30) | (S.idx[i] & ((1u << 30) - 1u));
			masks[S.idx[i]] = S.mask[s];
		}
	}
	__syncthreads();
	// branch attributes bottom-up
	for (int d = static_cast<int>(levels) - 1; d >= 0; --d)
	{
		for (uint32_t s = S.levelStart[d] + t; s < S.levelStart[d + 1]; s += kThreads)
		{
			if (!S.left[s]) continue;
			const Attr m = add(loadAttr(S.attr + 9 * static_cast<size_t>(S.left[s])),
				loadAttr(S.attr + 9 * static_cast<size_t>(S.left[s] + 1)));
			storeAttr(S.attr + 9 * static_cast<size_t>(s), m);
			PackedNode& p = nodes[S.pre[s]];
			for (int k = 0; k < 3; ++k) p.mean[k] = m.mean[k];
			p.variance = m.variance;
			p.direction = octEncodeU32(mk(m.dir[0], m.dir[1], m.dir[2]));
			p.sharpness = m.sharpness;
			p.flux = m.flux;
		}
		__syncthreads();
	}
	// camera-relative means (the host builder subtracts in double at the end)
	for (uint32_t i = t; i < total; i += kThreads)
		for (int k = 0; k < 3; ++k)
			nodes[i].mean[k] = static_cast<float>(static_cast<double>(nodes[i].mean[k]) - cam[k]);
	if (t == 0) *nodeCount = total;
}
constexpr size_t kSmemBins = sizeof(WarpBins) * kWarps;
} // namespace ltg
} // namespace rb

extern "C" size_t rb_k_build_light_tree_scratch_bytes(uint32_t n) { return rb::ltg::scratchBytes(n); }

extern "C" int rb_k_build_light_tree(uint32_t n, const float* world, const float* flux, const uint32_t* material,
	const uint32_t* primitive, const float* uvs, const double* camera, void* scratch, void* triangles, void* nodes, uint32_t* pointers,
	uint64_t* bitmasks, uint32_t* node_count, void* stream)
{
	if (!camera || !node_count) return RB_ERR_INVALID;
	if (n == 0) return RB_OK;
	if (!world || !flux || !material || !primitive || !scratch || !triangles || !nodes || !pointers || !bitmasks)
		return RB_ERR_INVALID;
	if (n > (1u << 27) - 1u) return RB_ERR_INVALID;
	const cudaStream_t st = static_cast<cudaStream_t>(stream);
	static_assert(rb::ltg::kSmemBins + 4 * rb::ltg::kThreads + 64 <= 227 * 1024, "bins fit in shared memory");
	if (cudaFuncSetAttribute(rb::ltg::kBuildLightTree, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(rb::ltg::kSmemBins)) != cudaSuccess)
		return RB_ERR_CUDA;
	rb::ltg::kBuildLightTree<<<1, rb::ltg::kThreads, rb::ltg::kSmemBins, st>>>(n, world, flux, material, primitive, uvs,
		static_cast<float>(camera[0]), static_cast<float>(camera[1]), static_cast<float>(camera[2]), camera[0], camera[1],
		camera[2], scratch, static_cast<rb::EmissiveTri*>(triangles), static_cast<rb::PackedNode*>(nodes), pointers,
		bitmasks, node_count);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}
