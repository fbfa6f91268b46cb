// Device refit of the flattened geometry after the instances move (the
// counterpart of updateInstanceAccelerationStructure,
// src/core/rendering_interface.cpp:943-1063, which the reference runs on every
// camera move because its scene is camera-relative).
//
// 1. kRetransform: per triangle, world vertices from the object-space
//    vertices and the instance's new 3x4 transform, and the encoded geometric
//    normal from the instance's world-to-object matrix, with the float
//    operations of the host upload (and of the reference's closest-hit
//    program, src/kernels/pathtrace.cu:102-148) in the same order. This
//    translation unit is built without multiply-add contraction.
// 2. kRefitLevel: the BVH keeps its topology; nodes are refit bottom-up one
//    depth level per launch, each child's exact box (double) recomputed from
//    its triangles or from the child node's box, and requantized with the
//    builder's own quantizer (rb_bvh_quant.h).

#include <cstdint>

#include "rb_bvh_quant.h"
#include "rb_launch.cuh"
#include "rb_light.cuh"
#include "rb_refit.h"
#include "ratbite_b200.h"

namespace rb
{
namespace
{
RB_D float world1(const float* W, float x, float y, float z, int row)
{
	const float* w = W + 4 * row;
	return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, w[0]), __fmul_rn(y, w[1])), __fmul_rn(z, w[2])), w[3]);
}

__global__ void kRetransform(uint32_t triCount, const float4* __restrict__ objVerts, const float* __restrict__ xf,
	const float* __restrict__ wi, float4* triVerts, uint2* triAux, uint32_t* status)
{
	for (uint32_t t = gtid(); t < triCount; t += gstride())
	{
		const float4 o0 = objVerts[3 * t], o1 = objVerts[3 * t + 1], o2 = objVerts[3 * t + 2];
		float4 a = triVerts[3 * t], b = triVerts[3 * t + 1], c = triVerts[3 * t + 2];
		const uint32_t inst = __float_as_uint(b.w);
		const float* W = xf + 12u * inst;
		a.x = world1(W, o0.x, o0.y, o0.z, 0); a.y = world1(W, o0.x, o0.y, o0.z, 1); a.z = world1(W, o0.x, o0.y, o0.z, 2);
		b.x = world1(W, o1.x, o1.y, o1.z, 0); b.y = world1(W, o1.x, o1.y, o1.z, 1); b.z = world1(W, o1.x, o1.y, o1.z, 2);
		c.x = world1(W, o2.x, o2.y, o2.z, 0); c.y = world1(W, o2.x, o2.y, o2.z, 1); c.z = world1(W, o2.x, o2.y, o2.z, 2);
		if (!isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z) || !isfinite(b.x) || !isfinite(b.y) || !isfinite(b.z)
			|| !isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z))
			atomicOr(status, RB_DEV_BAD_GEOMETRY);
		triVerts[3 * t] = a; triVerts[3 * t + 1] = b; triVerts[3 * t + 2] = c;
		// object-space cross product, transposed inverse, rounded 1/sqrt, octahedral code
		const float* Wi = wi + 12u * inst;
		const float ux = o1.x - o0.x, uy = o1.y - o0.y, uz = o1.z - o0.z;
		const float vx = o2.x - o0.x, vy = o2.y - o0.y, vz = o2.z - o0.z;
		const float gx = uy * vz - uz * vy, gy = uz * vx - ux * vz, gz = ux * vy - uy * vx;
		const float nx = gx * Wi[0] + gy * Wi[4] + gz * Wi[8];
		const float ny = gx * Wi[1] + gy * Wi[5] + gz * Wi[9];
		const float nz = gx * Wi[2] + gy * Wi[6] + gz * Wi[10];
		const float s = nx * nx + ny * ny + nz * nz;
		const float r = static_cast<float>(1.0 / sqrt(static_cast<double>(s)));
		triAux[t].x = octEncodeU32(mk(nx * r, ny * r, nz * r));
	}
}

__global__ void kRefitLevel(const uint32_t* __restrict__ order, uint32_t begin, uint32_t end, BvhNode* nodes,
	const float4* __restrict__ triVerts, double* nodeBox)
{
	for (uint32_t k = begin + gtid(); k < end; k += gstride())
	{
		const uint32_t i = order[k];
		BvhNode node = nodes[i];
		uint32_t slots = 0;
		double lo[8][3], hi[8][3];
		for (int c = 0; c < 8; ++c)
		{
			const uint32_t ref = node.child[c];
			if (ref == kEmptyChild) continue;
			slots |= 1u << c;
			if (ref & kLeafBit)
			{
				const uint32_t first = ref & 0x0FFFFFFFu;
				const uint32_t count = ((ref >> 28) & 0x7u) + 1u;
				for (int a = 0; a < 3; ++a) { lo[c][a] = INFINITY; hi[c][a] = -INFINITY; }
				for (uint32_t t = first; t < first + count; ++t)
					for (int v = 0; v < 3; ++v)
					{
						const float4 p = triVerts[3 * t + v];
						lo[c][0] = fmin(lo[c][0], static_cast<double>(p.x)); hi[c][0] = fmax(hi[c][0], static_cast<double>(p.x));
						lo[c][1] = fmin(lo[c][1], static_cast<double>(p.y)); hi[c][1] = fmax(hi[c][1], static_cast<double>(p.y));
						lo[c][2] = fmin(lo[c][2], static_cast<double>(p.z)); hi[c][2] = fmax(hi[c][2], static_cast<double>(p.z));
					}
			}
			else
			{
				const double* bx = nodeBox + 6u * ref;
				for (int a = 0; a < 3; ++a) { lo[c][a] = bx[a]; hi[c][a] = bx[3 + a]; }
			}
		}
		quantizeChildren(slots, lo, hi, node);
		nodes[i] = node;
		double* me = nodeBox + 6u * i;
		for (int a = 0; a < 3; ++a)
		{
			double l = INFINITY, h = -INFINITY;
			for (int c = 0; c < 8; ++c)
				if ((slots >> c) & 1u) { l = fmin(l, lo[c][a]); h = fmax(h, hi[c][a]); }
			me[a] = l;
			me[3 + a] = h;
		}
	}
}
} // namespace

namespace
{
__global__ void __launch_bounds__(256) kInstanceBoxes(const float4* __restrict__ objVerts, const uint32_t* __restrict__ range,
	const float* __restrict__ xf, float* __restrict__ boxes)
{
	const uint32_t i = blockIdx.x;
	const uint32_t first = range[2 * i], count = range[2 * i + 1];
	const float* W = xf + 12u * i;
	float lo[3] = { INFINITY, INFINITY, INFINITY }, hi[3] = { -INFINITY, -INFINITY, -INFINITY };
	for (uint32_t v = threadIdx.x; v < 3u * count; v += blockDim.x)
	{
		const float4 o = objVerts[3u * first + v];
		for (int k = 0; k < 3; ++k)
		{
			const float w = world1(W, o.x, o.y, o.z, k);
			lo[k] = fminf(lo[k], w);
			hi[k] = fmaxf(hi[k], w);
		}
	}
	__shared__ float red[6][8];
	for (int k = 0; k < 3; ++k)
	{
		for (int o = 16; o > 0; o >>= 1)
		{
			lo[k] = fminf(lo[k], __shfl_xor_sync(0xFFFFFFFFu, lo[k], o));
			hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xFFFFFFFFu, hi[k], o));
		}
	}
	const int warp = threadIdx.x >> 5;
	if ((threadIdx.x & 31) == 0)
		for (int k = 0; k < 3; ++k) { red[k][warp] = lo[k]; red[3 + k][warp] = hi[k]; }
	__syncthreads();
	if (threadIdx.x < 6)
	{
		float r = red[threadIdx.x][0];
		for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w)
			r = threadIdx.x < 3 ? fminf(r, red[threadIdx.x][w]) : fmaxf(r, red[threadIdx.x][w]);
		boxes[6u * i + threadIdx.x] = r;
	}
}
} // namespace

void launchInstanceBoxes(const float4* objVerts, const uint32_t* range, const float* xf, float* boxes, uint32_t n,
	cudaStream_t st)
{
	if (n) kInstanceBoxes<<<n, 256, 0, st>>>(objVerts, range, xf, boxes);
}

void launchRefit(const RefitData& r, DevGeometry& g, const float* xf, const float* wi, uint32_t* status, int smCount,
	cudaStream_t st)
{
	if (g.triCount == 0) return;
	const int cap = (smCount > 0 ? smCount : 148) * 8;
	const int gridT = gridFor(g.triCount) < cap ? gridFor(g.triCount) : cap;
	kRetransform<<<gridT, kThreads, 0, st>>>(g.triCount, r.objVerts, xf, wi, const_cast<float4*>(g.triVerts),
		const_cast<uint2*>(g.triAux), status);
	for (size_t l = 0; l + 1 < r.levelStart.size(); ++l)
	{
		const uint32_t b = r.levelStart[l], e = r.levelStart[l + 1];
		if (e <= b) continue;
		const int grid = gridFor(e - b) < cap ? gridFor(e - b) : cap;
		kRefitLevel<<<grid, kThreads, 0, st>>>(r.order, b, e, const_cast<BvhNode*>(g.nodes), g.triVerts, r.nodeBox);
	}
}
} // namespace rb
