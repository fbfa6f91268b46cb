// Two-level geometry (RB_ACCEL_INSTANCED): the world-space form of an
// instance's triangle, computed with the float operations of the host's
// flat upload (rb_context.cpp: toWorld, encodedNormal) in the same order and
// with explicit rounding, so that the traversal intersects, and the shading
// reconstructs, exactly the triangle the flat structure stores.
#pragma once

#include "rb_light.cuh"
#include "rb_math.cuh"
#include "rb_scene.h"

namespace rb
{
// Row `row` of W (3x4, row-major) applied to the point (x, y, z).
RB_D float xfRow(const float* W, float x, float y, float z, int row)
{
	const float* w = W + 4 * row;
	return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, w[0]), __fmul_rn(y, w[1])), __fmul_rn(z, w[2])), w[3]);
}
RB_D f3 xfPoint(const float* W, float4 p)
{
	return mk(xfRow(W, p.x, p.y, p.z, 0), xfRow(W, p.x, p.y, p.z, 1), xfRow(W, p.x, p.y, p.z, 2));
}
// Direction (no translation) through the 3x3 part of W.
RB_D f3 xfDir(const float* W, f3 d)
{
	return mk(d.x * W[0] + d.y * W[1] + d.z * W[2], d.x * W[4] + d.y * W[5] + d.z * W[6],
	          d.x * W[8] + d.y * W[9] + d.z * W[10]);
}
// The encoded world-space geometric normal of an object-space triangle under
// the world-to-object matrix Wi (transposed inverse, correctly rounded
// reciprocal square root, octahedral code).
RB_D uint32_t encodedNormalOf(float4 o0, float4 o1, float4 o2, const float* Wi)
{
	const float ux = __fsub_rn(o1.x, o0.x), uy = __fsub_rn(o1.y, o0.y), uz = __fsub_rn(o1.z, o0.z);
	const float vx = __fsub_rn(o2.x, o0.x), vy = __fsub_rn(o2.y, o0.y), vz = __fsub_rn(o2.z, o0.z);
	const float gx = __fsub_rn(__fmul_rn(uy, vz), __fmul_rn(uz, vy));
	const float gy = __fsub_rn(__fmul_rn(uz, vx), __fmul_rn(ux, vz));
	const float gz = __fsub_rn(__fmul_rn(ux, vy), __fmul_rn(uy, vx));
	const float nx = __fadd_rn(__fadd_rn(__fmul_rn(gx, Wi[0]), __fmul_rn(gy, Wi[4])), __fmul_rn(gz, Wi[8]));
	const float ny = __fadd_rn(__fadd_rn(__fmul_rn(gx, Wi[1]), __fmul_rn(gy, Wi[5])), __fmul_rn(gz, Wi[9]));
	const float nz = __fadd_rn(__fadd_rn(__fmul_rn(gx, Wi[2]), __fmul_rn(gy, Wi[6])), __fmul_rn(gz, Wi[10]));
	const float s = __fadd_rn(__fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)), __fmul_rn(nz, nz));
	const float r = __double2float_rn(__drcp_rn(__dsqrt_rn(static_cast<double>(s))));
	return octEncodeU32(mk(__fmul_rn(nx, r), __fmul_rn(ny, r), __fmul_rn(nz, r)));
}

// The world vertices of triangle `tri` (leaf order) of instance position
// `pos`, with the w lanes of the flat layout (canonical id, instance index,
// hit-group data): what the traversal intersects.
RB_D void instancedVerts(const DevGeometry& g, uint32_t tri, uint32_t pos, float4& a, float4& b, float4& c)
{
	const DevInstance& in = g.instances[pos];
	const float4 o0 = __ldg(g.triVerts + 3 * tri), o1 = __ldg(g.triVerts + 3 * tri + 1), o2 = __ldg(g.triVerts + 3 * tri + 2);
	const f3 w0 = xfPoint(in.xf, o0), w1 = xfPoint(in.xf, o1), w2 = xfPoint(in.xf, o2);
	a = make_float4(w0.x, w0.y, w0.z, __uint_as_float(__ldg(&in.canonBase) + __float_as_uint(o0.w)));
	b = make_float4(w1.x, w1.y, w1.z, __uint_as_float(__ldg(&in.index)));
	c = make_float4(w2.x, w2.y, w2.z, o2.w);
}
// The hit triangle as the flat structure stores it: the world vertices and
// (encoded normal, primitive index).
RB_D void instancedTriangle(const DevGeometry& g, uint32_t tri, uint32_t pos, float4& a, float4& b, float4& c, uint2& aux)
{
	instancedVerts(g, tri, pos, a, b, c);
	const float4 o0 = __ldg(g.triVerts + 3 * tri), o1 = __ldg(g.triVerts + 3 * tri + 1), o2 = __ldg(g.triVerts + 3 * tri + 2);
	aux = make_uint2(encodedNormalOf(o0, o1, o2, g.instances[pos].wi), __ldg(g.triAux + tri).y);
}
} // namespace rb
