// Quantization of a wide node's child boxes, shared by the host builder
// (rb_bvh_build.cpp) and the device refit (rb_refit.cu) so both write the
// same bytes for the same boxes.
//
// Per axis the node gets a power-of-two scale covering the union of its
// children in 250 steps and at least two float ulps of its coordinates, and an
// origin that is a multiple of the scale, so every decoded plane
// origin + q * scale is exact in float. Child boxes are rounded outward and
// padded by one step, so the quantized box always contains the exact one.
#pragma once

#include <cmath>
#include <cstdint>

#include "rb_scene.h"

#ifndef RB_HD
#define RB_HD __host__ __device__ __forceinline__
#endif

namespace rb
{
// Exponent e (scale 2^e) covering `extent` in 250 steps and at least two ulps of `mag`.
RB_HD int scaleExponent(double extent, double mag)
{
	double need = extent / 250.0;
	const double ulp2 = mag > 0.0 ? ::ldexp(1.0, ::ilogb(mag) - 22) : ::ldexp(1.0, -126);
	need = ::fmax(need, ulp2);
	int e = static_cast<int>(::ceil(::log2(need)));
	while (::ldexp(1.0, e) < need) ++e;
	return e > 127 ? 127 : (e < -126 ? -126 : e);
}

// Fills origin, exponents, child count and the quantized planes of `node`
// from the child boxes lo[c][axis], hi[c][axis] of the slots set in `slots`
// (bit c: slot c holds a child; at least one bit set); child references are
// left to the caller. An empty slot gets an inverted box (low planes 255
// steps, high planes 0), which no ray enters: for either sign of a
// direction component the far-plane distance is then below the near one.
RB_HD void quantizeChildren(uint32_t slots, const double (*lo)[3], const double (*hi)[3], BvhNode& node)
{
	double alo[3] = { INFINITY, INFINITY, INFINITY }, ahi[3] = { -INFINITY, -INFINITY, -INFINITY };
	int n = 0;
	for (int c = 0; c < 8; ++c)
	{
		if (!((slots >> c) & 1u)) continue;
		++n;
		for (int a = 0; a < 3; ++a) { alo[a] = ::fmin(alo[a], lo[c][a]); ahi[a] = ::fmax(ahi[a], hi[c][a]); }
	}
	double origin[3], scale[3];
	for (int a = 0; a < 3; ++a)
	{
		const double mag = ::fmax(::fabs(alo[a]), ::fabs(ahi[a]));
		const int e = scaleExponent(ahi[a] - alo[a], mag);
		scale[a] = ::ldexp(1.0, e);
		origin[a] = ::floor(alo[a] / scale[a]) * scale[a] - scale[a];
		node.origin[a] = static_cast<float>(origin[a]);
		node.exponent[a] = static_cast<uint8_t>(e + 127);
	}
	node.childCount = static_cast<uint8_t>(n);
	for (int c = 0; c < 8; ++c)
		for (int a = 0; a < 3; ++a) { node.qlo[a][c] = 255; node.qhi[a][c] = 0; }
	for (int c = 0; c < 8; ++c)
	{
		if (!((slots >> c) & 1u)) continue;
		for (int a = 0; a < 3; ++a)
		{
			const double ql = ::floor((lo[c][a] - origin[a]) / scale[a]) - 1.0;
			const double qh = ::ceil((hi[c][a] - origin[a]) / scale[a]) + 1.0;
			node.qlo[a][c] = static_cast<uint8_t>(::fmin(::fmax(ql, 0.0), 255.0));
			node.qhi[a][c] = static_cast<uint8_t>(::fmin(::fmax(qh, 0.0), 255.0));
		}
	}
}
} // namespace rb
