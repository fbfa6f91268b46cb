// Material texture sampling: tex2D<float4> on the reference's material
// textures (CudaCombinedTexture, src/core/texture.h:280-380, sampled at
// src/kernels/pathtrace.cu:1217-1228, 1437-1560, 1640-1650). Normalized
// coordinates with texel centres at (i + 0.5) / width, the texture's
// address mode (wrap, clamp, mirror) and filter (nearest, bilinear), 8-bit
// channels read as normalized floats, the sRGB curve applied per texel
// before filtering (a 256-entry table of IEC 61966-2-1's decode, computed on
// the host in double precision; r alone of a one-channel texture, the colour
// channel of an R8 sRGB format), a one-channel texture read as (r, 0, 0, 0)
// as the texture unit returns it (alpha 0: measured on B200 through a CUDA
// texture object).
// Bilinear weights are FP32 (the texture hardware rounds them to 8-bit
// fixed point; the oracle's parity mode uses FP32 as here).
#pragma once

#include "rb_math.cuh"
#include "rb_scene.h"

namespace rb
{
// Texel index along one axis for the address mode.
RB_D int texAddress(int i, int n, uint32_t mode)
{
	if (mode == RB_TEXADDR_WRAP)
	{
		const int m = i % n;
		return m < 0 ? m + n : m;
	}
	if (mode == RB_TEXADDR_MIRROR)
	{
		int m = i % (2 * n);
		if (m < 0) m += 2 * n;
		return m < n ? m : 2 * n - 1 - m;
	}
	return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
}
// The coordinate the filter works on: wrap takes the fraction, mirror
// reflects into [0, 1], clamp keeps it.
RB_D float texCoord(float u, uint32_t mode)
{
	if (mode == RB_TEXADDR_WRAP) return __fsub_rn(u, floorf(u));
	if (mode == RB_TEXADDR_MIRROR)
	{
		const float f = __fsub_rn(u, __fmul_rn(2.0f, floorf(__fmul_rn(u, 0.5f))));
		return f <= 1.0f ? f : __fsub_rn(2.0f, f);
	}
	return u;
}
RB_D float4 texel(const DevTexture& t, const float* srgb, int x, int y)
{
	const size_t i = static_cast<size_t>(y) * t.width + static_cast<size_t>(x);
	if (t.channels == 1)
		return make_float4(t.srgb ? srgb[t.data[i]] : static_cast<float>(t.data[i]) / 255.0f, 0.0f, 0.0f, 0.0f);
	const uchar4 c = reinterpret_cast<const uchar4*>(t.data)[i];
	if (t.srgb) return make_float4(srgb[c.x], srgb[c.y], srgb[c.z], static_cast<float>(c.w) / 255.0f);
	return make_float4(static_cast<float>(c.x) / 255.0f, static_cast<float>(c.y) / 255.0f,
		static_cast<float>(c.z) / 255.0f, static_cast<float>(c.w) / 255.0f);
}
RB_D float lerpT(float a, float b, float w) { return __fadd_rn(a, __fmul_rn(w, __fsub_rn(b, a))); }

RB_D float4 texSample(const DevScene& sc, uint32_t index, float u, float v)
{
	const DevTexture& t = sc.textures[index];
	const int w = static_cast<int>(t.width), h = static_cast<int>(t.height);
	const float cu = texCoord(u, t.addrU), cv = texCoord(v, t.addrV);
	if (t.filter == RB_TEXFILTER_NEAREST)
	{
		const int x = texAddress(static_cast<int>(floorf(__fmul_rn(cu, static_cast<float>(w)))), w, t.addrU);
		const int y = texAddress(static_cast<int>(floorf(__fmul_rn(cv, static_cast<float>(h)))), h, t.addrV);
		return texel(t, sc.srgbLut, x, y);
	}
	const float x = __fsub_rn(__fmul_rn(cu, static_cast<float>(w)), 0.5f);
	const float y = __fsub_rn(__fmul_rn(cv, static_cast<float>(h)), 0.5f);
	const float fx = floorf(x), fy = floorf(y);
	const float a = __fsub_rn(x, fx), b = __fsub_rn(y, fy);
	const int x0 = texAddress(static_cast<int>(fx), w, t.addrU), x1 = texAddress(static_cast<int>(fx) + 1, w, t.addrU);
	const int y0 = texAddress(static_cast<int>(fy), h, t.addrV), y1 = texAddress(static_cast<int>(fy) + 1, h, t.addrV);
	const float4 t00 = texel(t, sc.srgbLut, x0, y0), t10 = texel(t, sc.srgbLut, x1, y0);
	const float4 t01 = texel(t, sc.srgbLut, x0, y1), t11 = texel(t, sc.srgbLut, x1, y1);
	return make_float4(lerpT(lerpT(t00.x, t10.x, a), lerpT(t01.x, t11.x, a), b),
		lerpT(lerpT(t00.y, t10.y, a), lerpT(t01.y, t11.y, a), b),
		lerpT(lerpT(t00.z, t10.z, a), lerpT(t01.z, t11.z, a), b),
		lerpT(lerpT(t00.w, t10.w, a), lerpT(t01.w, t11.w, a), b));
}
// Texture slot `slot` of a material at the record's coordinates (x, y: set
// 1; z, w: set 2), by the slot's coordinate-set flag.
RB_D float4 materialTexture(const DevScene& sc, const DevMaterial& m, uint32_t slot, uint32_t setOf, float4 uv)
{
	const bool second = (m.texSets >> setOf) & 1u;
	return texSample(sc, m.tex[slot], second ? uv.z : uv.x, second ? uv.w : uv.y);
}
} // namespace rb
