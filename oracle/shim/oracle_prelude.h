// Oracle test infrastructure (not product code).
//
// Force-included (g++ -include) before every reference translation unit that
// the oracle compiles host-side. It maps the CUDA language keywords and the
// device intrinsics the reference uses onto plain C++ so the reference's own
// device code (src/device/*.h, src/kernels/pathtrace.cu) runs on the CPU:
//   __brev / __clz            (src/device/quasi_random.h:103-110)
//   __float_as_uint & co.     (src/kernels/pathtrace.cu:125-148, src/device/util.h:22-24)
//   __fmaf_rn                 (src/device/surface.h:323,346)
//   __frsqrt_rn / rsqrt       (src/kernels/pathtrace.cu:110,989)
//   tex2D / tex3D             (src/kernels/pathtrace.cu:646-658, src/device/surface.h:48)
// Texture fetches go to a registry of host arrays with normalized
// coordinates: linear filtering and clamp addressing, the sampler state the
// reference creates for its LUTs and environment map
// (src/core/rendering_interface.cpp: 540-616, 1358-1360), or the material
// textures' own address modes (wrap, clamp, mirror) and filter (nearest,
// linear; src/core/texture.h:280-380), their texels already decoded to
// floats (8-bit / 255, the sRGB curve where the texture is sRGB).
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#undef __global__
#undef __device__
#undef __host__
#undef __constant__
#undef __shared__
#undef __forceinline__
#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__
#define __forceinline__ inline

inline unsigned int __float_as_uint(float f) { unsigned int u; std::memcpy(&u, &f, 4); return u; }
inline float __uint_as_float(unsigned int u) { float f; std::memcpy(&f, &u, 4); return f; }
inline int __float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
inline unsigned int __brev(unsigned int x)
{
	unsigned int r = 0;
	for (int i = 0; i < 32; ++i) { r = (r << 1) | (x & 1u); x >>= 1; }
	return r;
}
inline int __clz(int x) { return x == 0 ? 32 : __builtin_clz(static_cast<unsigned int>(x)); }
inline float __fmaf_rn(float a, float b, float c) { return std::fma(a, b, c); }
// Correctly rounded reciprocal square root (the _rn suffix): computed in double.
inline float __frsqrt_rn(float x) { return static_cast<float>(1.0 / std::sqrt(static_cast<double>(x))); }
inline float rsqrt(float x) { return static_cast<float>(1.0 / std::sqrt(static_cast<double>(x))); }

namespace oracle_tex
{
	// A texture is a dense float array of w*h*d texels with c channels (1 or 4).
	struct Texture
	{
		const float* data;
		int w, h, d, c;
		int addrU = 1, addrV = 1;   // 0 wrap, 1 clamp, 2 mirror
		int linear = 1;             // 0 nearest
	};
	// Registry lookups (implemented in ref_harness.cpp). Handles start at 1.
	const Texture& get(cudaTextureObject_t handle);
	// 0: FP32 interpolation weights (parity mode); 1: 8-bit fixed-point
	// weights as documented for CUDA's linear filtering hardware.
	extern int weightMode;

	inline float weight(float frac)
	{
		if (weightMode == 1)
			return std::nearbyint(frac * 256.0f) / 256.0f;
		return frac;
	}
	// Texel index along one axis for the address mode.
	inline int address(int i, int n, int mode)
	{
		if (mode == 0) { int m = i % n; return m < 0 ? m + n : m; }
		if (mode == 2) { int m = i % (2 * n); if (m < 0) m += 2 * n; return m < n ? m : 2 * n - 1 - m; }
		return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
	}
	// The coordinate the filter works on: wrap takes the fraction, mirror
	// reflects into [0, 1], clamp keeps it.
	inline float coord(float u, int mode)
	{
		if (mode == 0) return u - std::floor(u);
		if (mode == 2) { float f = u - 2.0f * std::floor(u * 0.5f); return f <= 1.0f ? f : 2.0f - f; }
		return u;
	}
	// Texel coordinate setup of linear filtering with normalized coordinates:
	// x = u*N - 0.5, i0 = floor(x), a = frac(x), the taps addressed by the
	// mode (clamp: both clamped to [0, N-1]).
	inline void taps(float u, int n, int& i0, int& i1, float& a, int mode = 1)
	{
		float x = coord(u, mode) * static_cast<float>(n) - 0.5f;
		float fl = std::floor(x);
		a = weight(x - fl);
		int i = static_cast<int>(fl);
		i0 = address(i, n, mode);
		i1 = address(i + 1, n, mode);
	}
	inline void fetch2D(const Texture& t, float u, float v, float* out)
	{
		if (!t.linear)
		{
			const int x = address(static_cast<int>(std::floor(coord(u, t.addrU) * static_cast<float>(t.w))), t.w, t.addrU);
			const int y = address(static_cast<int>(std::floor(coord(v, t.addrV) * static_cast<float>(t.h))), t.h, t.addrV);
			for (int ch = 0; ch < t.c; ++ch) out[ch] = t.data[(y * t.w + x) * t.c + ch];
			return;
		}
		int x0, x1, y0, y1; float a, b;
		taps(u, t.w, x0, x1, a, t.addrU);
		taps(v, t.h, y0, y1, b, t.addrV);
		for (int ch = 0; ch < t.c; ++ch)
		{
			float t00 = t.data[(y0 * t.w + x0) * t.c + ch];
			float t10 = t.data[(y0 * t.w + x1) * t.c + ch];
			float t01 = t.data[(y1 * t.w + x0) * t.c + ch];
			float t11 = t.data[(y1 * t.w + x1) * t.c + ch];
			float r0 = t00 + a * (t10 - t00);
			float r1 = t01 + a * (t11 - t01);
			out[ch] = r0 + b * (r1 - r0);
		}
	}
	inline float fetch3D(const Texture& t, float u, float v, float s)
	{
		int x0, x1, y0, y1, z0, z1; float a, b, g;
		taps(u, t.w, x0, x1, a);
		taps(v, t.h, y0, y1, b);
		taps(s, t.d, z0, z1, g);
		auto T = [&](int x, int y, int z) { return t.data[(z * t.h + y) * t.w + x]; };
		float c00 = T(x0, y0, z0) + a * (T(x1, y0, z0) - T(x0, y0, z0));
		float c10 = T(x0, y1, z0) + a * (T(x1, y1, z0) - T(x0, y1, z0));
		float c01 = T(x0, y0, z1) + a * (T(x1, y0, z1) - T(x0, y0, z1));
		float c11 = T(x0, y1, z1) + a * (T(x1, y1, z1) - T(x0, y1, z1));
		float c0 = c00 + b * (c10 - c00);
		float c1 = c01 + b * (c11 - c01);
		return c0 + g * (c1 - c0);
	}
}

template<typename T> T tex2D(cudaTextureObject_t, float, float);
template<> inline float tex2D<float>(cudaTextureObject_t h, float u, float v)
{
	float r[4]; oracle_tex::fetch2D(oracle_tex::get(h), u, v, r); return r[0];
}
template<> inline float4 tex2D<float4>(cudaTextureObject_t h, float u, float v)
{
	float r[4] = { 0, 0, 0, 0 };
	const oracle_tex::Texture& t = oracle_tex::get(h);
	oracle_tex::fetch2D(t, u, v, r);
	if (t.c == 1) { r[1] = 0; r[2] = 0; r[3] = 0; }
	return float4{ r[0], r[1], r[2], r[3] };
}
template<typename T> T tex3D(cudaTextureObject_t, float, float, float);
template<> inline float tex3D<float>(cudaTextureObject_t h, float u, float v, float s)
{
	return oracle_tex::fetch3D(oracle_tex::get(h), u, v, s);
}
