// Sample generation: owen-scrambled Sobol (Burley 2020, Cycles' layout),
// hero wavelengths, dense spectra, the pixel filter and camera rays.
#pragma once

#include "rb_math.cuh"
#include "rb_scene.h"

namespace rb
{
// ---------------------------------------------------------------- QRNG
// Dimension offsets and per-bounce stride (src/device/quasi_random.h:13-29).
enum Dim : uint32_t
{
	DIM_FILTER = 0, DIM_LENS = 1,
	DIM_WAVELENGTH = 0, DIM_LIGHT = 1, DIM_BXDF_0 = 2, DIM_BXDF_1 = 3,
	DIM_ALPHA_BLEND = 7, DIM_ROULETTE = 8,
	DIM_STRIDE = 16,
};

// Sobol direction numbers of dimensions 1..3 in the reversed-bit layout of
// Burley's formulation (dimension 0 is the van der Corput sequence, a bit
// reversal). The sequence is only reproducible with exactly these numbers;
// the reference holds the same table at src/device/quasi_random.h:137-179.
// Kept in global memory and read through the read-only cache: lanes index it
// divergently, which the constant cache would serialise.
__device__ uint32_t kSobolDirections[3][32] = {
	{ 0x00000001, 0x00000003, 0x00000005, 0x0000000f, 0x00000011, 0x00000033, 0x00000055, 0x000000ff,
	  0x00000101, 0x00000303, 0x00000505, 0x00000f0f, 0x00001111, 0x00003333, 0x00005555, 0x0000ffff,
	  0x00010001, 0x00030003, 0x00050005, 0x000f000f, 0x00110011, 0x00330033, 0x00550055, 0x00ff00ff,
	  0x01010101, 0x03030303, 0x05050505, 0x0f0f0f0f, 0x11111111, 0x33333333, 0x55555555, 0xffffffff },
	{ 0x00000001, 0x00000003, 0x00000006, 0x00000009, 0x00000017, 0x0000003a, 0x00000071, 0x000000a3,
	  0x00000116, 0x00000339, 0x00000677, 0x000009aa, 0x00001601, 0x00003903, 0x00007706, 0x0000aa09,
	  0x00010117, 0x0003033a, 0x00060671, 0x000909a3, 0x00171616, 0x003a3939, 0x00717777, 0x00a3aaaa,
	  0x01170001, 0x033a0003, 0x06710006, 0x09a30009, 0x16160017, 0x3939003a, 0x77770071, 0xaaaa00a3 },
	{ 0x00000001, 0x00000003, 0x00000004, 0x0000000a, 0x0000001f, 0x0000002e, 0x00000045, 0x000000c9,
	  0x0000011b, 0x000002a4, 0x0000079a, 0x00000b67, 0x0000101e, 0x0000302d, 0x00004041, 0x0000a0c3,
	  0x0001f104, 0x0002e28a, 0x000457df, 0x000c9bae, 0x0011a105, 0x002a7289, 0x0079e7db, 0x00b6dba4,
	  0x0100011a, 0x030002a7, 0x0400079e, 0x0a000b6d, 0x1f001001, 0x2e003003, 0x45004004, 0xc900a00a },
};

// Per-pixel decorrelation hash (src/device/quasi_random.h:30-37, seed 0).
RB_HD uint32_t pixelHash(uint32_t x, uint32_t y)
{
	const uint32_t qx = 1103515245u * ((x >> 1u) ^ y);
	const uint32_t qy = 1103515245u * ((y >> 1u) ^ x);
	return 1103515245u * (qx ^ (qy >> 3u));
}
// Dimension hash (quasi_random.h:102-111).
RB_D uint32_t dimHash(uint32_t i)
{
	i ^= i >> 16; i *= 0x21f0aaadu;
	i ^= i >> 15; i *= 0xd35a2d97u;
	i ^= i >> 15;
	return i ^ 0xe6fe3bebu;
}
// Laine-Karras style Owen scramble in reversed-bit space (quasi_random.h:119-127).
RB_D uint32_t owenReversed(uint32_t n, uint32_t seed)
{
	n ^= n * 0x3d20adeau;
	n += seed;
	n *= (seed >> 16) | 1u;
	n ^= n * 0x05526c56u;
	n ^= n * 0x53a22864u;
	return n;
}
RB_D float u32ToUnitExclusive(uint32_t x) { return static_cast<float>(x) * (1.0f / 4294967808.0f); }

RB_D float sobolBurley(uint32_t revIndex, uint32_t dim, uint32_t scramble)
{
	uint32_t result = 0;
	if (dim == 0)
	{
		result = __brev(revIndex);
	}
	else
	{
		const uint32_t* table = kSobolDirections[dim - 1];
		uint32_t i = 0;
		while (revIndex != 0)
		{
			const uint32_t j = __clz(revIndex);
			result ^= __ldg(table + i + j);
			i += j + 1;
			revIndex <<= j;
			revIndex <<= 1;
		}
	}
	return u32ToUnitExclusive(__brev(owenReversed(result, scramble)));
}

// QRNG state of one path: sample index, pixel hash and the current
// dimension base (16 per bounce, starting at 16; QRNG::State, :38-64).
struct Qrng
{
	uint32_t sample, hash, base;
};
RB_D Qrng qrngAt(uint32_t sample, uint32_t hash, uint32_t bounce)
{
	return Qrng{ sample, hash, DIM_STRIDE * (bounce + 1u) };
}
RB_D float sample1D(const Qrng& q, uint32_t dim)
{
	const uint32_t seed = q.hash ^ dimHash(q.base + dim);
	const uint32_t idx = owenReversed(__brev(q.sample), seed ^ 0xbff95bfeu);
	return sobolBurley(idx, 0, seed ^ 0x635c77bdu);
}
RB_D void sample2D(const Qrng& q, uint32_t dim, float& a, float& b)
{
	const uint32_t seed = q.hash ^ dimHash(q.base + dim);
	const uint32_t idx = owenReversed(__brev(q.sample), seed ^ 0xf8ade99au);
	a = sobolBurley(idx, 0, seed ^ 0xe0aaaf76u);
	b = sobolBurley(idx, 1, seed ^ 0x94964d4eu);
}
RB_D f3 sample3D(const Qrng& q, uint32_t dim)
{
	const uint32_t seed = q.hash ^ dimHash(q.base + dim);
	const uint32_t idx = owenReversed(__brev(q.sample), seed ^ 0xcaa726acu);
	return f3{ sobolBurley(idx, 0, seed ^ 0x9e78e391u), sobolBurley(idx, 1, seed ^ 0x67c33241u),
	           sobolBurley(idx, 2, seed ^ 0x78c395c5u) };
}
// The third component of sample3D(q, dim) alone (the components are
// independent, so this is bit-identical to sample3D(q, dim).z).
RB_D float sample3DZ(const Qrng& q, uint32_t dim)
{
	const uint32_t seed = q.hash ^ dimHash(q.base + dim);
	const uint32_t idx = owenReversed(__brev(q.sample), seed ^ 0xcaa726acu);
	return sobolBurley(idx, 2, seed ^ 0x78c395c5u);
}

// ------------------------------------------------------------ wavelengths
// Hero-wavelength sampling of the visible range with the atanh warp of
// Radziszewski et al. (SampledWavelengths::sampleVisible, src/device/spectral.h:227-241, 289-299).
struct Wavelengths
{
	S4 lambda;
	S4 pdf;
	float active;
};
RB_D float visibleWavelengthPdf(float lambda)
{
	if (lambda < 360.0f || lambda > 830.0f) return 0.0f;
	const float c = coshf(0.0072f * (lambda - 538.0f));
	return 0.0039398042f / (c * c);
}
RB_D Wavelengths sampleVisible(float u)
{
	Wavelengths w;
	for (int i = 0; i < 4; ++i)
	{
		float up = u + static_cast<float>(i) / 4.0f;
		if (up > 1.0f) up -= 1.0f;
		w.lambda.v[i] = 538.0f - 138.888889f * atanhf(0.85691062f - 1.82750197f * up);
		w.pdf.v[i] = visibleWavelengthPdf(w.lambda.v[i]);
	}
	w.active = 4.0f;
	return w;
}

// Dense 471-bin spectrum lookup at the nearest nanometre (DenseSpectrum::sample, :313-327).
RB_D int lambdaBin(float lambda) { return static_cast<int>(lroundf(lambda)) - kLambdaMin; }
RB_D float denseAt(const float* table, float lambda) { return __ldg(table + lambdaBin(lambda)); }
RB_D S4 denseSample(const float* table, const S4& lambda)
{
	S4 r;
	for (int i = 0; i < 4; ++i) r.v[i] = denseAt(table, lambda.v[i]);
	return r;
}
// RGB to spectrum through the spectral basis (color::RGBtoSpectrum, src/device/color.h:31-43).
RB_D S4 rgbToSpectrum(const float* basis, f3 rgb, const S4& lambda)
{
	S4 r;
	for (int i = 0; i < 4; ++i)
	{
		const int b = lambdaBin(lambda.v[i]);
		r.v[i] = __ldg(basis + b) * rgb.x + __ldg(basis + kSpectrumBins + b) * rgb.y
			+ __ldg(basis + 2 * kSpectrumBins + b) * rgb.z;
	}
	return r;
}

// ------------------------------------------------------------- sampling
// Polar disk mapping (src/device/sampling.h:53-58).
RB_D void diskPolar(float u, float v, float& x, float& y)
{
	const float r = sqrtf(u);
	const float theta = 2.0f * kPi * v;
	x = r * cosf(theta);
	y = r * sinf(theta);
}
// Cosine-weighted hemisphere (src/device/surface.h:18-32).
RB_D f3 cosWeightedSample(float u, float v)
{
	float x, y;
	diskPolar(u, v, x, y);
	return f3{ x, y, sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y)) };
}
RB_D float cosWeightedPdf(float cosTheta) { return cosTheta / kPi; }

// Truncated Gaussian pixel filter, radius 1.5 px, sigma 0.25 (src/device/filter.h:14-27).
RB_D void gaussianFilterSample(float u, float v, float& dx, float& dy)
{
	const float rad = 1.5f, sigma = 0.25f;
	const float uTH = expf(-(rad * rad) / (2.0f * sigma * sigma));
	const float uu = fmaxf(0.00001f, u * (1.0f - uTH) + uTH);
	const float m = sigma * sqrtf(-2.0f * logf(uu));
	dx = m * cosf(2.0f * kPi * v);
	dy = m * sinf(2.0f * kPi * v);
}

// Camera ray for sub-pixel position (sx, sy): pinhole (src/device/dir_gen.h:19-30)
// or thin lens (:31-47). The camera sits at the origin.
RB_D void cameraRay(const DevLaunch& L, float sx, float sy, float lu, float lv, f3& o, f3& d)
{
	const f3 U = mk(L.camU[0], L.camU[1], L.camU[2]);
	const f3 V = mk(L.camV[0], L.camV[1], L.camV[2]);
	const f3 W = mk(L.camW[0], L.camW[1], L.camW[2]);
	if (L.dof)
	{
		const float xs = (2.0f * sx * L.invWidth - 1.0f) * L.perspW;
		const float zs = (2.0f * sy * L.invHeight - 1.0f) * L.perspH;
		const f3 focus = mk(xs, zs, 1.0f) * L.focusDistance;
		float px, py;
		diskPolar(lu, lv, px, py);
		px *= L.aperture;
		py *= L.aperture;
		o = U * px + W * py;
		const f3 dl = normalize(focus - mk(px, py, 0.0f));
		d = U * dl.x + W * dl.y + V * dl.z;
	}
	else
	{
		const float xs = 2.0f * sx * L.invWidth - 1.0f;
		const float zs = 2.0f * sy * L.invHeight - 1.0f;
		o = mk(0.0f);
		d = normalize(V + U * xs * L.perspW + W * zs * L.perspH);
	}
}
} // namespace rb
