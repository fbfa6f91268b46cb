// Monte Carlo regeneration of the multiple-scattering compensation tables
// that the BxDFs read (the reference ships them as data, bin/*.bin, with no
// generator). Each texel is the directional albedo of one microfacet lobe,
// integrated with the lobe formulas of rb_bxdf.cuh, on the axes the BxDFs
// look it up with (bxdfComplexSurface), sampled at i / 31 for i = 0..31 (the
// reference's tables are generated on these end-inclusive grids, although its
// texture lookup puts texel i at (i + 0.5) / 32; matching them showed it):
//   x: |cos theta_o| = i / 31 (at least kMinCos), y: roughness r = j / 31 (at
//   least 0.001, as the BxDFs clamp it), alpha = r^2 (isotropic GGX), z (3D
//   tables): w = k / 31 = sqrt(|f0Sr|) with f0Sr = (1 - eta) / (1 + eta), so
//   eta = (1 + w^2) / (1 - w^2) for the outer tables (eta > 1) and
//   (1 - w^2) / (1 + w^2) for the inner ones.
// Tables (definitions found by matching the reference's data, see below):
//   conductor  = albedo of GGX reflection with F = 1;
//   dielectric = albedo of reflection plus transmission, Schlick Fresnel
//                with total internal reflection (F = 1 where no refracted
//                direction exists), transmitted energy not scaled by eta^2;
//   reflective = albedo of the Schlick-Fresnel reflection alone, Schlick
//                without the total-internal-reflection override, divided by
//                the dielectric albedo (the share of the compensated
//                specular layer, which the BxDF scales by 1 / dielectric);
//   at w = 0 (eta = 1, no interface) dielectric = 1 and reflective = 0.
// Against the reference's bin/*.bin, away from the |cos| = 0 column that it
// fills in its own way, the regenerated conductor, dielectric and reflective
// tables agree to a few 1e-4 (Monte Carlo noise). Microfacet normals are drawn from the visible-normal
// distribution (spherical-cap sampling, the BxDFs' own sampler), so each
// sample weighs G2 / G1 times the lobe's Fresnel factor; a Hammersley point
// set with a per-texel rotation gives the (u, v) pairs.

#include <cstdint>

#include "rb_bxdf.cuh"
#include "rb_launch.cuh"
#include "ratbite_b200_kernels.h"

namespace rb
{
namespace
{
constexpr uint32_t kLut2 = kLutN * kLutN, kLut3 = kLutN * kLutN * kLutN;
constexpr float kMinCos = 1e-4f;
RB_D float lutAxis(uint32_t i) { return static_cast<float>(i) / static_cast<float>(kLutN - 1); }

struct LutOut
{
	float* conductor;
	float* dielOuter;
	float* dielInner;
	float* reflOuter;
	float* reflInner;
};

// texel t: [0, kLut2) conductor, then 2 x kLut3 (outer, inner) for the
// dielectric and reflective tables (one pass computes both).
__global__ void __launch_bounds__(kThreads) kGenerateLuts(LutOut o, uint32_t samples)
{
	for (uint32_t t = gtid(); t < kLut2 + 2 * kLut3; t += gstride())
	{
		const bool cond = t < kLut2;
		const uint32_t u3 = cond ? t : (t - kLut2) % kLut3;
		const bool inner = !cond && (t - kLut2) >= kLut3;
		const uint32_t ix = u3 % kLutN, iy = (u3 / kLutN) % kLutN, iz = u3 / kLut2;
		const float mu = fmaxf(lutAxis(ix), kMinCos);
		const float r = fmaxf(lutAxis(iy), 0.001f);
		const float alpha = r * r;
		const f3 wo = mk(sqrtf(fmaxf(0.0f, 1.0f - mu * mu)), 0.0f, mu);
		const CtxDir co = ctxDir(wo);
		const float g1 = G1(co, alpha, alpha);
		float eta = 1.0f, f0 = 0.0f;
		if (!cond)
		{
			const float w = lutAxis(iz), w2 = w * w;
			eta = inner ? (1.0f - w2) / (1.0f + w2) : (1.0f + w2) / (1.0f - w2);
			f0 = w2 * w2;
		}
		const uint32_t h = mix32(t * 0x9E3779B9u + 0x85EBCA6Bu);
		const float ru = static_cast<float>(h >> 8) * (1.0f / 16777216.0f);
		const float rv = static_cast<float>(mix32(h) >> 8) * (1.0f / 16777216.0f);
		double accR = 0.0, accT = 0.0, accS = 0.0;   // reflection (with TIR), transmission, Schlick reflection
		for (uint32_t s = 0; s < samples; ++s)
		{
			float u = (static_cast<float>(s) + 0.5f) / static_cast<float>(samples) + ru;
			float v = static_cast<float>(__brev(s) >> 8) * (1.0f / 16777216.0f) + rv;
			u -= floorf(u);
			v -= floorf(v);
			const f3 m = vndfSampleCap(wo, alpha, alpha, u, v);
			const float ad = fabsf(dot(wo, m));
			float F = 1.0f, Fs = 1.0f;
			if (!cond)
			{
				Fs = fresnelSchlick(f0, ad);
				const float s2t = fmaxf(0.0f, 1.0f - ad * ad) / (eta * eta);
				F = s2t >= 1.0f ? 1.0f : Fs;
			}
			const f3 wi = normalize(reflectAbout(wo, m));
			if (wi.z > 0.0f)
			{
				const float g = G2(ctxDir(wi), co, alpha, alpha) / g1;
				accR += static_cast<double>(F * g);
				accS += static_cast<double>(Fs * g);
			}
			if (!cond && F < 1.0f)
			{
				const f3 wt = refractSimple(wo, m, eta);
				if (wt.z < 0.0f) accT += static_cast<double>((1.0f - F) * G2(ctxDir(wt), co, alpha, alpha) / g1);
			}
		}
		if (cond)
		{
			o.conductor[u3] = static_cast<float>(accR / samples);
		}
		else
		{
			const double diel = (accR + accT) / samples;
			const bool noInterface = iz == 0;
			(inner ? o.dielInner : o.dielOuter)[u3] = noInterface ? 1.0f : static_cast<float>(diel);
			(inner ? o.reflInner : o.reflOuter)[u3] =
				noInterface || diel <= 0.0 ? 0.0f : static_cast<float>(accS / samples / diel);
		}
	}
}
} // namespace
} // namespace rb

extern "C" int rb_k_generate_luts(uint32_t samples, float* conductor, float* dielectric_outer, float* dielectric_inner,
	float* reflective_outer, float* reflective_inner, void* stream)
{
	if (samples == 0 || !conductor || !dielectric_outer || !dielectric_inner || !reflective_outer || !reflective_inner)
		return RB_ERR_INVALID;
	rb::LutOut o{ conductor, dielectric_outer, dielectric_inner, reflective_outer, reflective_inner };
	const uint32_t texels = rb::kLut2 + 2 * rb::kLut3;
	rb::kGenerateLuts<<<rb::gridFor(texels), rb::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(o, samples);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}
