// Surface scattering: GGX microfacet terms, spherical-cap VNDF sampling
// (Dupuy & Benyoub 2023; bounded variant of Eto & Tokuyoshi 2023), LTC sheen
// (Zeltner et al. 2022), multiple-scattering compensation LUTs (Turquin 2019)
// and the two BxDF callables of the reference (src/kernels/pathtrace.cu:
// 464-547, 548-905). The math follows src/device/surface.h term for term so
// results match the reference within float rounding on identical inputs.
#pragma once

#include <cuda/std/complex>

#include "rb_math.cuh"
#include "rb_qrng.cuh"
#include "rb_scene.h"

namespace rb
{
// ------------------------------------------------------- local frame math
// LocalTransform statics (src/device/local_transform.h:34-50).
RB_D float cos2Theta(f3 w) { return w.z * w.z; }
RB_D float sin2ThetaFromCos2(float c2) { return fmaxf(0.0f, 1.0f - c2); }
RB_D float tan2Theta(f3 w) { return sin2ThetaFromCos2(cos2Theta(w)) / cos2Theta(w); }
RB_D float sinThetaFromCos2(float c2) { return sqrtf(fmaxf(0.0f, 1.0f - c2)); }
RB_D float sinTheta(f3 w) { return sinThetaFromCos2(cos2Theta(w)); }
RB_D float cosPhiWith(f3 w, float st) { return st == 0.0f ? 1.0f : clampf(w.x / st, -1.0f, 1.0f); }
RB_D float sinPhiWith(f3 w, float st) { return st == 0.0f ? 0.0f : clampf(w.y / st, -1.0f, 1.0f); }
RB_D float cosPhi(f3 w) { return cosPhiWith(w, sinTheta(w)); }
RB_D float sinPhi(f3 w) { return sinPhiWith(w, sinTheta(w)); }

// Shading frame with columns t, b, n (LocalTransform(frameMat), :22-25).
struct Frame
{
	f3 t, b, n;
	RB_D f3 toLocal(f3 v) const { return f3{ dot(t, v), dot(b, v), dot(n, v) }; }
	RB_D f3 fromLocal(f3 v) const
	{
		return f3{ t.x * v.x + b.x * v.y + n.x * v.z, t.y * v.x + b.y * v.y + n.y * v.z,
		           t.z * v.x + b.z * v.y + n.z * v.z };
	}
};

RB_D f3 reflectAbout(f3 v, f3 n) { return -v + 2.0f * dot(v, n) * n; }   // src/device/util.h:49-52
// Refraction without inverting eta for back-facing input (src/device/util.h:53-70).
RB_D f3 refractSimple(f3 v, f3 n, float eta)
{
	float c = dot(v, n);
	if (c < 0.0f) { c = -c; n = -n; }
	const float s2i = fmaxf(0.0f, 1.0f - c * c);
	const float s2t = s2i / (eta * eta);
	if (s2t >= 1.0f) return mk(0.0f);
	return -v / eta + (c / eta - sqrtf(1.0f - s2t)) * n;
}

// --------------------------------------------------------------- GGX
struct CtxDir
{
	float tan2, cosPhi, sinPhi;
};
RB_D CtxDir ctxDir(f3 w) { return CtxDir{ tan2Theta(w), cosPhi(w), sinPhi(w) }; }
struct CtxM
{
	float cos2, tan2, cosPhi, sinPhi;
};
RB_D CtxM ctxM(f3 w) { return CtxM{ cos2Theta(w), tan2Theta(w), cosPhi(w), sinPhi(w) }; }

RB_D float lambdaG(float ax, float ay, float cp, float sp, float tan2)
{
	if (isinf(tan2)) return 0.0f;
	const float a = cp * ax, b = sp * ay;
	const float alpha2 = a * a + b * b;
	return (sqrtf(1.0f + alpha2 * tan2) - 1.0f) / 2.0f;
}
RB_D float G1(const CtxDir& o, float ax, float ay) { return 1.0f / (1.0f + lambdaG(ax, ay, o.cosPhi, o.sinPhi, o.tan2)); }
RB_D float G2(const CtxDir& i, const CtxDir& o, float ax, float ay)
{
	return 1.0f / (1.0f + lambdaG(ax, ay, i.cosPhi, i.sinPhi, i.tan2) + lambdaG(ax, ay, o.cosPhi, o.sinPhi, o.tan2));
}
RB_D float ggxD(const CtxM& m, float ax, float ay)
{
	if (isinf(m.tan2)) return 0.0f;
	const float cos4 = m.cos2 * m.cos2;
	if (cos4 < 1e-16f) return 0.0f;
	const float cx = m.cosPhi / ax, sy = m.sinPhi / ay;
	const float e = m.tan2 * (cx * cx + sy * sy);
	const float ope = 1.0f + e;
	return 1.0f / (kPi * ax * ay * cos4 * ope * ope);
}

RB_D float fresnelSchlick(float f0, float mu) { return f0 + (1.0f - f0) * powf(1.0f - mu, 5.0f); }
RB_D f3 fresnelSchlick3(f3 f0, float mu)
{
	const float p = powf(1.0f - mu, 5.0f);
	return f0 + (mk(1.0f) - f0) * p;
}
// F82 with specular colour and weight 1 (src/device/surface.h:254-264): the
// tint term then vanishes and the value equals Schlick's, computed the same way.
RB_D f3 fresnelF82(f3 f0, float mu)
{
	const float muDash = 1.0f / 7.0f;
	const f3 f = fresnelSchlick3(f0, mu);
	const f3 fDash = fresnelSchlick3(f0, muDash);
	const float k = (mu * powf(1.0f - mu, 6.0f)) / (muDash * powf(1.0f - muDash, 6.0f));
	return 1.0f * (f - k * (fDash - mk(1.0f) * fDash));
}
RB_D f3 fresnelAvgF82(f3 f0)
{
	return 0.877105f * f0 + (mk(0.0648148f) + 0.0752755f * f0) * mk(1.0f) - mk(0.0171958f);
}
// Complex Fresnel per wavelength for conductors (surface.h:176-195).
RB_D S4 fresnelComplex(float cosTheta, const S4& eta, const S4& k)
{
	using C = cuda::std::complex<float>;
	S4 r;
	for (int i = 0; i < 4; ++i)
	{
		const C ceta{ eta.v[i], k.v[i] };
		const float c = clampf(cosTheta, 0.0f, 1.0f);
		const float s2 = 1.0f - c * c;
		const C s2t = s2 / (ceta * ceta);
		const C ct = cuda::std::sqrt(1.0f - s2t);
		const C parl = (ceta * c - ct) / (ceta * c + ct);
		const C perp = (c - ceta * ct) / (c + ceta * ct);
		r.v[i] = (cuda::std::norm(parl) + cuda::std::norm(perp)) / 2.0f;
	}
	return r;
}

// Spherical-cap VNDF sampling (surface.h:313-328) and its pdf (:352-356).
RB_D f3 vndfSampleCap(f3 wo, float ax, float ay, float u, float v)
{
	f3 woStd = normalize(mk(wo.x * ax, wo.y * ay, wo.z));
	if (woStd.z < 0.0f) woStd = -woStd;
	const float phi = 2.0f * kPi * u;
	const float b = woStd.z;
	const float z = __fmaf_rn(1.0f - v, 1.0f + b, -b);
	const float st = sqrtf(clampf(1.0f - z * z, 0.0f, 1.0f));
	const f3 wiStd = mk(st * cosf(phi), st * sinf(phi), z);
	const f3 wmStd = woStd + wiStd;
	return normalize(mk(wmStd.x * ax, wmStd.y * ay, wmStd.z));
}
RB_D float vndfPdfCap(f3 wo, float absDotWoWm, const CtxDir& o, const CtxM& m, float ax, float ay)
{
	return G1(o, ax, ay) / fabsf(wo.z) * ggxD(m, ax, ay) * absDotWoWm;
}
// Bounded spherical-cap sampling for reflection (surface.h:329-345, 358-374).
RB_D f3 vndfSampleBounded(f3 wo, float ax, float ay, float u, float v)
{
	const f3 woStd = normalize(mk(wo.x * ax, wo.y * ay, wo.z));
	const float phi = 2.0f * kPi * u;
	const float a1 = fminf(ax, ay);
	const float s = 1.0f + sqrtf(wo.x * wo.x + wo.y * wo.y);
	const float a2 = a1 * a1, s2 = s * s;
	const float k = (1.0f - a2) * s2 / (s2 + a2 * wo.z * wo.z);
	const float b = wo.z > 0.0f ? k * woStd.z : woStd.z;
	const float z = __fmaf_rn(1.0f - v, 1.0f + b, -b);
	const float st = sqrtf(clampf(1.0f - z * z, 0.0f, 1.0f));
	const f3 wiStd = mk(st * cosf(phi), st * sinf(phi), z);
	const f3 wmStd = woStd + wiStd;
	return normalize(mk(wmStd.x * ax, wmStd.y * ay, wmStd.z));
}
RB_D float vndfPdfBounded(f3 wo, float absDotWoWm, const CtxM& m, float ax, float ay)
{
	const float ndf = ggxD(m, ax, ay);
	const float aox = wo.x * ax, aoy = wo.y * ay;
	const float len2 = aox * aox + aoy * aoy;
	const float t = sqrtf(len2 + wo.z * wo.z);
	if (wo.z >= 0.0f)
	{
		const float a1 = clampf(fminf(ax, ay), 0.0f, 1.0f);
		const float s = 1.0f + sqrtf(wo.x * wo.x + wo.y * wo.y);
		const float a2 = a1 * a1, s2 = s * s;
		const float k = (1.0f - a2) * s2 / (s2 + a2 * wo.z * wo.z);
		return ndf * 2.0f * absDotWoWm / (k * wo.z + t);
	}
	return ndf * (t - wo.z) * 2.0f * absDotWoWm / len2;
}

// ----------------------------------------------------------- LUT access
// Linear filtering with normalized coordinates and clamp addressing, in
// FP32 (the reference samples these tables through CUDA textures created at
// src/core/rendering_interface.cpp:536-616).
RB_D void lutTaps(float u, int n, int& i0, int& i1, float& a)
{
	const float x = u * static_cast<float>(n) - 0.5f;
	const float fl = floorf(x);
	a = x - fl;
	const int i = static_cast<int>(fl);
	i0 = min(max(i, 0), n - 1);
	i1 = min(max(i + 1, 0), n - 1);
}
RB_D float lut2D(const float* t, float u, float v)
{
	int x0, x1, y0, y1; float a, b;
	lutTaps(u, kLutN, x0, x1, a);
	lutTaps(v, kLutN, y0, y1, b);
	const float t00 = __ldg(t + y0 * kLutN + x0), t10 = __ldg(t + y0 * kLutN + x1);
	const float t01 = __ldg(t + y1 * kLutN + x0), t11 = __ldg(t + y1 * kLutN + x1);
	const float r0 = t00 + a * (t10 - t00);
	const float r1 = t01 + a * (t11 - t01);
	return r0 + b * (r1 - r0);
}
RB_D float4 lut2D4(const float4* t, float u, float v)
{
	int x0, x1, y0, y1; float a, b;
	lutTaps(u, kLutN, x0, x1, a);
	lutTaps(v, kLutN, y0, y1, b);
	const float4 t00 = __ldg(t + y0 * kLutN + x0), t10 = __ldg(t + y0 * kLutN + x1);
	const float4 t01 = __ldg(t + y1 * kLutN + x0), t11 = __ldg(t + y1 * kLutN + x1);
	float4 r;
	r.x = (t00.x + a * (t10.x - t00.x)) + b * ((t01.x + a * (t11.x - t01.x)) - (t00.x + a * (t10.x - t00.x)));
	r.y = (t00.y + a * (t10.y - t00.y)) + b * ((t01.y + a * (t11.y - t01.y)) - (t00.y + a * (t10.y - t00.y)));
	r.z = (t00.z + a * (t10.z - t00.z)) + b * ((t01.z + a * (t11.z - t01.z)) - (t00.z + a * (t10.z - t00.z)));
	r.w = (t00.w + a * (t10.w - t00.w)) + b * ((t01.w + a * (t11.w - t01.w)) - (t00.w + a * (t10.w - t00.w)));
	return r;
}
RB_D float lut3D(const float* t, float u, float v, float s)
{
	int x0, x1, y0, y1, z0, z1; float a, b, g;
	lutTaps(u, kLutN, x0, x1, a);
	lutTaps(v, kLutN, y0, y1, b);
	lutTaps(s, kLutN, z0, z1, g);
	auto T = [&](int x, int y, int z) { return __ldg(t + (z * kLutN + y) * kLutN + x); };
	const float c00 = T(x0, y0, z0) + a * (T(x1, y0, z0) - T(x0, y0, z0));
	const float c10 = T(x0, y1, z0) + a * (T(x1, y1, z0) - T(x0, y1, z0));
	const float c01 = T(x0, y0, z1) + a * (T(x1, y0, z1) - T(x0, y0, z1));
	const float c11 = T(x0, y1, z1) + a * (T(x1, y1, z1) - T(x0, y1, z1));
	const float c0 = c00 + b * (c10 - c00);
	const float c1 = c01 + b * (c11 - c01);
	return c0 + g * (c1 - c0);
}

// ------------------------------------------------------------- LTC sheen
// src/device/surface.h:34-90.
RB_D f3 ltcSample(f3 wo, float A, float B, float u, float v)
{
	const f3 w0 = cosWeightedSample(u, v);
	const f3 ws = mk(w0.x / A - w0.z * B / A, w0.y / A, w0.z);
	const float st = sinThetaFromCos2(wo.z * wo.z);
	const float cp = cosPhiWith(wo, st), sp = sinPhiWith(wo, st);
	const f3 wi = mk(cp * ws.x - sp * ws.y, cp * ws.y + sp * ws.x, ws.z);
	return normalize(wo.z > 0.0f ? wi : -wi);
}
RB_D void ltcEvaluate(f3 wo, f3 wi, float A, float B, float& f, float& pdf)
{
	const float st = sinThetaFromCos2(wo.z * wo.z);
	const float cp = cosPhiWith(wo, st), sp = sinPhiWith(wo, st);
	const f3 ws = mk(cp * wi.x + sp * wi.y, cp * wi.y - sp * wi.x, wi.z);
	f3 w0 = mk(A * ws.x + B * ws.z, A * ws.y, ws.z);
	const float len = length(w0);
	w0 = w0 / len;
	const float det = A * A;
	const float jac = det / (len * len * len);
	const float r = cosWeightedPdf(w0.z) * jac;
	f = r / fabsf(wi.z);
	pdf = r;
}

RB_D float powerHeuristic(float f, float g)   // MIS::powerHeuristic(1, f, 1, g), src/device/mis.h:14-21
{
	const float ff = 1.0f * f, gg = 1.0f * g;
	const float sf = ff * ff, sg = gg * gg;
	return sf / (sf + sg);
}

// ---------------------------------------------------------------- BxDFs
// Surface description built by the shading step (microsurface::Surface, surface.h:380-418).
struct Surface
{
	uint32_t layers;      // 1 base, 2 sheen
	f3 baseColor;
	float metalness;
	float ior;
	float roughness;
	float transmission;
	f3 sheenColor;
	float sheenAlpha;
};
RB_D Surface defaultSurface()
{
	Surface s;
	s.layers = 1u;
	s.baseColor = mk(1.0f);
	s.metalness = 1.0f;
	s.ior = 1.5f;
	s.roughness = 1.0f;
	s.transmission = 0.0f;
	s.sheenColor = mk(1.0f);
	s.sheenAlpha = 0.0f;
	return s;
}

// Light sample handed to the BxDF (DirectLightSampleData, pathtrace.cu:77-83).
struct LightSample
{
	S4 spectrum;
	f3 dir;
	float pdf;
	bool occluded;
};

// In/out path state the callables update. Where the reference adds the
// light sample's contribution to L inside the callable, this state returns
// it in `nee` (hasNee set); the caller adds it once the shadow ray is known to
// be unoccluded (L += nee is the same float operation, done later).
struct BxdfState
{
	S4 nee;
	bool hasNee;
	Wavelengths wl;
	S4 T;
	float pdf;
	f3 dir;
	uint32_t flags;
	float refractionScale;
};

// Which part of a BxDF callable runs: the evaluation of the light sample
// (the callable's direct-lighting block), the BxDF sample and everything
// after it, or the whole body. The two parts read disjoint outputs of each
// other: the light part writes only `nee`/`hasNee`, the sample part never
// reads them, so running the parts in two kernels gives the whole body's
// results bit for bit.
enum BxdfPart : int { kBxdfAll = 0, kBxdfLight = 1, kBxdfSample = 2 };

// __direct_callable__PureConductorBxDF (pathtrace.cu:464-547).
template<int PART>
RB_D void bxdfPureConductor(const DevScene& sc, const DevMaterial& mat, const LightSample& dl, const Qrng& q,
	const Frame& local, BxdfState& s)
{
	f3 wo = local.toLocal(-s.dir);
	const f3 li = local.toLocal(dl.dir);
	if (wo.z == 0.0f) { s.flags |= PF_PATH_TERMINATED; return; }
	const float* etaT = sc.spectra.extra + static_cast<size_t>(mat.iorSpectrum) * kSpectrumBins;
	const float* kT = sc.spectra.extra + static_cast<size_t>(mat.absorpSpectrum) * kSpectrumBins;
	const S4 eta = denseSample(etaT, s.wl.lambda);
	const S4 k = denseSample(kT, s.wl.lambda);
	const float alpha = mat.mfRoughness * mat.mfRoughness;
	float ax = alpha, ay = alpha;
	if (s.flags & PF_REGULARIZED)
	{
		if (ax < 0.3f) ax = clampf(2.0f * ax, 0.1f, 0.3f);
		if (ay < 0.3f) ay = clampf(2.0f * ay, 0.1f, 0.3f);
	}
	const CtxDir co = ctxDir(wo);
	if (alpha < 0.001f)
	{
		const f3 wi = mk(-wo.x, -wo.y, wo.z);
		s.T *= fresnelComplex(fabsf(wi.z), eta, k);
		s.pdf = 1.0f;
		s.flags |= PF_CURRENT_HIT_SPECULAR;
		s.dir = normalize(local.fromLocal(wi));
		return;
	}
	if (PART != kBxdfSample && !dl.occluded)
	{
		const f3 wi = li;
		if (wo.z * wi.z > 0.0f)
		{
			const CtxDir ci = ctxDir(wi);
			f3 wm = normalize(wi + wo);
			const CtxM cm = ctxM(wm);
			const float ad = fabsf(dot(wo, wm));
			const S4 f = ggxD(cm, ax, ay) * fresnelComplex(ad, eta, k) * G2(ci, co, ax, ay)
				/ fabsf(4.0f * wo.z * wi.z);
			const float cosF = fabsf(wi.z);
			wm = wm.z > 0.0f ? wm : -wm;
			const float lp = vndfPdfBounded(wo, ad, cm, ax, ay) / (4.0f * ad);
			s.nee = dl.spectrum * f * s.T * cosF * powerHeuristic(dl.pdf, lp) / dl.pdf;
			s.hasNee = true;
		}
	}
	if (PART == kBxdfLight) return;
	float u, v;
	sample2D(q, DIM_BXDF_0, u, v);
	const f3 wm = vndfSampleBounded(wo, ax, ay, u, v);
	const CtxM cm = ctxM(wm);
	const f3 wi = reflectAbout(wo, wm);
	const CtxDir ci = ctxDir(wi);
	if (wo.z * wi.z <= 0.0f) { s.flags |= PF_PATH_TERMINATED; return; }
	const float ad = fabsf(dot(wo, wm));
	const S4 f = ggxD(cm, ax, ay) * fresnelComplex(ad, eta, k) * G2(ci, co, ax, ay) / fabsf(4.0f * wo.z * wi.z);
	const float cosF = fabsf(wi.z);
	s.pdf = vndfPdfBounded(wo, ad, cm, ax, ay) / (4.0f * ad);
	s.T *= f * cosF / s.pdf;
	s.dir = normalize(local.fromLocal(wi));
}

// __direct_callable__ComplexSurface_BxDF (pathtrace.cu:548-905): sheen over a
// metal / dielectric-specular / translucent / glossy-diffuse base.
template<int PART>
RB_D void bxdfComplexSurface(const DevScene& sc, const LightSample& dl, const Qrng& q, const Frame& local,
	const Surface& surf, BxdfState& s)
{
	const f3 wo = local.toLocal(-s.dir);
	const f3 li = local.toLocal(dl.dir);
	if (wo.z == 0.0f) { s.flags |= PF_PATH_TERMINATED; return; }
	const CtxDir co = ctxDir(wo);

	float roughness = surf.roughness;
	bool perfectSpecular = false;
	if (roughness < 0.001f) { roughness = 0.001f; perfectSpecular = true; }
	const float alpha = roughness * roughness;
	const float ax = alpha, ay = alpha;

	const float eta = wo.z > 0.0f ? surf.ior / 1.0f : 1.0f / surf.ior;
	const float f0Sr = (1.0f - eta) / (1.0f + eta);
	const float f0 = f0Sr * f0Sr;
	const float absCosO = fabsf(wo.z);
	const float lutW = sqrtf(fabsf(f0Sr));
	const float ecDielectric = 1.0f / lut3D(eta > 1.0f ? sc.luts.dielOuter : sc.luts.dielInner, absCosO, roughness, lutW);
	const float epDiffuse = 1.0f - lut3D(eta > 1.0f ? sc.luts.reflOuter : sc.luts.reflInner, absCosO, roughness, lutW);
	const float albedoConductor = lut2D(sc.luts.conductor, absCosO, roughness);
	float albedoSheen = 0.0f;
	float ltcA = 0.0f, ltcB = 0.0f;
	if (surf.layers & 2u)
	{
		const float4 d = lut2D4(sc.luts.sheen, absCosO, surf.sheenAlpha);
		ltcA = d.x; ltcB = d.y; albedoSheen = d.z;
		if (albedoSheen < 0.0001f) albedoSheen = 0.0f;
	}
	const float* basis = sc.spectra.basis;

	// Direct lighting (pathtrace.cu:660-771).
	if (PART != kBxdfSample && !dl.occluded)
	{
		const f3 wi = li;
		const CtxDir ci = ctxDir(wi);
		const float cosI = wi.z, cosO = wo.z;
		const float cosF = fabsf(cosI);
		const bool refl = cosI * cosO > 0.0f;
		const float etaR = refl ? 1.0f : eta;
		f3 wm = normalize(wi * etaR + wo);
		if (wm.z < 0.0f) wm = -wm;
		const CtxM cm = ctxM(wm);
		const float dmo = dot(wm, wo), dmi = dot(wm, wi);
		const float ad = fabsf(dot(wo, wm));
		const float Fd = fresnelSchlick(f0, ad);
		const float Ds = ggxD(cm, ax, ay);
		const float Gs = G2(ci, co, ax, ay);
		const float sheen = albedoSheen;
		const float base = 1.0f - sheen;
		const float metal = surf.metalness;
		const float transl = surf.transmission;
		const float wSheen = sheen;
		const float wCSpec = base * metal;
		const float wDSpec = base * (1.0f - metal) * Fd;
		const float wDTrans = base * (1.0f - metal) * transl * (1.0f - Fd);
		const float wDiff = base * (1.0f - metal) * (1.0f - transl) * (1.0f - Fd);
		S4 flSheen = s4(0.0f);
		float pSheen = 1.0f;
		if (sheen != 0.0f)
		{
			float fNo = 0.0f;
			ltcEvaluate(wo, wi, ltcA, ltcB, fNo, pSheen);
			flSheen = rgbToSpectrum(basis, surf.sheenColor, s.wl.lambda) * fNo;
		}
		if (refl)
		{
			S4 flCond = s4(0.0f);
			float flDiel = 0.0f, pSpec = 0.0f;
			if (!perfectSpecular)
			{
				const S4 Fc = rgbToSpectrum(basis, fresnelF82(surf.baseColor, ad)
					* (mk(1.0f) + fresnelAvgF82(surf.baseColor) * ((1.0f - albedoConductor) / albedoConductor)), s.wl.lambda);
				flCond = Ds * Gs * Fc / fabsf(4.0f * wo.z * wi.z);
				flDiel = Ds * Gs * ecDielectric / fabsf(4.0f * wo.z * wi.z);
				pSpec = vndfPdfCap(wo, ad, co, cm, ax, ay) / (4.0f * ad);
			}
			const S4 flDiff = epDiffuse * rgbToSpectrum(basis, surf.baseColor, s.wl.lambda) / kPi;
			const float pDiff = cosWeightedPdf(wi.z);
			const float pdf = wSheen * pSheen + wCSpec * pSpec + wDSpec * pSpec + wDiff * pDiff;
			const float mis = powerHeuristic(dl.pdf, pdf);
			s.nee = dl.spectrum * s.T * cosF * mis
				* (wSheen * flSheen + wCSpec * flCond + s4(wDSpec * flDiel) + wDiff * flDiff) / dl.pdf;
			s.hasNee = true;
		}
		else if (surf.transmission != 0.0f && !(dmo * cosO <= 0.0f || dmi * cosI <= 0.0f))
		{
			float pTrans = 0.0f;
			S4 flTrans = s4(0.0f);
			if (!perfectSpecular)
			{
				const float t = dmi + dmo / eta;
				const float denom = t * t;
				const float dwm = fabsf(dmi) / denom;
				pTrans = vndfPdfCap(wo, ad, co, cm, ax, ay) * dwm;
				flTrans = rgbToSpectrum(basis, surf.baseColor, s.wl.lambda)
					* Ds * (1.0f - Fd) * Gs * ecDielectric * fabsf(dmo * dmi / (cosO * cosI * denom));
			}
			const float pdf = wSheen * pSheen + wDTrans * pTrans;
			const float mis = powerHeuristic(dl.pdf, pdf);
			flTrans /= (eta * eta);
			s.nee = dl.spectrum * s.T * cosF * mis * (wSheen * flSheen + wDTrans * flTrans) / dl.pdf;
			s.hasNee = true;
		}
	}

	if (PART == kBxdfLight) return;
	// BxDF sampling (pathtrace.cu:773-892).
	f3 wi;
	{
		const f3 r = sample3D(q, DIM_BXDF_0);
		const float sheen = albedoSheen;
		const float base = 1.0f - sheen;
		const float sheenP = sheen, baseP = base;
		const float baseCorr = 1.0f - albedoSheen;
		if (r.z > baseP)
		{
			float fNo = 0.0f, pP = 0.0f;
			wi = ltcSample(wo, ltcA, ltcB, r.x, r.y);
			ltcEvaluate(wo, wi, ltcA, ltcB, fNo, pP);
			const S4 f = rgbToSpectrum(basis, surf.sheenColor, s.wl.lambda) * fNo * sheen;
			s.pdf = pP * sheenP;
			s.T *= f * fabsf(wi.z) / s.pdf;
		}
		else
		{
			const f3 wm = vndfSampleCap(wo, ax, ay, r.x, r.y);
			const CtxM cm = ctxM(wm);
			const float ad = fabsf(dot(wo, wm));
			const float Ds = ggxD(cm, ax, ay);
			float Fd = fresnelSchlick(f0, ad);
			const float s2i = fmaxf(0.0f, 1.0f - ad * ad);
			const float s2t = s2i / (eta * eta);
			if (s2t >= 1.0f) Fd = 1.0f;
			const float metal = surf.metalness;
			const float transl = surf.transmission;
			const float pCond = base * metal;
			const float pDSpec = base * (1.0f - metal) * Fd;
			const float pTrans = base * transl * (1.0f - metal) * (1.0f - Fd);
			if (r.z < pCond + pDSpec)
			{
				wi = normalize(reflectAbout(wo, wm));
				const CtxDir ci = ctxDir(wi);
				if (wo.z * wi.z <= 0.0f) { s.flags |= PF_PATH_TERMINATED; return; }
				const float Gs = G2(ci, co, ax, ay);
				const float spec = Ds * Gs / fabsf(4.0f * wo.z * wi.z);
				S4 f;
				float pP;
				if (r.z < pCond)
				{
					const S4 Fc = rgbToSpectrum(basis, fresnelF82(surf.baseColor, ad)
						* (mk(1.0f) + fresnelAvgF82(surf.baseColor) * ((1.0f - albedoConductor) / albedoConductor)), s.wl.lambda);
					f = spec * Fc * metal;
					pP = pCond;
				}
				else
				{
					f = s4(spec * Fd * ecDielectric * (1.0f - metal));
					pP = pDSpec;
				}
				const float cosF = fabsf(wi.z);
				s.pdf = vndfPdfCap(wo, ad, co, cm, ax, ay) / (4.0f * ad) * pP;
				s.T *= f * cosF * baseCorr / s.pdf;
			}
			else if (r.z < pCond + pDSpec + pTrans)
			{
				wi = refractSimple(wo, wm, eta);
				s.refractionScale *= eta;
				if (wo.z * wi.z >= 0.0f) { s.flags |= PF_PATH_TERMINATED; return; }
				const CtxDir ci = ctxDir(wi);
				const float Gs = G2(ci, co, ax, ay);
				const float cosI = wi.z, cosO = wo.z;
				const float dmo = dot(wm, wo), dmi = dot(wm, wi);
				const float t = dmi + dmo / eta;
				const float denom = t * t;
				const float dwm = fabsf(dmi) / denom;
				float f = Ds * (1.0f - Fd) * Gs * (1.0f - metal) * transl * fabsf(dmo * dmi / (cosO * cosI * denom));
				f /= (eta * eta);
				s.pdf = vndfPdfCap(wo, ad, co, cm, ax, ay) * dwm * pTrans;
				const float cosF = fabsf(cosI);
				s.T *= rgbToSpectrum(basis, surf.baseColor, s.wl.lambda) * f * ecDielectric * cosF * baseCorr / s.pdf;
				s.flags |= PF_RAY_REFRACTED;
			}
			else
			{
				float u, v;
				sample2D(q, DIM_BXDF_1, u, v);
				wi = cosWeightedSample(u, v);
				if (wo.z * wi.z <= 0.0f) { s.flags |= PF_PATH_TERMINATED; return; }
				const float cosF = fabsf(wi.z);
				const S4 f = rgbToSpectrum(basis, surf.baseColor, s.wl.lambda) / kPi * (1.0f - metal) * (1.0f - transl);
				s.pdf = cosWeightedPdf(wi.z) * (base * (1.0f - transl) * (1.0f - metal) * (1.0f - Fd));
				s.T *= f * epDiffuse * cosF * baseCorr / s.pdf;
			}
		}
	}
	if (s.pdf <= 0.0f || isinf(s.pdf)) { s.flags |= PF_PATH_TERMINATED; return; }
	s.dir = normalize(local.fromLocal(wi));
}

// Dispatch on the material's callable index, as optixDirectCall does with
// MaterialData::bxdfIndexSBT (pathtrace.cu:1724-1733). Index 1 (the pure
// dielectric callable) has an empty body in the reference and changes nothing.
template<int PART = kBxdfAll>
RB_D void evalBxdf(const DevScene& sc, const DevMaterial& mat, const LightSample& dl, const Qrng& q,
	const Frame& local, const Surface& surf, BxdfState& s)
{
	if (mat.bxdf == 2u)
		bxdfComplexSurface<PART>(sc, dl, q, local, surf, s);
	else if (mat.bxdf == 0u)
		bxdfPureConductor<PART>(sc, mat, dl, q, local, s);
}
} // namespace rb
