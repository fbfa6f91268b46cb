// Light selection and emission: spherical-Gaussian light-tree importance
// (Tokuyoshi et al. 2024, as in src/core/math_util.h:229-588), light-tree
// sampling and pdf replay (src/kernels/pathtrace.cu:974-1112), environment
// map lookup and inverted-CDF sampling (:1234-1256, 1655-1694), plus the
// octahedral codes and ray-origin offset shared by the shading step.
#pragma once

#include <cfloat>

#include "rb_math.cuh"
#include "rb_qrng.cuh"
#include "rb_scene.h"

namespace rb
{
// ------------------------------------------------------------- octahedral
// Octohedral::decode (src/core/math_util.h:176-191).
RB_HD f3 octDecode(float u, float v)
{
	f3 r;
	r.z = 1.0f - fabsf(u) - fabsf(v);
	r.x = u;
	r.y = v;
	const float t = fmaxf(0.0f, -r.z);
	r.x += r.x >= 0.0f ? -t : t;
	r.y += r.y >= 0.0f ? -t : t;
	return normalize(r);
}
// Octohedral::decodeU32 (:217-224).
RB_HD f3 octDecodeU32(uint32_t e)
{
	const float n = 1.0f / 65535.0f;
	const float px = static_cast<float>(e & 0xFFFFu) * n;
	const float py = static_cast<float>(e >> 16) * n;
	return octDecode(px * 2.0f - 1.0f, py * 2.0f - 1.0f);
}
// Octohedral::encodeU32 (:199-212).
RB_HD uint32_t octEncodeU32(f3 v)
{
	const float inv = 1.0f / (fabsf(v.x) + fabsf(v.y) + fabsf(v.z));
	float px = v.x * inv, py = v.y * inv;
	if (v.z <= 0.0f)
	{
		const float ox = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f);
		const float oy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
		px = ox; py = oy;
	}
	const float q = 65535.99f;
	const uint32_t x = static_cast<uint32_t>(clampf(px * 0.5f + 0.5f, 0.0f, 1.0f) * q);
	const uint32_t y = static_cast<uint32_t>(clampf(py * 0.5f + 0.5f, 0.0f, 1.0f) * q) << 16;
	return y | x;
}

// utility::offsetPoint (src/device/util.h:15-30): move a surface point off
// the surface along n by 256 float ulps (1/65536 absolute near the origin).
RB_D f3 offsetPoint(f3 p, f3 n)
{
	const float interval = 1.0f / 32.0f, fscale = 1.0f / 65536.0f, iscale = 256.0f;
	const int ix = static_cast<int>(iscale * n.x), iy = static_cast<int>(iscale * n.y), iz = static_cast<int>(iscale * n.z);
	const float ox = __int_as_float(__float_as_int(p.x) + (p.x < 0.0f ? -ix : ix));
	const float oy = __int_as_float(__float_as_int(p.y) + (p.y < 0.0f ? -iy : iy));
	const float oz = __int_as_float(__float_as_int(p.z) + (p.z < 0.0f ? -iz : iz));
	return f3{ fabsf(p.x) < interval ? p.x + fscale * n.x : ox,
	           fabsf(p.y) < interval ? p.y + fscale * n.y : oy,
	           fabsf(p.z) < interval ? p.z + fscale * n.z : oz };
}

// --------------------------------------------------------- SG toolkit
namespace sg
{
constexpr float kPiSG = 3.14159265359f;   // SphericalGaussian::Math::PI
RB_D float mulsign(float x, float y) { return __uint_as_float((__float_as_uint(y) & 0x80000000u) ^ __float_as_uint(x)); }
// exp(x) - 1 and (exp(x) - 1)/x with Higham's cancellation trick;
// expm1cOf takes u = expf(x) already computed.
RB_D float expm1cOf(float x, float u)
{
	if (u == 1.0f) return x;
	const float y = u - 1.0f;
	if (fabsf(x) < 1.0f) return y * x / logf(u);
	return y;
}
RB_D float expm1c(float x) { return expm1cOf(x, expf(x)); }
RB_D float expm1OverX(float x)
{
	const float u = expf(x);
	if (u == 1.0f) return 1.0f;
	const float y = u - 1.0f;
	if (fabsf(x) < 1.0f) return y / logf(u);
	return y / x;
}
// Polynomial erf approximation (math_util.h:292-327).
RB_D float erfApprox(float x)
{
	if (fabsf(x) >= 4.0f) return mulsign(1.0f, x);
	if (fabsf(x) > 1.0f)
	{
		const float A1 = 1.628459513f, A2 = 9.15674746e-1f, A3 = 1.54329389e-1f, A4 = -3.51759829e-2f,
			A5 = 5.66795561e-3f, A6 = -5.64874616e-4f, A7 = 2.58907676e-5f;
		const float a = fabsf(x);
		const float y = 1.0f - exp2f(-(((((((A7 * a + A6) * a + A5) * a + A4) * a + A3) * a + A2) * a + A1) * a));
		return mulsign(y, x);
	}
	const float A1 = 1.128379121f, A2 = -3.76123011e-1f, A3 = 1.12799220e-1f, A4 = -2.67030653e-2f,
		A5 = 4.90735564e-3f, A6 = -5.58853149e-4f;
	const float x2 = x * x;
	return (((((A6 * x2 + A5) * x2 + A4) * x2 + A3) * x2 + A2) * x2 + A1) * x;
}
RB_D float erfcApprox(float x) { return 1.0f - erfApprox(x); }
RB_D float integral(float s) { return 4.0f * kPiSG * expm1OverX(-2.0f * s); }

struct Lobe
{
	f3 axis;
	float sharpness;
	float logAmplitude;
};
RB_D Lobe product(f3 a1, float s1, f3 a2, float s2)
{
	const f3 axis = a1 * s1 + a2 * s2;
	const float sharp = length(axis);
	// (cosine - 1) below cancels for nearly aligned lobes: keep the dot
	// product uncontracted so it rounds as the reference's does.
	const float cosine = clampf(dotRn(a1, a2), -1.0f, 1.0f);
	const float sMin = fminf(s1, s2);
	const float ratio = sMin / fmaxf(fmaxf(s1, s2), FLT_MIN);
	const float logAmp = 2.0f * sMin * (cosine - 1.0f) / (sqrtf(2.0f * ratio * cosine + ratio * ratio + 1.0f) + ratio + 1.0f);
	return Lobe{ axis / fmaxf(sharp, FLT_MIN), sharp, logAmp };
}
// SG x clamped-cosine product integral / pi (Tokuyoshi et al. 2024, Listing 7; math_util.h:508-534).
RB_D float clampedCosineProductOverPi2024(float cosine, float s)
{
	const float A = 2.7360831611272558028247203765204f, B = 17.02129778174187535455530451145f,
		C = 4.0100826728510421403939290030394f, D = 15.219156263147210594866010069381f,
		E = 76.087896272360737270901154261082f;
	const float t = s * sqrtf(0.5f * ((s + A) * s + B) / (((s + C) * s + D) * s + E));
	const float tz = t * cosine;
	const float invSqrtPi = 0.56418958354775628694807945156077f;
	const float clampTh = 0.5f * FLT_EPSILON;
	const float lerp = clampf(fmaxf(0.5f * (cosine * erfcApprox(-tz) + erfcApprox(t))
		- 0.5f * invSqrtPi * expf(-tz * tz) * expm1c(t * t * (cosine * cosine - 1.0f)) / t, clampTh), 0.0f, 1.0f);
	// LowerClampedCosineIntegralOverTwoPi(s) and
	// UpperClampedCosineIntegralOverTwoPi(s) (math_util.h:464-506), with
	// exp(-s) and expm1c(-s) evaluated once for both: the same operations on
	// the same values.
	const float e = expf(-s);
	float lo, up;
	if (s <= 0.5f)
	{
		lo = e * (((((((((1.0f / 403200.0f) * s - 1.0f / 45360.0f) * s + 1.0f / 5760.0f) * s - 1.0f / 840.0f) * s
			+ 1.0f / 144.0f) * s - 1.0f / 30.0f) * s + 1.0f / 8.0f) * s - 1.0f / 3.0f) * s + 0.5f);
		up = (((((((-1.0f / 362880.0f) * s + 1.0f / 40320.0f) * s - 1.0f / 5040.0f) * s + 1.0f / 720.0f) * s
			- 1.0f / 120.0f) * s + 1.0f / 24.0f) * s - 1.0f / 6.0f) * s + 0.5f;
	}
	else
	{
		const float m = expm1cOf(-s, e);
		lo = e * (-m - s * e) / (s * s);
		up = (m + s) / (s * s);
	}
	return 2.0f * mixf(lo, up, lerp);
}
} // namespace sg

// ------------------------------------------------------------- light tree
struct TreeNode
{
	f3 mean;
	float variance;
	f3 direction;
	float sharpness;
	float flux;
	bool leaf;
	uint32_t a;   // branch: right child; leaf: light count
	uint32_t b;   // leaf: light offset
};
// LightTree::unpackNode (src/core/light_tree_types.h:165-189). The average
// direction is decoded from the raw [0,1] code pair exactly as the
// reference's unpackNode does it (without the [-1,1] remap of decodeU32).
RB_D TreeNode unpackNode(const PackedNode* nodes, uint32_t i)
{
	const float4 q0 = __ldg(reinterpret_cast<const float4*>(nodes + i));
	const float4 q1 = __ldg(reinterpret_cast<const float4*>(nodes + i) + 1);
	TreeNode n;
	n.mean = mk(q0.x, q0.y, q0.z);
	n.variance = q0.w;
	const uint32_t dir = __float_as_uint(q1.x);
	n.sharpness = q1.y;
	n.flux = q1.z;
	const uint32_t core = __float_as_uint(q1.w);
	n.direction = octDecode(static_cast<float>(dir & 0xFFFFu) / 65535.0f, static_cast<float>(dir >> 16) / 65535.0f);
	n.leaf = (core >> 31) != 0u;
	if (n.leaf)
	{
		n.a = (core >> 27) & 0xFu;
		n.b = core & ((1u << 27) - 1u);
	}
	else
	{
		n.a = core;
		n.b = 0;
	}
	return n;
}
// evaluateNodeImportance (pathtrace.cu:974-1001).
RB_D float nodeImportance(const TreeNode& n, f3 p, f3 nrm)
{
	f3 ld = n.mean - p;
	const float d2 = dotRn(ld, ld);
	ld *= __frsqrt_rn(d2);
	const float var = fmaxf(n.variance, 0x1.0p-31f * d2);
	const float sharp = d2 / var;
	const sg::Lobe lobe = sg::product(n.direction, n.sharpness, ld, sharp);
	const float amp = expf(lobe.logAmplitude);
	const float cosine = clampf(dot(lobe.axis, nrm), -1.0f, 1.0f);
	return (n.flux / (var * sg::integral(n.sharpness))) * amp * sg::clampedCosineProductOverPi2024(cosine, lobe.sharpness);
}

// Light-tree node unpacked once per tree on the device (kUnpackLightTree,
// TreeNodeU in rb_scene.h): the decoded average direction and the SG integral
// of the node's sharpness are stored, so the per-sample descent does only the
// point-dependent part, with three 16-B loads per node.
RB_D TreeNodeU makeNodeU(const PackedNode* nodes, uint32_t i)
{
	const TreeNode n = unpackNode(nodes, i);
	TreeNodeU u;
	u.meanVar = make_float4(n.mean.x, n.mean.y, n.mean.z, n.variance);
	u.dirSharp = make_float4(n.direction.x, n.direction.y, n.direction.z, n.sharpness);
	u.fluxInt = make_float4(n.flux, sg::integral(n.sharpness), __uint_as_float(n.a),
		__uint_as_float(n.b | (n.leaf ? 0x80000000u : 0u)));
	return u;
}
RB_D bool nodeLeaf(const TreeNodeU& u) { return (__float_as_uint(u.fluxInt.w) >> 31) != 0u; }
RB_D uint32_t nodeA(const TreeNodeU& u) { return __float_as_uint(u.fluxInt.z); }
RB_D uint32_t nodeB(const TreeNodeU& u) { return __float_as_uint(u.fluxInt.w) & 0x7FFFFFFFu; }
// Node load from global memory through the read-only cache, or (SHARED)
// from a copy of the tree in shared memory.
template<bool SHARED = false>
RB_D TreeNodeU loadNodeU(const TreeNodeU* nodes, uint32_t i)
{
	if (SHARED) return nodes[i];
	TreeNodeU u;
	u.meanVar = __ldg(&nodes[i].meanVar);
	u.dirSharp = __ldg(&nodes[i].dirSharp);
	u.fluxInt = __ldg(&nodes[i].fluxInt);
	return u;
}
// nodeImportance on an unpacked node: the same float operations in the same order.
RB_D float nodeImportanceU(const TreeNodeU& n, f3 p, f3 nrm)
{
	f3 ld = f3_of(n.meanVar) - p;
	const float d2 = dotRn(ld, ld);
	ld *= __frsqrt_rn(d2);
	const float var = fmaxf(n.meanVar.w, 0x1.0p-31f * d2);
	const float sharp = d2 / var;
	const sg::Lobe lobe = sg::product(f3_of(n.dirSharp), n.dirSharp.w, ld, sharp);
	const float amp = expf(lobe.logAmplitude);
	const float cosine = clampf(dot(lobe.axis, nrm), -1.0f, 1.0f);
	return (n.fluxInt.x / (var * n.fluxInt.y)) * amp * sg::clampedCosineProductOverPi2024(cosine, lobe.sharpness);
}

// traverseLightTree: pdf of picking light (type, index) from p with normal n.
RB_D float lightTreePdf(const DevScene& sc, uint32_t type, uint32_t index, f3 p, f3 nrm)
{
	const float envImp = sc.env.enabled ? kEnvMapImportance : 0.0f;
	if (type == kLightTypeSky) return envImp;
	float pdf = 1.0f - envImp;
	const uint64_t mask = sc.lights.bitmasks[index];
	const TreeNodeU* nodes = sc.lights.unpacked;
	uint32_t cur = 0;
	TreeNodeU node = loadNodeU(nodes, 0);
	for (int depth = 0; depth < 64; ++depth)
	{
		if (nodeLeaf(node)) break;
		const TreeNodeU l = loadNodeU(nodes, cur + 1);
		const float li = nodeImportanceU(l, p, nrm);
		const TreeNodeU r = loadNodeU(nodes, nodeA(node));
		const float ri = nodeImportanceU(r, p, nrm);
		const bool right = (mask >> depth) & 1ull;
		cur = right ? nodeA(node) : cur + 1;
		node = right ? r : l;
		pdf *= right ? ri / (li + ri) : li / (li + ri);
	}
	pdf *= 1.0f / static_cast<float>(nodeA(node));
	return pdf;
}

// sampleLightTree: pick the environment (0.3 when both exist) or descend the
// tree choosing children by importance with rescaled `rand`. `nodes` is the
// unpacked tree in shared or global memory.
template<bool SHARED = false>
RB_D void lightTreeSample(const DevScene& sc, const TreeNodeU* nodes, float rand, f3 p, f3 nrm, uint32_t& type,
	uint32_t& index, float& pdf)
{
	const bool envPresent = sc.env.enabled != 0;
	const bool treePresent = sc.lights.nodes != nullptr;
	const float envImp = envPresent ? (treePresent ? kEnvMapImportance : 1.0f) : 0.0f;
	if (rand < envImp)
	{
		type = kLightTypeSky; index = 0; pdf = envImp;
		return;
	}
	rand = clampf((rand - envImp) / (1.0f - envImp), 0.0f, 1.0f);
	pdf = 1.0f - envImp;
	uint32_t cur = 0;
	TreeNodeU node = loadNodeU<SHARED>(nodes, 0);
	while (!nodeLeaf(node))
	{
		const TreeNodeU l = loadNodeU<SHARED>(nodes, cur + 1);
		const TreeNodeU r = loadNodeU<SHARED>(nodes, nodeA(node));
		const float li = nodeImportanceU(l, p, nrm);
		const float ri = nodeImportanceU(r, p, nrm);
		const float sep = li / (li + ri);
		const bool right = rand > sep;
		cur = right ? nodeA(node) : cur + 1;
		node = right ? r : l;
		pdf *= right ? 1.0f - sep : sep;
		rand = right ? clampf((rand - sep) / (1.0f - sep), 0.0f, 1.0f) : clampf(rand / sep, 0.0f, 1.0f);
	}
	const uint32_t count = nodeA(node);
	const uint32_t k = static_cast<uint32_t>(static_cast<float>(count) * rand);
	const uint32_t slot = nodeB(node) + (k == count ? count - 1u : k);
	pdf *= 1.0f / static_cast<float>(count);
	const uint32_t ptr = __ldg(sc.lights.pointers + slot);
	type = ptr >> 30;
	index = ptr & ((1u << 30) - 1u);
	if (isnan(pdf) || isinf(pdf) || pdf == 0.0f) type = kLightTypeNone;
}

// ---------------------------------------------------------- environment
// Bilinear fetch with normalized coordinates and clamp addressing.
RB_D float4 envFetch(const DevEnvMap& e, float u, float v)
{
	auto taps = [](float c, int n, int& i0, int& i1, float& a) {
		const float x = c * static_cast<float>(n) - 0.5f;
		const float fl = floorf(x);
		a = x - fl;
		const int i = static_cast<int>(fl);
		i0 = min(max(i, 0), n - 1);
		i1 = min(max(i + 1, 0), n - 1);
	};
	int x0, x1, y0, y1; float a, b;
	taps(u, static_cast<int>(e.w), x0, x1, a);
	taps(v, static_cast<int>(e.h), y0, y1, b);
	const float4 t00 = __ldg(e.texels + static_cast<size_t>(y0) * e.w + x0);
	const float4 t10 = __ldg(e.texels + static_cast<size_t>(y0) * e.w + x1);
	const float4 t01 = __ldg(e.texels + static_cast<size_t>(y1) * e.w + x0);
	const float4 t11 = __ldg(e.texels + static_cast<size_t>(y1) * e.w + x1);
	auto lerp2 = [&](float c00, float c10, float c01, float c11) {
		const float r0 = c00 + a * (c10 - c00);
		const float r1 = c01 + a * (c11 - c01);
		return r0 + b * (r1 - r0);
	};
	return make_float4(lerp2(t00.x, t10.x, t01.x, t11.x), lerp2(t00.y, t10.y, t01.y, t11.y),
		lerp2(t00.z, t10.z, t01.z, t11.z), lerp2(t00.w, t10.w, t01.w, t11.w));
}
// Radiance seen along d when a ray escapes, and its light-sampling pdf
// (pathtrace.cu:1236-1249).
RB_D void envEmission(const DevScene& sc, f3 d, const S4& lambda, S4& Le, float& lightPdf)
{
	const float phi = atan2f(d.y, d.x);
	const float theta = acosf(d.z);
	const float4 c = envFetch(sc.env, 0.5f - phi / (2.0f * kPi), theta / kPi);
	const float surfacePdf = 1.0f / (4.0f * kPi);
	lightPdf = surfacePdf * ((c.x + c.y + c.z) / 3.0f) * sinf(theta) / __ldg(sc.env.integral);
	Le = rgbToSpectrum(sc.spectra.basis, mk(c.x, c.y, c.z), lambda);
}
// Importance sample of the map from interpolated inverted-CDF indices (pathtrace.cu:1657-1689).
RB_D void envSample(const DevScene& sc, float rx, float ry, const S4& lambda, f3& dir, S4& spectrum, float& lightPdf)
{
	const DevEnvMap& e = sc.env;
	const float fx = fminf(rx * (e.width - 1.0f), e.width - 1.0001f);
	const float fy = fminf(ry * (e.height - 1.0f), e.height - 1.0001f);
	const float flx = floorf(fx), fly = floorf(fy);
	const float frx = fx - flx, fry = fy - fly;
	const uint32_t ix = static_cast<uint32_t>(flx), iy = static_cast<uint32_t>(fly);
	const float m0 = static_cast<float>(__ldg(e.marginal + iy));
	const float m1 = static_cast<float>(__ldg(e.marginal + iy + 1));
	const uint32_t row = static_cast<uint32_t>(m0 * e.width);
	const float c0 = static_cast<float>(__ldg(e.conditional + row + ix));
	const float c1 = static_cast<float>(__ldg(e.conditional + row + ix + 1));
	const float sx = mixf(c0, c1, frx) * (1.0f / e.width);
	const float sy = mixf(m0, m1, fry) * (1.0f / e.height);
	const float phi = 2.0f * kPi * sx;
	const float theta = kPi * sy;
	dir = mk(-sinf(theta) * cosf(phi), sinf(theta) * sinf(phi), cosf(theta));
	const float4 c = envFetch(e, sx, sy);
	spectrum = rgbToSpectrum(sc.spectra.basis, mk(c.x, c.y, c.z), lambda);
	const float surfacePdf = 1.0f / (4.0f * kPi);
	lightPdf = surfacePdf * ((c.x + c.y + c.z) / 3.0f) * sinf(theta) / __ldg(e.integral);
}
} // namespace rb
