// Wavefront rendering kernels and per-function batch kernels.
//
// One wave renders whole sample planes of the image. Per bounce:
//   extend  - closest hit of every active path (rb_bvh.cuh)
//   shade   - the body of the reference's bounce loop
//             (src/kernels/pathtrace.cu:1179-1785): hit emission with MIS,
//             shading frame and material, light-tree / environment light
//             sample, BxDF sample, Russian roulette, next ray; continuing
//             paths go to the next queue, light samples to the shadow queue
//   shadow  - any-hit test of the light samples; unoccluded ones add their
//             contribution to L
// and after the last bounce
//   resolve - L / pdf -> XYZ, summed into the FP64 accumulation in sample
//             order per pixel (pathtrace.cu:1789-1812), so the result does
//             not depend on the order in which paths were processed.
// Kernels are persistent: the grid is sized from the SM count and occupancy,
// and each one reads its work count from device memory, so a whole wave is a
// fixed launch sequence with no host round trip.

#include <cfloat>

#include "rb_bvh.cuh"
#include "rb_bxdf.cuh"
#include "rb_light.cuh"
#include "rb_launch.cuh"
#include "rb_qrng.cuh"
#include "rb_texture.cuh"
#include "rb_wavefront.h"
#include "ratbite_b200_kernels.h"
#include "ratbite_b200_nrc.h"

namespace rb
{
namespace
{
RB_D f3 mulMat(const float* m, f3 v)   // rows of 3
{
	return f3{ m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
	           m[6] * v.x + m[7] * v.y + m[8] * v.z };
}

// Rotation matrix columns of a unit quaternion (glm::mat3_cast order of operations).
RB_D void quatColumns(float4 q, f3& c0, f3& c2)
{
	const float qxx = q.x * q.x, qyy = q.y * q.y, qzz = q.z * q.z;
	const float qxz = q.x * q.z, qxy = q.x * q.y, qyz = q.y * q.z;
	const float qwx = q.w * q.x, qwy = q.w * q.y, qwz = q.w * q.z;
	c0 = mk(1.0f - 2.0f * (qyy + qzz), 2.0f * (qxy + qwz), 2.0f * (qxz - qwy));
	c2 = mk(2.0f * (qxz + qwy), 2.0f * (qyz - qwx), 1.0f - 2.0f * (qxx + qyy));
}

// Branchless orthonormal tangent of a unit normal (pathtrace.cu:1374-1377, 1408-1413).
RB_D f3 tangentOf(f3 n)
{
	const float sign = copysignf(1.0f, n.z);
	const float a = -1.0f / (sign + n.z);
	const float b = n.x * n.y * a;
	return mk(1.0f + sign * (n.x * n.x) * a, sign * b, -sign * n.x);
}

// Surface interaction reconstructed from a hit (unpackInteractionData,
// pathtrace.cu:908-953, with the closest-hit program's payload, :86-149).
struct Interaction
{
	f3 hitPos, hitPosInterp, gn;
	f3 v0, v1, v2;
	float b1, b2;
	uint32_t lightType, lightIndex, material, prim;
	uint32_t instance;
	bool backHit;
};

RB_D void unpackHit(const DevScene& sc, float4 h, f3 rayD, Interaction& it)
{
	const int tri = __float_as_int(h.x);
	if (tri < 0)
	{
		it.lightType = kLightTypeSky;
		it.lightIndex = 0;
		it.material = 0;
		it.gn = octDecodeU32(0u);
		it.backHit = dot(it.gn, rayD) > 0.0f;
		return;
	}
	float4 a, b, c;
	uint2 aux;
	if (sc.geo.instanced)
	{
		// two-level: h.y holds the hit's instance (its position in the top level)
		instancedTriangle(sc.geo, static_cast<uint32_t>(tri), __float_as_uint(h.y), a, b, c, aux);
	}
	else
	{
		a = __ldg(sc.geo.triVerts + 3 * tri);
		b = __ldg(sc.geo.triVerts + 3 * tri + 1);
		c = __ldg(sc.geo.triVerts + 3 * tri + 2);
		aux = __ldg(sc.geo.triAux + tri);
	}
	it.v0 = f3_of(a); it.v1 = f3_of(b); it.v2 = f3_of(c);
	it.instance = __float_as_uint(b.w);
	const uint32_t sbt = __float_as_uint(c.w);
	it.gn = octDecodeU32(aux.x);
	it.prim = aux.y;
	if (sbt == 0xFFFFFFFFu)
	{
		it.lightType = kLightTypeTriangle;
		it.lightIndex = aux.y;
		const EmissiveTri& et = sc.lights.triangles[aux.y];
		it.prim = et.prim;
		it.material = et.material;
	}
	else
	{
		it.lightType = kLightTypeNone;
		it.lightIndex = 0;
		it.material = sbt;
	}
	it.b1 = h.z; it.b2 = h.w;
	const float w0 = 1.0f - it.b1 - it.b2;
	it.hitPos = mk(it.v0.x * w0 + it.v1.x * it.b1 + it.v2.x * it.b2,
	               it.v0.y * w0 + it.v1.y * it.b1 + it.v2.y * it.b2,
	               it.v0.z * w0 + it.v1.z * it.b1 + it.v2.z * it.b2);
	it.hitPosInterp = it.hitPos;
	it.backHit = dot(it.gn, rayD) > 0.0f;
}

RB_D uint32_t readIndex(const DevMaterial& m, uint32_t i)
{
	return m.indexType == 0 ? static_cast<uint32_t>(reinterpret_cast<const uint16_t*>(m.indices)[i])
	                        : reinterpret_cast<const uint32_t*>(m.indices)[i];
}

// Texture coordinates of a textured material's hit (x, y: set 1; z, w: set
// 2; zero where the mesh has none), and the normal texture's direction in
// the frame ((0, 0, 1) without one).
RB_D void textureFrameInputs(const DevScene& sc, const DevMaterial& mat, uint32_t idx0, uint32_t idx1,
	uint32_t idx2, float w0, float w1, float w2, float4& uv, f3& nm)
{
	for (uint32_t set = 0; set < 2; ++set)
	{
		if (!(mat.attributes & (set ? RB_ATTR_TEX_COORD_2 : RB_ATTR_TEX_COORD_1))) continue;
		const uint8_t* at = mat.attributeData + mat.texcoordOffset[set];
		const float2 c0 = *reinterpret_cast<const float2*>(at + mat.attributeStride * idx0);
		const float2 c1 = *reinterpret_cast<const float2*>(at + mat.attributeStride * idx1);
		const float2 c2 = *reinterpret_cast<const float2*>(at + mat.attributeStride * idx2);
		const float tu = w0 * c0.x + w1 * c1.x + w2 * c2.x, tv = w0 * c0.y + w1 * c1.y + w2 * c2.y;
		if (set) { uv.z = tu; uv.w = tv; } else { uv.x = tu; uv.y = tv; }
	}
	if (mat.textures & (1u << RB_TEXTURE_NORMAL))
	{
		const float4 t = materialTexture(sc, mat, RB_TEXTURE_NORMAL, RB_TEXTURE_NORMAL, uv);
		nm = normalize(mk(t.x * 2.0f - 1.0f, t.y * 2.0f - 1.0f, t.z * 2.0f - 1.0f));
	}
}

// Shading frame and shadow-terminator offset (pathtrace.cu:1279-1461), and
// the texture coordinates at the hit (x, y: set 1; z, w: set 2; zero where
// the mesh has none), with the normal texture applied to the frame.
// Four floats from an 8-byte-aligned address.
RB_D float4 load8x2(const uint8_t* p)
{
	const float2 a = reinterpret_cast<const float2*>(p)[0], b = reinterpret_cast<const float2*>(p)[1];
	return make_float4(a.x, a.y, b.x, b.y);
}

template<bool TEX>
RB_D void shadingFrame(const DevScene& sc, const DevMaterial& mat, Interaction& it, f3 rayD, Frame& frame,
	f3& lastNormal, float4& uv)
{
	const float w0 = 1.0f - it.b1 - it.b2, w1 = it.b1, w2 = it.b2;
	const float* M = sc.geo.normalMatrix + 9u * it.instance;
	f3 normal, tangent;
	bool flipTangent = false;
	const uint32_t idx0 = readIndex(mat, it.prim * 3 + 0);
	const uint32_t idx1 = readIndex(mat, it.prim * 3 + 1);
	const uint32_t idx2 = readIndex(mat, it.prim * 3 + 2);
	if (mat.attributes & (RB_ATTR_NORMAL | RB_ATTR_FRAME))
	{
		f3 sn, st, n0, n1, n2;
		const uint8_t* base = mat.attributeData;
		const uint32_t stride = mat.attributeStride;
		if (mat.attributes & RB_ATTR_FRAME)
		{
			// 8-byte loads: a frame sits at a multiple of 8 bytes (a 24-byte
			// vertex, frame + one coordinate set, puts every other one off 16)
			const uint8_t* at = base + mat.frameOffset;
			const float4 q0 = load8x2(at + stride * idx0);
			const float4 q1 = load8x2(at + stride * idx1);
			const float4 q2 = load8x2(at + stride * idx2);
			flipTangent = signbit(q0.w);
			f3 t0, t1, t2;
			quatColumns(q0, t0, n0);
			quatColumns(q1, t1, n1);
			quatColumns(q2, t2, n2);
			sn = w0 * n0 + w1 * n1 + w2 * n2;
			st = w0 * t0 + w1 * t1 + w2 * t2;
		}
		else
		{
			const uint8_t* at = base + mat.normalOffset;
			const float2 e0 = *reinterpret_cast<const float2*>(at + stride * idx0);
			const float2 e1 = *reinterpret_cast<const float2*>(at + stride * idx1);
			const float2 e2 = *reinterpret_cast<const float2*>(at + stride * idx2);
			n0 = octDecode(e0.x, e0.y);
			n1 = octDecode(e1.x, e1.y);
			n2 = octDecode(e2.x, e2.y);
			sn = w0 * n0 + w1 * n1 + w2 * n2;
			st = tangentOf(sn);
		}
		// Shadow-terminator offset (Hanika 2021), pathtrace.cu:1380-1399.
		const f3 nA = normalize(mulMat(M, n0));
		const f3 nB = normalize(mulMat(M, n1));
		const f3 nC = normalize(mulMat(M, n2));
		f3 tu = it.hitPos - it.v0, tv = it.hitPos - it.v1, tw = it.hitPos - it.v2;
		const float du = fminf(0.0f, dot(tu, nA));
		const float dv = fminf(0.0f, dot(tv, nB));
		const float dw = fminf(0.0f, dot(tw, nC));
		tu -= du * nA;
		tv -= dv * nB;
		tw -= dw * nC;
		it.hitPosInterp = it.hitPos + w0 * tu + w1 * tv + w2 * tw;
		normal = normalize(mulMat(M, sn));
		// inverse(transpose(M)) with glm's cofactor formula; M is stored by rows.
		const float m00 = M[0], m01 = M[3], m02 = M[6];   // column-major view m[c][r] of M
		const float m10 = M[1], m11 = M[4], m12 = M[7];
		const float m20 = M[2], m21 = M[5], m22 = M[8];
		// T = transpose(M): T[c][r] = M[r][c]
		const float t00 = m00, t01 = m10, t02 = m20, t10 = m01, t11 = m11, t12 = m21, t20 = m02, t21 = m12, t22 = m22;
		const float inv = 1.0f / (+t00 * (t11 * t22 - t21 * t12) - t10 * (t01 * t22 - t21 * t02) + t20 * (t01 * t12 - t11 * t02));
		const float i00 = +(t11 * t22 - t21 * t12) * inv, i10 = -(t10 * t22 - t20 * t12) * inv, i20 = +(t10 * t21 - t20 * t11) * inv;
		const float i01 = -(t01 * t22 - t21 * t02) * inv, i11 = +(t00 * t22 - t20 * t02) * inv, i21 = -(t00 * t21 - t20 * t01) * inv;
		const float i02 = +(t01 * t12 - t11 * t02) * inv, i12 = -(t00 * t12 - t10 * t02) * inv, i22 = +(t00 * t11 - t10 * t01) * inv;
		const f3 vt = mk(i00 * st.x + i10 * st.y + i20 * st.z, i01 * st.x + i11 * st.y + i21 * st.z,
		                 i02 * st.x + i12 * st.y + i22 * st.z);
		tangent = normalize(vt);
	}
	else
	{
		normal = it.gn;
		tangent = tangentOf(it.gn);
	}
	// texture coordinates (pathtrace.cu:1414-1430), read only for textured
	// materials; without TEX (a scene without textures) the code is not compiled in
	uv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	f3 nm = mk(0.0f, 0.0f, 1.0f);
	if (TEX && mat.textures) textureFrameInputs(sc, mat, idx0, idx1, idx2, w0, w1, w2, uv, nm);
	// Frame, normal texture and shading-normal correction (pathtrace.cu:1434-1461).
	const f3 bitangent = cross(normal, tangent) * (flipTangent ? -1.0f : 1.0f);
	f3 n = mk(tangent.x * nm.x + bitangent.x * nm.y + normal.x * nm.z,
	          tangent.y * nm.x + bitangent.y * nm.y + normal.y * nm.z,
	          tangent.z * nm.x + bitangent.z * nm.y + normal.z * nm.z);
	const float dNs = dot(n, rayD), dNg = dot(it.gn, rayD);
	const bool fromOutside = dNs > 0.0f && dNg < 0.0f;
	const bool fromInside = dNs < 0.0f && dNg > 0.0f;
	if (fromOutside || fromInside)
		n = normalize(n - rayD * (dNs + (fromOutside ? 0.001f : -0.001f)));
	f3 sb = normalize(cross(n, tangent));
	const f3 stn = normalize(cross(sb, n));
	sb *= flipTangent ? -1.0f : 1.0f;
	frame = Frame{ stn, sb, n };
	lastNormal = n;
}

// Surface description from the material factors (pathtrace.cu:1463-1560),
// for a material without textures.
RB_D Surface surfaceOf(const DevMaterial& mat)
{
	Surface surf = defaultSurface();
	if (mat.factors & RB_FACTOR_BASE_COLOR) surf.baseColor = mk(mat.baseColor[0], mat.baseColor[1], mat.baseColor[2]);
	if (mat.factors & RB_FACTOR_METALNESS) surf.metalness = mat.metalness;
	if (mat.factors & RB_FACTOR_ROUGHNESS) surf.roughness = mat.roughness;
	if (mat.factors & RB_FACTOR_TRANSMISSION) surf.transmission = mat.transmission;
	surf.ior = mat.ior;
	if (mat.sheenPresent)
	{
		surf.layers |= 2u;
		if (mat.factors & RB_FACTOR_SHEEN_COLOR) surf.sheenColor = mk(mat.sheenColor[0], mat.sheenColor[1], mat.sheenColor[2]);
		if (mat.factors & RB_FACTOR_SHEEN_ROUGH) surf.sheenAlpha = mat.sheenRoughness;
	}
	return surf;
}

// Surface description with the material's textures at the record's
// coordinates (pathtrace.cu:1463-1560). The base-colour texture is read
// with the normal texture's coordinate set, as the reference does (:1468).
RB_D Surface surfaceTextured(const DevScene& sc, const DevMaterial& mat, float4 uv)
{
	Surface surf = surfaceOf(mat);
	const uint32_t T = mat.textures;
	if (T & (1u << RB_TEXTURE_BASE_COLOR))
	{
		const float4 t = materialTexture(sc, mat, RB_TEXTURE_BASE_COLOR, RB_TEXTURE_NORMAL, uv);
		surf.baseColor = mk(t.x, t.y, t.z);
		if (mat.factors & RB_FACTOR_BASE_COLOR)
			surf.baseColor = mk(surf.baseColor.x * mat.baseColor[0], surf.baseColor.y * mat.baseColor[1],
				surf.baseColor.z * mat.baseColor[2]);
	}
	if (T & (1u << RB_TEXTURE_MET_ROUGH))
	{
		const float4 t = materialTexture(sc, mat, RB_TEXTURE_MET_ROUGH, RB_TEXTURE_MET_ROUGH, uv);
		surf.metalness = t.z * ((mat.factors & RB_FACTOR_METALNESS) ? mat.metalness : 1.0f);
		surf.roughness = t.y * ((mat.factors & RB_FACTOR_ROUGHNESS) ? mat.roughness : 1.0f);
	}
	if (T & (1u << RB_TEXTURE_TRANSMISSION))
	{
		const float4 t = materialTexture(sc, mat, RB_TEXTURE_TRANSMISSION, RB_TEXTURE_TRANSMISSION, uv);
		surf.transmission = t.x * ((mat.factors & RB_FACTOR_TRANSMISSION) ? mat.transmission : 1.0f);
	}
	if (mat.sheenPresent)
	{
		if (T & (1u << RB_TEXTURE_SHEEN_COLOR))
		{
			const float4 t = materialTexture(sc, mat, RB_TEXTURE_SHEEN_COLOR, RB_TEXTURE_SHEEN_COLOR, uv);
			const bool f = (mat.factors & RB_FACTOR_SHEEN_COLOR) != 0;
			surf.sheenColor = mk(t.x * (f ? mat.sheenColor[0] : 1.0f), t.y * (f ? mat.sheenColor[1] : 1.0f),
				t.z * (f ? mat.sheenColor[2] : 1.0f));
		}
		if (T & (1u << RB_TEXTURE_SHEEN_ROUGH))
		{
			// the texture's fourth channel, squared (the factor alone is taken as is)
			const float4 t = materialTexture(sc, mat, RB_TEXTURE_SHEEN_ROUGH, RB_TEXTURE_SHEEN_ROUGH, uv);
			const float r = t.w * ((mat.factors & RB_FACTOR_SHEEN_ROUGH) ? mat.sheenRoughness : 1.0f);
			surf.sheenAlpha = r * r;
		}
	}
	return surf;
}
template<bool TEX>
RB_D Surface surfaceAt(const DevScene& sc, const DevMaterial& mat, float4 uv)
{
	return (TEX && mat.textures) ? surfaceTextured(sc, mat, uv) : surfaceOf(mat);
}

// Alpha of a base-colour texture, times the factor's (pathtrace.cu:1466-1477).
RB_D float texturedAlpha(const DevScene& sc, const DevMaterial& mat, float4 uv)
{
	float alpha = materialTexture(sc, mat, RB_TEXTURE_BASE_COLOR, RB_TEXTURE_NORMAL, uv).w;
	if (mat.factors & RB_FACTOR_BASE_COLOR) alpha *= mat.baseColor[3];
	return alpha;
}
// Alpha cutoff or stochastic alpha blending (pathtrace.cu:1470-1496): true
// if the interaction is skipped and the path continues through the surface.
template<bool TEX>
RB_D bool alphaSkipped(const DevScene& sc, const DevMaterial& mat, float4 uv, const Qrng& q)
{
	float alpha = (mat.factors & RB_FACTOR_BASE_COLOR) ? mat.baseColor[3] : 0.0f;
	if (TEX && (mat.textures & (1u << RB_TEXTURE_BASE_COLOR))) alpha = texturedAlpha(sc, mat, uv);
	if (mat.factors & RB_FACTOR_CUTOFF) return alpha < mat.alphaCutoff;
	if (mat.factors & RB_FACTOR_BLEND) return sample1D(q, DIM_ALPHA_BLEND) > alpha;
	return false;
}
// Emitted RGB of an emissive triangle at barycentrics (w1, w2) (the
// emissive factor, times the emission texture at the triangle's
// coordinates: pathtrace.cu:1215-1228, 1638-1648).
RB_D f3 texturedEmission(const DevScene& sc, const EmissiveTri& et, const DevMaterial& em, f3 e,
	float w1, float w2)
{
	const float w0 = 1.0f - w1 - w2;
	const float u = w0 * et.uv[0] + w1 * et.uv[2] + w2 * et.uv[4];
	const float v = w0 * et.uv[1] + w1 * et.uv[3] + w2 * et.uv[5];
	const float4 t = texSample(sc, em.tex[RB_TEXTURE_EMISSION], u, v);
	return mk(e.x * t.x, e.y * t.y, e.z * t.z);
}
template<bool TEX>
RB_D f3 emissionAt(const DevScene& sc, const EmissiveTri& et, float w1, float w2)
{
	const DevMaterial& em = sc.materials[et.material];
	const f3 e = mk(em.emissive[0], em.emissive[1], em.emissive[2]);
	return (TEX && (em.textures & (1u << RB_TEXTURE_EMISSION))) ? texturedEmission(sc, et, em, e, w1, w2) : e;
}

// Pixel (x, y) of path slot `slot` (0 .. W x H - 1) of a plane: slots run
// over tiles of 8 x 4 pixels, so the 32 paths of a warp share a compact
// tile (more coherent primary rays and hit points than a 32 x 1 row
// strip), tiles row-major within bands of 4 rows. Where W or H is not a
// multiple of the tile, the last tile of a band is narrower and the last
// band lower. A bijection onto the pixels, so every pixel still gets
// exactly one path per plane with the same sample sequence.
RB_D uint2 slotPixel(uint32_t slot, uint32_t W, uint32_t H)
{
	const uint32_t band = slot / (4u * W);
	const uint32_t hb = min(4u, H - 4u * band);
	const uint32_t s = slot - band * 4u * W;
	const uint32_t c = s / (8u * hb);
	const uint32_t r = s - c * 8u * hb;
	const uint32_t cw = min(8u, W - 8u * c);
	return make_uint2(8u * c + r % cw, 4u * band + r / cw);
}

// Shared wavefront (rb_render_jobs): the chunk holding path slot `slot`, or
// pixel slot `px` of the resolve (the last chunk starting at or before it).
RB_D uint32_t chunkOfSlot(const WaveParams& w, uint32_t slot)
{
	uint32_t lo = 0, hi = w.nChunks;
	while (hi - lo > 1)
	{
		const uint32_t mid = (lo + hi) >> 1;
		if (w.chunks[mid].slot <= slot) lo = mid; else hi = mid;
	}
	return lo;
}
RB_D uint32_t chunkOfPixel(const WaveParams& w, uint32_t px)
{
	uint32_t lo = 0, hi = w.nChunks;
	while (hi - lo > 1)
	{
		const uint32_t mid = (lo + hi) >> 1;
		if (w.chunks[mid].pixel <= px) lo = mid; else hi = mid;
	}
	return lo;
}
// The scene of path p: the kernel's own, or in a shared wavefront its job's.
template<bool JOBS>
RB_D const DevScene& pathScene(const DevScene& own, const PathSoA& s, uint32_t p)
{
	return JOBS ? s.jobs[s.job[p]].scene : own;
}

// ------------------------------------------------------------- kernels
template<bool JOBS>
__global__ void __launch_bounds__(kThreads) kGenerate(const __grid_constant__ DevScene scK, PathSoA s, WaveParams w)
{
	for (uint32_t p = gtid(); p < w.paths; p += gstride())
	{
		uint32_t x, y, sample;
		const DevScene* scp = &scK;
		if (JOBS)
		{
			const WaveChunk c = w.chunks[chunkOfSlot(w, p)];
			const uint32_t local = p - c.slot;
			const uint2 px = slotPixel(local % c.pixels, c.width, c.height);
			x = px.x; y = px.y;
			sample = c.sample + local / c.pixels;
			s.job[p] = c.job;
			s.key[p] = make_uint2(x | (y << 16), sample);
			scp = &s.jobs[c.job].scene;
		}
		else
		{
			const uint2 px = slotPixel(p % w.pixels, scK.launch.width, scK.launch.height);
			x = px.x; y = px.y;
			sample = waveSampleBase(w) + p / w.pixels;
		}
		const DevScene& sc = *scp;
		const Qrng q = qrngAt(sample, pixelHash(x, y), 0);
		const Wavelengths wl = sampleVisible(sample1D(q, DIM_WAVELENGTH));
		float fu, fv, dx, dy, lu = 0.0f, lv = 0.0f;
		sample2D(q, DIM_FILTER, fu, fv);
		gaussianFilterSample(fu, fv, dx, dy);
		if (sc.launch.dof) sample2D(q, DIM_LENS, lu, lv);
		f3 o, d;
		cameraRay(sc.launch, static_cast<float>(x) + dx, static_cast<float>(y) + dy, lu, lv, o, d);
		s.rayO[p] = f4_of(o, 1.0f);
		s.rayD[p] = f4_of(d, 1.0f);
		s.lambda[p] = f4(wl.lambda);
		s.lpdf[p] = f4(wl.pdf);
		s.nrm[p] = make_float4(0.0f, 0.0f, 0.0f, wl.active);
		s.L[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		s.T[p] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
		s.fd[p] = make_uint2(0u, 0u);
		s.queue[0][p] = p;
		if (w.cached)
		{
			s.spread[p] = make_float2(0.0f, 0.0f);
			s.trainRec[p] = w.trainOneIn && mix32(p ^ w.trainSeed) % w.trainOneIn == 0 ? kNoRecord : kNotTraining;
		}
	}
	if (gtid() == 0)
	{
		// the first extension queue holds every path of the wave
		s.counts[0] = w.paths;
		if (w.paths > s.queueCap) atomicOr(scK.status, RB_DEV_QUEUE_OVERFLOW);
	}
}

// Minimum resident blocks per SM requested for the shading kernels, which
// caps their registers per thread (65536 / (128 x blocks)): 85, 64 and 64.
// These kernels are latency-bound, and on B200 (at-scale frame) the extra
// warps outweigh the spilled bytes, which stay in L1: surface -8%, light
// sample -6% against the compiler's own choice. The BxDF stage runs as two
// kernels (light-sample evaluation, BxDF sample; 94 and 109 registers
// uncapped), both at 8 blocks: 188 ms per frame, against 202 / 216 / 220 /
// 203 ms at 12 / 4 / 5 / 6 blocks, and 229 ms for the single kernel at its
// best cap (16 blocks, 32 registers, 1.2 KB of spills per thread).
// Re-swept with the records at their queue position (frame ms): surface 4 /
// 6 / 8 blocks 976 / 970 / 970, BxDF 6 / 8 / 12 982 / 970 / 974, light
// sample 6 / 8 / 12 970 / 970 / 971.
#ifndef RB_SURFACE_MIN_BLOCKS
#define RB_SURFACE_MIN_BLOCKS 6
#endif
#ifndef RB_NEE_MIN_BLOCKS
#define RB_NEE_MIN_BLOCKS 8
#endif
#ifndef RB_BSDF_MIN_BLOCKS
#define RB_BSDF_MIN_BLOCKS 8
#endif

// Block size of the shared-memory light-sample kernel: two blocks of 512
// per SM hold two copies of a tree of up to kNeeSharedMaxBytes.
#ifndef RB_NEE_SHARED_MAX_BYTES
#define RB_NEE_SHARED_MAX_BYTES (100u * 1024u)
#endif
constexpr int kNeeSharedThreads = 512;
constexpr uint32_t kNeeSharedMaxBytes = RB_NEE_SHARED_MAX_BYTES;

// Surface-record bits (PathSoA::sfPi.w); bits 8..15 hold the path's depth,
// so the light-sample kernels need not read the path's flags for it.
constexpr uint32_t kSfBackHit = 1u << 0;
constexpr uint32_t kSfSkipped = 1u << 1;
constexpr uint32_t kSfTriangle = 1u << 2;
constexpr uint32_t kSfOccluded = 1u << 3;
constexpr uint32_t kSfDepthShift = 8;
static_assert(kMaxBounces <= 255, "depth fits bits 8..15");
RB_D uint32_t sfDepth(uint32_t bits) { return (bits >> kSfDepthShift) & 0xFFu; }


RB_D Qrng pathQrng(const DevScene& sc, const WaveParams& w, uint32_t p, uint32_t depth)
{
	const uint2 px = slotPixel(p % w.pixels, sc.launch.width, sc.launch.height);
	return qrngAt(waveSampleBase(w) + p / w.pixels, pixelHash(px.x, px.y), depth);
}
// ... of a path of either kind of wave (a shared wavefront keeps the keys).
template<bool JOBS>
RB_D Qrng pathQrngT(const DevScene& sc, const WaveParams& w, const PathSoA& s, uint32_t p, uint32_t depth)
{
	if (JOBS)
	{
		const uint2 k = s.key[p];
		return qrngAt(k.y, pixelHash(k.x & 0xFFFFu, k.x >> 16), depth);
	}
	return pathQrng(sc, w, p, depth);
}

// wavelength range of the hero sampling, for the cache's normalised input
constexpr float kLambdaMin = 360.0f, kLambdaMax = 830.0f;

// Radiance-cache form at a shaded vertex (Mueller et al. 2021, sec. 4):
// the path spread of eq. 3 -- the first shaded vertex sets the footprint
// a0 = d^2 / (4 pi cos), each later vertex adds sqrt(d^2 / (pdf cos)) for
// the direction that reached it (nothing after a specular vertex). A path
// that is not a training path terminates into the cache once
// (summed spread)^2 > c a0 at a surface rough enough to cache (queued as a
// query; returns true); a training path records the vertex (inputs,
// radiance so far, throughput) instead.
RB_D bool cacheVertex(const PathSoA& s, const WaveParams& w, uint32_t* status, uint32_t p, uint32_t& flags,
	const f3& rayO, const f3& rayD, float bxdfPdf, const f3& hitPos, const f3& gn, const f3& nrm, float lambda0,
	bool rough)
{
	const f3 toHit = hitPos - rayO;
	const float d2 = dot(toHit, toHit);
	const float cosHit = fmaxf(fabsf(dot(rayD, gn)), 1e-4f);
	float2 sp = s.spread[p];
	if (sp.x == 0.0f) sp.x = d2 / (4.0f * kPi * cosHit);   // first shaded vertex
	else if (!(flags & PF_PREVIOUS_HIT_SPECULAR) && bxdfPdf > 0.0f) sp.y += sqrtf(d2 / (bxdfPdf * cosHit));
	s.spread[p] = sp;
	const uint32_t tr = s.trainRec[p];
	const bool atQuery = rough && sp.y > 0.0f && sp.y * sp.y > w.spreadC * sp.x;
	const bool terminate = tr == kNotTraining && atQuery;
	if (tr == kNotTraining && !terminate) return false;
	float in[kNrcInputs];
	in[0] = (hitPos.x - w.posMin[0]) * w.posScale[0];
	in[1] = (hitPos.y - w.posMin[1]) * w.posScale[1];
	in[2] = (hitPos.z - w.posMin[2]) * w.posScale[2];
	in[3] = -rayD.x; in[4] = -rayD.y; in[5] = -rayD.z;
	in[6] = nrm.x; in[7] = nrm.y; in[8] = nrm.z;
	in[9] = (lambda0 - kLambdaMin) / (kLambdaMax - kLambdaMin);
	if (terminate)
	{
		const uint32_t q = appendSlot(s.counts + kCacheQueryCount, s.queueCap, status);
		if (q != kNoSlot)
		{
			s.cPath[q] = p | ((flags & kPathLitPrefix) ? kLitPrefixBit : 0u);
			for (int k = 0; k < kNrcInputs; ++k) s.cIn[static_cast<size_t>(kNrcInputs) * q + k] = in[k];
		}
		return true;
	}
	// a training path's vertex where the cache would have ended it: the
	// records the drop bias of the path's class (camera ray hit an emitter
	// or not) is measured on
	const bool queryRecord = atQuery && !(flags & kPathQueryPassed);
	const uint32_t recordBits = !queryRecord ? 0u : ((flags & kPathLitPrefix) ? kLitPrefixBit : kQueryRecordBit);
	if (atQuery) flags |= kPathQueryPassed;
	const uint32_t r = appendIndex(s.counts + kTrainRecordCount);
	if (r < s.trainCapacity)
	{
		s.tPath[r] = p | recordBits;
		for (int k = 0; k < kNrcInputs; ++k) s.tIn[static_cast<size_t>(kNrcInputs) * r + k] = in[k];
		s.tL[r] = s.L[p];
		s.tT[r] = s.T[p];
	}
	s.trainRec[p] = r < s.trainCapacity ? r : kNoRecord;
	return false;
}

// Stage 1 of shading: the hit record, hit emission with MIS
// (pathtrace.cu:1185-1274), the shading frame and the alpha test. Paths that
// continue get a surface record and join the surface queue, which the light
// sampling and BxDF stages read.
// counters (optional): [6] surface records.
template<bool JOBS, bool TEX>
__global__ void __launch_bounds__(kThreads, RB_SURFACE_MIN_BLOCKS) kSurface(const __grid_constant__ DevScene scK, PathSoA s,
	WaveParams w, int bounce, unsigned long long* counters)
{
	const uint32_t n = min(s.counts[bounce], s.queueCap);
	const uint32_t* queue = s.queue[bounce & 1];
	unsigned long long* regions = reinterpret_cast<unsigned long long*>(s.counts + kRegionCounts + 2 * bounce);
	uint32_t records = 0;
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const uint32_t p = queue[i];
		const DevScene& sc = pathScene<JOBS>(scK, s, p);
		const float4 ro = s.rayO[p], rd = s.rayD[p];
		const f3 rayO = f3_of(ro), rayD = f3_of(rd);
		const float bxdfPdf = rd.w;
		const float4 nv = s.nrm[p];
		f3 lastNormal = f3_of(nv);
		uint2 fd = s.fd[p];
		uint32_t flags = fd.x;
		const uint32_t depth = fd.y;

		Interaction it;
		unpackHit(sc, s.hit[p], rayD, it);
		if (it.lightType == kLightTypeTriangle || it.lightType == kLightTypeNone) flags |= PF_TRIANGULAR_GEOMETRY;

		if (it.lightType != kLightTypeNone)
		{
			const S4 lambda = s4(s.lambda[p]);
			const bool prevNee = depth != 0 && !(flags & PF_PREVIOUS_HIT_SPECULAR);
			// The light-tree pdf of an emitter hit replays ~2 SG importances
			// per tree level; few lanes need it, so it is deferred to kEmission
			// over a compacted queue. The sky's tree pdf is a constant: the
			// environment's share, lightTreePdf's first return.
			const bool deferTree = prevNee && it.lightType == kLightTypeTriangle;
			const float treePdf = prevNee && !deferTree ? (sc.env.enabled ? kEnvMapImportance : 0.0f) : 1.0f;
			float lightPdf = 0.0f;
			S4 Le = s4(0.0f);
			bool noEmission = false;
			const f3 toHit = it.hitPos - rayO;
			const float d2 = toHit.x * toHit.x + toHit.y * toHit.y + toHit.z * toHit.z;
			if (it.lightType == kLightTypeTriangle)
			{
				const EmissiveTri& et = sc.lights.triangles[it.lightIndex];
				const f3 a = mk(et.v[0], et.v[1], et.v[2]), b = mk(et.v[3], et.v[4], et.v[5]), c = mk(et.v[6], et.v[7], et.v[8]);
				f3 nn = cross(b - a, c - a);
				const float nl = length(nn);
				nn = nn / nl;
				const float area = nl / 2.0f;
				const float lCos = -dot(rayD, nn);
				noEmission = lCos <= 0.0f;
				lightPdf = (1.0f / area) * d2 / lCos;
				Le = rgbToSpectrum(sc.spectra.basis, emissionAt<TEX>(sc, et, it.b1, it.b2), lambda);
			}
			else
			{
				if (sc.env.enabled)
					envEmission(sc, rayD, lambda, Le, lightPdf);
				else
					noEmission = true;
				flags |= PF_FINISHED;
			}
			if (!noEmission && deferTree)
			{
				const uint32_t slot = appendSlot(s.counts + kEmissionCounts + bounce, s.queueCap, sc.status);
				if (slot != kNoSlot)
				{
					s.emQueue[slot] = p;
					s.emA[slot] = f4_of(rayO, bxdfPdf);
					s.emB[slot] = f4_of(lastNormal, lightPdf);
					s.emC[slot] = f4(Le);
					s.emLight[slot] = it.lightIndex;
				}
			}
			else if (!noEmission)
			{
				lightPdf *= treePdf;
				const float wgt = prevNee ? powerHeuristic(bxdfPdf, lightPdf) : 1.0f;
				S4 L = s4(s.L[p]);
				L += s4(s.T[p]) * Le * wgt;
				s.L[p] = f4(L);
			}
		}
		if (!(flags & PF_FINISHED))
		{
			const DevMaterial& mat = sc.materials[it.material];
			Frame frame{};
			bool skipped = false;
			float4 uv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			if (flags & PF_TRIANGULAR_GEOMETRY)
			{
				shadingFrame<TEX>(sc, mat, it, rayD, frame, lastNormal, uv);
				skipped = alphaSkipped<TEX>(sc, mat, uv, pathQrngT<JOBS>(sc, w, s, p, depth));
			}
			if (w.cached)
			{
				if (!skipped && (flags & PF_TRIANGULAR_GEOMETRY))
				{
					const Surface sf = surfaceAt<TEX>(sc, mat, uv);
					const bool rough = (sf.metalness == 0.0f && sf.transmission == 0.0f) || sf.roughness >= w.minRoughness;
					if (depth == 0 && it.lightType == kLightTypeTriangle) flags |= kPathLitPrefix;
					if (cacheVertex(s, w, sc.status, p, flags, rayO, rayD, bxdfPdf, it.hitPos, it.gn, lastNormal,
							s.lambda[p].x, rough))
					{
						s.fd[p] = make_uint2(flags | PF_FINISHED, depth);
						continue;
					}
				}
				else if (s.trainRec[p] != kNotTraining)
				{
					s.trainRec[p] = kNoRecord;
				}
			}
			const uint32_t bits = (it.backHit ? kSfBackHit : 0u) | (skipped ? kSfSkipped : 0u)
				| ((flags & PF_TRIANGULAR_GEOMETRY) ? kSfTriangle : 0u) | (depth << kSfDepthShift);
			s.nrm[p] = f4_of(lastNormal, nv.w);
			// The light choice of the record's light sample (pathtrace.cu:
			// 1572-1590: the environment with probability envImp, else the
			// tree) decides its region: tree picks from record 0 up, the rest
			// (environment picks and skipped surfaces, which take no light
			// sample) from queueCap - 1 down, so each light-sample launch
			// reads its records densely.
			bool sky = true;
			if (!skipped)
			{
				const bool envPresent = sc.env.enabled != 0;
				const bool treePresent = sc.lights.nodes != nullptr;
				const float envImp = envPresent ? (treePresent ? kEnvMapImportance : 1.0f) : 0.0f;
				if (envPresent || treePresent) sky = sample3DZ(pathQrngT<JOBS>(sc, w, s, p, depth), DIM_LIGHT) < envImp;
			}
			uint32_t order = 0;
			const uint32_t r = appendRegion(regions, sky, s.queueCap, sc.status, order);
			if (r != kNoSlot)
			{
				s.recOrder[order] = r;
				s.surfQueue[r] = p;
				s.sfP[r] = f4_of(it.hitPos, __uint_as_float(it.material));
				s.sfPi[r] = f4_of(it.hitPosInterp, __uint_as_float(bits));
				s.sfGn[r] = f4_of(it.gn, 0.0f);
				s.sfT[r] = f4_of(frame.t, 0.0f);
				s.sfB[r] = f4_of(frame.b, 0.0f);
				s.sfN[r] = f4_of(lastNormal, 0.0f);
				s.sfL[r] = s.lambda[p];
				if (TEX && mat.textures) s.sfUV[r] = uv;
			}
			++records;
		}
		else if (w.cached && s.trainRec[p] != kNotTraining)
		{
			s.trainRec[p] = kNoRecord;
		}
		s.fd[p] = make_uint2(flags, depth);
	}
	if (counters) warpAdd(counters + 6, records);
}

// Emission MIS of emitter hits whose previous vertex sampled a light
// (pathtrace.cu:1185-1274): the light-tree pdf of the hit light replayed from
// the previous vertex, the power heuristic, and the contribution, with the
// values kSurface queued for it; the same arithmetic as the inline case.
template<bool JOBS>
__global__ void __launch_bounds__(kThreads) kEmission(const __grid_constant__ DevScene scK, PathSoA s, int bounce)
{
	const uint32_t n = min(s.counts[kEmissionCounts + bounce], s.queueCap);
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const uint32_t p = s.emQueue[i];
		const DevScene& sc = pathScene<JOBS>(scK, s, p);
		const float4 a = s.emA[i], b = s.emB[i];
		const float treePdf = lightTreePdf(sc, kLightTypeTriangle, s.emLight[i], f3_of(a), f3_of(b));
		float lightPdf = b.w;
		lightPdf *= treePdf;
		const float wgt = powerHeuristic(a.w, lightPdf);
		const S4 c = s4(s.T[p]) * s4(s.emC[i]) * wgt;
		S4 L = s4(s.L[p]);
		L += c;
		s.L[p] = f4(L);
		if (s.trainRec)
		{
			// a training record of this vertex counts the emission on arrival
			const uint32_t r = s.trainRec[p];
			if (r < kNoRecord)
			{
				S4 R = s4(s.tL[r]);
				R += c;
				s.tL[r] = f4(R);
			}
		}
	}
}

// Stage 2 of shading: the light sample (pathtrace.cu:1572-1721) for every
// surface that is not skipped: pick a light from the light tree (held in the
// read-only cache: it is read by every thread) or the environment, sample a
// point on it and write the shadow ray and the light sample.
// SHARED: the block first copies the unpacked tree into shared memory
// (dynamic, nodeCount x 48 B) and descends it there; used when the tree fits.
// The records come from one region of the record arrays (`which`: 0 the
// tree picks, records 0 ..; 1 the environment picks, records queueCap - 1
// down), which kSurface chose with the light choice of sampleLightTree
// (pathtrace.cu:1064-1076: the same sample dimension and comparison as the
// body below), so a warp's lanes take the same branch of the light choice
// and read their records densely; the body is the same for both.
// JOBS (a shared wavefront; never with SHARED): each record's tree is its job's.
template<bool SHARED, bool JOBS, bool TEX>
__global__ void __launch_bounds__(SHARED ? kNeeSharedThreads : kThreads, SHARED ? 2 : RB_NEE_MIN_BLOCKS)
kNee(const __grid_constant__ DevScene scK, PathSoA s, WaveParams w, int bounce, int which)
{
	extern __shared__ float4 sharedTree[];
	const uint2 nr = regionCounts(s.counts + kRegionCounts + 2 * bounce, s.queueCap);
	const uint32_t n = which ? nr.y : nr.x;
	const TreeNodeU* sharedNodes = scK.lights.unpacked;
	if (SHARED)
	{
		const float4* src = reinterpret_cast<const float4*>(scK.lights.unpacked);
		const uint32_t words = 3u * scK.lights.nodeCount;
		for (uint32_t k = threadIdx.x; k < words; k += blockDim.x) sharedTree[k] = __ldg(src + k);
		__syncthreads();
		sharedNodes = reinterpret_cast<const TreeNodeU*>(sharedTree);
	}
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const uint32_t rec = which ? s.queueCap - 1u - i : i;
		const float4 pi = s.sfPi[rec];
		uint32_t bits = __float_as_uint(pi.w);
		if (bits & kSfSkipped) continue;              // environment region only: no light sample
		const uint32_t p = s.surfQueue[rec];
		const DevScene& sc = pathScene<JOBS>(scK, s, p);
		const TreeNodeU* nodes = JOBS ? sc.lights.unpacked : sharedNodes;
		const bool envPresent = sc.env.enabled != 0;
		const bool treePresent = sc.lights.nodes != nullptr;
		const float4 hp = s.sfP[rec];
		const f3 hitPos = f3_of(hp), hitPosInterp = f3_of(pi), gn = f3_of(s.sfGn[rec]), sn = f3_of(s.sfN[rec]);
		f3 dir = mk(0.0f), shadowO = mk(0.0f);
		S4 spectrum = s4(0.0f);
		float pdf = 0.0f, dToL = 0.0f;
		bool occluded = false;
		if (!envPresent && !treePresent)
		{
			occluded = true;
		}
		else
		{
			const DevMaterial& mat = sc.materials[__float_as_uint(hp.w)];
			const bool canTransmit = surfaceAt<TEX>(sc, mat, (TEX && mat.textures) ? s.sfUV[rec] : make_float4(0.0f, 0.0f, 0.0f, 0.0f)).transmission != 0.0f;
			const Qrng q = pathQrngT<JOBS>(sc, w, s, p, sfDepth(bits));
			const f3 r = sample3D(q, DIM_LIGHT);
			const bool tri = (bits & kSfTriangle) != 0;
			const S4 lambda = s4(s.sfL[rec]);
			uint32_t type = 0, index = 0;
			float treePdf = 0.0f, lightPdf = 0.0f;
			lightTreeSample<SHARED>(sc, nodes, r.z, hitPos, sn, type, index, treePdf);
			if (type == kLightTypeTriangle)
			{
				const EmissiveTri& et = sc.lights.triangles[index];
				const f3 a = mk(et.v[0], et.v[1], et.v[2]), b = mk(et.v[3], et.v[4], et.v[5]), c = mk(et.v[6], et.v[7], et.v[8]);
				f3 nn = cross(b - a, c - a);
				const float nl = length(nn);
				nn = nn / nl;
				const float area = nl / 2.0f;
				float u = r.x, v = r.y;
				if (u + v > 1.0f) { u = 1.0f - u; v = 1.0f - v; }
				const f3 lp = a + (b - a) * u + (c - a) * v;
				const f3 sr = lp - hitPos;
				const bool inSample = dot(sn, sr) < 0.0f;
				if ((inSample && !canTransmit) || (inSample && dot(gn, sr) > 0.0f)) occluded = true;
				shadowO = offsetPoint(inSample || !tri ? hitPos : hitPosInterp, inSample ? -gn : gn);
				const f3 rl = lp - shadowO;
				const float d2 = rl.x * rl.x + rl.y * rl.y + rl.z * rl.z;
				dToL = sqrtf(d2);
				dir = rl / dToL;
				const float lCos = -dot(nn, dir);
				// the reference overwrites the flag set above here (pathtrace.cu:1633)
				occluded = lCos <= 0.0f;
				lightPdf = (1.0f / area) * d2 / lCos;
				spectrum = rgbToSpectrum(sc.spectra.basis, emissionAt<TEX>(sc, et, u, v), lambda);
			}
			else if (type == kLightTypeSky)
			{
				envSample(sc, r.x, r.y, lambda, dir, spectrum, lightPdf);
				dToL = FLT_MAX;
				shadowO = offsetPoint(!tri ? hitPos : hitPosInterp, (bits & kSfBackHit) ? -gn : gn);
			}
			else
			{
				occluded = true;
			}
			pdf = lightPdf * treePdf;
		}
		if (occluded) reinterpret_cast<float*>(s.sfPi + rec)[3] = __uint_as_float(bits | kSfOccluded);
		s.shO[rec] = f4_of(shadowO, dToL - 0.1f);
		s.shD[rec] = f4_of(dir, pdf);
		s.shC[rec] = f4(spectrum);
	}
}

// Stage 3a of shading: the BxDF callable's evaluation of the light sample
// (pathtrace.cu:1724-1733 calling the direct-lighting block, :660-771 of the
// complex surface, :498-520 of the conductor). Its contribution replaces the
// light's spectrum in the record; a light sample that gets none is marked
// occluded, so the next stage queues no shadow ray for it. Split from the
// BxDF sample (stage 3b) so neither kernel holds both parts' registers.
template<bool JOBS, bool TEX>
__global__ void __launch_bounds__(kThreads, RB_BSDF_MIN_BLOCKS) kBsdfLight(const __grid_constant__ DevScene scK, PathSoA s,
	WaveParams w, int bounce)
{
	const uint2 nr = regionCounts(s.counts + kRegionCounts + 2 * bounce, s.queueCap);
	const uint32_t n = nr.x + nr.y;
	for (uint32_t j = gtid(); j < n; j += gstride())
	{
		const uint32_t i = s.recOrder[j];
		const uint32_t bits = __float_as_uint(lastWord(s.sfPi + i));
		if (bits & (kSfSkipped | kSfOccluded)) continue;
		const uint32_t p = s.surfQueue[i];
		const DevScene& sc = pathScene<JOBS>(scK, s, p);
		const DevMaterial& mat = sc.materials[__float_as_uint(lastWord(s.sfP + i))];
		const float4 rd = s.rayD[p], dd = s.shD[i];
		const uint2 fd = s.fd[p];
		BxdfState st;
		st.hasNee = false;
		st.wl.lambda = s4(s.sfL[i]);
		st.T = s4(s.T[p]);
		st.pdf = rd.w;
		st.dir = f3_of(rd);
		st.flags = fd.x;
		st.refractionScale = lastWord(s.rayO + p);
		LightSample dl;
		dl.spectrum = s4(s.shC[i]);
		dl.dir = f3_of(dd);
		dl.pdf = dd.w;
		dl.occluded = false;
		const Frame frame{ f3_of(s.sfT[i]), f3_of(s.sfB[i]), f3_of(s.sfN[i]) };
		evalBxdf<kBxdfLight>(sc, mat, dl, pathQrngT<JOBS>(sc, w, s, p, fd.y), frame,
			(TEX && mat.textures) ? surfaceAt<TEX>(sc, mat, s.sfUV[i]) : surfaceOf(mat), st);
		if (st.hasNee) s.shC[i] = f4(st.nee);
		else reinterpret_cast<float*>(s.sfPi + i)[3] = __uint_as_float(bits | kSfOccluded);
	}
}

// Stage 3b of shading: the BxDF sample (the rest of the callable,
// pathtrace.cu:773-905 / :521-547), Russian roulette, the next ray and the
// depth limits (:1736-1785). Continuing paths go to the next extend queue,
// light samples that passed stage 3a to the shadow queue.
template<bool JOBS, bool TEX>
__global__ void __launch_bounds__(kThreads, RB_BSDF_MIN_BLOCKS) kBsdf(const __grid_constant__ DevScene scK, PathSoA s,
	WaveParams w, int bounce)
{
	const uint2 nr = regionCounts(s.counts + kRegionCounts + 2 * bounce, s.queueCap);
	const uint32_t n = nr.x + nr.y;
	uint32_t* nextQueue = s.queue[(bounce + 1) & 1];
	uint32_t* nextCount = s.counts + bounce + 1;
	uint32_t* shadowCount = s.counts + kShadowCounts + bounce;
	for (uint32_t j = gtid(); j < n; j += gstride())
	{
		const uint32_t i = s.recOrder[j];
		const uint32_t p = s.surfQueue[i];
		const DevScene& sc = pathScene<JOBS>(scK, s, p);
		// Only the words the BxDF sample needs are read before it; the hit
		// points, the geometric normal and the ray origin are read after it,
		// so they are not live (and spilled) across the call.
		const uint32_t bits = __float_as_uint(lastWord(s.sfPi + i));
		const bool skipped = (bits & kSfSkipped) != 0, backHit = (bits & kSfBackHit) != 0;
		const float4 rd = s.rayD[p];
		const uint2 fd = s.fd[p];
		uint32_t flags = fd.x, depth = fd.y;
		const Qrng q = pathQrngT<JOBS>(sc, w, s, p, depth);
		const DevMaterial& mat = sc.materials[__float_as_uint(lastWord(s.sfP + i))];

		// The BxDF reads the wavelengths and changes none of them: only
		// their values are loaded, and nothing is written back.
		BxdfState st;
		st.hasNee = false;
		st.wl.lambda = s4(s.sfL[i]);
		st.T = s4(s.T[p]);
		st.pdf = rd.w;
		st.dir = f3_of(rd);
		st.flags = flags;
		st.refractionScale = lastWord(s.rayO + p);
		bool hasShadow = false;
		if (!skipped)
		{
			LightSample dl;
			dl.occluded = true;      // not read by the sample part
			const Frame frame{ f3_of(s.sfT[i]), f3_of(s.sfB[i]), f3_of(s.sfN[i]) };
			evalBxdf<kBxdfSample>(sc, mat, dl, q, frame,
				(TEX && mat.textures) ? surfaceAt<TEX>(sc, mat, s.sfUV[i]) : surfaceOf(mat), st);
			hasShadow = !(bits & kSfOccluded) && !(st.flags & PF_PATH_TERMINATED);
		}
		flags = st.flags;
		S4 T = st.T;
		f3 rayO = f3_of(s.rayO[p]), rayD = st.dir;
		const float refrScale = st.refractionScale;
		bool done = false;
		if (flags & PF_PATH_TERMINATED)
		{
			done = true;
			hasShadow = false;
		}
		else
		{
			// Russian roulette (pathtrace.cu:1736-1744).
			const float tMax = s4max(T) * refrScale;
			bool killed = false;
			if (tMax < 1.0f && depth > 0)
			{
				float qq = fmaxf(0.0f, 1.0f - tMax);
				qq = qq * qq;
				if (sample1D(q, DIM_ROULETTE) < qq) killed = true;
				else T /= (1.0f - qq);
			}
			if (killed)
			{
				done = true;
			}
			else
			{
				// Next origin and direction fix-up (:1747-1766).
				const bool refracted = (flags & PF_RAY_REFRACTED) != 0;
				const bool triGeo = (flags & PF_TRIANGULAR_GEOMETRY) != 0;
				const bool in = refracted || skipped;
				const f3 hitPos = f3_of(s.sfP[i]), hitPosInterp = f3_of(s.sfPi[i]), gn = f3_of(s.sfGn[i]);
				const f3 origin = (in == backHit) && triGeo ? hitPosInterp : hitPos;
				const f3 offset = in == backHit ? gn : -gn;
				rayO = offsetPoint(origin, offset);
				const float dNg = dot(gn, rayD);
				if (dNg > 0.0f && (backHit != refracted) && !skipped)
					rayD = normalize(rayD - (gn * (dNg + 0.001f)));
				// Depth limits (:1769-1779).
				++depth;
				bool cont = depth < sc.launch.maxDepth;
				if (!(flags & PF_CURRENT_HIT_SPECULAR) && !skipped)
					cont = (flags & PF_REFRACTION_HAPPENED) ? depth < sc.launch.maxTransmitted : depth < sc.launch.maxReflected;
				if (!cont) flags |= PF_FINISHED;
				// updateStateFlags (:954-972).
				uint32_t inc = 0;
				if (flags & PF_CURRENT_HIT_SPECULAR) inc |= PF_PREVIOUS_HIT_SPECULAR; else inc |= PF_REGULARIZED;
				if (flags & PF_RAY_REFRACTED) inc |= PF_REFRACTION_HAPPENED;
				flags = (flags & ~(PF_CURRENT_HIT_SPECULAR | PF_PREVIOUS_HIT_SPECULAR | PF_TRIANGULAR_GEOMETRY
					| PF_RIGHT_HANDED_FRAME | PF_RAY_REFRACTED)) | inc;
				done = (flags & PF_FINISHED) != 0;
			}
		}
		s.T[p] = f4(T);
		s.fd[p] = make_uint2(flags, depth);
		s.rayO[p] = f4_of(rayO, refrScale);
		s.rayD[p] = f4_of(rayD, st.pdf);
		if (hasShadow)
		{
			const uint32_t slot = appendSlot(shadowCount, s.queueCap, sc.status);
			if (slot != kNoSlot) s.shadowQueue[slot] = i;
		}
		if (!done)
		{
			const uint32_t slot = appendSlot(nextCount, s.queueCap, sc.status);
			if (slot != kNoSlot) nextQueue[slot] = p;
		}
	}
}

__global__ void kSetWaveDyn(uint32_t* dyn, uint32_t offset, uint32_t fresh)
{
	dyn[0] = offset;
	dyn[1] = fresh;
}

// Camera-relative light data (the reference's fillLightDataBuffer /
// fillLightTreeDataBuffers): one float subtraction per coordinate.
__global__ void kLightOrigin(const EmissiveTri* __restrict__ worldTris, EmissiveTri* __restrict__ tris, uint32_t nTris,
	const PackedNode* __restrict__ worldNodes, PackedNode* __restrict__ nodes, uint32_t nNodes, float ox, float oy,
	float oz)
{
	for (uint32_t i = gtid(); i < nTris + nNodes; i += gstride())
	{
		if (i < nTris)
		{
			EmissiveTri t = worldTris[i];
			for (int k = 0; k < 3; ++k)
			{
				t.v[3 * k] = __fsub_rn(t.v[3 * k], ox);
				t.v[3 * k + 1] = __fsub_rn(t.v[3 * k + 1], oy);
				t.v[3 * k + 2] = __fsub_rn(t.v[3 * k + 2], oz);
			}
			tris[i] = t;
		}
		else
		{
			PackedNode n = worldNodes[i - nTris];
			n.mean[0] = __fsub_rn(n.mean[0], ox);
			n.mean[1] = __fsub_rn(n.mean[1], oy);
			n.mean[2] = __fsub_rn(n.mean[2], oz);
			nodes[i - nTris] = n;
		}
	}
}

// Unpacks the light tree once per upload (TreeNodeU).
__global__ void kUnpackLightTree(const PackedNode* in, TreeNodeU* out, uint32_t n)
{
	for (uint32_t i = gtid(); i < n; i += gstride()) out[i] = makeNodeU(in, i);
}

// Sample resolve and FP64 accumulation (pathtrace.cu:1789-1812, color::toRGB).
template<bool JOBS>
__global__ void __launch_bounds__(kThreads) kResolve(const __grid_constant__ DevScene scK, PathSoA s, WaveParams w,
	double4* accumK)
{
	const uint32_t slots = JOBS ? w.pixelSlots : w.pixels;
	for (uint32_t slot = gtid(); slot < slots; slot += gstride())
	{
		// the pixel, its planes' path slots (first + k stride) and its job
		const DevScene* scp = &scK;
		double4* accum = accumK;
		uint32_t first, stride, planes, pix;
		bool fresh, keepFailed;
		if (JOBS)
		{
			const WaveChunk c = w.chunks[chunkOfPixel(w, slot)];
			const uint32_t local = slot - c.pixel;
			const uint2 px = slotPixel(local, c.width, c.height);
			pix = px.y * c.width + px.x;
			first = c.slot + local;
			stride = c.pixels;
			planes = c.planes;
			fresh = c.fresh != 0;
			const DevJob& job = s.jobs[c.job];
			scp = &job.scene;
			accum = job.accum;
			keepFailed = job.keepFailed != 0;
		}
		else
		{
			const uint2 px = slotPixel(slot, scK.launch.width, scK.launch.height);
			pix = px.y * scK.launch.width + px.x;
			first = slot;
			stride = w.pixels;
			planes = w.paths / w.pixels;
			fresh = waveFresh(w);
			keepFailed = w.keepFailed != 0;
		}
		const DevScene& sc = *scp;
		const float* X = sc.spectra.sensor;
		const float* Y = X + kSpectrumBins;
		const float* Z = Y + kSpectrumBins;
		double4 acc = fresh ? make_double4(0.0, 0.0, 0.0, 0.0) : accum[pix];
		for (uint32_t k = 0; k < planes; ++k)
		{
			const uint32_t p = first + k * stride;
			const uint32_t flags = s.fd[p].x;
			if (!(flags & PF_PATH_TERMINATED) || keepFailed)
			{
				S4 L = s4(s.L[p]);
				const S4 pdf = s4(s.lpdf[p]);
				const S4 lam = s4(s.lambda[p]);
				for (int i = 0; i < 4; ++i) L.v[i] = pdf.v[i] != 0.0f ? L.v[i] / pdf.v[i] : 0.0f;
				float cx = __fmul_rn(denseAt(X, lam.v[0]), L.v[0]);
				float cy = __fmul_rn(denseAt(Y, lam.v[0]), L.v[0]);
				float cz = __fmul_rn(denseAt(Z, lam.v[0]), L.v[0]);
				for (int i = 1; i < 4; ++i)
				{
					cx = __fadd_rn(cx, __fmul_rn(denseAt(X, lam.v[i]), L.v[i]));
					cy = __fadd_rn(cy, __fmul_rn(denseAt(Y, lam.v[i]), L.v[i]));
					cz = __fadd_rn(cz, __fmul_rn(denseAt(Z, lam.v[i]), L.v[i]));
				}
				cx /= 4.0f; cy /= 4.0f; cz /= 4.0f;
				if (!isfinite(cx) || !isfinite(cy) || !isfinite(cz)) atomicOr(sc.status, RB_DEV_NAN_RADIANCE);
				acc.x += static_cast<double>(cx);
				acc.y += static_cast<double>(cy);
				acc.z += static_cast<double>(cz);
				acc.w += 1.0;
			}
			else
			{
				acc.w += 1.0;
			}
		}
		accum[pix] = acc;
	}
}

// ------------------------------------------------ per-function kernels
__global__ void kSobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash, const uint32_t* bounce,
	const uint32_t* dim, float* out)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const Qrng q = qrngAt(sample[i], hash[i], bounce[i]);
		if (dims == 1) out[i] = sample1D(q, dim[i]);
		else if (dims == 2) sample2D(q, dim[i], out[2 * i], out[2 * i + 1]);
		else
		{
			const f3 v = sample3D(q, dim[i]);
			out[3 * i] = v.x; out[3 * i + 1] = v.y; out[3 * i + 2] = v.z;
		}
	}
}
__global__ void kPixelHash(uint32_t n, const uint32_t* x, const uint32_t* y, uint32_t* out)
{
	for (uint32_t i = gtid(); i < n; i += gstride()) out[i] = pixelHash(x[i], y[i]);
}
__global__ void kWavelengths(uint32_t n, const float* u, float* lambda, float* pdf)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const Wavelengths w = sampleVisible(u[i]);
		for (int k = 0; k < 4; ++k) { lambda[4 * i + k] = w.lambda.v[k]; pdf[4 * i + k] = w.pdf.v[k]; }
	}
}
__global__ void kCameraRay(DevScene sc, uint32_t n, const float* pixel, const float* fuv, const float* luv, float* out)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		float dx, dy;
		gaussianFilterSample(fuv[2 * i], fuv[2 * i + 1], dx, dy);
		f3 o, d;
		cameraRay(sc.launch, pixel[2 * i] + dx, pixel[2 * i + 1] + dy, luv[2 * i], luv[2 * i + 1], o, d);
		out[6 * i] = o.x; out[6 * i + 1] = o.y; out[6 * i + 2] = o.z;
		out[6 * i + 3] = d.x; out[6 * i + 4] = d.y; out[6 * i + 5] = d.z;
	}
}
__global__ void kBxdfCases(DevScene sc, uint32_t n, rb_bxdf_case* cases)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		rb_bxdf_case c = cases[i];
		const DevMaterial& mat = sc.materials[c.material];
		LightSample dl;
		for (int k = 0; k < 4; ++k) dl.spectrum.v[k] = c.light_spectrum[k];
		dl.dir = mk(c.light_dir[0], c.light_dir[1], c.light_dir[2]);
		dl.pdf = c.light_pdf;
		dl.occluded = c.occluded != 0;
		const Qrng q = qrngAt(c.sample, c.hash, c.bounce);
		const Frame fr{ mk(c.frame_t[0], c.frame_t[1], c.frame_t[2]), mk(c.frame_b[0], c.frame_b[1], c.frame_b[2]),
		                mk(c.frame_n[0], c.frame_n[1], c.frame_n[2]) };
		Surface sf;
		sf.layers = c.layers;
		sf.baseColor = mk(c.base_color[0], c.base_color[1], c.base_color[2]);
		sf.metalness = c.metalness;
		sf.ior = c.ior;
		sf.roughness = c.roughness;
		sf.transmission = c.transmission;
		sf.sheenColor = mk(c.sheen_color[0], c.sheen_color[1], c.sheen_color[2]);
		sf.sheenAlpha = c.sheen_alpha;
		BxdfState st;
		st.hasNee = false;
		for (int k = 0; k < 4; ++k)
		{
			st.wl.lambda.v[k] = c.lambda[k]; st.wl.pdf.v[k] = c.lambda_pdf[k]; st.T.v[k] = c.throughput[k];
		}
		st.wl.active = c.active_count;
		st.pdf = c.bxdf_pdf;
		st.dir = mk(c.dir[0], c.dir[1], c.dir[2]);
		st.flags = c.flags;
		st.refractionScale = c.refraction_scale;
		evalBxdf(sc, mat, dl, q, fr, sf, st);
		S4 L;
		for (int k = 0; k < 4; ++k) L.v[k] = c.L[k];
		if (st.hasNee) L += st.nee;
		for (int k = 0; k < 4; ++k)
		{
			c.L[k] = L.v[k]; c.throughput[k] = st.T.v[k]; c.lambda[k] = st.wl.lambda.v[k]; c.lambda_pdf[k] = st.wl.pdf.v[k];
		}
		c.active_count = st.wl.active;
		c.bxdf_pdf = st.pdf;
		c.dir[0] = st.dir.x; c.dir[1] = st.dir.y; c.dir[2] = st.dir.z;
		c.flags = st.flags;
		c.refraction_scale = st.refractionScale;
		cases[i] = c;
	}
}
__global__ void kLightCases(DevScene sc, uint32_t n, rb_light_case* cases)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		rb_light_case c = cases[i];
		const f3 p = mk(c.position[0], c.position[1], c.position[2]);
		const f3 nn = mk(c.normal[0], c.normal[1], c.normal[2]);
		lightTreeSample(sc, sc.lights.unpacked, c.rand, p, nn, c.type, c.index, c.pdf);
		c.q_pdf = lightTreePdf(sc, c.q_type, c.q_index, p, nn);
		cases[i] = c;
	}
}
__global__ void kOffsetPoint(uint32_t n, const float* p, const float* nrm, float* out)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const f3 r = offsetPoint(mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]), mk(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]));
		out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
	}
}
__global__ void kOctEncode(uint32_t n, const float* v, uint32_t* out)
{
	for (uint32_t i = gtid(); i < n; i += gstride()) out[i] = octEncodeU32(mk(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
}
__global__ void kOctDecode(uint32_t n, const uint32_t* code, float* out)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const f3 r = octDecodeU32(code[i]);
		out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
	}
}
} // namespace

LaunchShape queryLaunchShape()
{
	LaunchShape ls{};
	int dev = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&ls.smCount, cudaDevAttrMultiProcessorCount, dev);
	auto occ = [&](const void* fn) {
		int b = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kThreads, 0);
		return (b < 1 ? 1 : b) * ls.smCount;
	};
	ls.threads = kThreads;
	ls.blocksGenerate = occ(reinterpret_cast<const void*>(kGenerate<false>));
	ls.blocksSurface = occ(reinterpret_cast<const void*>(kSurface<false, false>));
	ls.blocksNee = occ(reinterpret_cast<const void*>(kNee<false, false, false>));
	ls.blocksEmission = occ(reinterpret_cast<const void*>(kEmission<false>));
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kNee<true, false, false>), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kNeeSharedMaxBytes));
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kNee<true, false, true>), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kNeeSharedMaxBytes));
	ls.blocksBsdf = occ(reinterpret_cast<const void*>(kBsdf<false, false>));
	ls.blocksBsdfLight = occ(reinterpret_cast<const void*>(kBsdfLight<false, false>));
	ls.blocksResolve = occ(reinterpret_cast<const void*>(kResolve<false>));
	queryTraceShape(ls);
	return ls;
}

// The launchers run the shared-wavefront variants when the path arrays
// carry a job table (rb_render_jobs).
void launchGenerate(const DevScene& sc, const PathSoA& s, const WaveParams& w, const LaunchShape& ls, cudaStream_t st)
{
	const int g = capBlocks(ls.blocksGenerate, ls.items, kThreads);
	if (s.jobs) kGenerate<true><<<g, kThreads, 0, st>>>(sc, s, w);
	else kGenerate<false><<<g, kThreads, 0, st>>>(sc, s, w);
}
void launchSurface(const DevScene& sc, const PathSoA& s, const WaveParams& w, int bounce, const LaunchShape& ls, cudaStream_t st,
	unsigned long long* counters)
{
	const int g = capBlocks(ls.blocksSurface, ls.items, kThreads);
	if (s.jobs)
	{
		if (w.textured) kSurface<true, true><<<g, kThreads, 0, st>>>(sc, s, w, bounce, counters);
		else kSurface<true, false><<<g, kThreads, 0, st>>>(sc, s, w, bounce, counters);
	}
	else if (w.textured) kSurface<false, true><<<g, kThreads, 0, st>>>(sc, s, w, bounce, counters);
	else kSurface<false, false><<<g, kThreads, 0, st>>>(sc, s, w, bounce, counters);
}
void launchEmission(const DevScene& sc, const PathSoA& s, int bounce, const LaunchShape& ls, cudaStream_t st)
{
	const int g = capBlocks(ls.blocksEmission, ls.items, kThreads);
	if (s.jobs) kEmission<true><<<g, kThreads, 0, st>>>(sc, s, bounce);
	else kEmission<false><<<g, kThreads, 0, st>>>(sc, s, bounce);
}
template<bool TEX>
void launchNeeT(const DevScene& sc, const PathSoA& s, const WaveParams& w, int bounce, const LaunchShape& ls, cudaStream_t st)
{
	const int g = capBlocks(ls.blocksNee, ls.items, kThreads);
	if (s.jobs)
	{
		kNee<false, true, TEX><<<g, kThreads, 0, st>>>(sc, s, w, bounce, 0);
		kNee<false, true, TEX><<<g, kThreads, 0, st>>>(sc, s, w, bounce, 1);
		return;
	}
	const size_t treeBytes = sizeof(TreeNodeU) * sc.lights.nodeCount;
	if (sc.lights.unpacked && treeBytes <= kNeeSharedMaxBytes)
	{
		int b = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, reinterpret_cast<const void*>(kNee<true, false, TEX>),
			kNeeSharedThreads, treeBytes);
		kNee<true, false, TEX><<<capBlocks((b < 1 ? 1 : b) * ls.smCount, ls.items, kNeeSharedThreads), kNeeSharedThreads,
			treeBytes, st>>>(sc, s, w, bounce, 0);
	}
	else
	{
		kNee<false, false, TEX><<<g, kThreads, 0, st>>>(sc, s, w, bounce, 0);
	}
	kNee<false, false, TEX><<<g, kThreads, 0, st>>>(sc, s, w, bounce, 1);
}
void launchNee(const DevScene& sc, const PathSoA& s, const WaveParams& w, int bounce, const LaunchShape& ls, cudaStream_t st)
{
	if (w.textured) launchNeeT<true>(sc, s, w, bounce, ls, st);
	else launchNeeT<false>(sc, s, w, bounce, ls, st);
}
void launchBsdf(const DevScene& sc, const PathSoA& s, const WaveParams& w, int bounce, const LaunchShape& ls, cudaStream_t st)
{
	const int gl = capBlocks(ls.blocksBsdfLight, ls.items, kThreads), gs = capBlocks(ls.blocksBsdf, ls.items, kThreads);
	if (s.jobs && w.textured)
	{
		kBsdfLight<true, true><<<gl, kThreads, 0, st>>>(sc, s, w, bounce);
		kBsdf<true, true><<<gs, kThreads, 0, st>>>(sc, s, w, bounce);
	}
	else if (s.jobs)
	{
		kBsdfLight<true, false><<<gl, kThreads, 0, st>>>(sc, s, w, bounce);
		kBsdf<true, false><<<gs, kThreads, 0, st>>>(sc, s, w, bounce);
	}
	else if (w.textured)
	{
		kBsdfLight<false, true><<<gl, kThreads, 0, st>>>(sc, s, w, bounce);
		kBsdf<false, true><<<gs, kThreads, 0, st>>>(sc, s, w, bounce);
	}
	else
	{
		kBsdfLight<false, false><<<gl, kThreads, 0, st>>>(sc, s, w, bounce);
		kBsdf<false, false><<<gs, kThreads, 0, st>>>(sc, s, w, bounce);
	}
}
void launchSetWaveDyn(uint32_t* dyn, uint32_t offset, uint32_t fresh, cudaStream_t st)
{
	kSetWaveDyn<<<1, 1, 0, st>>>(dyn, offset, fresh);
}
void launchLightOrigin(const EmissiveTri* worldTris, EmissiveTri* tris, uint32_t nTris, const PackedNode* worldNodes,
	PackedNode* nodes, uint32_t nNodes, float ox, float oy, float oz, cudaStream_t st)
{
	if (nTris + nNodes == 0) return;
	kLightOrigin<<<gridFor(nTris + nNodes), kThreads, 0, st>>>(worldTris, tris, nTris, worldNodes, nodes, nNodes, ox, oy, oz);
}
void launchUnpackLightTree(const PackedNode* in, TreeNodeU* out, uint32_t n, cudaStream_t st)
{
	kUnpackLightTree<<<gridFor(n), kThreads, 0, st>>>(in, out, n);
}
void launchResolve(const DevScene& sc, const PathSoA& s, const WaveParams& w, double4* accum, const LaunchShape& ls, cudaStream_t st)
{
	if (s.jobs)
		kResolve<true><<<capBlocks(ls.blocksResolve, w.pixelSlots, kThreads), kThreads, 0, st>>>(sc, s, w, accum);
	else
		kResolve<false><<<capBlocks(ls.blocksResolve, w.pixels, kThreads), kThreads, 0, st>>>(sc, s, w, accum);
}

void launchSobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash, const uint32_t* bounce,
	const uint32_t* dim, float* out, cudaStream_t st)
{
	kSobol<<<gridFor(n), kThreads, 0, st>>>(n, dims, sample, hash, bounce, dim, out);
}
void launchPixelHash(uint32_t n, const uint32_t* x, const uint32_t* y, uint32_t* out, cudaStream_t st)
{
	kPixelHash<<<gridFor(n), kThreads, 0, st>>>(n, x, y, out);
}
void launchWavelengths(uint32_t n, const float* u, float* lambda, float* pdf, cudaStream_t st)
{
	kWavelengths<<<gridFor(n), kThreads, 0, st>>>(n, u, lambda, pdf);
}
namespace
{
// The software sampler and the texture unit on the same texture and
// coordinates (a check of the sampler's semantics against the hardware the
// reference samples with).
__global__ void kTextureSample(const __grid_constant__ DevScene sc, uint32_t texture, cudaTextureObject_t hw,
	uint32_t n, const float* __restrict__ uv, float4* __restrict__ soft, float4* __restrict__ hwOut)
{
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		const float u = uv[2 * i], v = uv[2 * i + 1];
		soft[i] = texSample(sc, texture, u, v);
		hwOut[i] = tex2D<float4>(hw, u, v);
	}
}
} // namespace

void launchTextureSample(const DevScene& sc, uint32_t texture, cudaTextureObject_t hw, uint32_t n, const float* uv,
	float* soft, float* hwOut, cudaStream_t st)
{
	kTextureSample<<<gridFor(n), kThreads, 0, st>>>(sc, texture, hw, n, uv, reinterpret_cast<float4*>(soft),
		reinterpret_cast<float4*>(hwOut));
}

void launchCameraRay(const DevScene& sc, uint32_t n, const float* pixel, const float* fuv, const float* luv, float* out, cudaStream_t st)
{
	kCameraRay<<<gridFor(n), kThreads, 0, st>>>(sc, n, pixel, fuv, luv, out);
}
void launchBxdfCases(const DevScene& sc, uint32_t n, void* cases, cudaStream_t st)
{
	kBxdfCases<<<gridFor(n), kThreads, 0, st>>>(sc, n, static_cast<rb_bxdf_case*>(cases));
}
void launchLightCases(const DevScene& sc, uint32_t n, void* cases, cudaStream_t st)
{
	kLightCases<<<gridFor(n), kThreads, 0, st>>>(sc, n, static_cast<rb_light_case*>(cases));
}
void launchOffsetPoint(uint32_t n, const float* p, const float* nrm, float* out, cudaStream_t st)
{
	kOffsetPoint<<<gridFor(n), kThreads, 0, st>>>(n, p, nrm, out);
}
void launchOctEncode(uint32_t n, const float* v, uint32_t* out, cudaStream_t st)
{
	kOctEncode<<<gridFor(n), kThreads, 0, st>>>(n, v, out);
}
void launchOctDecode(uint32_t n, const uint32_t* code, float* out, cudaStream_t st)
{
	kOctDecode<<<gridFor(n), kThreads, 0, st>>>(n, code, out);
}
} // namespace rb
