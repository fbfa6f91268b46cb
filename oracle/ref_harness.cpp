// Oracle test infrastructure (not product code).
//
// Runs the reference's own per-sample rendering code on the CPU. The patched
// copy of src/kernels/pathtrace.cu (see stage_ref.sh) is included below as a
// C++ source, so __raygen__main, __closesthit__triangle, __miss__miss, the
// BxDF callables and every src/device/*.h function it calls are the
// reference's code compiled by g++. This file supplies only what OptiX and
// the CUDA runtime would: a CPU BVH behind optixTrace/optixTraverse
// (cpu_bvh.h), texture fetches from host arrays, the LaunchParameters
// contents and a thread pool that plays the role of optixLaunch(W, H, 1)
// (src/core/rendering_interface.cpp:1875).
//
// The exported rbref_* functions take the same boundary records as the
// product's C ABI (include/ratbite_b200.h, include/ratbite_b200_kernels.h), so
// tests can hand identical inputs to both. Only tests/, the smoke check and
// the CPU baseline of bench.py load this library.

#include "_ref/src/kernels/pathtrace.cu"
#include "_ref/src/core/light_tree.h"
#include "_ref/src/core/scene.h"
#include "_ref/src/core/spectral.h"
#include "_ref/src/core/color.h"

#include "../include/ratbite_b200.h"
#include "../include/ratbite_b200_kernels.h"
#include "cpu_bvh.h"

#include <array>
#include <atomic>
#include <memory>
#include <thread>
#include <vector>

std::filesystem::path getExePath() { return {}; }
std::filesystem::path getExeDir() { return {}; }

namespace oracle_optix
{
	thread_local ThreadState tls;
	void* callables[3] = {
		reinterpret_cast<void*>(&__direct_callable__PureConductorBxDF),
		reinterpret_cast<void*>(&__direct_callable__PureDielectricBxDF),
		reinterpret_cast<void*>(&__direct_callable__ComplexSurface_BxDF),
	};
}

namespace
{
	// ---------------------------------------------------------------- textures
	struct OwnedTexture
	{
		std::vector<float> data;
		oracle_tex::Texture view;
	};
	std::vector<std::unique_ptr<OwnedTexture>> g_textures;

	cudaTextureObject_t addTexture(const float* src, int w, int h, int d, int c)
	{
		auto t = std::make_unique<OwnedTexture>();
		t->data.assign(src, src + static_cast<size_t>(w) * h * d * c);
		t->view = oracle_tex::Texture{ t->data.data(), w, h, d, c };
		g_textures.push_back(std::move(t));
		return static_cast<cudaTextureObject_t>(g_textures.size()); // handles start at 1
	}

	// ------------------------------------------------------------ scene state
	struct alignas(16) DenseStorage { float v[SpectralSettings::KSampledWavelengthsNumber]; };
	std::vector<DenseStorage> g_sensor(3), g_basis(3), g_extra;

	std::vector<MaterialData> g_materials;
	std::vector<std::vector<uint8_t>> g_materialBuffers;
	std::vector<cudaTextureObject_t> g_materialTextures;   // rb_set_textures index -> registry handle

	struct TriRecord
	{
		uint32_t primitiveIndex;
		uint32_t sbtData;
		uint32_t instance;
		float obj[9];
	};
	std::vector<TriRecord> g_tris;
	std::vector<std::array<float, 12>> g_objToWorld, g_worldToObj;
	oracle_bvh::BVH g_bvh;

	std::vector<EmissiveTriangleLightData> g_lightTris;
	std::vector<LightTree::PackedNode> g_nodes;
	std::vector<LightTree::LightPointer> g_pointers;
	std::vector<uint64_t> g_bitmasks;

	std::vector<uint16_t> g_envCond, g_envMarg;

	std::vector<glm::dvec4> g_renderData;

	void refreshSpectraPointers()
	{
		parameters.sensorSpectralCurveA = reinterpret_cast<DenseSpectrum*>(&g_sensor[0]);
		parameters.sensorSpectralCurveB = reinterpret_cast<DenseSpectrum*>(&g_sensor[1]);
		parameters.sensorSpectralCurveC = reinterpret_cast<DenseSpectrum*>(&g_sensor[2]);
		parameters.spectralBasisR = reinterpret_cast<DenseSpectrum*>(&g_basis[0]);
		parameters.spectralBasisG = reinterpret_cast<DenseSpectrum*>(&g_basis[1]);
		parameters.spectralBasisB = reinterpret_cast<DenseSpectrum*>(&g_basis[2]);
		parameters.spectra = g_extra.empty() ? nullptr : reinterpret_cast<DenseSpectrum*>(g_extra.data());
	}

	// Row-major 3x4 inverse, computed in double and rounded once.
	std::array<float, 12> invert3x4(const float* m)
	{
		const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
		const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
		const double r = 1.0 / det;
		double inv[9] = {
			(e * i - f * h) * r, (c * h - b * i) * r, (b * f - c * e) * r,
			(f * g - d * i) * r, (a * i - c * g) * r, (c * d - a * f) * r,
			(d * h - e * g) * r, (b * g - a * h) * r, (a * e - b * d) * r };
		const double t[3] = { m[3], m[7], m[11] };
		std::array<float, 12> out{};
		for (int row = 0; row < 3; ++row)
		{
			out[row * 4 + 0] = static_cast<float>(inv[row * 3 + 0]);
			out[row * 4 + 1] = static_cast<float>(inv[row * 3 + 1]);
			out[row * 4 + 2] = static_cast<float>(inv[row * 3 + 2]);
			out[row * 4 + 3] = static_cast<float>(-(inv[row * 3 + 0] * t[0] + inv[row * 3 + 1] * t[1] + inv[row * 3 + 2] * t[2]));
		}
		return out;
	}

	// World-space vertex exactly as __closesthit__triangle forms it
	// (src/kernels/pathtrace.cu:125-127): ((x*W0 + y*W1) + z*W2) + W3 in float.
	void toWorld(const float* W, const float* p, float* out)
	{
		out[0] = p[0] * W[0] + p[1] * W[1] + p[2] * W[2] + W[3];
		out[1] = p[0] * W[4] + p[1] * W[5] + p[2] * W[6] + W[7];
		out[2] = p[0] * W[8] + p[1] * W[9] + p[2] * W[10] + W[11];
	}

	uint32_t readIndex(const void* indices, uint32_t type, size_t i)
	{
		return type == RB_INDEX_U16 ? static_cast<const uint16_t*>(indices)[i] : static_cast<const uint32_t*>(indices)[i];
	}

	QRNG::State makeState(uint32_t sample, uint32_t hash, uint32_t bounce)
	{
		QRNG::State s{ sample, hash };
		for (uint32_t b = 0; b < bounce; ++b) s.advanceBounce();
		return s;
	}
}

namespace oracle_tex
{
	int weightMode = 0;
	const Texture& get(cudaTextureObject_t handle)
	{
		return g_textures.at(static_cast<size_t>(handle) - 1)->view;
	}
}

namespace oracle_optix
{
	bool traceClosest(float3 o, float3 d, float tmin, float tmax, HitState& out)
	{
		float t, b1, b2;
		const int id = g_bvh.closest({ o.x, o.y, o.z }, { d.x, d.y, d.z }, tmin, tmax, t, b1, b2);
		if (id < 0) return false;
		const TriRecord& r = g_tris[id];
		out.primitiveIndex = r.primitiveIndex;
		out.barycentrics = float2{ b1, b2 };
		out.sbtData = r.sbtData;
		for (int k = 0; k < 3; ++k)
			out.objectVertices[k] = float3{ r.obj[k * 3 + 0], r.obj[k * 3 + 1], r.obj[k * 3 + 2] };
		for (int k = 0; k < 12; ++k)
		{
			out.objectToWorld[k] = g_objToWorld[r.instance][k];
			out.worldToObject[k] = g_worldToObj[r.instance][k];
		}
		tls.lastT = t;
		tls.lastTri = id;
		return true;
	}
	bool traceAny(float3 o, float3 d, float tmin, float tmax)
	{
		return g_bvh.any({ o.x, o.y, o.z }, { d.x, d.y, d.z }, tmin, tmax);
	}
}

extern "C"
{

int rbref_abi_version() { return RB_ABI_VERSION; }

void rbref_reset()
{
	g_textures.clear();
	g_materialTextures.clear();
	g_materials.clear();
	g_materialBuffers.clear();
	g_tris.clear();
	g_objToWorld.clear();
	g_worldToObj.clear();
	g_bvh = oracle_bvh::BVH{};
	g_lightTris.clear();
	g_nodes.clear();
	g_pointers.clear();
	g_bitmasks.clear();
	g_envCond.clear();
	g_envMarg.clear();
	g_renderData.clear();
	g_extra.clear();
	parameters = LaunchParameters{};
	refreshSpectraPointers();
}

void rbref_set_texture_weight_mode(int mode) { oracle_tex::weightMode = mode; }

// ---- reference data tables (src/core/spectral.cpp) ----------------------
// out: 3*471 floats X, Y, Z (SpectralData::CIE::X/Y/Z, spectral.cpp:1488-1502).
void rbref_cie_xyz(float* out)
{
	const DenselySampledSpectrum* s[3] = { &SpectralData::CIE::X(), &SpectralData::CIE::Y(), &SpectralData::CIE::Z() };
	for (int k = 0; k < 3; ++k)
		std::memcpy(out + k * RB_SPECTRUM_BINS, s[k], sizeof(float) * RB_SPECTRUM_BINS);
}
// out: 3*471 floats R, G, B basis (SpectralData::CIE::BasisR/G/B, spectral.cpp:1507-1521).
void rbref_basis_rgb(float* out)
{
	const DenselySampledSpectrum* s[3] = { &SpectralData::CIE::BasisR(), &SpectralData::CIE::BasisG(), &SpectralData::CIE::BasisB() };
	for (int k = 0; k < 3; ++k)
		std::memcpy(out + k * RB_SPECTRUM_BINS, s[k], sizeof(float) * RB_SPECTRUM_BINS);
}
// SpectralData::loadSpectrum for a SpectralDataType value (spectral.cpp:1524+).
int rbref_named_spectrum(int type, float* out)
{
	if (type <= 0 || type >= static_cast<int>(SpectralData::SpectralDataType::DESC)) return RB_ERR_INVALID;
	DenselySampledSpectrum s{ SpectralData::loadSpectrum(static_cast<SpectralData::SpectralDataType>(type)) };
	std::memcpy(out, &s, sizeof(float) * RB_SPECTRUM_BINS);
	return RB_OK;
}

// ---- uploads mirroring the product ABI ----------------------------------
int rbref_set_spectra(const float* sensor, const float* basis, const float* extra, uint32_t nExtra)
{
	for (int k = 0; k < 3; ++k)
	{
		std::memcpy(g_sensor[k].v, sensor + k * RB_SPECTRUM_BINS, sizeof(float) * RB_SPECTRUM_BINS);
		std::memcpy(g_basis[k].v, basis + k * RB_SPECTRUM_BINS, sizeof(float) * RB_SPECTRUM_BINS);
	}
	g_extra.assign(nExtra, DenseStorage{});
	for (uint32_t k = 0; k < nExtra; ++k)
		std::memcpy(g_extra[k].v, extra + k * RB_SPECTRUM_BINS, sizeof(float) * RB_SPECTRUM_BINS);
	refreshSpectraPointers();
	return RB_OK;
}

int rbref_set_luts(const float* conductor, const float* dielOuter, const float* dielInner,
	const float* reflOuter, const float* reflInner, const float* sheen)
{
	constexpr int N = RB_LUT_SIZE;
	parameters.LUTs.conductorAlbedo = addTexture(conductor, N, N, 1, 1);
	parameters.LUTs.dielectricOuterAlbedo = addTexture(dielOuter, N, N, N, 1);
	parameters.LUTs.dielectricInnerAlbedo = addTexture(dielInner, N, N, N, 1);
	parameters.LUTs.reflectiveDielectricOuterAlbedo = addTexture(reflOuter, N, N, N, 1);
	parameters.LUTs.reflectiveDielectricInnerAlbedo = addTexture(reflInner, N, N, N, 1);
	parameters.LUTs.sheenLTC = addTexture(sheen, N, N, 1, 4);
	return RB_OK;
}

// Material textures (the product's rb_set_textures table): texels decoded
// to floats as the texture hardware reads them (8-bit / 255; the sRGB curve
// for r, g, b of sRGB textures, r of a one-channel one, IEC 61966-2-1 in
// double precision), a one-channel texture stored as (r, 0, 0, 0), which
// is what the texture unit returns for it; handles registered for
// rbref_set_materials to use. Call after rbref_set_luts.
int rbref_set_textures(const rb_texture* tex, uint32_t count)
{
	g_materialTextures.clear();
	float lut[256];
	for (int c = 0; c < 256; ++c)
	{
		const double x = c / 255.0;
		lut[c] = static_cast<float>(x <= 0.04045 ? x / 12.92 : std::pow((x + 0.055) / 1.055, 2.4));
	}
	for (uint32_t i = 0; i < count; ++i)
	{
		const rb_texture& t = tex[i];
		if (t.format > RB_TEXFMT_RGBA8 || !t.data || t.width == 0 || t.height == 0) return RB_ERR_INVALID;
		const size_t n = static_cast<size_t>(t.width) * t.height;
		const uint8_t* src = static_cast<const uint8_t*>(t.data);
		std::vector<float> texels(n * 4);
		for (size_t k = 0; k < n; ++k)
		{
			if (t.format == RB_TEXFMT_R8)
			{
				texels[4 * k] = t.srgb ? lut[src[k]] : static_cast<float>(src[k]) / 255.0f;
				texels[4 * k + 1] = 0.0f; texels[4 * k + 2] = 0.0f; texels[4 * k + 3] = 0.0f;
				continue;
			}
			for (int ch = 0; ch < 4; ++ch)
			{
				const uint8_t b = src[4 * k + ch];
				texels[4 * k + ch] = (t.srgb && ch < 3) ? lut[b] : static_cast<float>(b) / 255.0f;
			}
		}
		const cudaTextureObject_t h = addTexture(texels.data(), static_cast<int>(t.width), static_cast<int>(t.height), 1, 4);
		oracle_tex::Texture& view = g_textures.back()->view;
		view.addrU = static_cast<int>(t.address_u == RB_TEXADDR_WRAP ? 0 : (t.address_u == RB_TEXADDR_CLAMP ? 1 : 2));
		view.addrV = static_cast<int>(t.address_v == RB_TEXADDR_WRAP ? 0 : (t.address_v == RB_TEXADDR_CLAMP ? 1 : 2));
		view.linear = t.filter == RB_TEXFILTER_LINEAR ? 1 : 0;
		g_materialTextures.push_back(h);
	}
	return RB_OK;
}

int rbref_set_materials(const rb_material* mats, uint32_t count)
{
	g_materials.assign(count, MaterialData{});
	g_materialBuffers.clear();
	g_materialBuffers.reserve(count * 2);
	for (uint32_t i = 0; i < count; ++i)
	{
		const rb_material& m = mats[i];
		if (m.textures >> RB_TEXTURE_SLOTS) return RB_ERR_INVALID;
		for (uint32_t t = 0; t < RB_TEXTURE_SLOTS; ++t)
			if (((m.textures >> t) & 1u) && m.texture_index[t] >= g_materialTextures.size()) return RB_ERR_INVALID;
		MaterialData& d = g_materials[i];
		d.bxdfIndexSBT = m.bxdf;
		d.doubleSided = m.double_sided != 0;
		d.sheenPresent = m.sheen_present != 0;
		d.indexType = m.index_type == RB_INDEX_U16 ? IndexType::UINT_16 : IndexType::UINT_32;
		const size_t ib = static_cast<size_t>(m.triangle_count) * 3 * (m.index_type == RB_INDEX_U16 ? 2 : 4);
		g_materialBuffers.emplace_back(static_cast<const uint8_t*>(m.indices), static_cast<const uint8_t*>(m.indices) + ib);
		d.indices = g_materialBuffers.back().data();
		d.attributes = static_cast<MaterialData::AttributeTypeBitfield>(m.attributes);
		d.attributeStride = static_cast<uint8_t>(m.attribute_stride);
		d.normalOffset = static_cast<uint8_t>(m.normal_offset);
		d.frameOffset = static_cast<uint8_t>(m.frame_offset);
		d.colorOffset = static_cast<uint8_t>(m.color_offset);
		d.texCoord1Offset = static_cast<uint8_t>(m.texcoord1_offset);
		d.texCoord2Offset = static_cast<uint8_t>(m.texcoord2_offset);
		const size_t ab = static_cast<size_t>(m.vertex_count) * m.attribute_stride;
		if (m.attribute_data != nullptr && ab != 0)
			g_materialBuffers.emplace_back(static_cast<const uint8_t*>(m.attribute_data), static_cast<const uint8_t*>(m.attribute_data) + ab);
		else
			g_materialBuffers.emplace_back(16, 0);
		d.attributeData = g_materialBuffers.back().data();
		d.indexOfRefractSpectrumDataIndex = static_cast<uint16_t>(m.ior_spectrum);
		d.absorpCoefSpectrumDataIndex = static_cast<uint16_t>(m.absorp_spectrum);
		d.emissionSpectrumDataIndex = static_cast<uint16_t>(m.emission_spectrum);
		d.mfRoughnessValue = m.mf_roughness;
		d.ior = m.ior;
		d.alphaCutoff = m.alpha_cutoff;
		d.textures = static_cast<MaterialData::TextureTypeBitfield>(m.textures);
		auto handle = [&](uint32_t slot) -> cudaTextureObject_t {
			return ((m.textures >> slot) & 1u) ? g_materialTextures[m.texture_index[slot]] : 0;
		};
		auto set2 = [&](uint32_t slot) { return ((m.texcoord_sets >> slot) & 1u) != 0; };
		d.baseColorTexture = handle(RB_TEXTURE_BASE_COLOR);
		d.normalTexture = handle(RB_TEXTURE_NORMAL);
		d.pbrMetalRoughnessTexture = handle(RB_TEXTURE_MET_ROUGH);
		d.transmissionTexture = handle(RB_TEXTURE_TRANSMISSION);
		d.sheenColorTexture = handle(RB_TEXTURE_SHEEN_COLOR);
		d.sheenRoughTexture = handle(RB_TEXTURE_SHEEN_ROUGH);
		d.emissiveTexture = handle(RB_TEXTURE_EMISSION);
		d.bcTexCoordSetIndex = set2(RB_TEXTURE_BASE_COLOR);
		d.nmTexCoordSetIndex = set2(RB_TEXTURE_NORMAL);
		d.mrTexCoordSetIndex = set2(RB_TEXTURE_MET_ROUGH);
		d.trTexCoordSetIndex = set2(RB_TEXTURE_TRANSMISSION);
		d.shcTexCoordSetIndex = set2(RB_TEXTURE_SHEEN_COLOR);
		d.shrTexCoordSetIndex = set2(RB_TEXTURE_SHEEN_ROUGH);
		d.emTexCoordSetIndex = set2(RB_TEXTURE_EMISSION);
		d.factors = static_cast<MaterialData::FactorTypeBitfield>(m.factors);
		for (int k = 0; k < 4; ++k) d.baseColorFactor[k] = m.base_color[k];
		d.metalnessFactor = m.metalness;
		d.roughnessFactor = m.roughness;
		d.transmissionFactor = m.transmission;
		for (int k = 0; k < 3; ++k) d.sheenColorFactor[k] = m.sheen_color[k];
		d.sheenRoughnessFactor = m.sheen_roughness;
		for (int k = 0; k < 3; ++k) d.emissiveFactor[k] = m.emissive[k];
	}
	parameters.materials = g_materials.data();
	return RB_OK;
}

// Canonical triangle order (shared with the product for closest-hit tie
// breaks): emissive subsets first, then instances x submeshes x triangles,
// mirroring the IAS instance order (src/core/rendering_interface.cpp:964-1012).
int rbref_set_geometry(const rb_geometry* g)
{
	g_tris.clear();
	g_objToWorld.clear();
	g_worldToObj.clear();
	std::vector<float> world;
	uint32_t emissivePrim = 0;
	for (uint32_t s = 0; s < g->emissive_subset_count; ++s)
	{
		const rb_emissive_subset& es = g->emissive_subsets[s];
		const uint32_t inst = static_cast<uint32_t>(g_objToWorld.size());
		g_objToWorld.push_back({});
		std::memcpy(g_objToWorld.back().data(), es.transform, sizeof(float) * 12);
		g_worldToObj.push_back(invert3x4(es.transform));
		for (uint32_t t = 0; t < es.triangle_count; ++t)
		{
			TriRecord r{};
			r.primitiveIndex = emissivePrim++;
			r.sbtData = 0xFFFFFFFFu;
			r.instance = inst;
			std::memcpy(r.obj, es.vertices + t * 9, sizeof(float) * 9);
			float w[9];
			for (int k = 0; k < 3; ++k) toWorld(es.transform, r.obj + k * 3, w + k * 3);
			world.insert(world.end(), w, w + 9);
			g_tris.push_back(r);
		}
	}
	for (uint32_t i = 0; i < g->instance_count; ++i)
	{
		const rb_instance& in = g->instances[i];
		if (in.mesh >= g->mesh_count) return RB_ERR_INVALID;
		const uint32_t inst = static_cast<uint32_t>(g_objToWorld.size());
		g_objToWorld.push_back({});
		std::memcpy(g_objToWorld.back().data(), in.transform, sizeof(float) * 12);
		g_worldToObj.push_back(invert3x4(in.transform));
		const rb_mesh& mesh = g->meshes[in.mesh];
		for (uint32_t s = 0; s < mesh.submesh_count; ++s)
		{
			const rb_submesh& sm = mesh.submeshes[s];
			std::vector<uint8_t> discarded(sm.triangle_count, 0);
			for (uint32_t k = 0; k < sm.discarded_count; ++k)
				if (sm.discarded[k] < sm.triangle_count) discarded[sm.discarded[k]] = 1;
			for (uint32_t t = 0; t < sm.triangle_count; ++t)
			{
				TriRecord r{};
				r.primitiveIndex = t;
				r.sbtData = sm.material;
				r.instance = inst;
				for (int k = 0; k < 3; ++k)
				{
					const uint32_t vi = discarded[t] ? 0u : readIndex(sm.indices, sm.index_type, static_cast<size_t>(t) * 3 + k);
					if (vi >= sm.vertex_count) return RB_ERR_INVALID;
					r.obj[k * 3 + 0] = sm.vertices[vi * 4 + 0];
					r.obj[k * 3 + 1] = sm.vertices[vi * 4 + 1];
					r.obj[k * 3 + 2] = sm.vertices[vi * 4 + 2];
				}
				float w[9];
				for (int k = 0; k < 3; ++k) toWorld(in.transform, r.obj + k * 3, w + k * 3);
				world.insert(world.end(), w, w + 9);
				g_tris.push_back(r);
			}
		}
	}
	g_bvh.build(world.data(), static_cast<int>(g_tris.size()));
	parameters.traversable = 1;
	return RB_OK;
}

int rbref_set_lights(const rb_light_tree* lt)
{
	g_lightTris.resize(lt->triangle_count);
	std::memcpy(g_lightTris.data(), lt->triangles, sizeof(EmissiveTriangleLightData) * lt->triangle_count);
	g_nodes.resize(lt->node_count);
	std::memcpy(static_cast<void*>(g_nodes.data()), lt->nodes, sizeof(LightTree::PackedNode) * lt->node_count);
	g_pointers.resize(lt->pointer_count);
	std::memcpy(g_pointers.data(), lt->pointers, sizeof(uint32_t) * lt->pointer_count);
	g_bitmasks.assign(lt->bitmasks, lt->bitmasks + lt->triangle_count);
	parameters.lightTree.nodes = lt->node_count ? g_nodes.data() : nullptr;
	parameters.lightTree.lightPointers = g_pointers.data();
	parameters.lightTree.triangles = g_lightTris.data();
	parameters.lightTree.bitmasks[KTriangleLightsArrayIndex] = g_bitmasks.data();
	return RB_OK;
}

// Environment map with CDF tables computed elsewhere (the reference's
// cdf.cu on the GPU, or the C restatement): integral already divided by w*h.
int rbref_set_envmap(const float* rgba, uint32_t w, uint32_t h, const uint16_t* cond, const uint16_t* marg, float integral)
{
	auto& e = parameters.lightTree.envMap;
	e.enabled = true;
	e.width = static_cast<float>(w);
	e.height = static_cast<float>(h);
	e.environmentTexture = addTexture(rgba, static_cast<int>(w), static_cast<int>(h), 1, 4);
	g_envCond.assign(cond, cond + static_cast<size_t>(w) * h);
	g_envMarg.assign(marg, marg + h);
	e.conditionalCDFIndices = g_envCond.data();
	e.marginalCDFIndices = g_envMarg.data();
	e.integral = integral;
	return RB_OK;
}
void rbref_clear_envmap() { parameters.lightTree.envMap = {}; }

int rbref_set_launch(const rb_launch* l)
{
	auto& r = parameters.resolutionState;
	r.filmWidth = l->width;
	r.filmHeight = l->height;
	r.invFilmWidth = l->inv_width;
	r.invFilmHeight = l->inv_height;
	r.perspectiveScaleW = l->perspective_scale_w;
	r.perspectiveScaleH = l->perspective_scale_h;
	parameters.pathState.maxPathDepth = l->max_path_depth;
	parameters.pathState.maxReflectedPathDepth = static_cast<uint16_t>(l->max_reflected_depth);
	parameters.pathState.maxTransmittedPathDepth = static_cast<uint16_t>(l->max_transmitted_depth);
	auto& c = parameters.cameraState;
	c.camU = glm::vec3{ l->cam_u[0], l->cam_u[1], l->cam_u[2] };
	c.camV = glm::vec3{ l->cam_v[0], l->cam_v[1], l->cam_v[2] };
	c.camW = glm::vec3{ l->cam_w[0], l->cam_w[1], l->cam_w[2] };
	c.depthOfFieldEnabled = l->dof_enabled != 0;
	c.appertureSize = l->aperture;
	c.focusDistance = l->focus_distance;
	g_renderData.assign(static_cast<size_t>(l->width) * l->height, glm::dvec4{ 0.0 });
	parameters.renderData = g_renderData.data();
	return RB_OK;
}

// optixLaunch(W, H, 1) on `threads` CPU threads (rows interleaved). Renders
// samples [offset, offset+count) into the FP64 accumulation buffer. If
// rowBegin/rowEnd select a band, only those rows are rendered (used for
// bounded CPU-baseline timing).
int rbref_render_rows(uint32_t offset, uint32_t count, int threads, uint32_t rowBegin, uint32_t rowEnd)
{
	if (parameters.renderData == nullptr || parameters.traversable == 0) return RB_ERR_NO_SCENE;
	parameters.samplingState.offset = offset;
	parameters.samplingState.count = count;
	const uint32_t W = parameters.resolutionState.filmWidth;
	rowEnd = std::min(rowEnd, parameters.resolutionState.filmHeight);
	if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
	std::atomic<uint32_t> nextRow{ rowBegin };
	auto worker = [&]() {
		for (;;)
		{
			const uint32_t y = nextRow.fetch_add(1);
			if (y >= rowEnd) break;
			for (uint32_t x = 0; x < W; ++x)
			{
				oracle_optix::tls.launchIndex = uint3{ x, y, 0 };
				__raygen__main();
			}
		}
	};
	std::vector<std::thread> pool;
	for (int i = 0; i < threads; ++i) pool.emplace_back(worker);
	for (auto& t : pool) t.join();
	return RB_OK;
}
// Bounded CPU sample of a frame for timing: rows first, first + stride,
// first + 2 stride, ... (every column of each), samples [offset,
// offset + count). Work is handed out in 64-pixel row segments so that
// `threads` stay busy whatever the rows cost. Returns the number of pixels
// rendered (>= 0) or an error code (< 0).
int64_t rbref_render_strided(uint32_t offset, uint32_t count, int threads, uint32_t first, uint32_t stride)
{
	if (parameters.renderData == nullptr || parameters.traversable == 0) return RB_ERR_NO_SCENE;
	if (stride == 0) return RB_ERR_INVALID;
	parameters.samplingState.offset = offset;
	parameters.samplingState.count = count;
	const uint32_t W = parameters.resolutionState.filmWidth;
	const uint32_t H = parameters.resolutionState.filmHeight;
	const uint32_t rows = first < H ? (H - first + stride - 1) / stride : 0;
	const uint32_t segs = (W + 63) / 64;
	const uint64_t units = static_cast<uint64_t>(rows) * segs;
	if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
	std::atomic<uint64_t> next{ 0 };
	auto worker = [&]() {
		for (;;)
		{
			const uint64_t u = next.fetch_add(1);
			if (u >= units) break;
			const uint32_t y = first + static_cast<uint32_t>(u / segs) * stride;
			const uint32_t x0 = static_cast<uint32_t>(u % segs) * 64;
			const uint32_t x1 = std::min(W, x0 + 64);
			for (uint32_t x = x0; x < x1; ++x)
			{
				oracle_optix::tls.launchIndex = uint3{ x, y, 0 };
				__raygen__main();
			}
		}
	};
	std::vector<std::thread> pool;
	for (int i = 0; i < threads; ++i) pool.emplace_back(worker);
	for (auto& t : pool) t.join();
	return static_cast<int64_t>(rows) * W;
}
int rbref_render(uint32_t offset, uint32_t count, int threads)
{
	return rbref_render_rows(offset, count, threads, 0, parameters.resolutionState.filmHeight);
}
void rbref_read_accum(double* out)
{
	std::memcpy(out, g_renderData.data(), sizeof(glm::dvec4) * g_renderData.size());
}
void rbref_write_accum(const double* in)
{
	std::memcpy(g_renderData.data(), in, sizeof(glm::dvec4) * g_renderData.size());
}

// ---- per-function entry points (host arrays) -----------------------------
void rbref_sobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash,
	const uint32_t* bounce, const uint32_t* dim, float* out)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		const QRNG::State s = makeState(sample[i], hash[i], bounce[i]);
		const auto d = static_cast<QRNG::DimensionOffset>(dim[i]);
		if (dims == 1)
			out[i] = QRNG::Sobol::sample1D(s, d);
		else if (dims == 2)
		{
			glm::vec2 v = QRNG::Sobol::sample2D(s, d);
			out[i * 2] = v.x; out[i * 2 + 1] = v.y;
		}
		else
		{
			glm::vec3 v = QRNG::Sobol::sample3D(s, d);
			out[i * 3] = v.x; out[i * 3 + 1] = v.y; out[i * 3 + 2] = v.z;
		}
	}
}
void rbref_pixel_hash(uint32_t n, const uint32_t* x, const uint32_t* y, uint32_t* out)
{
	for (uint32_t i = 0; i < n; ++i) out[i] = QRNG::getPixelHash(x[i], y[i]);
}
void rbref_wavelengths(uint32_t n, const float* u, float* lambda, float* pdf)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		SampledWavelengths w = SampledWavelengths::sampleVisible(u[i]);
		for (int k = 0; k < 4; ++k) { lambda[i * 4 + k] = w[k]; pdf[i * 4 + k] = w.getPDF()[k]; }
	}
}
// Camera ray exactly as __raygen__main forms it (pathtrace.cu:1136-1156).
void rbref_camera_ray(uint32_t n, const float* pixel, const float* filterUV, const float* lensUV, float* out)
{
	const auto& rs = parameters.resolutionState;
	const auto& cs = parameters.cameraState;
	for (uint32_t i = 0; i < n; ++i)
	{
		const glm::vec2 pc{ pixel[i * 2], pixel[i * 2 + 1] };
		const glm::vec2 sub{ pc + filter::gaussian::sampleDistribution(glm::vec2{ filterUV[i * 2], filterUV[i * 2 + 1] }) };
		Ray ray;
		if (cs.depthOfFieldEnabled)
			ray = generateThinLensCamera(sub, glm::vec2{ lensUV[i * 2], lensUV[i * 2 + 1] }, cs.focusDistance, cs.appertureSize,
				glm::vec2{ rs.invFilmWidth, rs.invFilmHeight }, glm::vec2{ rs.perspectiveScaleW, rs.perspectiveScaleH }, cs.camU, cs.camV, cs.camW);
		else
			ray = generatePinholeCameraDirection(sub, glm::vec2{ rs.invFilmWidth, rs.invFilmHeight },
				glm::vec2{ rs.perspectiveScaleW, rs.perspectiveScaleH }, cs.camU, cs.camV, cs.camW);
		out[i * 6 + 0] = ray.o.x; out[i * 6 + 1] = ray.o.y; out[i * 6 + 2] = ray.o.z;
		out[i * 6 + 3] = ray.d.x; out[i * 6 + 4] = ray.d.y; out[i * 6 + 5] = ray.d.z;
	}
}

// One BxDF callable invocation per case (pathtrace.cu:1724-1733).
void rbref_bxdf(uint32_t n, rb_bxdf_case* cases)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		rb_bxdf_case& c = cases[i];
		const MaterialData& mat = g_materials.at(c.material);
		DirectLightSampleData dl{};
		for (int k = 0; k < 4; ++k) dl.spectrumSample[k] = c.light_spectrum[k];
		dl.lightDir = glm::vec3{ c.light_dir[0], c.light_dir[1], c.light_dir[2] };
		dl.lightSamplePDF = c.light_pdf;
		dl.occluded = c.occluded != 0;
		const QRNG::State qs = makeState(c.sample, c.hash, c.bounce);
		const glm::mat3 frame{ glm::vec3{ c.frame_t[0], c.frame_t[1], c.frame_t[2] },
			glm::vec3{ c.frame_b[0], c.frame_b[1], c.frame_b[2] },
			glm::vec3{ c.frame_n[0], c.frame_n[1], c.frame_n[2] } };
		const LocalTransform local{ frame };
		microsurface::Surface surface{};
		surface.layers = c.layers;
		surface.base.color = glm::vec3{ c.base_color[0], c.base_color[1], c.base_color[2] };
		surface.base.metalness = c.metalness;
		surface.specular.ior = c.ior;
		surface.specular.roughness = c.roughness;
		surface.transmission.weight = c.transmission;
		surface.sheen.color = glm::vec3{ c.sheen_color[0], c.sheen_color[1], c.sheen_color[2] };
		surface.sheen.alpha = c.sheen_alpha;
		SampledSpectrum L; for (int k = 0; k < 4; ++k) L[k] = c.L[k];
		// SampledWavelengths has private members; rebuild its state through
		// the public interface: sample, then overwrite via byte copy of the
		// same layout (lambda[4], pdf[4], activeCount).
		SampledWavelengths wl{};
		struct WLayout { float lambda[4]; float pdf[4]; float active; } wlay{};
		static_assert(sizeof(WLayout) == sizeof(SampledWavelengths));
		for (int k = 0; k < 4; ++k) { wlay.lambda[k] = c.lambda[k]; wlay.pdf[k] = c.lambda_pdf[k]; }
		wlay.active = c.active_count;
		std::memcpy(&wl, &wlay, sizeof(wlay));
		SampledSpectrum T; for (int k = 0; k < 4; ++k) T[k] = c.throughput[k];
		float pdf = c.bxdf_pdf;
		glm::vec3 rD{ c.dir[0], c.dir[1], c.dir[2] };
		PathStateBitfield flags = static_cast<PathStateBitfield>(c.flags);
		float refr = c.refraction_scale;
		optixDirectCall<void,
			const MaterialData&, const DirectLightSampleData&, const QRNG::State&,
			const LocalTransform&, const microsurface::Surface&,
			SampledSpectrum&, SampledWavelengths&, SampledSpectrum&,
			float&, glm::vec3&, PathStateBitfield&, float&>
			(mat.bxdfIndexSBT, mat, dl, qs, local, surface, L, wl, T, pdf, rD, flags, refr);
		for (int k = 0; k < 4; ++k) { c.L[k] = L[k]; c.throughput[k] = T[k]; }
		std::memcpy(&wlay, &wl, sizeof(wlay));
		for (int k = 0; k < 4; ++k) { c.lambda[k] = wlay.lambda[k]; c.lambda_pdf[k] = wlay.pdf[k]; }
		c.active_count = wlay.active;
		c.bxdf_pdf = pdf;
		c.dir[0] = rD.x; c.dir[1] = rD.y; c.dir[2] = rD.z;
		c.flags = static_cast<uint32_t>(flags);
		c.refraction_scale = refr;
	}
}

void rbref_light_tree(uint32_t n, rb_light_case* cases)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		rb_light_case& c = cases[i];
		const glm::vec3 p{ c.position[0], c.position[1], c.position[2] };
		const glm::vec3 nn{ c.normal[0], c.normal[1], c.normal[2] };
		LightType type{};
		uint32_t index{};
		float pdf{};
		sampleLightTree(parameters.lightTree, c.rand, p, nn, type, index, pdf);
		c.type = static_cast<uint32_t>(type);
		c.index = index;
		c.pdf = pdf;
		c.q_pdf = traverseLightTree(parameters.lightTree, static_cast<LightType>(c.q_type), c.q_index, p, nn);
	}
}

void rbref_offset_point(uint32_t n, const float* p, const float* nrm, float* out)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		glm::vec3 r = utility::offsetPoint(glm::vec3{ p[i * 3], p[i * 3 + 1], p[i * 3 + 2] },
			glm::vec3{ nrm[i * 3], nrm[i * 3 + 1], nrm[i * 3 + 2] });
		out[i * 3] = r.x; out[i * 3 + 1] = r.y; out[i * 3 + 2] = r.z;
	}
}
void rbref_oct_encode(uint32_t n, const float* v, uint32_t* out)
{
	for (uint32_t i = 0; i < n; ++i)
		out[i] = Octohedral::encodeU32(glm::vec3{ v[i * 3], v[i * 3 + 1], v[i * 3 + 2] });
}
void rbref_oct_decode(uint32_t n, const uint32_t* code, float* out)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		glm::vec3 r = Octohedral::decodeU32(code[i]);
		out[i * 3] = r.x; out[i * 3 + 1] = r.y; out[i * 3 + 2] = r.z;
	}
}

// Closest hit with the reference's closest-hit / miss programs filling the
// 24-word payload (pathtrace.cu:1162-1177).
void rbref_trace(uint32_t n, const float* rays, uint32_t* payload, float* t, int32_t* tri)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		uint32_t* pl = payload + static_cast<size_t>(i) * 24;
		oracle_optix::tls.lastTri = -1;
		oracle_optix::tls.lastT = INFINITY;
		optixTrace(OPTIX_PAYLOAD_TYPE_ID_0, parameters.traversable,
			float3{ rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2] },
			float3{ rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5] },
			0.0f, FLT_MAX, 0.0f, 0xFF, 0, 0, 1, 0,
			pl[0], pl[1], pl[2], pl[3], pl[4], pl[5], pl[6], pl[7], pl[8], pl[9], pl[10], pl[11],
			pl[12], pl[13], pl[14], pl[15], pl[16], pl[17], pl[18], pl[19], pl[20], pl[21], pl[22], pl[23]);
		t[i] = oracle_optix::tls.lastT;
		tri[i] = oracle_optix::tls.lastTri;
	}
}
void rbref_occluded(uint32_t n, const float* rays, const float* tmax, uint32_t* out)
{
	for (uint32_t i = 0; i < n; ++i)
		out[i] = oracle_optix::traceAny(float3{ rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2] },
			float3{ rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5] }, 0.0f, tmax[i]) ? 1u : 0u;
}

// ---- light tree builder (src/core/light_tree.cpp, driven as
// RenderingInterface::buildLightTree does, src/core/rendering_interface.cpp:1065-1167)
// Input per emissive triangle: world-space vertices (9 floats), object
// vertices are not needed; flux already multiplied by transformFluxCorrection;
// material index and primitive index for EmissiveTriangleLightData; uvs.
// Outputs: camera-relative EmissiveTriangleLightData (68 B each), nodes
// (capacity 2*n), pointers (n), bitmasks (n). Returns the node count.
int rbref_build_light_tree(uint32_t n, const float* worldVerts, const float* flux,
	const uint32_t* materialIndex, const uint32_t* primIndex, const double* cameraPos,
	void* outTriangles, void* outNodes, uint32_t* outPointers, uint64_t* outBitmasks)
{
	if (n == 0) return 0;
	SceneData scene{};
	scene.models.emplace_back();
	SceneData::Model& model = scene.models.back();
	model.instancedEmissiveMeshSubsets.emplace_back();
	auto& subset = model.instancedEmissiveMeshSubsets.back();
	subset.transformFluxCorrection = 1.0f;
	std::vector<LightTree::Builder::SortData> sortData(n);
	std::vector<EmissiveTriangleLightData> tris(n);
	const glm::dvec3 cam{ cameraPos[0], cameraPos[1], cameraPos[2] };
	for (uint32_t k = 0; k < n; ++k)
	{
		SceneData::EmissiveMeshSubset::TriangleData td{};
		const float* v = worldVerts + k * 9;
		td.v0WS = glm::vec3{ v[0], v[1], v[2] };
		td.v1WS = glm::vec3{ v[3], v[4], v[5] };
		td.v2WS = glm::vec3{ v[6], v[7], v[8] };
		td.primIndex = primIndex[k];
		td.flux = flux[k];
		subset.triangles.push_back(td);

		EmissiveTriangleLightData& ld = tris[k];
		for (int q = 0; q < 9; ++q) ld.vertices[q] = v[q];
		ld.primitiveDataIndex = primIndex[k];
		ld.materialIndex = materialIndex[k];
		glm::vec3 triCamWVerts[3]{
			{ static_cast<float>(td.v0WS.x - cam.x), static_cast<float>(td.v0WS.y - cam.y), static_cast<float>(td.v0WS.z - cam.z) },
			{ static_cast<float>(td.v1WS.x - cam.x), static_cast<float>(td.v1WS.y - cam.y), static_cast<float>(td.v1WS.z - cam.z) },
			{ static_cast<float>(td.v2WS.x - cam.x), static_cast<float>(td.v2WS.y - cam.y), static_cast<float>(td.v2WS.z - cam.z) } };
		auto& sd = sortData[k];
		sd.lightType = LightType::TRIANGLE;
		sd.lightIndex = k;
		glm::vec3 normal{ glm::normalize(glm::cross(triCamWVerts[1] - triCamWVerts[0], triCamWVerts[2] - triCamWVerts[0])) };
		for (int a = 0; a < 3; ++a)
		{
			sd.bounds.min[a] = std::min(triCamWVerts[0][a], std::min(triCamWVerts[1][a], triCamWVerts[2][a]));
			sd.bounds.max[a] = std::max(triCamWVerts[0][a], std::max(triCamWVerts[1][a], triCamWVerts[2][a]));
			if (sd.bounds.max[a] <= sd.bounds.min[a])
			{
				sd.bounds.min[a] = sd.bounds.max[a] - std::numeric_limits<float>::epsilon();
				sd.bounds.max[a] = sd.bounds.max[a] + std::numeric_limits<float>::epsilon();
			}
		}
		sd.coneDirection[0] = normal.x; sd.coneDirection[1] = normal.y; sd.coneDirection[2] = normal.z;
		sd.cosConeAngle = 1.0f;
		sd.flux = td.flux * subset.transformFluxCorrection;
		sd.lightDataRef.triangleRef.modelIndex = 0;
		sd.lightDataRef.triangleRef.subsetIndex = 0;
		sd.lightDataRef.triangleRef.triangleIndex = k;
	}
	// fillLightDataBuffer: camera-relative vertices (rendering_interface.cpp:1440-1452)
	for (uint32_t k = 0; k < n; ++k)
		for (int q = 0; q < 9; ++q)
			tris[k].vertices[q] -= cam[q % 3];
	LightTree::Builder builder{};
	LightTree::Tree tree = builder.build(scene, sortData.data(), static_cast<int>(n), static_cast<int>(n));
	// fillLightTreeDataBuffers: camera-relative node means (:1478-1484)
	auto* nodes = static_cast<LightTree::PackedNode*>(outNodes);
	for (int i = 0; i < tree.nodeCount; ++i)
	{
		nodes[i] = tree.nodes[i];
		nodes[i].spatialMean[0] -= cam.x;
		nodes[i].spatialMean[1] -= cam.y;
		nodes[i].spatialMean[2] -= cam.z;
	}
	for (uint32_t k = 0; k < n; ++k)
	{
		outPointers[k] = tree.lightPointers[k].lptr;
		outBitmasks[k] = tree.bitmaskSets[KTriangleLightsArrayIndex][k];
	}
	std::memcpy(outTriangles, tris.data(), sizeof(EmissiveTriangleLightData) * n);
	const int count = tree.nodeCount;
	tree.clear();
	return count;
}

// Color::generateColorspaceConversionMatrix (src/core/color.h:60-99): the
// XYZ -> RGB matrix of colorspace `cs` (0 sRGB, 1 DCI-P3, 2 Rec.2020) with the
// D65 white point from the reference's own illuminant spectrum; out is
// column-major (glm::mat3).
void rbref_colorspace_matrix(int cs, float* out)
{
	const glm::mat3 m = Color::generateColorspaceConversionMatrix(static_cast<Color::RGBColorspace>(cs));
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r) out[3 * c + r] = m[c][r];
}

uint32_t rbref_sizeof_material_data() { return sizeof(MaterialData); }
uint32_t rbref_sizeof_launch_parameters() { return sizeof(LaunchParameters); }

} // extern "C"
