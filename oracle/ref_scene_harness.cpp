// Oracle test infrastructure (not product code).
//
// The reference's own glTF loader (SceneData::loadModel and loadGLTF,
// src/core/scene.cpp:92-656, on the vendored cgltf) compiled host-side, with
// plain C getters over the SceneData it fills, so the project's loader
// (ratbite_b200/gltf.py) can be compared with it on the same files, and the
// reference's tangent-frame packing (src/core/rendering_interface.cpp:258-284)
// for the FRAME vertex attribute.

#define STB_IMAGE_IMPLEMENTATION
#include <stb/stb_image.h>
#undef STB_IMAGE_IMPLEMENTATION

#include "_ref/src/core/scene.h"

#include <cstring>
#include <glm/gtc/quaternion.hpp>

namespace
{
SceneData* g_scene = nullptr;

const SceneData::Model* model()
{
	return g_scene && !g_scene->models.empty() ? &g_scene->models.back() : nullptr;
}
}

extern "C" {

struct rbref_submesh_info
{
	int32_t material;
	int32_t index_type;           // 0 u16, 1 u32
	uint32_t primitive_count;
	uint32_t vertex_count;
	const void* indices;
	const float* vertices;        // vec4 per vertex
	const float* normals;         // vec4 per vertex or null
	const float* tangents;        // vec4 per vertex or null
	const float* texcoords0;      // vec2 per vertex or null
	uint32_t discarded_count;
	const uint32_t* discarded;
	const float* texcoords1;      // vec2 per vertex or null
};

struct rbref_material_info
{
	int32_t bxdf, double_sided, sheen_present;
	float ior;
	int32_t bc_factor_present;
	float base_color[4];
	int32_t alpha_mode;           // AlphaInterpretation: 0 none, 1 cutoff, 2 blend
	float alpha_cutoff;
	int32_t met_factor_present;
	float metalness;
	int32_t rough_factor_present;
	float roughness;
	int32_t transmit_factor_present;
	float transmission;
	int32_t sheen_color_present;
	float sheen_color[3];
	int32_t sheen_rough_present;
	float sheen_roughness;
	int32_t emissive_present;
	float emissive[3];
	int32_t textures;             // bit per texture slot that is set
	int32_t tex_index[7];         // bc, mr, nm, tr, shc, shr, em (-1: none)
	int32_t tex_coord[7];         // the slots' texture-coordinate sets
};

// Loads `path` into a fresh SceneData with the identity model transform.
int rbref_scene_load(const char* path)
{
	delete g_scene;
	g_scene = new SceneData();
	g_scene->loadModel(path);
	return model() ? 0 : -1;
}

// [meshes, instances, materials, emissive subsets, triangle count]
void rbref_scene_counts(int64_t* out)
{
	const SceneData::Model* m = model();
	out[0] = m ? m->meshes.size() : 0;
	out[1] = m ? m->instances.size() : 0;
	out[2] = m ? m->materialDescriptors.size() : 0;
	out[3] = m ? m->instancedEmissiveMeshSubsets.size() : 0;
	out[4] = m ? m->triangleCount : 0;
}

int rbref_scene_submesh_count(int mesh)
{
	const SceneData::Model* m = model();
	return m && mesh >= 0 && mesh < static_cast<int>(m->meshes.size()) ? m->meshes[mesh].submeshes.size() : -1;
}

int rbref_scene_submesh(int mesh, int sub, rbref_submesh_info* out)
{
	if (rbref_scene_submesh_count(mesh) <= sub || sub < 0) return -1;
	const SceneData::Submesh& s = model()->meshes[mesh].submeshes[sub];
	std::memset(out, 0, sizeof(*out));
	out->material = s.materialIndex;
	out->index_type = s.indexType == IndexType::UINT_16 ? 0 : 1;
	out->primitive_count = s.primitiveCount;
	out->vertex_count = s.vertexCount;
	out->indices = s.indices;
	out->vertices = s.vertices.empty() ? nullptr : &s.vertices[0].x;
	out->normals = s.normals.empty() ? nullptr : &s.normals[0].x;
	out->tangents = s.tangents.empty() ? nullptr : &s.tangents[0].x;
	out->texcoords0 = s.texCoordsSets.empty() || s.texCoordsSets[0].empty() ? nullptr : &s.texCoordsSets[0][0].x;
	out->discarded_count = s.discardedPrimitives.size();
	out->discarded = s.discardedPrimitives.empty() ? nullptr : s.discardedPrimitives.data();
	out->texcoords1 = s.texCoordsSets.size() < 2 || s.texCoordsSets[1].empty() ? nullptr : &s.texCoordsSets[1][0].x;
	return 0;
}

int rbref_scene_material(int i, rbref_material_info* out)
{
	const SceneData::Model* m = model();
	if (!m || i < 0 || i >= static_cast<int>(m->materialDescriptors.size())) return -1;
	const SceneData::MaterialDescriptor& d = m->materialDescriptors[i];
	std::memset(out, 0, sizeof(*out));
	out->bxdf = static_cast<int32_t>(d.bxdf);
	out->double_sided = d.doubleSided;
	out->sheen_present = d.sheenPresent;
	out->ior = d.ior;
	out->bc_factor_present = d.bcFactorPresent;
	for (int k = 0; k < 4; ++k) out->base_color[k] = d.baseColorFactor[k];
	out->alpha_mode = static_cast<int32_t>(d.alphaInterpretation);
	out->alpha_cutoff = d.alphaCutoff;
	out->met_factor_present = d.metFactorPresent;
	out->metalness = d.metalnessFactor;
	out->rough_factor_present = d.roughFactorPresent;
	out->roughness = d.roughnessFactor;
	out->transmit_factor_present = d.transmitFactorPresent;
	out->transmission = d.transmitFactor;
	out->sheen_color_present = d.sheenColorFactorPresent;
	for (int k = 0; k < 3; ++k) out->sheen_color[k] = d.sheenColorFactor[k];
	out->sheen_rough_present = d.sheenRoughnessFactorPresent;
	out->sheen_roughness = d.sheenRoughnessFactor;
	out->emissive_present = d.emissiveFactorPresent;
	for (int k = 0; k < 3; ++k) out->emissive[k] = d.emissiveFactor[k];
	const int tex[7] = { d.baseColorTextureIndex, d.metalRoughnessTextureIndex, d.normalTextureIndex,
		d.transmissionTextureIndex, d.sheenColorTextureIndex, d.sheenRoughTextureIndex, d.emissiveTextureIndex };
	const int crd[7] = { d.bcTexCoordIndex, d.mrTexCoordIndex, d.nmTexCoordIndex, d.trTexCoordIndex,
		d.shcTexCoordIndex, d.shrTexCoordIndex, d.emTexCoordIndex };
	for (int k = 0; k < 7; ++k)
	{
		if (tex[k] >= 0) out->textures |= 1 << k;
		out->tex_index[k] = tex[k];
		out->tex_coord[k] = crd[k];
	}
	return 0;
}

// mesh index and the 4x3 transform (glm::mat4x3: 4 columns of 3 floats)
int rbref_scene_instance(int i, int32_t* mesh, float* transform12)
{
	const SceneData::Model* m = model();
	if (!m || i < 0 || i >= static_cast<int>(m->instances.size())) return -1;
	*mesh = m->instances[i].meshIndex;
	for (int c = 0; c < 4; ++c)
		for (int r = 0; r < 3; ++r) transform12[3 * c + r] = m->instances[i].transform[c][r];
	return 0;
}

// instance, submesh, flux correction and triangle count of emissive subset i
int rbref_scene_emissive(int i, int32_t* instance, int32_t* submesh, float* fluxCorrection, int32_t* triangles)
{
	const SceneData::Model* m = model();
	if (!m || i < 0 || i >= static_cast<int>(m->instancedEmissiveMeshSubsets.size())) return -1;
	const SceneData::EmissiveMeshSubset& e = m->instancedEmissiveMeshSubsets[i];
	*instance = e.instanceIndex;
	*submesh = e.submeshIndex;
	*fluxCorrection = e.transformFluxCorrection;
	*triangles = static_cast<int32_t>(e.triangles.size());
	return 0;
}

// 20 floats: v0WS v1WS v2WS (9), v0 v1 v2 (9), primIndex (as float bits), flux
int rbref_scene_emissive_triangle(int i, int k, float* out)
{
	const SceneData::Model* m = model();
	if (!m || i < 0 || i >= static_cast<int>(m->instancedEmissiveMeshSubsets.size())) return -1;
	const auto& tris = m->instancedEmissiveMeshSubsets[i].triangles;
	if (k < 0 || k >= static_cast<int>(tris.size())) return -1;
	const auto& t = tris[k];
	const glm::vec3 v[6] = { t.v0WS, t.v1WS, t.v2WS, t.v0, t.v1, t.v2 };
	for (int j = 0; j < 6; ++j) { out[3 * j] = v[j].x; out[3 * j + 1] = v[j].y; out[3 * j + 2] = v[j].z; }
	const uint32_t prim = t.primIndex;
	std::memcpy(out + 18, &prim, 4);
	out[19] = t.flux;
	return 0;
}

// [images, textures]
void rbref_scene_texture_counts(int64_t* out)
{
	const SceneData::Model* m = model();
	out[0] = m ? m->imageData.size() : 0;
	out[1] = m ? m->textureData.size() : 0;
}

// width, height, channels and the 8-bit texels of image i
int rbref_scene_image(int i, int32_t* dims3, const uint8_t** data)
{
	const SceneData::Model* m = model();
	if (!m || i < 0 || i >= static_cast<int>(m->imageData.size())) return -1;
	const auto& im = m->imageData[i];
	dims3[0] = im.width;
	dims3[1] = im.height;
	dims3[2] = im.channelCount;
	*data = static_cast<const uint8_t*>(im.data);
	return 0;
}

// image index, sRGB, filter, address x, address y of texture i
int rbref_scene_texture(int i, int32_t* out5)
{
	const SceneData::Model* m = model();
	if (!m || i < 0 || i >= static_cast<int>(m->textureData.size())) return -1;
	const auto& t = m->textureData[i];
	out5[0] = t.imageIndex;
	out5[1] = t.sRGB;
	out5[2] = static_cast<int32_t>(t.filter);
	out5[3] = static_cast<int32_t>(t.addressX);
	out5[4] = static_cast<int32_t>(t.addressY);
	return 0;
}

// uv0, uv1, uv2 of triangle k of emissive subset i
int rbref_scene_emissive_uvs(int i, int k, float* out6)
{
	const SceneData::Model* m = model();
	if (!m || i < 0 || i >= static_cast<int>(m->instancedEmissiveMeshSubsets.size())) return -1;
	const auto& tris = m->instancedEmissiveMeshSubsets[i].triangles;
	if (k < 0 || k >= static_cast<int>(tris.size())) return -1;
	const glm::vec2 uv[3] = { tris[k].uv0, tris[k].uv1, tris[k].uv2 };
	for (int j = 0; j < 3; ++j) { out6[2 * j] = uv[j].x; out6[2 * j + 1] = uv[j].y; }
	return 0;
}

// The FRAME attribute of n vertices (normals and tangents as vec4): the
// quaternion (x, y, z, w) of the frame (tangent, normal x tangent, normal),
// w signed by the tangent's handedness, as the reference packs it
// (src/core/rendering_interface.cpp:258-284, glm::quat_cast).
void rbref_pack_frames(int n, const float* normals4, const float* tangents4, float* out4)
{
	for (int i = 0; i < n; ++i)
	{
		const glm::vec4 nv{ normals4[4 * i], normals4[4 * i + 1], normals4[4 * i + 2], normals4[4 * i + 3] };
		const glm::vec4 tv{ tangents4[4 * i], tangents4[4 * i + 1], tangents4[4 * i + 2], tangents4[4 * i + 3] };
		glm::quat q{ glm::quat_cast(glm::mat3{ tv, glm::cross(glm::vec3{ nv }, glm::vec3{ tv }), nv }) };
		if (q.w == 0.0f)
			q.w = tv.w > 0.0f ? 0.0f : -0.0f;
		else if (q.w * tv.w < 0.0f)
			q = -q;
		out4[4 * i] = q.x; out4[4 * i + 1] = q.y; out4[4 * i + 2] = q.z; out4[4 * i + 3] = q.w;
	}
}

} // extern "C"
