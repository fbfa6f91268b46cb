// Device-resident scene layout shared by the host context (rb_context.cpp)
// and the kernels. All pointers are device pointers owned by the context.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ratbite_b200.h"

namespace rb
{
constexpr int kSpectrumBins = 471;   // 360..830 nm (src/core/spectral_settings.h:5-9)
constexpr int kLambdaMin = 360;
constexpr int kLutN = 32;
constexpr float kEnvMapImportance = 0.3f;   // src/core/light_tree_types.h:55
constexpr uint32_t kLightTypeTriangle = 0, kLightTypeSky = 1, kLightTypeNone = 2;

// PathStateBitfield (src/kernels/pathtrace.cu:25-37).
enum PathFlag : uint32_t
{
	PF_PREVIOUS_HIT_SPECULAR = 1u << 0,
	PF_CURRENT_HIT_SPECULAR = 1u << 1,
	PF_REGULARIZED = 1u << 2,
	PF_RAY_REFRACTED = 1u << 3,
	PF_PATH_TERMINATED = 1u << 4,
	PF_TRIANGULAR_GEOMETRY = 1u << 5,
	PF_RIGHT_HANDED_FRAME = 1u << 6,
	PF_REFRACTION_HAPPENED = 1u << 7,
	PF_FINISHED = 1u << 8,
};

// Material record as the shading kernels read it: the MaterialData fields
// (src/core/material.h:62-107) the device path uses, 16-byte aligned.
struct alignas(16) DevMaterial
{
	uint32_t bxdf;
	uint32_t sheenPresent;
	uint32_t indexType;          // 0 u16, 1 u32
	uint32_t attributes;
	uint32_t attributeStride;
	uint32_t normalOffset;
	uint32_t frameOffset;
	uint32_t factors;
	uint32_t iorSpectrum;
	uint32_t absorpSpectrum;
	float mfRoughness;
	float ior;
	float alphaCutoff;
	float metalness;
	float roughness;
	float transmission;
	float baseColor[4];
	float sheenColor[3];
	float sheenRoughness;
	float emissive[3];
	uint32_t triangleCount;
	const uint8_t* indices;
	const uint8_t* attributeData;
	uint32_t vertexCount;
	uint32_t textures;           // RB_TEXTURE_* bits (TextureTypeBitfield)
	uint32_t texSets;            // bit t: texture slot t reads texture coordinate set 2
	uint32_t texcoordOffset[2];  // byte offsets of TEXCOORD_1 / TEXCOORD_2 in a vertex
	uint16_t tex[8];             // texture table index per slot
};

// One texture of the material texture table (rb_set_textures).
struct DevTexture
{
	const uint8_t* data;         // width x height texels, 1 or 4 bytes each
	uint32_t width, height;
	uint32_t channels;           // 1 (R8) or 4 (RGBA8)
	uint32_t srgb;
	uint32_t addrU, addrV;       // RB_TEXADDR_*
	uint32_t filter;             // RB_TEXFILTER_*
	uint32_t pad;
};

// Reference light-tree records, byte compatible with
// src/core/light_tree_types.h:40-46 and :119-163.
struct EmissiveTri
{
	float v[9];
	float uv[6];
	uint32_t material;
	uint32_t prim;
};
static_assert(sizeof(EmissiveTri) == 68, "EmissiveTriangleLightData is 68 B");
struct alignas(16) PackedNode
{
	float mean[3];
	float variance;
	uint32_t direction;
	float sharpness;
	float flux;
	uint32_t core;
};
static_assert(sizeof(PackedNode) == 32, "PackedNode is 32 B");

// Wide BVH node: 8 children with boxes quantized to 8 bits per plane against
// the node's origin and power-of-two per-axis scale (conservative rounding:
// lo down, hi up). 96 bytes = six 16-byte loads.
struct alignas(16) BvhNode
{
	float origin[3];
	uint8_t exponent[3];         // scale = 2^(exponent - 127)
	uint8_t childCount;
	uint32_t child[8];           // interior: node index; leaf: kLeafBit | (count-1) << 24 | first triangle; empty: kEmpty
	uint8_t qlo[3][8];           // [axis][child]
	uint8_t qhi[3][8];
};
static_assert(sizeof(BvhNode) == 96, "BVH node is 96 B");
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kEmptyChild = 0xFFFFFFFFu;
constexpr int kLeafMaxTris = 4;
// Limits of the traversal's node-group stack entries (24-bit node index) and
// depth (one entry per level); rb_set_geometry rejects trees beyond them.
constexpr uint32_t kMaxBvhNodes = 1u << 24;
constexpr int kMaxBvhDepth = 48;
// Entries of a ray's traversal stack (one per entered child still owed).
constexpr int kTraversalStackEntries = 64;

// An instance of the two-level structure (RB_ACCEL_INSTANCED), in the
// top-level BVH's leaf order: object-to-world and world-to-object 3x4
// transforms, the reference of its unit's BVH root (node index, or a leaf
// reference for units of <= kLeafMaxTris triangles), the canonical id of its
// first triangle, and its index in the flat numbering (emissive subsets,
// then instances), which the normal matrices and hit records use.
struct alignas(16) DevInstance
{
	float xf[12];
	float wi[12];
	uint32_t root;
	uint32_t canonBase;
	uint32_t index;
	uint32_t pad;
};

// Per-triangle hit data in BVH leaf order. Flat: v[0..2] are the world-space
// vertices; their w lanes carry the canonical triangle id (v0.w), the
// instance index (v1.w) and the hit-group data (v2.w: material index, or
// 0xFFFFFFFF for emissive triangles) as raw bits. Instanced: the triangles
// of every unit (mesh or emissive subset) in object space, v0.w the
// canonical id within the unit, v1.w unused, v2.w as flat; triAux.x unused
// (the encoded normal depends on the instance).
struct DevGeometry
{
	const BvhNode* nodes;        // instanced: the units' BVHs, then the top level
	const float4* triVerts;      // 3 per triangle
	const uint2* triAux;         // (encoded geometric normal, primitive index)
	const float* normalMatrix;   // 9 per instance: payload words 9..17 (src/kernels/pathtrace.cu:134-142)
	const DevInstance* instances;  // instanced: top-level leaf order
	uint32_t nodeCount;
	uint32_t triCount;
	uint32_t rootIsLeaf;         // scenes of <= kLeafMaxTris triangles
	uint32_t stackLimit;         // traversal stack entries in use (kTraversalStackEntries unless injected)
	uint32_t instanced;          // 1: two-level structure
	uint32_t topRoot;            // instanced: reference of the top-level root
	uint32_t instanceCount;      // instanced: entries of `instances`
	uint32_t pad;
};

// A light-tree node unpacked for the descent (48 B): mean and variance,
// decoded average direction and sharpness, then flux, the SG integral of the
// sharpness, and the child / leaf words (a; b with the leaf bit in bit 31).
struct alignas(16) TreeNodeU
{
	float4 meanVar;
	float4 dirSharp;
	float4 fluxInt;
};

struct DevLights
{
	const PackedNode* nodes;     // nullptr when there is no light tree
	const TreeNodeU* unpacked;   // nodes unpacked on the device (same indexing)
	const uint32_t* pointers;
	const EmissiveTri* triangles;
	const uint64_t* bitmasks;
	uint32_t nodeCount;
	uint32_t triangleCount;
};

struct DevEnvMap
{
	uint32_t enabled;
	uint32_t w, h;
	float width, height;         // as floats, as LaunchParameters stores them
	const float* integral;       // device scalar: integral divided by w*h (rebuilt on the device)
	const float4* texels;
	const uint16_t* conditional;
	const uint16_t* marginal;
};

struct DevLuts
{
	const float* conductor;      // 32x32
	const float* dielOuter;      // 32^3, x fastest
	const float* dielInner;
	const float* reflOuter;
	const float* reflInner;
	const float4* sheen;         // 32x32
};

struct DevSpectra
{
	const float* sensor;         // 3 x 471: X, Y, Z
	const float* basis;          // 3 x 471: R, G, B
	const float* extra;          // n x 471
	uint32_t extraCount;
};

struct DevLaunch
{
	uint32_t width, height;
	float invWidth, invHeight;
	float perspW, perspH;
	uint32_t maxDepth, maxReflected, maxTransmitted;
	float camU[3], camV[3], camW[3];
	uint32_t dof;
	float aperture, focusDistance;
};

// Everything a kernel reads about the scene, passed by value as a kernel
// parameter (fits the 32 KB parameter space of sm_100).
struct DevScene
{
	DevGeometry geo;
	DevLights lights;
	DevEnvMap env;
	DevLuts luts;
	DevSpectra spectra;
	DevLaunch launch;
	const DevMaterial* materials;
	uint32_t materialCount;
	uint32_t textureCount;
	const DevTexture* textures;
	const float* srgbLut;        // 256 entries: the sRGB decode of each 8-bit code
	uint32_t* status;            // device status word (RB_DEV_* bits), [0] flags, [1] detail
};
} // namespace rb
