// Device refit of the flattened geometry (rb_refit.cu).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "rb_scene.h"

namespace rb
{
struct RefitData
{
	const float4* objVerts = nullptr;      // device: 3 object-space vertices per triangle, BVH order
	const uint32_t* order = nullptr;       // device: node indices, deepest level first
	std::vector<uint32_t> levelStart;      // host: level k is order[levelStart[k] .. levelStart[k+1])
	double* nodeBox = nullptr;             // device scratch: exact box (lo xyz, hi xyz) per node
};

// xf, wi: device, 12 floats per flattened instance (emissive subsets, then
// instances): the new object-to-world 3x4 transform and its inverse.
void launchRefit(const RefitData& r, DevGeometry& g, const float* xf, const float* wi, uint32_t* status,
	int smCount, cudaStream_t st);

// Two-level structure: the world box of each of n instances, over its unit's
// triangles (range: 2 per instance, first triangle and count in objVerts;
// count 0 for an instance without triangles) through its 3x4 transform xf,
// with the flat upload's vertex arithmetic. boxes: 6 floats per instance
// (lo xyz, hi xyz). One block per instance.
void launchInstanceBoxes(const float4* objVerts, const uint32_t* range, const float* xf, float* boxes, uint32_t n,
	cudaStream_t st);
} // namespace rb
