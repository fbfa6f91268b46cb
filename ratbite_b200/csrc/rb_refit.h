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
} // namespace rb
