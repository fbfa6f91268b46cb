// Oracle test infrastructure (not product code): host-side stand-in for the
// OptiX SDK's optix_types.h, written for this project. It declares only the
// names the reference's device code (src/kernels/pathtrace.cu,
// src/core/launch_parameters.h, src/core/scene.h) uses, so that code can be
// compiled by g++ as a CPU path tracer.
#pragma once
#include <cstdint>
#include <cuda.h>

typedef unsigned long long OptixTraversableHandle;
typedef unsigned int OptixVisibilityMask;

enum OptixPayloadTypeID
{
	OPTIX_PAYLOAD_TYPE_DEFAULT = 0,
	OPTIX_PAYLOAD_TYPE_ID_0 = (1 << 0u),
};

enum OptixRayFlags
{
	OPTIX_RAY_FLAG_NONE = 0u,
	OPTIX_RAY_FLAG_TERMINATE_ON_FIRST_HIT = 1u << 2,
};

enum OptixResult
{
	OPTIX_SUCCESS = 0,
};

struct OptixAabb
{
	float minX, minY, minZ;
	float maxX, maxY, maxZ;
};
