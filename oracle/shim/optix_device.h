// Oracle test infrastructure (not product code).
//
// Host-side stand-in for the OptiX device API, written for this project so the
// reference's own OptiX programs (src/kernels/pathtrace.cu) run unchanged on
// the CPU. Semantics follow the OptiX programming model the reference relies
// on:
//   * optixTrace (pathtrace.cu:1162) runs a closest-hit query on a CPU BVH and
//     then calls the reference's __closesthit__triangle (pathtrace.cu:86) or
//     __miss__miss (pathtrace.cu:230); payload registers are written through
//     optixSetPayload_N into the caller's 24 payload words.
//   * optixTraverse + optixHitObjectIsHit (pathtrace.cu:1708-1719) run an
//     any-hit occlusion query (OPTIX_RAY_FLAG_TERMINATE_ON_FIRST_HIT).
//   * optixDirectCall (pathtrace.cu:1724) dispatches on the callable index to
//     the three BxDF callables in the order the reference's SBT uses
//     (src/core/rendering_interface.cpp:1291-1309: 0 conductor, 1 dielectric,
//     2 complex surface).
// All per-launch state is thread-local so a launch can run on many threads.
#pragma once

#include <cstdint>
#include <vector_types.h>
#include "optix_types.h"

namespace oracle_optix
{
	// Result of a closest-hit query, filled by the CPU BVH in ref_harness.cpp.
	struct HitState
	{
		uint32_t primitiveIndex;   // index inside the build input (optixGetPrimitiveIndex)
		float2 barycentrics;       // (b1, b2) of vertices 1 and 2
		uint32_t sbtData;          // hit-group record data: material index or 0xFFFFFFFF
		float3 objectVertices[3];  // optixGetTriangleVertexData
		float objectToWorld[12];   // row-major 3x4
		float worldToObject[12];   // row-major 3x4
	};
	struct ThreadState
	{
		uint3 launchIndex;
		uint32_t* payload[24];
		HitState hit;
		bool shadowHit;
		float lastT;   // distance of the last closest hit (harness diagnostics)
		int lastTri;   // canonical triangle id of the last closest hit, -1 on a miss
	};
	extern thread_local ThreadState tls;

	// Implemented by the harness: closest hit and any hit over the CPU BVH.
	bool traceClosest(float3 o, float3 d, float tmin, float tmax, HitState& out);
	bool traceAny(float3 o, float3 d, float tmin, float tmax);

	// Callable table: filled by the harness after the reference programs are defined.
	extern void* callables[3];
}

inline void optixSetPayloadTypes(unsigned int) {}
inline uint3 optixGetLaunchIndex() { return oracle_optix::tls.launchIndex; }
inline void* optixGetSbtDataPointer() { return &oracle_optix::tls.hit.sbtData; }
inline unsigned int optixGetPrimitiveIndex() { return oracle_optix::tls.hit.primitiveIndex; }
inline float2 optixGetTriangleBarycentrics() { return oracle_optix::tls.hit.barycentrics; }
inline OptixTraversableHandle optixGetGASTraversableHandle() { return 0; }
inline unsigned int optixGetSbtGASIndex() { return 0; }
inline void optixGetTriangleVertexData(OptixTraversableHandle, unsigned int, unsigned int, float, float3 data[3])
{
	data[0] = oracle_optix::tls.hit.objectVertices[0];
	data[1] = oracle_optix::tls.hit.objectVertices[1];
	data[2] = oracle_optix::tls.hit.objectVertices[2];
}
inline void optixGetObjectToWorldTransformMatrix(float m[12])
{
	for (int i = 0; i < 12; ++i) m[i] = oracle_optix::tls.hit.objectToWorld[i];
}
inline void optixGetWorldToObjectTransformMatrix(float m[12])
{
	for (int i = 0; i < 12; ++i) m[i] = oracle_optix::tls.hit.worldToObject[i];
}

#define ORACLE_PAYLOAD_SETTER(N) \
	inline void optixSetPayload_##N(unsigned int v) { *oracle_optix::tls.payload[N] = v; }
ORACLE_PAYLOAD_SETTER(0)  ORACLE_PAYLOAD_SETTER(1)  ORACLE_PAYLOAD_SETTER(2)  ORACLE_PAYLOAD_SETTER(3)
ORACLE_PAYLOAD_SETTER(4)  ORACLE_PAYLOAD_SETTER(5)  ORACLE_PAYLOAD_SETTER(6)  ORACLE_PAYLOAD_SETTER(7)
ORACLE_PAYLOAD_SETTER(8)  ORACLE_PAYLOAD_SETTER(9)  ORACLE_PAYLOAD_SETTER(10) ORACLE_PAYLOAD_SETTER(11)
ORACLE_PAYLOAD_SETTER(12) ORACLE_PAYLOAD_SETTER(13) ORACLE_PAYLOAD_SETTER(14) ORACLE_PAYLOAD_SETTER(15)
ORACLE_PAYLOAD_SETTER(16) ORACLE_PAYLOAD_SETTER(17) ORACLE_PAYLOAD_SETTER(18) ORACLE_PAYLOAD_SETTER(19)
ORACLE_PAYLOAD_SETTER(20) ORACLE_PAYLOAD_SETTER(21) ORACLE_PAYLOAD_SETTER(22) ORACLE_PAYLOAD_SETTER(23)
#undef ORACLE_PAYLOAD_SETTER

// The two programs a trace can end in; defined by the reference source that
// includes this header.
extern "C" void __closesthit__triangle();
extern "C" void __miss__miss();

template<typename... Payload>
inline void optixTrace(OptixPayloadTypeID, OptixTraversableHandle, float3 origin, float3 direction,
	float tmin, float tmax, float /*time*/, OptixVisibilityMask, unsigned int /*flags*/,
	unsigned int /*sbtOffset*/, unsigned int /*sbtStride*/, unsigned int /*missIndex*/, Payload&... p)
{
	static_assert(sizeof...(Payload) == 24, "the reference traces with 24 payload words");
	uint32_t* ptrs[24] = { &p... };
	for (int i = 0; i < 24; ++i)
	{
		oracle_optix::tls.payload[i] = ptrs[i];
		*ptrs[i] = 0u; // deterministic contents for words a program does not write
	}
	if (oracle_optix::traceClosest(origin, direction, tmin, tmax, oracle_optix::tls.hit))
		__closesthit__triangle();
	else
		__miss__miss();
}

inline void optixTraverse(OptixTraversableHandle, float3 origin, float3 direction, float tmin, float tmax,
	float /*time*/, OptixVisibilityMask, unsigned int /*flags*/, unsigned int, unsigned int, unsigned int)
{
	oracle_optix::tls.shadowHit = oracle_optix::traceAny(origin, direction, tmin, tmax);
}
inline bool optixHitObjectIsHit() { return oracle_optix::tls.shadowHit; }

template<typename ReturnT, typename... ArgTypes>
inline ReturnT optixDirectCall(unsigned int sbtIndex, ArgTypes... args)
{
	using Fn = ReturnT (*)(ArgTypes...);
	return reinterpret_cast<Fn>(oracle_optix::callables[sbtIndex])(args...);
}
