// Wavefront path state and the host-side launchers of the rendering kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rb_scene.h"

namespace rb
{
// Structure-of-arrays state of the paths of one wave, one slot per path.
// A wave holds `samplesPerWave` whole sample planes of the image, so slot p
// renders pixel p % (W*H), sample sampleBase + p / (W*H). Every array is
// 16-byte aligned and read/written with vector accesses.
struct PathSoA
{
	float4* rayO;      // origin, w: refraction scale
	float4* rayD;      // direction, w: BxDF pdf of the last bounce
	float4* lambda;    // hero wavelengths
	float4* lpdf;      // wavelength pdfs
	float4* nrm;       // last shading normal, w: active wavelength count
	float4* L;         // radiance
	float4* T;         // throughput
	uint2* fd;         // flags, depth
	float4* hit;       // closest hit: triangle (bits, -1 miss), t, b1, b2
	// Surface records of the current bounce, and their light samples, are
	// indexed by record, not by path slot: kSurface takes a record in one of
	// two regions by the record's light choice (tree picks from 0 up, the
	// rest from queueCap - 1 down; see kRegionCounts), a warp's records of
	// one region adjacent, so the shading kernels move them in whole sectors
	// and each light-sample launch reads one region densely.
	// surfQueue[record] is the path slot.
	float4* shO;       // shadow ray origin, w: tmax
	float4* shD;       // shadow ray direction
	float4* shC;       // light sample spectrum, then the pending light-sample contribution
	float4* sfP;       // hit position, w: material index (bits)
	float4* sfPi;      // shadow-terminator-offset position, w: surface bits (kSf*)
	float4* sfGn;      // geometric normal
	float4* sfT;       // shading frame tangent
	float4* sfB;       // shading frame bitangent
	float4* sfN;       // shading normal (the path keeps its own copy in nrm for the next bounce)
	float4* sfL;       // the path's hero wavelengths (a copy of lambda)
	float4* sfUV;      // texture coordinates (sets 1 and 2), written for textured materials
	uint32_t* queue[2];// active path slots, ping-pong by bounce parity
	uint32_t* surfQueue;   // per record: its path slot
	uint32_t* recOrder;    // records in order of arrival (both regions): the BxDF kernels take them in
	                       // this order, which follows the paths' queue order, so the path state they
	                       // read and write by slot, and the next queue they fill, keep that order
	// emitter hits whose MIS weight needs the light-tree pdf (kEmission),
	// indexed by queue position: path, (previous origin, BxDF pdf),
	// (previous normal, area pdf), emitted spectrum, light index
	uint32_t* emQueue;
	float4* emA;
	float4* emB;
	float4* emC;
	uint32_t* emLight;
	uint32_t* shadowQueue;  // records whose shadow ray is traced
	uint32_t* counts;  // kCountSlots words: see kShadowCounts, kRegionCounts
	uint32_t capacity;
	// jobs of a shared wavefront (rb_render_jobs; null for a single render):
	// the job table, and per path its job and key (x | y << 16, sample index)
	const struct DevJob* jobs;
	uint32_t* job;
	uint2* key;
	// entries a queue accepts per bounce (capacity, or the injected limit of
	// rb_config.inject_queue_limit); an append beyond it is dropped with
	// RB_DEV_QUEUE_OVERFLOW, and readers take at most this many
	uint32_t queueCap;
	// radiance-cache form (all null without a cache): per path, the spread
	// (primary footprint a0, summed spread) and, for training paths, the
	// record of the current vertex (kNoRecord: none this vertex; kNotTraining
	// for the other paths); cache queries (path, kNrcInputs floats); training
	// records (path, inputs, radiance at the vertex then the target,
	// throughput at the vertex)
	float2* spread;
	uint32_t* trainRec;
	uint32_t* cPath;
	float* cIn;
	uint32_t* tPath;
	float* tIn;
	float4* tL;
	float4* tT;
	uint32_t trainCapacity;
};
constexpr uint32_t kNotTraining = 0xFFFFFFFFu;
constexpr uint32_t kNoRecord = 0xFFFFFFFEu;
// Cached form, renderer-private path flags (fd.x bits above the
// reference's PF_ set): the camera ray hit an emitter, so the path's
// prefix holds that emitter's radiance ("lit prefix"); a training path
// has passed the vertex where the cache would have ended it.
constexpr uint32_t kPathLitPrefix = 1u << 16;
constexpr uint32_t kPathQueryPassed = 1u << 17;
// High bits of a query's path index (cPath): bit 31, a lit-prefix path's
// query. Of a record's (tPath): bit 31, a training record at the vertex
// where a lit-prefix path would have queried the cache; bit 30, the same
// for any other path. Path indices stay below 2^30.
constexpr uint32_t kLitPrefixBit = 1u << 31;
constexpr uint32_t kQueryRecordBit = 1u << 30;
constexpr uint32_t kRecordPathMask = kQueryRecordBit - 1u;
constexpr int kMaxBounces = 64;
// counts[b]: paths entering bounce b; counts[kShadowCounts + b]: shadow rays
// of bounce b; counts[kExtendFetch + b], counts[kShadowFetch + b]: work
// counters from which the persistent traversal warps take their next rays;
// counts[kEmissionCounts + b]: deferred emission-MIS records of bounce b;
// counts[kRegionCounts + 2 b], counts[kRegionCounts + 2 b + 1]: surface
// records of bounce b in the tree-pick region (records 0 ..) and in the
// other region (environment picks and skipped surfaces, records queueCap - 1
// down), one 64-bit word per bounce that kSurface adds to with one atomic
// per warp; counts[kCacheQueryCount], counts[kTrainRecordCount]:
// radiance-cache queries and training records of the wave (all bounces).
constexpr uint32_t kShadowCounts = kMaxBounces + 1;
constexpr uint32_t kExtendFetch = 3 * (kMaxBounces + 1);
constexpr uint32_t kShadowFetch = 4 * (kMaxBounces + 1);
constexpr uint32_t kEmissionCounts = 5 * (kMaxBounces + 1);
constexpr uint32_t kRegionCounts = 6 * (kMaxBounces + 1);
static_assert(kRegionCounts % 2 == 0, "64-bit region counters are 8-byte aligned");
constexpr uint32_t kCacheQueryCount = 8 * (kMaxBounces + 1);
constexpr uint32_t kTrainRecordCount = kCacheQueryCount + 1;
constexpr uint32_t kCountSlots = kCacheQueryCount + 2;

// One render job of a shared wavefront (rb_render_jobs): its scene, its
// accumulation buffer and whether its failed samples keep their radiance.
struct DevJob
{
	DevScene scene;
	double4* accum;
	uint32_t keepFailed;
	uint32_t pad[3];
};
// A run of sample planes of one job inside a wave: path slots [slot, slot +
// planes x pixels) (plane-major, slotPixel order within a plane), pixel
// slots [pixel, pixel + pixels) of the wave's resolve, sample indices
// [sample, sample + planes); fresh: the job's accumulation restarts here.
struct WaveChunk
{
	uint32_t job, slot, pixel, planes, sample, fresh, pixels, width, height, pad[3];
};

struct WaveParams
{
	uint32_t paths;        // slots in this wave
	uint32_t pixels;       // W*H
	uint32_t sampleBase;   // absolute sample index of plane 0 of the wave
	uint32_t fresh;        // 1: accumulation starts from zero (first wave of a launch at offset 0)
	uint32_t keepFailed;   // 1: a path with the terminated flag keeps its radiance (RB_FAILED_KEEP)
	// replayed waves (rb_render_graph): dyn[0] is the call's first sample
	// index, added to sampleBase, and dyn[1] is 1 when the call starts at
	// sample 0 (fresh then also needs it); null for directly launched waves
	const uint32_t* dyn;
	// radiance-cache form
	uint32_t cached;       // 1: paths terminate into the cache (PathSoA cache arrays are set)
	uint32_t trainOneIn;   // one path in trainOneIn is a training path (0: none)
	uint32_t trainSeed;    // varies the training paths from wave to wave
	float spreadC;         // terminate once (summed spread)^2 > spreadC * a0
	float minRoughness;    // ... at a surface that is not metallic or transmissive, or at least this rough
	float posMin[3], posScale[3];  // hit position -> [0,1]^3
	// shared wavefront (PathSoA::jobs set): the wave's chunks, sorted by slot
	// and by pixel slot, and the number of pixel slots the resolve covers
	const WaveChunk* chunks;
	uint32_t nChunks;
	uint32_t pixelSlots;
	// 1: some material of the wave's scene(s) samples textures; the shading
	// kernels then run their variants with the texture reads compiled in
	uint32_t textured;
};

struct LaunchShape
{
	int smCount;
	int blocksGenerate, blocksExtend, blocksSurface, blocksEmission, blocksNee, blocksBsdf, blocksBsdfLight, blocksShadow,
		blocksResolve;
	int threads;
	uint32_t items;   // paths of the wave (0: no limit): grids are capped at the blocks those need
};

// First sample index and fresh flag of a wave, reading dyn when set.
#ifdef __CUDACC__
__device__ __forceinline__ uint32_t waveSampleBase(const WaveParams& w)
{
	return w.dyn ? __ldg(w.dyn) + w.sampleBase : w.sampleBase;
}
__device__ __forceinline__ bool waveFresh(const WaveParams& w)
{
	return w.fresh && (!w.dyn || __ldg(w.dyn + 1) != 0u);
}
#endif

LaunchShape queryLaunchShape();
// dyn[0] = offset, dyn[1] = fresh, stream-ordered (one thread).
void launchSetWaveDyn(uint32_t* dyn, uint32_t offset, uint32_t fresh, cudaStream_t st);
void launchGenerate(const DevScene& sc, const PathSoA& s, const WaveParams& w, const LaunchShape& ls, cudaStream_t st);
// counters: nullptr, or 7 device uint64 (extend rays/nodes/tris, shadow rays/nodes/tris,
// surface records) to run the counting variants.
void launchExtend(const DevScene& sc, const PathSoA& s, int bounce, const LaunchShape& ls, cudaStream_t st,
	unsigned long long* counters);
// The shading stage as three kernels: surface record, light sample, BxDF.
void launchSurface(const DevScene& sc, const PathSoA& s, const WaveParams& w, int bounce, const LaunchShape& ls, cudaStream_t st,
	unsigned long long* counters);
void launchEmission(const DevScene& sc, const PathSoA& s, int bounce, const LaunchShape& ls, cudaStream_t st);
void launchNee(const DevScene& sc, const PathSoA& s, const WaveParams& w, int bounce, const LaunchShape& ls, cudaStream_t st);
void launchBsdf(const DevScene& sc, const PathSoA& s, const WaveParams& w, int bounce, const LaunchShape& ls, cudaStream_t st);
// Resolve + AgX tonemap of the accumulation into width*height RGBA8 words
// (rb_image.cu); colorspace: 9 floats, column-major XYZ -> RGB.
void launchResolveImage(uint32_t width, uint32_t height, const float* colorspace, float exposureScale,
	const double4* data, uint32_t* out, int smCount, cudaStream_t st);
void launchUnpackLightTree(const PackedNode* in, TreeNodeU* out, uint32_t n, cudaStream_t st);
// Camera-relative light data: tris[i].v = worldTris[i].v - origin, nodes[i].mean =
// worldNodes[i].mean - origin (all other fields copied).
void launchLightOrigin(const EmissiveTri* worldTris, EmissiveTri* tris, uint32_t nTris, const PackedNode* worldNodes,
	PackedNode* nodes, uint32_t nNodes, float ox, float oy, float oz, cudaStream_t st);
void queryTraceShape(LaunchShape& ls);   // fills blocksExtend, blocksShadow (rb_trace.cu)
void launchShadow(const DevScene& sc, const PathSoA& s, int bounce, const LaunchShape& ls, cudaStream_t st,
	unsigned long long* counters);
void launchResolve(const DevScene& sc, const PathSoA& s, const WaveParams& w, double4* accum, const LaunchShape& ls, cudaStream_t st);
// Radiance-cache form, after the last bounce of a wave: training targets
// (L_final - L_vertex) / T_vertex in place of the records' radiance (0 for a
// dropped path), then n training rows drawn from them (step: varies the
// draw) into in (kNrcInputs floats) and target (8 floats: radiance, drop
// flag, unused) with valid = n (or 0 without records). keepFailed:
// RB_FAILED_KEEP (a path with the terminated flag is not dropped).
void launchTrainTargets(const PathSoA& s, uint32_t keepFailed, int smCount, cudaStream_t st);
void launchTrainGather(const PathSoA& s, uint32_t keepFailed, uint32_t n, uint32_t step, float* in, float* target,
	uint32_t* valid, cudaStream_t st);
// tally[0] += queries, tally[1] += training records of the wave.
// Folds the wave's sums of the cached form's correction state
// (rb::nrc::kCorr* layout, rb_nrc_internal.h) into its corrections and
// clears the sums.
void launchCacheCorrectionUpdate(float* state, cudaStream_t st);
void launchCacheTally(const PathSoA& s, unsigned long long* tally, cudaStream_t st);

// Per-function batch kernels (include/ratbite_b200_kernels.h).
void launchSobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash, const uint32_t* bounce,
	const uint32_t* dim, float* out, cudaStream_t st);
void launchPixelHash(uint32_t n, const uint32_t* x, const uint32_t* y, uint32_t* out, cudaStream_t st);
void launchWavelengths(uint32_t n, const float* u, float* lambda, float* pdf, cudaStream_t st);
void launchCameraRay(const DevScene& sc, uint32_t n, const float* pixel, const float* fuv, const float* luv, float* out, cudaStream_t st);
void launchTextureSample(const DevScene& sc, uint32_t texture, cudaTextureObject_t hw, uint32_t n, const float* uv,
	float* soft, float* hwOut, cudaStream_t st);
void launchBxdfCases(const DevScene& sc, uint32_t n, void* cases, cudaStream_t st);
void launchLightCases(const DevScene& sc, uint32_t n, void* cases, cudaStream_t st);
void launchOffsetPoint(uint32_t n, const float* p, const float* nrm, float* out, cudaStream_t st);
void launchOctEncode(uint32_t n, const float* v, uint32_t* out, cudaStream_t st);
void launchOctDecode(uint32_t n, const uint32_t* code, float* out, cudaStream_t st);
void launchTrace(const DevScene& sc, uint32_t n, const float* rays, uint32_t* payload, float* t, int32_t* tri, cudaStream_t st);
void launchOccluded(const DevScene& sc, uint32_t n, const float* rays, const float* tmax, uint32_t* out, cudaStream_t st);
} // namespace rb
