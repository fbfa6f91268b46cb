// C ABI of the renderer (include/ratbite_b200.h): context, scene upload,
// geometry preparation, wavefront scheduling and readback.
//
// Compiled with -ffp-contract=off: the per-triangle values prepared here
// (world-space vertices, encoded geometric normals, inverse transforms)
// must be bitwise what the reference's closest-hit program computes from
// the same inputs (src/kernels/pathtrace.cu:94-148).

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "ratbite_b200.h"
#include "ratbite_b200_kernels.h"
#include "ratbite_b200_nrc.h"
#include "rb_bvh_build.h"
#include "rb_envmap.h"
#include "rb_launch.cuh"
#include "rb_light.cuh"
#include "rb_nrc_internal.h"
#include "rb_refit.h"
#include "rb_scene.h"
#include "rb_wavefront.h"

struct rb_ctx
{
	int device = 0;
	cudaStream_t stream = nullptr;
	std::string error;
	rb::DevScene scene{};
	rb::LaunchShape shape{};
	uint32_t* status = nullptr;          // [0] flags, [1] detail
	// owned device buffers by role
	std::vector<void*> lutBufs, spectraBufs, materialBufs, geoBufs, lightBufs, envBufs, textureBufs;
	// wavefront state
	rb::PathSoA soa{};
	std::vector<void*> soaBufs;
	uint32_t capacity = 0;
	uint32_t requestedCapacity = 0;
	uint32_t cdfMode = RB_CDF_FP64;
	uint32_t failedMode = RB_FAILED_DROP;
	// shared wavefront of rb_render_jobs (this context hosts it): per-path job
	// index and key, the job table and the chunk table of a call
	std::vector<void*> jobBufs;
	uint32_t* jobIdx = nullptr;
	uint2* jobKey = nullptr;
	uint32_t jobPathCap = 0;
	rb::DevJob* jobTable = nullptr;
	uint32_t jobTableCap = 0;
	rb::WaveChunk* chunkTable = nullptr;
	uint32_t chunkCap = 0;
	// fault injection (rb_config.inject_*; tests only)
	uint32_t injectQueueLimit = 0, injectAllocFailure = 0, injectStackLimit = 0;
	uint64_t allocCount = 0;                    // device allocations made so far
	uint32_t texturesNeeded = 0;                // 1 + the largest texture index the materials use
	void* envScratch = nullptr;                 // CDF scratch of the current map (in envBufs)
	float* envIntegral = nullptr;               // device scalar (in envBufs)
	double4* accum = nullptr;
	size_t accumPixels = 0;
	uint32_t* image = nullptr;                  // resolved RGBA8 (rb_resolve)
	size_t imagePixels = 0;
	bool haveLaunch = false, haveGeometry = false;
	uint64_t pathsTraced = 0;
	// cross-table references checked before any kernel reads them
	// refit of moved instances (rb_update_instances)
	rb::RefitData refit;
	// two-level structure (RB_ACCEL_INSTANCED): per flat instance its unit
	// (-1: no triangles) and canonical base; per unit its root; the top
	// level's node slots, the instance table and the world-box inputs on the
	// device
	bool instanced = false;
	std::vector<int32_t> instUnit;
	std::vector<uint32_t> instCanon;
	std::vector<uint32_t> unitRoot;
	uint32_t* instRangeDev = nullptr;           // per flat instance: its unit's first triangle and count
	float* instXfDev = nullptr;                 // per flat instance: 12 floats
	float* instBoxDev = nullptr;                // per flat instance: world box (6 floats)
	rb::BvhNode* topNodes = nullptr;            // the top level's slots inside scene.geo.nodes
	uint32_t topBase = 0, topCapacity = 0;
	rb::DevInstance* instDev = nullptr;
	uint32_t geoInstances = 0, geoSubsets = 0;
	float* xfDev = nullptr;                     // 12 floats per flattened instance (in geoBufs)
	float* wiDev = nullptr;
	uint32_t geoEmissive = 0;                   // emissive triangles traced by the geometry
	uint32_t geoMaxMaterial = 0;                // 1 + largest material index of the geometry
	uint32_t lightMaxMaterial = 0;              // 1 + largest material index of the light records
	// progressive schedule (rb_progressive_*)
	uint32_t progOffset = 0, progCount = 0, progTotal = 0;
	int progMode = RB_MODE_IMMEDIATE;
	// instrumentation (rb_set_stats)
	uint32_t statsMode = 0;
	unsigned long long* counters = nullptr;     // 7 device counters
	struct Timed { int stage; cudaEvent_t a, b; };
	std::vector<Timed> timed;
	std::vector<cudaEvent_t> eventPool;
	uint32_t launches[9] = {};   // generate, extend, surface, shadow, resolve, nee, bsdf, cache queries, cache training
	double stageMs[9] = {};      // device time drained from `timed`
	uint64_t waves = 0;
	// light data as given to rb_set_lights (in lightBufs), and the light origin
	const rb::EmissiveTri* lightWorldTris = nullptr;
	const rb::PackedNode* lightWorldNodes = nullptr;
	float lightOrigin[3] = { 0.0f, 0.0f, 0.0f };
	// geometry bounds at upload (radiance-cache position normalisation)
	float geoMin[3] = {}, geoMax[3] = {};
	// radiance-cache form (rb_attach_radiance_cache)
	rb_nrc* cache = nullptr;
	rb_cache_params cacheParams{};
	rb::PathSoA cacheArrays{};           // only the cache fields are used
	std::vector<void*> cacheBufs;
	uint32_t cacheCapacity = 0;          // paths the per-path arrays hold
	uint32_t cacheBatchRows = 0;         // rows of the training batch buffers
	float* batchIn = nullptr;
	float* batchTarget = nullptr;
	uint32_t* batchValid = nullptr;
	unsigned long long* cacheTally = nullptr;   // device: queries, records
	float* cacheCorr = nullptr;                 // device: the cached form's correction state (rb::nrc::kCorr*)
	uint64_t cacheWaves = 0, cacheSteps = 0, cacheStepsReported = 0;
	// replayed wave sequences (rb_render_graph): one per call shape and scene
	// state; dyn holds the replayed call's offset and fresh flag
	struct GraphKey
	{
		rb::DevScene scene;
		rb::PathSoA soa;
		double4* accum;
		uint32_t count;
	};
	struct Graph
	{
		GraphKey key;
		cudaGraphExec_t exec;
		uint32_t launches[9];
		uint64_t paths, waves;
	};
	std::vector<Graph> graphs;
	uint32_t* dyn = nullptr;
};

// NVTX range over a host-side phase (render calls, structure builds), for
// timeline tools; free when no tool is attached.
struct NvtxRange
{
	explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
	~NvtxRange() { nvtxRangePop(); }
	NvtxRange(const NvtxRange&) = delete;
	NvtxRange& operator=(const NvtxRange&) = delete;
};

namespace
{
int fail(rb_ctx* ctx, int code, const std::string& msg)
{
	if (ctx) ctx->error = msg;
	return code;
}
int cudaFail(rb_ctx* ctx, cudaError_t e, const char* what)
{
	return fail(ctx, e == cudaErrorMemoryAllocation ? RB_ERR_OOM : RB_ERR_CUDA,
		std::string(what) + ": " + cudaGetErrorString(e));
}
void freeAll(std::vector<void*>& bufs)
{
	for (void* p : bufs) cudaFree(p);
	bufs.clear();
}
// Allocates and uploads `bytes` from host `src` (may be null: zero fill).
// Every device allocation of a context goes through here, so that a test can
// make the n-th one fail (rb_config.inject_alloc_failure) the way an
// exhausted device would.
cudaError_t devMalloc(rb_ctx* ctx, void** p, size_t bytes)
{
	++ctx->allocCount;
	if (ctx->injectAllocFailure && ctx->allocCount == ctx->injectAllocFailure)
	{
		*p = nullptr;
		return cudaErrorMemoryAllocation;
	}
	return cudaMalloc(p, bytes);
}
template<typename T>
int upload(rb_ctx* ctx, std::vector<void*>& owner, const void* src, size_t bytes, T*& out)
{
	void* d = nullptr;
	cudaError_t e = devMalloc(ctx, &d, std::max<size_t>(bytes, 16));
	if (e != cudaSuccess) return cudaFail(ctx, e, "cudaMalloc");
	owner.push_back(d);
	e = src ? cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, ctx->stream)
	        : cudaMemsetAsync(d, 0, std::max<size_t>(bytes, 16), ctx->stream);
	if (e != cudaSuccess) return cudaFail(ctx, e, "upload");
	out = static_cast<T*>(d);
	return RB_OK;
}
cudaStream_t pick(rb_ctx* ctx, void* s) { return s ? static_cast<cudaStream_t>(s) : ctx->stream; }

// Buffers a render call allocates on demand (the wave, the cache arrays, a
// shared wavefront's job tables) are zero-filled on the context's own
// stream (upload). A call that renders on a caller's stream waits for those
// fills before it enqueues anything that writes the buffers, or a fill that
// runs late would overwrite what the render wrote (a zeroed job table has
// null scene and accumulation pointers). `allocs0`: the context's allocation
// count at the start of the call.
int settleFills(rb_ctx* ctx, uint64_t allocs0, cudaStream_t st)
{
	if (ctx->allocCount == allocs0 || st == ctx->stream) return RB_OK;
	const cudaError_t e = cudaStreamSynchronize(ctx->stream);
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "zero-fill of new buffers");
}

// Setters are transactional: new tables are uploaded into `fresh` first, and
// only when every upload succeeded does the context switch to them, after
// all queued work (renders may run on caller streams) has finished with the
// old ones. A rejected or failed call leaves the context exactly as it was.
int commit(rb_ctx* ctx, std::vector<void*>& owned, std::vector<void*>& fresh, int rc)
{
	if (rc != RB_OK)
	{
		freeAll(fresh);
		return rc;
	}
	const cudaError_t e = cudaDeviceSynchronize();
	if (e != cudaSuccess)
	{
		freeAll(fresh);
		return cudaFail(ctx, e, "synchronize before replacing scene data");
	}
	freeAll(owned);
	owned.swap(fresh);
	return RB_OK;
}

// Row-major 3x4 inverse in double, rounded once to float.
void invert3x4(const float* m, float* out)
{
	const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
	const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
	const double r = 1.0 / det;
	const double inv[9] = {
		(e * i - f * h) * r, (c * h - b * i) * r, (b * f - c * e) * r,
		(f * g - d * i) * r, (a * i - c * g) * r, (c * d - a * f) * r,
		(d * h - e * g) * r, (b * g - a * h) * r, (a * e - b * d) * r };
	const double t[3] = { m[3], m[7], m[11] };
	for (int row = 0; row < 3; ++row)
	{
		out[row * 4 + 0] = static_cast<float>(inv[row * 3 + 0]);
		out[row * 4 + 1] = static_cast<float>(inv[row * 3 + 1]);
		out[row * 4 + 2] = static_cast<float>(inv[row * 3 + 2]);
		out[row * 4 + 3] = static_cast<float>(-(inv[row * 3 + 0] * t[0] + inv[row * 3 + 1] * t[1] + inv[row * 3 + 2] * t[2]));
	}
}
// Object to world as the closest-hit program forms it: ((x*W0 + y*W1) + z*W2) + W3.
void toWorld(const float* W, const float* p, float* o)
{
	o[0] = p[0] * W[0] + p[1] * W[1] + p[2] * W[2] + W[3];
	o[1] = p[0] * W[4] + p[1] * W[5] + p[2] * W[6] + W[7];
	o[2] = p[0] * W[8] + p[1] * W[9] + p[2] * W[10] + W[11];
}
// Encoded geometric normal of an object-space triangle under world-to-object
// matrix Wi (pathtrace.cu:102-112): object-space cross product, transposed
// inverse transform, correctly rounded reciprocal square root, octahedral code.
uint32_t encodedNormal(const float* obj, const float* Wi)
{
	const float ux = obj[3] - obj[0], uy = obj[4] - obj[1], uz = obj[5] - obj[2];
	const float vx = obj[6] - obj[0], vy = obj[7] - obj[1], vz = obj[8] - obj[2];
	float gx = uy * vz - uz * vy, gy = uz * vx - ux * vz, gz = ux * vy - uy * vx;
	const float nx = gx * Wi[0] + gy * Wi[4] + gz * Wi[8];
	const float ny = gx * Wi[1] + gy * Wi[5] + gz * Wi[9];
	const float nz = gx * Wi[2] + gy * Wi[6] + gz * Wi[10];
	const float s = nx * nx + ny * ny + nz * nz;
	const float r = static_cast<float>(1.0 / std::sqrt(static_cast<double>(s)));
	return rb::octEncodeU32(rb::mk(nx * r, ny * r, nz * r));
}
uint32_t readIndex(const void* p, uint32_t type, size_t i)
{
	return type == RB_INDEX_U16 ? static_cast<const uint16_t*>(p)[i] : static_cast<const uint32_t*>(p)[i];
}
bool degenerate(const float* w)
{
	return (w[0] == w[3] && w[1] == w[4] && w[2] == w[5]) || (w[0] == w[6] && w[1] == w[7] && w[2] == w[8])
		|| (w[3] == w[6] && w[4] == w[7] && w[5] == w[8]);
}

cudaEvent_t takeEvent(rb_ctx* ctx)
{
	if (!ctx->eventPool.empty())
	{
		cudaEvent_t e = ctx->eventPool.back();
		ctx->eventPool.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	cudaEventCreate(&e);
	return e;
}
// Runs `launch` bracketed by events when per-stage timing is on.
template<typename F>
void timedStage(rb_ctx* ctx, int stage, cudaStream_t st, F&& launch)
{
	++ctx->launches[stage];
	if (!(ctx->statsMode & RB_STATS_TIME))
	{
		launch();
		return;
	}
	rb_ctx::Timed t{ stage, takeEvent(ctx), takeEvent(ctx) };
	cudaEventRecord(t.a, st);
	launch();
	cudaEventRecord(t.b, st);
	ctx->timed.push_back(t);
}

// Adds the device time of the finished timed launches to stageMs (synchronized by the caller).
void drainTimed(rb_ctx* ctx)
{
	for (const auto& t : ctx->timed)
	{
		float v = 0.0f;
		if (cudaEventElapsedTime(&v, t.a, t.b) == cudaSuccess) ctx->stageMs[t.stage] += v;
		ctx->eventPool.push_back(t.a);
		ctx->eventPool.push_back(t.b);
	}
	ctx->timed.clear();
}

// Every index a kernel will follow must land inside its table.
int checkReferences(rb_ctx* ctx)
{
	if (ctx->geoMaxMaterial > ctx->scene.materialCount || ctx->lightMaxMaterial > ctx->scene.materialCount)
		return fail(ctx, RB_ERR_INVALID, "material index out of range of the material table");
	if (ctx->geoEmissive > ctx->scene.lights.triangleCount)
		return fail(ctx, RB_ERR_INVALID, "geometry traces more emissive triangles than the light data holds");
	if (ctx->texturesNeeded > ctx->scene.textureCount)
		return fail(ctx, RB_ERR_INVALID, "texture index out of range of the texture table");
	return RB_OK;
}

void releaseWave(rb_ctx* ctx)
{
	freeAll(ctx->soaBufs);
	ctx->soa = rb::PathSoA{};
	ctx->capacity = 0;
}
int ensureWave(rb_ctx* ctx, uint32_t paths)
{
	if (ctx->capacity >= paths) return RB_OK;
	releaseWave(ctx);
	rb::PathSoA& s = ctx->soa;
	int rc = RB_OK;
	auto alloc = [&](auto*& p, size_t elem) {
		if (rc != RB_OK) return;
		rc = upload(ctx, ctx->soaBufs, nullptr, elem * paths, p);
	};
	alloc(s.rayO, sizeof(float4)); alloc(s.rayD, sizeof(float4)); alloc(s.lambda, sizeof(float4));
	alloc(s.lpdf, sizeof(float4)); alloc(s.nrm, sizeof(float4)); alloc(s.L, sizeof(float4));
	alloc(s.T, sizeof(float4)); alloc(s.fd, sizeof(uint2)); alloc(s.hit, sizeof(float4));
	alloc(s.shO, sizeof(float4)); alloc(s.shD, sizeof(float4)); alloc(s.shC, sizeof(float4));
	alloc(s.sfP, sizeof(float4)); alloc(s.sfPi, sizeof(float4)); alloc(s.sfGn, sizeof(float4));
	alloc(s.sfT, sizeof(float4)); alloc(s.sfB, sizeof(float4)); alloc(s.sfN, sizeof(float4));
	alloc(s.sfL, sizeof(float4)); alloc(s.sfUV, sizeof(float4));
	alloc(s.queue[0], sizeof(uint32_t)); alloc(s.queue[1], sizeof(uint32_t)); alloc(s.shadowQueue, sizeof(uint32_t));
	alloc(s.surfQueue, sizeof(uint32_t)); alloc(s.recOrder, sizeof(uint32_t));
	alloc(s.emQueue, sizeof(uint32_t)); alloc(s.emA, sizeof(float4)); alloc(s.emB, sizeof(float4));
	alloc(s.emC, sizeof(float4)); alloc(s.emLight, sizeof(uint32_t));
	if (rc == RB_OK)
		rc = upload(ctx, ctx->soaBufs, nullptr, sizeof(uint32_t) * rb::kCountSlots, s.counts);
	if (rc != RB_OK) { releaseWave(ctx); return rc; }
	s.capacity = paths;
	s.queueCap = ctx->injectQueueLimit ? std::min(ctx->injectQueueLimit, paths) : paths;
	ctx->capacity = paths;
	return RB_OK;
}
// Radiance-cache arrays for waves of `paths` paths and up to `depth` vertices.
int ensureCache(rb_ctx* ctx, uint32_t paths, uint32_t depth)
{
	const rb_cache_params& P = ctx->cacheParams;
	const uint64_t oneIn = P.frozen ? 0 : P.train_one_in;
	const uint32_t want = oneIn ? static_cast<uint32_t>(std::min<uint64_t>((paths / oneIn + 1) * (depth + 1), 64u << 20)) : 1u;
	if (ctx->cacheCapacity >= paths && ctx->cacheArrays.trainCapacity >= want && ctx->cacheBatchRows >= P.batch)
		return RB_OK;
	cudaStreamSynchronize(ctx->stream);
	freeAll(ctx->cacheBufs);
	ctx->cacheArrays = rb::PathSoA{};
	ctx->cacheCapacity = ctx->cacheBatchRows = 0;
	rb::PathSoA& c = ctx->cacheArrays;
	int rc = RB_OK;
	auto alloc = [&](auto*& ptr, size_t bytes) {
		if (rc == RB_OK) rc = upload(ctx, ctx->cacheBufs, nullptr, bytes, ptr);
	};
	alloc(c.spread, sizeof(float2) * paths);
	alloc(c.trainRec, sizeof(uint32_t) * paths);
	alloc(c.cPath, sizeof(uint32_t) * paths);
	alloc(c.cIn, sizeof(float) * kNrcInputs * static_cast<size_t>(paths));
	alloc(c.tPath, sizeof(uint32_t) * want);
	alloc(c.tIn, sizeof(float) * kNrcInputs * static_cast<size_t>(want));
	alloc(c.tL, sizeof(float4) * want);
	alloc(c.tT, sizeof(float4) * want);
	alloc(ctx->batchIn, sizeof(float) * kNrcInputs * static_cast<size_t>(P.batch));
	alloc(ctx->batchTarget, 2 * sizeof(float4) * P.batch);   // radiance, drop (+3 unused)
	alloc(ctx->batchValid, sizeof(uint32_t));
	if (rc != RB_OK)
	{
		freeAll(ctx->cacheBufs);
		ctx->cacheArrays = rb::PathSoA{};
		return rc;
	}
	c.trainCapacity = want;
	ctx->cacheCapacity = paths;
	ctx->cacheBatchRows = P.batch;
	return RB_OK;
}

void releaseCache(rb_ctx* ctx)
{
	cudaStreamSynchronize(ctx->stream);
	freeAll(ctx->cacheBufs);
	ctx->cacheArrays = rb::PathSoA{};
	ctx->cacheCapacity = ctx->cacheBatchRows = 0;
	ctx->batchIn = ctx->batchTarget = nullptr;
	ctx->batchValid = nullptr;
}
} // namespace

extern "C" {

int rb_abi_version(void) { return RB_ABI_VERSION; }

int rb_attach_radiance_cache(rb_ctx* ctx, rb_nrc* cache, const rb_cache_params* params)
{
	if (!ctx) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	if (!cache)
	{
		releaseCache(ctx);
		ctx->cache = nullptr;
		return RB_OK;
	}
	if (rb::nrc::deviceOf(cache) != ctx->device)
		return fail(ctx, RB_ERR_INVALID, "rb_attach_radiance_cache: the cache lives on another device");
	rb_cache_params P = params ? *params : rb_cache_params{};
	if (!std::isfinite(P.spread_threshold) || P.spread_threshold < 0.0f)
		return fail(ctx, RB_ERR_INVALID, "rb_attach_radiance_cache: spread threshold must be finite and >= 0");
	for (int k = 0; k < 3; ++k)
		if (!std::isfinite(P.scene_min[k]) || !std::isfinite(P.scene_max[k]))
			return fail(ctx, RB_ERR_INVALID, "rb_attach_radiance_cache: non-finite bounds");
	if (!std::isfinite(P.min_roughness)) return fail(ctx, RB_ERR_INVALID, "rb_attach_radiance_cache: non-finite roughness");
	if (P.spread_threshold == 0.0f) P.spread_threshold = 0.01f;
	if (P.train_one_in == 0) P.train_one_in = 16;
	if (P.targets_per_sample == 0) P.targets_per_sample = 65536;
	if (P.batch == 0) P.batch = 131072;
	if (P.samples_per_wave == 0) P.samples_per_wave = 8;
	if (P.min_roughness == 0.0f) P.min_roughness = 0.25f;
	if (P.batch > (1u << 22)) return fail(ctx, RB_ERR_INVALID, "rb_attach_radiance_cache: batch above 2^22 rows");
	if (!ctx->cacheTally)
	{
		cudaError_t e = devMalloc(ctx, reinterpret_cast<void**>(&ctx->cacheTally), 2 * sizeof(unsigned long long));
		if (e == cudaSuccess) e = cudaMemset(ctx->cacheTally, 0, 2 * sizeof(unsigned long long));
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_attach_radiance_cache");
	}
	if (!ctx->cacheCorr)
	{
		const cudaError_t e = devMalloc(ctx, reinterpret_cast<void**>(&ctx->cacheCorr), rb::nrc::kCorrFloats * sizeof(float));
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_attach_radiance_cache");
	}
	// the corrections are measured anew for every attached cache
	cudaStreamSynchronize(ctx->stream);
	if (const cudaError_t e = cudaMemset(ctx->cacheCorr, 0, rb::nrc::kCorrFloats * sizeof(float)); e != cudaSuccess)
		return cudaFail(ctx, e, "rb_attach_radiance_cache");
	// per-path arrays are sized by the next render; batch buffers follow the new parameters
	ctx->cache = cache;
	ctx->cacheParams = P;
	return RB_OK;
}

int rb_get_cache_stats(rb_ctx* ctx, rb_cache_stats* out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	cudaError_t e = cudaStreamSynchronize(ctx->stream);
	if (e == cudaSuccess) e = cudaDeviceSynchronize();
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_get_cache_stats");
	drainTimed(ctx);
	*out = rb_cache_stats{};
	if (ctx->cacheTally)
	{
		unsigned long long t[2] = {};
		e = cudaMemcpy(t, ctx->cacheTally, sizeof(t), cudaMemcpyDeviceToHost);
		if (e == cudaSuccess) e = cudaMemset(ctx->cacheTally, 0, sizeof(t));
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_get_cache_stats");
		out->queries = t[0];
		out->records = t[1];
	}
	if (ctx->cache)
	{
		e = cudaMemcpy(&out->last_loss, rb::nrc::lossDevice(ctx->cache), sizeof(float), cudaMemcpyDeviceToHost);
		float corr[rb::nrc::kCorrFloats] = {};
		if (e == cudaSuccess && ctx->cacheCorr)
			e = cudaMemcpy(corr, ctx->cacheCorr, sizeof(corr), cudaMemcpyDeviceToHost);
		out->drop_bias = corr[rb::nrc::kCorrDropLit + 2];
		out->drop_bias_other = corr[rb::nrc::kCorrDropOther + 2];
		out->radiance_scale = corr[rb::nrc::kCorrRadiance + 3] > 0.0f ? corr[rb::nrc::kCorrRadiance + 2] : 1.0f;
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_get_cache_stats");
	}
	out->steps = ctx->cacheSteps - ctx->cacheStepsReported;
	ctx->cacheStepsReported = ctx->cacheSteps;
	out->launches = ctx->launches[7] + ctx->launches[8];
	out->ms_infer = ctx->stageMs[7];
	out->ms_train = ctx->stageMs[8];
	ctx->launches[7] = ctx->launches[8] = 0;
	ctx->stageMs[7] = ctx->stageMs[8] = 0.0;
	return RB_OK;
}

int rb_create(const rb_config* config, rb_ctx** out)
{
	if (!out) return RB_ERR_INVALID;
	*out = nullptr;
	rb_ctx* ctx = new (std::nothrow) rb_ctx();
	if (!ctx) return RB_ERR_OOM;
	ctx->device = config ? config->device : 0;
	ctx->requestedCapacity = config ? config->max_paths_in_flight : 0u;
	if (config && config->envmap_cdf_mode > RB_CDF_REFERENCE) { delete ctx; return RB_ERR_INVALID; }
	ctx->cdfMode = config ? config->envmap_cdf_mode : RB_CDF_FP64;
	if (config && config->failed_sample_mode > RB_FAILED_KEEP) { delete ctx; return RB_ERR_INVALID; }
	ctx->failedMode = config ? config->failed_sample_mode : RB_FAILED_DROP;
	if (config && config->acceleration > RB_ACCEL_INSTANCED) { delete ctx; return RB_ERR_INVALID; }
	ctx->instanced = config && config->acceleration == RB_ACCEL_INSTANCED;
	if (config)
	{
		ctx->injectQueueLimit = config->inject_queue_limit;
		ctx->injectAllocFailure = config->inject_alloc_failure;
		ctx->injectStackLimit = config->inject_stack_limit;
	}
	cudaError_t e = cudaSetDevice(ctx->device);
	if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
	if (e == cudaSuccess) e = devMalloc(ctx, reinterpret_cast<void**>(&ctx->status), 2 * sizeof(uint32_t));
	if (e == cudaSuccess) e = cudaMemset(ctx->status, 0, 2 * sizeof(uint32_t));
	if (e == cudaSuccess) e = devMalloc(ctx, reinterpret_cast<void**>(&ctx->dyn), 2 * sizeof(uint32_t));
	if (e != cudaSuccess)
	{
		const int rc = e == cudaErrorMemoryAllocation ? RB_ERR_OOM : RB_ERR_CUDA;
		if (ctx->stream) cudaStreamDestroy(ctx->stream);
		if (ctx->status) cudaFree(ctx->status);
		if (ctx->dyn) cudaFree(ctx->dyn);
		delete ctx;
		return rc;
	}
	ctx->scene.status = ctx->status;
	ctx->shape = rb::queryLaunchShape();
	*out = ctx;
	return RB_OK;
}

int rb_destroy(rb_ctx* ctx)
{
	if (!ctx) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	cudaStreamSynchronize(ctx->stream);
	for (auto* v : { &ctx->lutBufs, &ctx->spectraBufs, &ctx->materialBufs, &ctx->geoBufs, &ctx->lightBufs, &ctx->envBufs,
			&ctx->textureBufs })
		freeAll(*v);
	releaseWave(ctx);
	freeAll(ctx->jobBufs);
	freeAll(ctx->cacheBufs);
	if (ctx->cacheTally) cudaFree(ctx->cacheTally);
	if (ctx->cacheCorr) cudaFree(ctx->cacheCorr);
	for (const auto& t : ctx->timed) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
	for (cudaEvent_t e : ctx->eventPool) cudaEventDestroy(e);
	if (ctx->counters) cudaFree(ctx->counters);
	if (ctx->accum) cudaFree(ctx->accum);
	if (ctx->image) cudaFree(ctx->image);
	if (ctx->status) cudaFree(ctx->status);
	if (ctx->dyn) cudaFree(ctx->dyn);
	for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
	if (ctx->stream) cudaStreamDestroy(ctx->stream);
	delete ctx;
	return RB_OK;
}

const char* rb_last_error(const rb_ctx* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int rb_set_luts(rb_ctx* ctx, const float* conductor, const float* dOuter, const float* dInner,
	const float* rOuter, const float* rInner, const float* sheen)
{
	if (!ctx || !conductor || !dOuter || !dInner || !rOuter || !rInner || !sheen)
		return fail(ctx, RB_ERR_INVALID, "rb_set_luts: null table");
	cudaSetDevice(ctx->device);
	const size_t n2 = rb::kLutN * rb::kLutN, n3 = n2 * rb::kLutN;
	std::vector<void*> fresh;
	rb::DevLuts L{};
	int rc = upload(ctx, fresh, conductor, n2 * 4, L.conductor);
	if (rc == RB_OK) rc = upload(ctx, fresh, dOuter, n3 * 4, L.dielOuter);
	if (rc == RB_OK) rc = upload(ctx, fresh, dInner, n3 * 4, L.dielInner);
	if (rc == RB_OK) rc = upload(ctx, fresh, rOuter, n3 * 4, L.reflOuter);
	if (rc == RB_OK) rc = upload(ctx, fresh, rInner, n3 * 4, L.reflInner);
	if (rc == RB_OK) rc = upload(ctx, fresh, sheen, n2 * 16, L.sheen);
	rc = commit(ctx, ctx->lutBufs, fresh, rc);
	if (rc == RB_OK) ctx->scene.luts = L;
	return rc;
}

int rb_set_spectra(rb_ctx* ctx, const float* sensor, const float* basis, const float* extra, uint32_t nExtra)
{
	if (!ctx || !sensor || !basis || (nExtra && !extra)) return fail(ctx, RB_ERR_INVALID, "rb_set_spectra: null table");
	cudaSetDevice(ctx->device);
	const size_t b = sizeof(float) * rb::kSpectrumBins;
	std::vector<void*> fresh;
	rb::DevSpectra S{};
	int rc = upload(ctx, fresh, sensor, 3 * b, S.sensor);
	if (rc == RB_OK) rc = upload(ctx, fresh, basis, 3 * b, S.basis);
	if (rc == RB_OK) rc = upload(ctx, fresh, nExtra ? extra : nullptr, std::max<size_t>(nExtra, 1) * b, S.extra);
	S.extraCount = nExtra;
	rc = commit(ctx, ctx->spectraBufs, fresh, rc);
	if (rc == RB_OK) ctx->scene.spectra = S;
	return rc;
}

int rb_set_materials(rb_ctx* ctx, const rb_material* mats, uint32_t count)
{
	if (!ctx || (count && !mats)) return fail(ctx, RB_ERR_INVALID, "rb_set_materials: null materials");
	for (uint32_t i = 0; i < count; ++i)
	{
		const rb_material& m = mats[i];
		if (m.textures >> RB_TEXTURE_SLOTS) return fail(ctx, RB_ERR_INVALID, "rb_set_materials: unknown texture slot");
		for (uint32_t t = 0; t < RB_TEXTURE_SLOTS; ++t)
			if (((m.textures >> t) & 1u) && m.texture_index[t] >= ctx->scene.textureCount)
				return fail(ctx, RB_ERR_INVALID, "rb_set_materials: texture index beyond the rb_set_textures table");
		if (m.textures & ~(1u << RB_TEXTURE_EMISSION))
		{
			// the surface textures read vertex texture coordinates
			if (!m.attribute_data || m.attribute_stride == 0)
				return fail(ctx, RB_ERR_INVALID, "rb_set_materials: textures without attribute data");
			for (uint32_t set = 0; set < 2; ++set)
				if ((m.attributes & (set ? RB_ATTR_TEX_COORD_2 : RB_ATTR_TEX_COORD_1)) &&
					(set ? m.texcoord2_offset : m.texcoord1_offset) + 8u > m.attribute_stride)
					return fail(ctx, RB_ERR_INVALID, "rb_set_materials: texture coordinates outside the vertex");
		}
		if (m.bxdf > RB_BXDF_COMPLEX_SURFACE) return fail(ctx, RB_ERR_INVALID, "rb_set_materials: unknown bxdf");
		if (m.index_type > RB_INDEX_U32) return fail(ctx, RB_ERR_INVALID, "rb_set_materials: unknown index type");
		if ((m.attributes & (RB_ATTR_NORMAL | RB_ATTR_FRAME)) && (!m.attribute_data || m.attribute_stride == 0))
			return fail(ctx, RB_ERR_INVALID, "rb_set_materials: attributes declared without attribute data");
		// the vertex layout the shading step reads with 8-byte loads: stride and
		// field offsets multiples of 8, each field inside the vertex
		if (m.attributes)
		{
			bool ok = m.attribute_stride % 8u == 0;
			if (m.attributes & RB_ATTR_FRAME) ok = ok && m.frame_offset % 8u == 0 && m.frame_offset + 16u <= m.attribute_stride;
			else if (m.attributes & RB_ATTR_NORMAL)
				ok = ok && m.normal_offset % 8u == 0 && m.normal_offset + 8u <= m.attribute_stride;
			if (m.attributes & RB_ATTR_TEX_COORD_1) ok = ok && m.texcoord1_offset % 8u == 0 && m.texcoord1_offset + 8u <= m.attribute_stride;
			if (m.attributes & RB_ATTR_TEX_COORD_2) ok = ok && m.texcoord2_offset % 8u == 0 && m.texcoord2_offset + 8u <= m.attribute_stride;
			if (!ok) return fail(ctx, RB_ERR_INVALID, "rb_set_materials: vertex attributes not at multiples of 8 bytes inside the stride");
		}
		if (m.triangle_count && !m.indices) return fail(ctx, RB_ERR_INVALID, "rb_set_materials: null indices");
	}
	cudaSetDevice(ctx->device);
	std::vector<void*> fresh;
	std::vector<rb::DevMaterial> dm(std::max<uint32_t>(count, 1));
	for (uint32_t i = 0; i < count; ++i)
	{
		const rb_material& m = mats[i];
		rb::DevMaterial& d = dm[i];
		d = rb::DevMaterial{};
		d.bxdf = m.bxdf;
		d.sheenPresent = m.sheen_present;
		d.indexType = m.index_type;
		d.attributes = m.attributes;
		d.attributeStride = m.attribute_stride;
		d.normalOffset = m.normal_offset;
		d.frameOffset = m.frame_offset;
		d.factors = m.factors;
		d.iorSpectrum = m.ior_spectrum;
		d.absorpSpectrum = m.absorp_spectrum;
		d.mfRoughness = m.mf_roughness;
		d.ior = m.ior;
		d.alphaCutoff = m.alpha_cutoff;
		d.metalness = m.metalness;
		d.roughness = m.roughness;
		d.transmission = m.transmission;
		for (int k = 0; k < 4; ++k) d.baseColor[k] = m.base_color[k];
		for (int k = 0; k < 3; ++k) { d.sheenColor[k] = m.sheen_color[k]; d.emissive[k] = m.emissive[k]; }
		d.sheenRoughness = m.sheen_roughness;
		d.triangleCount = m.triangle_count;
		d.vertexCount = m.vertex_count;
		d.textures = m.textures;
		d.texSets = m.texcoord_sets;
		d.texcoordOffset[0] = m.texcoord1_offset;
		d.texcoordOffset[1] = m.texcoord2_offset;
		for (uint32_t t = 0; t < RB_TEXTURE_SLOTS; ++t)
			d.tex[t] = ((m.textures >> t) & 1u) ? static_cast<uint16_t>(m.texture_index[t]) : 0;
		const size_t ib = static_cast<size_t>(m.triangle_count) * 3 * (m.index_type == RB_INDEX_U16 ? 2 : 4);
		uint8_t* dptr = nullptr;
		int rc = upload(ctx, fresh, m.indices, ib, dptr);
		if (rc != RB_OK) return commit(ctx, ctx->materialBufs, fresh, rc);
		d.indices = dptr;
		const size_t ab = static_cast<size_t>(m.vertex_count) * m.attribute_stride;
		rc = upload(ctx, fresh, m.attribute_data && ab ? m.attribute_data : nullptr, ab, dptr);
		if (rc != RB_OK) return commit(ctx, ctx->materialBufs, fresh, rc);
		d.attributeData = dptr;
	}
	rb::DevMaterial* dptr = nullptr;
	int rc = upload(ctx, fresh, dm.data(), sizeof(rb::DevMaterial) * dm.size(), dptr);
	if (rc == RB_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = fail(ctx, RB_ERR_CUDA, "material upload");
	rc = commit(ctx, ctx->materialBufs, fresh, rc);
	if (rc != RB_OK) return rc;
	ctx->scene.materials = dptr;
	ctx->scene.materialCount = count;
	ctx->texturesNeeded = 0;
	for (uint32_t i = 0; i < count; ++i)
		for (uint32_t t = 0; t < RB_TEXTURE_SLOTS; ++t)
			if ((mats[i].textures >> t) & 1u) ctx->texturesNeeded = std::max(ctx->texturesNeeded, mats[i].texture_index[t] + 1u);
	return RB_OK;
}

int rb_set_textures(rb_ctx* ctx, const rb_texture* textures, uint32_t count)
{
	if (!ctx || (count && !textures)) return fail(ctx, RB_ERR_INVALID, "rb_set_textures: null textures");
	if (count > 65535u) return fail(ctx, RB_ERR_TOO_LARGE, "rb_set_textures: more than 65535 textures");
	for (uint32_t i = 0; i < count; ++i)
	{
		const rb_texture& t = textures[i];
		if (t.width == 0 || t.height == 0 || t.width > 32768u || t.height > 32768u || !t.data)
			return fail(ctx, RB_ERR_INVALID, "rb_set_textures: empty, oversized or null texture");
		if (t.format > RB_TEXFMT_RGBA8 || t.address_u > RB_TEXADDR_MIRROR || t.address_v > RB_TEXADDR_MIRROR ||
			t.filter > RB_TEXFILTER_LINEAR || t.srgb > 1u)
			return fail(ctx, RB_ERR_INVALID, "rb_set_textures: unknown format, address mode or filter");
	}
	cudaSetDevice(ctx->device);
	std::vector<void*> fresh;
	std::vector<rb::DevTexture> dt(std::max<uint32_t>(count, 1));
	int rc = RB_OK;
	for (uint32_t i = 0; i < count && rc == RB_OK; ++i)
	{
		const rb_texture& t = textures[i];
		rb::DevTexture& d = dt[i];
		d = rb::DevTexture{};
		d.width = t.width;
		d.height = t.height;
		d.channels = t.format == RB_TEXFMT_R8 ? 1u : 4u;
		d.srgb = t.srgb ? 1u : 0u;
		d.addrU = t.address_u;
		d.addrV = t.address_v;
		d.filter = t.filter;
		uint8_t* dptr = nullptr;
		rc = upload(ctx, fresh, t.data, static_cast<size_t>(t.width) * t.height * d.channels, dptr);
		d.data = dptr;
	}
	// the sRGB decode of each 8-bit code (IEC 61966-2-1), in double precision
	float lut[256];
	for (int c = 0; c < 256; ++c)
	{
		const double x = c / 255.0;
		lut[c] = static_cast<float>(x <= 0.04045 ? x / 12.92 : std::pow((x + 0.055) / 1.055, 2.4));
	}
	rb::DevTexture* table = nullptr;
	float* lutDev = nullptr;
	if (rc == RB_OK) rc = upload(ctx, fresh, dt.data(), sizeof(rb::DevTexture) * dt.size(), table);
	if (rc == RB_OK) rc = upload(ctx, fresh, lut, sizeof(lut), lutDev);
	if (rc == RB_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = fail(ctx, RB_ERR_CUDA, "texture upload");
	rc = commit(ctx, ctx->textureBufs, fresh, rc);
	if (rc != RB_OK) return rc;
	ctx->scene.textures = table;
	ctx->scene.textureCount = count;
	ctx->scene.srgbLut = lutDev;
	return RB_OK;
}

#ifndef RB_TOP_LEAF
#define RB_TOP_LEAF 4
#endif


namespace
{
// Relocates a unit's (or the top level's) BVH node into the shared node
// array: interior children by the node base, leaf references by the base of
// the unit's triangles (or of the instance table, which is 0).
void relocate(rb::BvhNode& n, uint32_t nodeBase, uint32_t leafBase)
{
	for (int c = 0; c < 8; ++c)
	{
		const uint32_t ref = n.child[c];
		if (ref == rb::kEmptyChild) continue;
		if (ref & rb::kLeafBit) n.child[c] = (ref & 0xF0000000u) | ((ref & 0x0FFFFFFFu) + leafBase);
		else n.child[c] = ref + nodeBase;
	}
}

// The instances' world boxes, exact over their world triangles (the flat
// upload's vertex arithmetic, on the device: the corners of the object box
// through a rotation bound a box up to sqrt(3) times as wide), copied back.
int instanceBoxes(rb_ctx* ctx, const std::vector<float>& xfAll, std::vector<float>& boxes, cudaStream_t st)
{
	const size_t n = ctx->instUnit.size();
	boxes.assign(6 * n, 0.0f);
	if (!n) return RB_OK;
	cudaError_t e = cudaMemcpyAsync(ctx->instXfDev, xfAll.data(), sizeof(float) * 12 * n, cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess)
	{
		rb::launchInstanceBoxes(ctx->scene.geo.triVerts, ctx->instRangeDev, ctx->instXfDev, ctx->instBoxDev,
			static_cast<uint32_t>(n), st);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess) e = cudaMemcpyAsync(boxes.data(), ctx->instBoxDev, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	return e == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}

// The top level over the instances' world boxes, as "triangles" (lo, hi,
// centre) that bound each box; the instance table in its leaf order.
int buildTopLevel(rb_ctx* ctx, const std::vector<float>& xfAll, const std::vector<float>& wiAll,
	const std::vector<float>& worldBoxes, std::vector<rb::BvhNode>& nodes, std::vector<rb::DevInstance>& table,
	uint32_t& root)
{
	std::vector<float> boxes;
	std::vector<uint32_t> flat;
	for (size_t i = 0; i < ctx->instUnit.size(); ++i)
	{
		if (ctx->instUnit[i] < 0) continue;
		const float* lo = worldBoxes.data() + 6 * i;
		const float* hi = lo + 3;
		for (int a = 0; a < 3; ++a)
			if (!std::isfinite(lo[a]) || !std::isfinite(hi[a]) || lo[a] > hi[a]) return RB_ERR_INVALID;
		const float tri[9] = { lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], 0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]),
			0.5f * (lo[2] + hi[2]) };
		boxes.insert(boxes.end(), tri, tri + 9);
		flat.push_back(static_cast<uint32_t>(i));
	}
	table.clear();
	nodes.clear();
	root = rb::kEmptyChild;
	if (flat.empty()) return RB_OK;
	// RB_TOP_LEAF instances per leaf at most (1: each instance's own box is
	// tested in its parent node, entered near to far, and skipped beyond the
	// closest hit so far)
	const rb::WideBvh top = rb::buildWideBvh(boxes, RB_TOP_LEAF);
	if (top.maxDepth + 1 > 8u) return RB_ERR_TOO_LARGE;
	nodes = top.nodes;
	for (rb::BvhNode& n : nodes) relocate(n, ctx->topBase, 0u);
	root = top.rootIsLeaf ? (rb::kLeafBit | (static_cast<uint32_t>(flat.size() - 1) << 28)) : ctx->topBase;
	for (uint32_t j = 0; j < flat.size(); ++j)
	{
		const uint32_t i = flat[top.triOrder[j]];
		rb::DevInstance d{};
		std::memcpy(d.xf, xfAll.data() + 12 * i, sizeof(d.xf));
		std::memcpy(d.wi, wiAll.data() + 12 * i, sizeof(d.wi));
		d.root = ctx->unitRoot[ctx->instUnit[i]];
		d.canonBase = ctx->instCanon[i];
		d.index = i;
		table.push_back(d);
	}
	return RB_OK;
}

// rb_set_geometry for RB_ACCEL_INSTANCED: one BVH per unit (each mesh an
// instance uses, each emissive subset) over its object-space triangles, the
// top level over the instances. Triangle numbering (canonical ids,
// primitive and emissive indices) and the skipped degenerate triangles are
// the flat upload's.
int setGeometryInstanced(rb_ctx* ctx, const rb_geometry* g)
{
	struct Unit
	{
		std::vector<float> obj;
		std::vector<uint32_t> canon, sbt, prim;
	};
	std::vector<Unit> units;
	std::vector<int32_t> meshUnit(g->mesh_count, -2);      // -2: not built yet
	std::vector<uint32_t> meshTris(g->mesh_count, 0);
	std::vector<int32_t> instUnit;
	std::vector<uint32_t> instCanon;
	std::vector<float> xfAll, wiAll, normalMatrix;
	uint32_t canonical = 0, emissivePrim = 0;
	auto addInstance = [&](const float* xf, int32_t unit, uint32_t canonBase) {
		for (int k = 0; k < 12; ++k)
			if (!std::isfinite(xf[k])) return false;
		float wi[12];
		invert3x4(xf, wi);
		const float nm[9] = { wi[0], wi[4], wi[8], wi[1], wi[5], wi[9], wi[2], wi[6], wi[10] };
		normalMatrix.insert(normalMatrix.end(), nm, nm + 9);
		xfAll.insert(xfAll.end(), xf, xf + 12);
		wiAll.insert(wiAll.end(), wi, wi + 12);
		instUnit.push_back(unit);
		instCanon.push_back(canonBase);
		return true;
	};
	auto keep = [&](Unit& u, const float* obj, uint32_t canon, uint32_t sbt, uint32_t prim) {
		for (int k = 0; k < 9; ++k)
			if (!std::isfinite(obj[k])) return false;
		if (degenerate(obj)) return true;
		u.obj.insert(u.obj.end(), obj, obj + 9);
		u.canon.push_back(canon);
		u.sbt.push_back(sbt);
		u.prim.push_back(prim);
		return true;
	};
	for (uint32_t s = 0; s < g->emissive_subset_count; ++s)
	{
		const rb_emissive_subset& es = g->emissive_subsets[s];
		if (es.triangle_count && !es.vertices) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null emissive vertices");
		Unit u;
		for (uint32_t t = 0; t < es.triangle_count; ++t)
			if (!keep(u, es.vertices + 9 * t, t, 0xFFFFFFFFu, emissivePrim++))
				return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: non-finite emissive vertex");
		const int32_t id = u.obj.empty() ? -1 : static_cast<int32_t>(units.size());
		if (!u.obj.empty()) units.push_back(std::move(u));
		if (!addInstance(es.transform, id, canonical)) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: non-finite transform");
		canonical += es.triangle_count;
	}
	for (uint32_t i = 0; i < g->instance_count; ++i)
	{
		const rb_instance& in = g->instances[i];
		if (in.mesh >= g->mesh_count) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: instance mesh out of range");
		if (meshUnit[in.mesh] == -2)
		{
			const rb_mesh& mesh = g->meshes[in.mesh];
			if (mesh.submesh_count && !mesh.submeshes) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null submeshes");
			Unit u;
			uint32_t local = 0;
			for (uint32_t s = 0; s < mesh.submesh_count; ++s)
			{
				const rb_submesh& sm = mesh.submeshes[s];
				if (sm.triangle_count && (!sm.indices || !sm.vertices)) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null submesh data");
				if (sm.index_type > RB_INDEX_U32) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: unknown index type");
				std::vector<uint8_t> discarded(sm.triangle_count, 0);
				for (uint32_t k = 0; k < sm.discarded_count; ++k)
					if (sm.discarded[k] < sm.triangle_count) discarded[sm.discarded[k]] = 1;
				for (uint32_t t = 0; t < sm.triangle_count; ++t)
				{
					float obj[9];
					for (int k = 0; k < 3; ++k)
					{
						const uint32_t vi = discarded[t] ? 0u : readIndex(sm.indices, sm.index_type, static_cast<size_t>(t) * 3 + k);
						if (vi >= sm.vertex_count) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: vertex index out of range");
						obj[3 * k + 0] = sm.vertices[4 * vi + 0];
						obj[3 * k + 1] = sm.vertices[4 * vi + 1];
						obj[3 * k + 2] = sm.vertices[4 * vi + 2];
					}
					if (!keep(u, obj, local++, sm.material, t)) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: non-finite vertex");
				}
			}
			meshTris[in.mesh] = local;
			meshUnit[in.mesh] = u.obj.empty() ? -1 : static_cast<int32_t>(units.size());
			if (!u.obj.empty()) units.push_back(std::move(u));
		}
		if (!addInstance(in.transform, meshUnit[in.mesh], canonical)) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: non-finite transform");
		canonical += meshTris[in.mesh];
	}
	// the units' BVHs in one node array and one triangle array
	std::vector<rb::BvhNode> nodes;
	std::vector<float4> triVerts;
	std::vector<uint2> triAux;
	std::vector<uint32_t> unitRoot(units.size());
	for (size_t u = 0; u < units.size(); ++u)
	{
		const Unit& U = units[u];
		const rb::WideBvh b = rb::buildWideBvh(U.obj);
		if (b.maxDepth + 1 > static_cast<uint32_t>(rb::kMaxBvhDepth) - 8u)
			return fail(ctx, RB_ERR_TOO_LARGE, "rb_set_geometry: BVH beyond the traversal limits");
		const uint32_t nodeBase = static_cast<uint32_t>(nodes.size()), triBase = static_cast<uint32_t>(triVerts.size() / 3);
		const size_t nt = U.canon.size();
		if (static_cast<size_t>(triBase) + nt >= (1u << 28)) return fail(ctx, RB_ERR_TOO_LARGE, "rb_set_geometry: more than 2^28 unique triangles");
		for (rb::BvhNode n : b.nodes)
		{
			relocate(n, nodeBase, triBase);
			nodes.push_back(n);
		}
		unitRoot[u] = b.rootIsLeaf ? (rb::kLeafBit | (static_cast<uint32_t>(nt - 1) << 28) | triBase) : nodeBase;
		for (size_t j = 0; j < nt; ++j)
		{
			const uint32_t t = b.triOrder[j];
			const float* o = U.obj.data() + 9 * t;
			float4 v[3];
			for (int k = 0; k < 3; ++k) v[k] = make_float4(o[3 * k], o[3 * k + 1], o[3 * k + 2], 0.0f);
			std::memcpy(&v[0].w, &U.canon[t], 4);
			std::memcpy(&v[2].w, &U.sbt[t], 4);
			triVerts.insert(triVerts.end(), v, v + 3);
			triAux.push_back(make_uint2(0u, U.prim[t]));
		}
	}
	ctx->instUnit = instUnit;
	ctx->instCanon = instCanon;
	ctx->unitRoot = unitRoot;
	const uint32_t nInst = static_cast<uint32_t>(instUnit.size());
	ctx->topBase = static_cast<uint32_t>(nodes.size());
	ctx->topCapacity = std::max<uint32_t>(nInst, 1u) + 1u;
	if (static_cast<size_t>(ctx->topBase) + ctx->topCapacity > rb::kMaxBvhNodes)
		return fail(ctx, RB_ERR_TOO_LARGE, "rb_set_geometry: BVH beyond the traversal limits (2^24 nodes)");
	nodes.resize(static_cast<size_t>(ctx->topBase) + ctx->topCapacity);   // top-level slots, filled below
	// world bounds over the kept triangles, as the flat upload computes them
	float lo[3] = { 0.0f, 0.0f, 0.0f }, hi[3] = { 0.0f, 0.0f, 0.0f };
	bool first = true;
	for (uint32_t i = 0; i < nInst; ++i)
	{
		if (instUnit[i] < 0) continue;
		const Unit& U = units[instUnit[i]];
		for (size_t j = 0; j < U.obj.size(); j += 3)
		{
			float w[3];
			toWorld(xfAll.data() + 12 * i, U.obj.data() + j, w);
			for (int k = 0; k < 3; ++k)
			{
				if (!std::isfinite(w[k])) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: non-finite vertex");
				lo[k] = first ? w[k] : std::min(lo[k], w[k]);
				hi[k] = first ? w[k] : std::max(hi[k], w[k]);
			}
			first = false;
		}
	}
	if (triVerts.empty()) { triVerts.resize(3); triAux.resize(1); }
	// per flat instance: its unit's triangle range, for the world boxes
	std::vector<uint32_t> range(2 * std::max<uint32_t>(nInst, 1u), 0u);
	{
		std::vector<uint32_t> unitFirst(units.size(), 0u);
		uint32_t acc = 0;
		for (size_t u = 0; u < units.size(); ++u) { unitFirst[u] = acc; acc += static_cast<uint32_t>(units[u].canon.size()); }
		for (uint32_t i = 0; i < nInst; ++i)
			if (instUnit[i] >= 0)
			{
				range[2 * i] = unitFirst[instUnit[i]];
				range[2 * i + 1] = static_cast<uint32_t>(units[instUnit[i]].canon.size());
			}
	}
	std::vector<void*> fresh;
	rb::DevGeometry G{};
	rb::BvhNode* nodeDev = nullptr;
	rb::DevInstance* instDev = nullptr;
	uint32_t* rangeDev = nullptr;
	float *xfDev = nullptr, *boxDev = nullptr;
	int rc = upload(ctx, fresh, nodes.data(), sizeof(rb::BvhNode) * nodes.size(), nodeDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, triVerts.data(), sizeof(float4) * triVerts.size(), G.triVerts);
	if (rc == RB_OK) rc = upload(ctx, fresh, triAux.data(), sizeof(uint2) * triAux.size(), G.triAux);
	if (rc == RB_OK) rc = upload(ctx, fresh, normalMatrix.empty() ? nullptr : normalMatrix.data(),
		sizeof(float) * std::max<size_t>(normalMatrix.size(), 9), G.normalMatrix);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(rb::DevInstance) * std::max<uint32_t>(nInst, 1u), instDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, range.data(), sizeof(uint32_t) * range.size(), rangeDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(float) * 12 * std::max<uint32_t>(nInst, 1u), xfDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(float) * 6 * std::max<uint32_t>(nInst, 1u), boxDev);
	// the top level over the instances' exact world boxes
	std::vector<rb::BvhNode> top;
	std::vector<rb::DevInstance> table;
	uint32_t topRoot = rb::kEmptyChild;
	if (rc == RB_OK)
	{
		rb::DevGeometry keepGeo = ctx->scene.geo;
		uint32_t* keepRange = ctx->instRangeDev;
		float *keepXf = ctx->instXfDev, *keepBox = ctx->instBoxDev;
		ctx->scene.geo.triVerts = G.triVerts;
		ctx->instRangeDev = rangeDev;
		ctx->instXfDev = xfDev;
		ctx->instBoxDev = boxDev;
		std::vector<float> boxes;
		rc = instanceBoxes(ctx, xfAll, boxes, ctx->stream);
		if (rc == RB_OK) rc = buildTopLevel(ctx, xfAll, wiAll, boxes, top, table, topRoot);
		if (rc == RB_OK && top.size() > ctx->topCapacity) rc = RB_ERR_TOO_LARGE;
		ctx->scene.geo = keepGeo;
		ctx->instRangeDev = keepRange;
		ctx->instXfDev = keepXf;
		ctx->instBoxDev = keepBox;
		if (rc != RB_OK) rc = fail(ctx, rc, "rb_set_geometry: top level (non-finite, too deep or too large)");
	}
	if (rc == RB_OK && !top.empty() &&
		cudaMemcpyAsync(nodeDev + ctx->topBase, top.data(), sizeof(rb::BvhNode) * top.size(), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
		rc = fail(ctx, RB_ERR_CUDA, "geometry upload");
	if (rc == RB_OK && !table.empty() &&
		cudaMemcpyAsync(instDev, table.data(), sizeof(rb::DevInstance) * table.size(), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
		rc = fail(ctx, RB_ERR_CUDA, "geometry upload");
	if (rc == RB_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = fail(ctx, RB_ERR_CUDA, "geometry upload");
	rc = commit(ctx, ctx->geoBufs, fresh, rc);
	if (rc != RB_OK) return rc;
	ctx->instRangeDev = rangeDev;
	ctx->instXfDev = xfDev;
	ctx->instBoxDev = boxDev;
	G.nodes = nodeDev;
	G.instances = instDev;
	G.nodeCount = static_cast<uint32_t>(nodes.size());
	G.triCount = static_cast<uint32_t>(triVerts.size() / 3);
	G.rootIsLeaf = 0u;
	G.stackLimit = static_cast<uint32_t>(rb::kTraversalStackEntries);
	if (ctx->injectStackLimit) G.stackLimit = std::min(ctx->injectStackLimit, G.stackLimit);
	G.instanced = 1u;
	G.topRoot = topRoot;
	G.instanceCount = static_cast<uint32_t>(table.size());
	ctx->scene.geo = G;
	ctx->topNodes = nodeDev + ctx->topBase;
	ctx->instDev = instDev;
	ctx->refit = rb::RefitData{};
	ctx->xfDev = ctx->wiDev = nullptr;
	ctx->geoInstances = g->instance_count;
	ctx->geoSubsets = g->emissive_subset_count;
	ctx->geoEmissive = emissivePrim;
	for (int k = 0; k < 3; ++k) { ctx->geoMin[k] = lo[k]; ctx->geoMax[k] = hi[k]; }
	ctx->geoMaxMaterial = 0;
	for (const Unit& U : units)
		for (uint32_t s : U.sbt)
			if (s != 0xFFFFFFFFu) ctx->geoMaxMaterial = std::max(ctx->geoMaxMaterial, s + 1);
	ctx->haveGeometry = true;
	return RB_OK;
}
} // namespace

int rb_set_geometry(rb_ctx* ctx, const rb_geometry* g)
{
	const NvtxRange range("rb_set_geometry");
	if (!ctx || !g) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null geometry");
	if ((g->mesh_count && !g->meshes) || (g->instance_count && !g->instances) ||
		(g->emissive_subset_count && !g->emissive_subsets))
		return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null array");
	cudaSetDevice(ctx->device);
	if (ctx->instanced) return setGeometryInstanced(ctx, g);
	// Triangles in canonical order: emissive subsets, then instances x submeshes.
	std::vector<float> world;          // 9 per kept triangle
	std::vector<float> objAll;         // 9 object-space floats per kept triangle
	std::vector<uint32_t> canon, inst, sbt, prim, enc;
	std::vector<float> normalMatrix;   // 9 per instance
	uint32_t instIndex = 0, canonical = 0, emissivePrim = 0;
	auto addInstance = [&](const float* xf, float* wi) {
		invert3x4(xf, wi);
		const float nm[9] = { wi[0], wi[4], wi[8], wi[1], wi[5], wi[9], wi[2], wi[6], wi[10] };
		normalMatrix.insert(normalMatrix.end(), nm, nm + 9);
	};
	auto addTriangle = [&](const float* obj, const float* xf, const float* wi, uint32_t instId, uint32_t sbtData, uint32_t primId) {
		float w[9];
		for (int k = 0; k < 3; ++k) toWorld(xf, obj + 3 * k, w + 3 * k);
		const uint32_t id = canonical++;
		for (float v : w) if (!std::isfinite(v)) return false;
		if (degenerate(w) || degenerate(obj)) return true;
		world.insert(world.end(), w, w + 9);
		objAll.insert(objAll.end(), obj, obj + 9);
		canon.push_back(id);
		inst.push_back(instId);
		sbt.push_back(sbtData);
		prim.push_back(primId);
		enc.push_back(encodedNormal(obj, wi));
		return true;
	};
	for (uint32_t s = 0; s < g->emissive_subset_count; ++s)
	{
		const rb_emissive_subset& es = g->emissive_subsets[s];
		if (es.triangle_count && !es.vertices) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null emissive vertices");
		float wi[12];
		addInstance(es.transform, wi);
		for (uint32_t t = 0; t < es.triangle_count; ++t)
			if (!addTriangle(es.vertices + 9 * t, es.transform, wi, instIndex, 0xFFFFFFFFu, emissivePrim++))
				return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: non-finite emissive vertex");
		++instIndex;
	}
	for (uint32_t i = 0; i < g->instance_count; ++i)
	{
		const rb_instance& in = g->instances[i];
		if (in.mesh >= g->mesh_count) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: instance mesh out of range");
		float wi[12];
		addInstance(in.transform, wi);
		const rb_mesh& mesh = g->meshes[in.mesh];
		if (mesh.submesh_count && !mesh.submeshes) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null submeshes");
		for (uint32_t s = 0; s < mesh.submesh_count; ++s)
		{
			const rb_submesh& sm = mesh.submeshes[s];
			if (sm.triangle_count && (!sm.indices || !sm.vertices)) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: null submesh data");
			if (sm.index_type > RB_INDEX_U32) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: unknown index type");
			std::vector<uint8_t> discarded(sm.triangle_count, 0);
			for (uint32_t k = 0; k < sm.discarded_count; ++k)
				if (sm.discarded[k] < sm.triangle_count) discarded[sm.discarded[k]] = 1;
			for (uint32_t t = 0; t < sm.triangle_count; ++t)
			{
				float obj[9];
				for (int k = 0; k < 3; ++k)
				{
					const uint32_t vi = discarded[t] ? 0u : readIndex(sm.indices, sm.index_type, static_cast<size_t>(t) * 3 + k);
					if (vi >= sm.vertex_count) return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: vertex index out of range");
					obj[3 * k + 0] = sm.vertices[4 * vi + 0];
					obj[3 * k + 1] = sm.vertices[4 * vi + 1];
					obj[3 * k + 2] = sm.vertices[4 * vi + 2];
				}
				if (!addTriangle(obj, in.transform, wi, instIndex, sm.material, t))
					return fail(ctx, RB_ERR_INVALID, "rb_set_geometry: non-finite vertex");
			}
		}
		++instIndex;
	}
	const rb::WideBvh bvh = rb::buildWideBvh(world);
	if (bvh.nodes.size() > rb::kMaxBvhNodes || bvh.maxDepth + 1 > static_cast<uint32_t>(rb::kMaxBvhDepth))
		return fail(ctx, RB_ERR_TOO_LARGE, "rb_set_geometry: BVH beyond the traversal limits (2^24 nodes, depth 48)");
	const size_t nt = canon.size();
	float lo[3] = { 0.0f, 0.0f, 0.0f }, hi[3] = { 0.0f, 0.0f, 0.0f };
	for (size_t j = 0; j < world.size(); j += 3)
		for (int k = 0; k < 3; ++k)
		{
			lo[k] = j ? std::min(lo[k], world[j + k]) : world[j + k];
			hi[k] = j ? std::max(hi[k], world[j + k]) : world[j + k];
		}
	std::vector<float4> triVerts(3 * std::max<size_t>(nt, 1)), objVerts(3 * std::max<size_t>(nt, 1));
	std::vector<uint2> triAux(std::max<size_t>(nt, 1));
	for (size_t j = 0; j < nt; ++j)
	{
		const uint32_t t = bvh.triOrder[j];
		const float* w = world.data() + 9 * t;
		float4 a, b, c;
		a.x = w[0]; a.y = w[1]; a.z = w[2]; std::memcpy(&a.w, &canon[t], 4);
		b.x = w[3]; b.y = w[4]; b.z = w[5]; std::memcpy(&b.w, &inst[t], 4);
		c.x = w[6]; c.y = w[7]; c.z = w[8]; std::memcpy(&c.w, &sbt[t], 4);
		triVerts[3 * j] = a; triVerts[3 * j + 1] = b; triVerts[3 * j + 2] = c;
		const float* ob = objAll.data() + 9 * t;
		for (int k = 0; k < 3; ++k) objVerts[3 * j + k] = make_float4(ob[3 * k], ob[3 * k + 1], ob[3 * k + 2], 0.0f);
		triAux[j] = make_uint2(enc[t], prim[t]);
	}
	std::vector<void*> fresh;
	rb::DevGeometry G{};
	int rc = upload(ctx, fresh, bvh.nodes.empty() ? nullptr : bvh.nodes.data(),
		sizeof(rb::BvhNode) * std::max<size_t>(bvh.nodes.size(), 1), G.nodes);
	if (rc == RB_OK) rc = upload(ctx, fresh, triVerts.data(), sizeof(float4) * triVerts.size(), G.triVerts);
	if (rc == RB_OK) rc = upload(ctx, fresh, triAux.data(), sizeof(uint2) * triAux.size(), G.triAux);
	if (rc == RB_OK) rc = upload(ctx, fresh, normalMatrix.empty() ? nullptr : normalMatrix.data(),
		sizeof(float) * std::max<size_t>(normalMatrix.size(), 9), G.normalMatrix);
	// refit data: object-space vertices, the bottom-up schedule, box scratch
	// and room for the flattened instances' transforms and inverses
	rb::RefitData refit{};
	float4* objDev = nullptr;
	uint32_t* orderDev = nullptr;
	double* boxDev = nullptr;
	float *xfDev = nullptr, *wiDev = nullptr;
	const size_t nInst = std::max<size_t>(instIndex, 1);
	if (rc == RB_OK) rc = upload(ctx, fresh, objVerts.data(), sizeof(float4) * objVerts.size(), objDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, bvh.refitOrder.empty() ? nullptr : bvh.refitOrder.data(),
		sizeof(uint32_t) * std::max<size_t>(bvh.refitOrder.size(), 1), orderDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(double) * 6 * std::max<size_t>(bvh.nodes.size(), 1), boxDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(float) * 12 * nInst, xfDev);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(float) * 12 * nInst, wiDev);
	if (rc == RB_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = fail(ctx, RB_ERR_CUDA, "geometry upload");
	rc = commit(ctx, ctx->geoBufs, fresh, rc);
	if (rc != RB_OK) return rc;
	refit.objVerts = objDev;
	refit.order = orderDev;
	refit.nodeBox = boxDev;
	refit.levelStart = bvh.levelStart;
	ctx->refit = refit;
	ctx->xfDev = xfDev;
	ctx->wiDev = wiDev;
	ctx->geoInstances = g->instance_count;
	ctx->geoSubsets = g->emissive_subset_count;
	G.nodeCount = static_cast<uint32_t>(bvh.nodes.size());
	G.triCount = static_cast<uint32_t>(nt);
	G.rootIsLeaf = bvh.rootIsLeaf ? 1u : 0u;
	G.stackLimit = static_cast<uint32_t>(rb::kTraversalStackEntries);
	if (ctx->injectStackLimit) G.stackLimit = std::min(ctx->injectStackLimit, G.stackLimit);
	ctx->scene.geo = G;
	ctx->geoEmissive = emissivePrim;
	for (int k = 0; k < 3; ++k) { ctx->geoMin[k] = lo[k]; ctx->geoMax[k] = hi[k]; }
	ctx->geoMaxMaterial = 0;
	for (uint32_t s : sbt)
		if (s != 0xFFFFFFFFu) ctx->geoMaxMaterial = std::max(ctx->geoMaxMaterial, s + 1);
	ctx->haveGeometry = true;
	return RB_OK;
}

int rb_update_instances(rb_ctx* ctx, const float* instXf, const float* subsetXf, void* stream)
{
	const NvtxRange range("rb_update_instances");
	if (!ctx) return RB_ERR_INVALID;
	if (!ctx->haveGeometry) return fail(ctx, RB_ERR_NO_SCENE, "rb_update_instances: no geometry");
	if ((ctx->geoInstances && !instXf) || (ctx->geoSubsets && !subsetXf))
		return fail(ctx, RB_ERR_INVALID, "rb_update_instances: null transforms");
	const uint32_t n = ctx->geoSubsets + ctx->geoInstances;
	std::vector<float> xf(12 * std::max<uint32_t>(n, 1), 0.0f), wi(12 * std::max<uint32_t>(n, 1), 0.0f),
		nm(9 * std::max<uint32_t>(n, 1), 0.0f);
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* src = i < ctx->geoSubsets ? subsetXf + 12 * i : instXf + 12 * (i - ctx->geoSubsets);
		for (int k = 0; k < 12; ++k)
			if (!std::isfinite(src[k])) return fail(ctx, RB_ERR_INVALID, "rb_update_instances: non-finite transform");
		std::memcpy(xf.data() + 12 * i, src, sizeof(float) * 12);
		float* w = wi.data() + 12 * i;
		invert3x4(src, w);
		const float m[9] = { w[0], w[4], w[8], w[1], w[5], w[9], w[2], w[6], w[10] };
		std::memcpy(nm.data() + 9 * i, m, sizeof(m));
	}
	cudaSetDevice(ctx->device);
	const cudaStream_t st = pick(ctx, stream);
	if (ctx->instanced)
	{
		// rebuild the top level over the moved instances; the units stay
		std::vector<rb::BvhNode> top;
		std::vector<rb::DevInstance> table;
		uint32_t root = rb::kEmptyChild;
		std::vector<float> boxes;
		int rc = instanceBoxes(ctx, xf, boxes, st);
		if (rc != RB_OK) return fail(ctx, rc, "rb_update_instances: instance boxes");
		rc = buildTopLevel(ctx, xf, wi, boxes, top, table, root);
		if (rc != RB_OK) return fail(ctx, rc, "rb_update_instances: top level (non-finite or too deep)");
		if (top.size() > ctx->topCapacity) return fail(ctx, RB_ERR_TOO_LARGE, "rb_update_instances: top level larger than its slots");
		cudaError_t e2 = cudaSuccess;
		if (!top.empty()) e2 = cudaMemcpyAsync(ctx->topNodes, top.data(), sizeof(rb::BvhNode) * top.size(), cudaMemcpyHostToDevice, st);
		if (e2 == cudaSuccess && !table.empty())
			e2 = cudaMemcpyAsync(ctx->instDev, table.data(), sizeof(rb::DevInstance) * table.size(), cudaMemcpyHostToDevice, st);
		if (e2 == cudaSuccess)
			e2 = cudaMemcpyAsync(const_cast<float*>(ctx->scene.geo.normalMatrix), nm.data(), sizeof(float) * 9 * n,
				cudaMemcpyHostToDevice, st);
		if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(st);
		if (e2 != cudaSuccess) return cudaFail(ctx, e2, "rb_update_instances");
		ctx->scene.geo.topRoot = root;
		ctx->scene.geo.instanceCount = static_cast<uint32_t>(table.size());
		return RB_OK;
	}
	cudaError_t e = cudaMemcpyAsync(ctx->xfDev, xf.data(), sizeof(float) * 12 * n, cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->wiDev, wi.data(), sizeof(float) * 12 * n, cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(const_cast<float*>(ctx->scene.geo.normalMatrix), nm.data(), sizeof(float) * 9 * n,
			cudaMemcpyHostToDevice, st);
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_update_instances: upload");
	rb::launchRefit(ctx->refit, ctx->scene.geo, ctx->xfDev, ctx->wiDev, ctx->status, ctx->shape.smCount, st);
	// the host copies above read pageable memory that goes away on return
	e = cudaStreamSynchronize(st);
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_update_instances");
}

int rb_set_lights(rb_ctx* ctx, const rb_light_tree* t)
{
	if (!ctx || !t) return fail(ctx, RB_ERR_INVALID, "rb_set_lights: null tree");
	if (t->triangle_count && (!t->triangles || !t->bitmasks)) return fail(ctx, RB_ERR_INVALID, "rb_set_lights: null triangles");
	if (t->node_count && (!t->nodes || !t->pointers)) return fail(ctx, RB_ERR_INVALID, "rb_set_lights: null nodes");
	cudaSetDevice(ctx->device);
	// Validate the node graph so device code never indexes out of range.
	const rb::PackedNode* nodes = static_cast<const rb::PackedNode*>(t->nodes);
	for (uint32_t i = 0; i < t->node_count; ++i)
	{
		const uint32_t core = nodes[i].core;
		if (core >> 31)
		{
			const uint32_t cnt = (core >> 27) & 0xFu, off = core & ((1u << 27) - 1u);
			if (cnt == 0 || off + cnt > t->pointer_count) return fail(ctx, RB_ERR_INVALID, "rb_set_lights: leaf out of range");
		}
		else if (core >= t->node_count || i + 1 >= t->node_count)
			return fail(ctx, RB_ERR_INVALID, "rb_set_lights: child index out of range");
	}
	for (uint32_t i = 0; i < t->pointer_count; ++i)
	{
		const uint32_t type = t->pointers[i] >> 30, idx = t->pointers[i] & ((1u << 30) - 1u);
		if (type == rb::kLightTypeTriangle && idx >= t->triangle_count)
			return fail(ctx, RB_ERR_INVALID, "rb_set_lights: light pointer out of range");
	}
	std::vector<void*> fresh;
	rb::DevLights L{};
	// the given (origin-independent) triangles and nodes, and their
	// camera-relative working copies: given - light origin
	rb::EmissiveTri *worldTris = nullptr, *tris = nullptr;
	rb::PackedNode *worldNodes = nullptr, *dn = nullptr;
	rb::TreeNodeU* du = nullptr;
	int rc = upload(ctx, fresh, t->triangles, sizeof(rb::EmissiveTri) * t->triangle_count, worldTris);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(rb::EmissiveTri) * std::max<uint32_t>(t->triangle_count, 1), tris);
	if (rc == RB_OK) rc = upload(ctx, fresh, t->bitmasks, sizeof(uint64_t) * t->triangle_count, L.bitmasks);
	if (rc == RB_OK) rc = upload(ctx, fresh, t->pointers, sizeof(uint32_t) * t->pointer_count, L.pointers);
	if (rc == RB_OK && t->node_count) rc = upload(ctx, fresh, t->nodes, sizeof(rb::PackedNode) * t->node_count, worldNodes);
	if (rc == RB_OK && t->node_count) rc = upload(ctx, fresh, nullptr, sizeof(rb::PackedNode) * t->node_count, dn);
	if (rc == RB_OK && t->node_count) rc = upload(ctx, fresh, nullptr, sizeof(rb::TreeNodeU) * t->node_count, du);
	if (rc == RB_OK)
		rb::launchLightOrigin(worldTris, tris, t->triangle_count, worldNodes, dn, t->node_count, ctx->lightOrigin[0],
			ctx->lightOrigin[1], ctx->lightOrigin[2], ctx->stream);
	if (rc == RB_OK && t->node_count) rb::launchUnpackLightTree(dn, du, t->node_count, ctx->stream);
	if (rc == RB_OK)
	{
		const cudaError_t e = cudaStreamSynchronize(ctx->stream);
		if (e != cudaSuccess) rc = cudaFail(ctx, e, "rb_set_lights: upload");
	}
	rc = commit(ctx, ctx->lightBufs, fresh, rc);
	if (rc != RB_OK) return rc;
	L.triangles = t->triangle_count ? tris : nullptr;
	L.nodes = dn;
	L.unpacked = du;
	L.nodeCount = t->node_count;
	L.triangleCount = t->triangle_count;
	ctx->scene.lights = L;
	ctx->lightWorldTris = worldTris;
	ctx->lightWorldNodes = worldNodes;
	ctx->lightMaxMaterial = 0;
	const rb::EmissiveTri* lt = static_cast<const rb::EmissiveTri*>(t->triangles);
	for (uint32_t i = 0; i < t->triangle_count; ++i) ctx->lightMaxMaterial = std::max(ctx->lightMaxMaterial, lt[i].material + 1);
	return RB_OK;
}

int rb_build_lights(rb_ctx* ctx, uint32_t n, const float* world, const float* flux, const uint32_t* material,
	const uint32_t* primitive, const float* uvs, void* stream)
{
	const NvtxRange range("rb_build_lights");
	if (!ctx) return RB_ERR_INVALID;
	if (n && (!world || !flux || !material || !primitive)) return fail(ctx, RB_ERR_INVALID, "rb_build_lights: null input");
	if (n > (1u << 27) - 1u) return fail(ctx, RB_ERR_INVALID, "rb_build_lights: too many emitters");
	cudaSetDevice(ctx->device);
	const cudaStream_t st = pick(ctx, stream);
	std::vector<void*> fresh;
	rb::DevLights L{};
	rb::EmissiveTri *worldTris = nullptr, *tris = nullptr;
	rb::PackedNode *worldNodes = nullptr, *dn = nullptr;
	rb::TreeNodeU* du = nullptr;
	void* scratch = nullptr;
	uint32_t* dCount = nullptr;
	const size_t nodesMax = std::max<size_t>(2 * static_cast<size_t>(n), 1);
	int rc = upload(ctx, fresh, nullptr, sizeof(rb::EmissiveTri) * std::max<uint32_t>(n, 1), worldTris);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(rb::EmissiveTri) * std::max<uint32_t>(n, 1), tris);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(uint64_t) * std::max<uint32_t>(n, 1), L.bitmasks);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(uint32_t) * std::max<uint32_t>(n, 1), L.pointers);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(rb::PackedNode) * nodesMax, worldNodes);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(rb::PackedNode) * nodesMax, dn);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(rb::TreeNodeU) * nodesMax, du);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, rb_k_build_light_tree_scratch_bytes(n), scratch);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(uint32_t), dCount);
	uint32_t nodeCount = 0;
	if (rc == RB_OK && n)
	{
		// origin-independent records (light origin 0), then the working copies as rb_set_lights makes them
		cudaStreamSynchronize(ctx->stream);
		const double zero[3] = { 0.0, 0.0, 0.0 };
		rc = rb_k_build_light_tree(n, world, flux, material, primitive, uvs, zero, scratch, worldTris, worldNodes,
			const_cast<uint32_t*>(L.pointers), const_cast<uint64_t*>(L.bitmasks), dCount, st);
		if (rc != RB_OK) rc = fail(ctx, rc, "rb_build_lights: build");
		if (rc == RB_OK && cudaMemcpyAsync(&nodeCount, dCount, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess)
			rc = fail(ctx, RB_ERR_CUDA, "rb_build_lights: node count");
		if (rc == RB_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(ctx, RB_ERR_CUDA, "rb_build_lights: build");
		if (rc == RB_OK && (nodeCount == 0 || nodeCount > nodesMax)) rc = fail(ctx, RB_ERR_CUDA, "rb_build_lights: bad tree");
	}
	if (rc == RB_OK && n)
	{
		rb::launchLightOrigin(worldTris, tris, n, worldNodes, dn, nodeCount, ctx->lightOrigin[0], ctx->lightOrigin[1],
			ctx->lightOrigin[2], ctx->stream);
		rb::launchUnpackLightTree(dn, du, nodeCount, ctx->stream);
		const cudaError_t e = cudaStreamSynchronize(ctx->stream);
		if (e != cudaSuccess) rc = cudaFail(ctx, e, "rb_build_lights: install");
	}
	// the largest material index, for the render-time cross-table check
	uint32_t maxMaterial = 0;
	if (rc == RB_OK && n)
	{
		std::vector<uint32_t> mats(n);
		if (cudaMemcpy(mats.data(), material, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = fail(ctx, RB_ERR_CUDA, "rb_build_lights: materials");
		for (uint32_t m : mats) maxMaterial = std::max(maxMaterial, m + 1);
	}
	// the scratch and the count are not kept
	if (rc == RB_OK)
	{
		fresh.erase(std::remove(fresh.begin(), fresh.end(), scratch), fresh.end());
		fresh.erase(std::remove(fresh.begin(), fresh.end(), static_cast<void*>(dCount)), fresh.end());
		cudaFree(scratch);
		cudaFree(dCount);
	}
	rc = commit(ctx, ctx->lightBufs, fresh, rc);
	if (rc != RB_OK) return rc;
	L.triangles = n ? tris : nullptr;
	L.nodes = n ? dn : nullptr;
	L.unpacked = n ? du : nullptr;
	L.nodeCount = nodeCount;
	L.triangleCount = n;
	ctx->scene.lights = L;
	ctx->lightWorldTris = worldTris;
	ctx->lightWorldNodes = worldNodes;
	ctx->lightMaxMaterial = maxMaterial;
	return RB_OK;
}

int rb_set_light_origin(rb_ctx* ctx, const float origin[3], void* stream)
{
	if (!ctx || !origin) return RB_ERR_INVALID;
	for (int k = 0; k < 3; ++k)
		if (!std::isfinite(origin[k])) return fail(ctx, RB_ERR_INVALID, "rb_set_light_origin: non-finite origin");
	cudaSetDevice(ctx->device);
	for (int k = 0; k < 3; ++k) ctx->lightOrigin[k] = origin[k];
	const rb::DevLights& L = ctx->scene.lights;
	if (L.triangleCount + L.nodeCount == 0) return RB_OK;
	const cudaStream_t st = pick(ctx, stream);
	rb::launchLightOrigin(ctx->lightWorldTris, const_cast<rb::EmissiveTri*>(L.triangles), L.triangleCount,
		ctx->lightWorldNodes, const_cast<rb::PackedNode*>(L.nodes), L.nodeCount, origin[0], origin[1], origin[2], st);
	if (L.nodeCount)
		rb::launchUnpackLightTree(L.nodes, const_cast<rb::TreeNodeU*>(L.unpacked), L.nodeCount, st);
	const cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_set_light_origin");
}

int rb_set_envmap(rb_ctx* ctx, const float* rgba, uint32_t w, uint32_t h)
{
	if (!ctx || !rgba) return fail(ctx, RB_ERR_INVALID, "rb_set_envmap: null image");
	if (w < 4 || h < 4 || (w % 4) != 0 || (h % 4) != 0)
		return fail(ctx, RB_ERR_INVALID, "rb_set_envmap: width and height must be multiples of 4");
	if (w > 32768 || h > 32768) return fail(ctx, RB_ERR_INVALID, "rb_set_envmap: image larger than 32768");
	cudaSetDevice(ctx->device);
	std::vector<void*> fresh;
	rb::DevEnvMap E{};
	float4* tex = nullptr;
	uint16_t *cond = nullptr, *marg = nullptr;
	float* integral = nullptr;
	void* scratch = nullptr;
	int rc = upload(ctx, fresh, rgba, sizeof(float4) * w * h, tex);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(uint16_t) * w * h, cond);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(uint16_t) * h, marg);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, sizeof(float), integral);
	if (rc == RB_OK) rc = upload(ctx, fresh, nullptr, rb_envmap_cdf_scratch_bytes(w, h), scratch);
	// kernel mode 0 is the reference order, 1 the float64 sums
	const int kmode = ctx->cdfMode == RB_CDF_REFERENCE ? 0 : 1;
	if (rc == RB_OK)
	{
		rc = rb_envmap_cdf(w, h, reinterpret_cast<const float*>(tex), kmode, scratch, cond, marg, integral, ctx->stream);
		if (rc != RB_OK) rc = fail(ctx, rc, "rb_set_envmap: CDF build failed");
	}
	if (rc == RB_OK)
	{
		const cudaError_t e = cudaStreamSynchronize(ctx->stream);
		if (e != cudaSuccess) rc = cudaFail(ctx, e, "rb_set_envmap");
	}
	rc = commit(ctx, ctx->envBufs, fresh, rc);
	if (rc != RB_OK) return rc;
	E.enabled = 1;
	E.w = w; E.h = h;
	E.width = static_cast<float>(w); E.height = static_cast<float>(h);
	E.integral = integral;
	E.texels = tex;
	E.conditional = cond;
	E.marginal = marg;
	ctx->scene.env = E;
	ctx->envScratch = scratch;
	ctx->envIntegral = integral;
	return RB_OK;
}

int rb_rebuild_envmap_cdf(rb_ctx* ctx, void* stream)
{
	if (!ctx) return RB_ERR_INVALID;
	if (!ctx->scene.env.enabled) return fail(ctx, RB_ERR_NO_SCENE, "rb_rebuild_envmap_cdf: no environment map");
	cudaSetDevice(ctx->device);
	rb::DevEnvMap& E = ctx->scene.env;
	const int kmode = ctx->cdfMode == RB_CDF_REFERENCE ? 0 : 1;
	const int rc = rb_envmap_cdf(E.w, E.h, reinterpret_cast<const float*>(E.texels), kmode, ctx->envScratch,
		const_cast<uint16_t*>(E.conditional), const_cast<uint16_t*>(E.marginal), ctx->envIntegral, pick(ctx, stream));
	return rc == RB_OK ? RB_OK : fail(ctx, rc, "rb_rebuild_envmap_cdf");
}

int rb_clear_envmap(rb_ctx* ctx)
{
	if (!ctx) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	cudaStreamSynchronize(ctx->stream);
	freeAll(ctx->envBufs);
	ctx->scene.env = rb::DevEnvMap{};
	return RB_OK;
}

int rb_set_launch(rb_ctx* ctx, const rb_launch* l)
{
	if (!ctx || !l) return fail(ctx, RB_ERR_INVALID, "rb_set_launch: null launch");
	if (l->width == 0 || l->height == 0) return fail(ctx, RB_ERR_INVALID, "rb_set_launch: empty film");
	if (static_cast<uint64_t>(l->width) * l->height > (1ull << 31)) return fail(ctx, RB_ERR_INVALID, "rb_set_launch: film too large");
	if (l->max_path_depth == 0 || l->max_path_depth > rb::kMaxBounces || l->max_reflected_depth > rb::kMaxBounces ||
		l->max_transmitted_depth > rb::kMaxBounces)
		return fail(ctx, RB_ERR_INVALID, "rb_set_launch: path depth must be in [1, 64]");
	cudaSetDevice(ctx->device);
	rb::DevLaunch& D = ctx->scene.launch;
	D.width = l->width; D.height = l->height;
	D.invWidth = l->inv_width; D.invHeight = l->inv_height;
	D.perspW = l->perspective_scale_w; D.perspH = l->perspective_scale_h;
	D.maxDepth = l->max_path_depth; D.maxReflected = l->max_reflected_depth; D.maxTransmitted = l->max_transmitted_depth;
	for (int k = 0; k < 3; ++k) { D.camU[k] = l->cam_u[k]; D.camV[k] = l->cam_v[k]; D.camW[k] = l->cam_w[k]; }
	D.dof = l->dof_enabled; D.aperture = l->aperture; D.focusDistance = l->focus_distance;
	const size_t pixels = static_cast<size_t>(l->width) * l->height;
	if (pixels != ctx->accumPixels)
	{
		cudaStreamSynchronize(ctx->stream);
		if (ctx->accum) cudaFree(ctx->accum);
		ctx->accum = nullptr;
		ctx->accumPixels = 0;
		const cudaError_t e = devMalloc(ctx, reinterpret_cast<void**>(&ctx->accum), sizeof(double4) * pixels);
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_set_launch: accumulation buffer");
		// finished before the call returns: a render on a caller's stream
		// that adds to the accumulation must not race the fill
		const cudaError_t f = cudaMemsetAsync(ctx->accum, 0, sizeof(double4) * pixels, ctx->stream);
		if (f != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
			return cudaFail(ctx, f != cudaSuccess ? f : cudaGetLastError(), "rb_set_launch: accumulation fill");
		ctx->accumPixels = pixels;
	}
	ctx->haveLaunch = true;
	return RB_OK;
}

} // extern "C"

namespace
{
// Checks shared by the render entry points.
int renderReady(rb_ctx* ctx)
{
	if (!ctx->haveLaunch || !ctx->haveGeometry || !ctx->scene.materials || !ctx->scene.spectra.sensor || !ctx->scene.luts.conductor)
		return fail(ctx, RB_ERR_NO_SCENE, "rb_render: launch, geometry, materials, spectra and LUTs must be set first");
	return RB_OK;
}

// Sample planes per wave of a call rendering `count` planes.
uint32_t planesPerWaveFor(const rb_ctx* ctx, uint32_t count)
{
	const uint32_t pixels = ctx->scene.launch.width * ctx->scene.launch.height;
	const uint64_t cap = ctx->requestedCapacity ? ctx->requestedCapacity : (16u << 20);
	uint32_t planes = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(count, cap / pixels)));
	if (ctx->cache) planes = std::min(planes, ctx->cacheParams.samples_per_wave);
	return planes;
}

// The wave sequence of one render call, launched on st. With dyn (replayed
// waves), the call's offset and fresh flag are read from dyn at run time and
// `offset` is ignored.
int renderWaves(rb_ctx* ctx, uint32_t offset, uint32_t count, cudaStream_t st, const uint32_t* dyn)
{
	const rb::DevScene& sc = ctx->scene;
	const uint32_t pixels = sc.launch.width * sc.launch.height;
	// Wave size: whole sample planes, up to the capacity (default 16M paths,
	// about 6.2 GB of path state).
	const bool cached = ctx->cache != nullptr;
	const rb_cache_params& CP = ctx->cacheParams;
	const uint32_t planesPerWave = planesPerWaveFor(ctx, count);
	const uint32_t wavePaths = planesPerWave * pixels;
	const uint64_t allocs0 = ctx->allocCount;
	int rc = ensureWave(ctx, wavePaths);
	if (rc != RB_OK) return rc;
	const int bounces = static_cast<int>(std::min<uint32_t>(rb::kMaxBounces,
		std::max({ sc.launch.maxDepth, sc.launch.maxReflected, sc.launch.maxTransmitted })));
	rb::PathSoA soa = ctx->soa;
	if (cached)
	{
		rc = ensureCache(ctx, wavePaths, static_cast<uint32_t>(bounces));
		if (rc != RB_OK) return rc;
		const rb::PathSoA& c = ctx->cacheArrays;
		soa.spread = c.spread; soa.trainRec = c.trainRec; soa.cPath = c.cPath; soa.cIn = c.cIn;
		soa.tPath = c.tPath; soa.tIn = c.tIn; soa.tL = c.tL; soa.tT = c.tT; soa.trainCapacity = c.trainCapacity;
	}
	rc = settleFills(ctx, allocs0, st);
	if (rc != RB_OK) return rc;
	// scene box -> [0,1]^3 (cache inputs): the cache's
	// given box, or the geometry's bounds grown by 1 %
	float posMin[3] = {}, posScale[3] = {};
	const bool given = cached && CP.scene_min[0] < CP.scene_max[0] && CP.scene_min[1] < CP.scene_max[1] &&
		CP.scene_min[2] < CP.scene_max[2];
	for (int k = 0; k < 3; ++k)
	{
		float lo = given ? CP.scene_min[k] : ctx->geoMin[k], hi = given ? CP.scene_max[k] : ctx->geoMax[k];
		if (!given)
		{
			const float pad = 0.005f * std::max(hi - lo, 1e-6f);
			lo -= pad;
			hi += pad;
		}
		posMin[k] = lo;
		posScale[k] = hi > lo ? 1.0f / (hi - lo) : 1.0f;
	}
	for (uint32_t done = 0; done < count;)
	{
		const uint32_t planes = std::min(planesPerWave, count - done);
		rb::WaveParams w{};
		w.paths = planes * pixels;
		w.pixels = pixels;
		w.dyn = dyn;
		w.sampleBase = dyn ? done : offset + done;
		w.fresh = dyn ? (done == 0 ? 1u : 0u) : ((offset == 0 && done == 0) ? 1u : 0u);
		w.keepFailed = ctx->failedMode == RB_FAILED_KEEP ? 1u : 0u;
		w.textured = ctx->texturesNeeded ? 1u : 0u;
		if (cached)
		{
			w.cached = 1;
			w.trainOneIn = CP.frozen ? 0u : CP.train_one_in;
			w.trainSeed = rb::mix32(static_cast<uint32_t>(ctx->cacheWaves++) * 0x9E3779B9u + 1u);
			w.spreadC = CP.spread_threshold;
			w.minRoughness = CP.min_roughness;
		}
		for (int k = 0; k < 3; ++k) { w.posMin[k] = posMin[k]; w.posScale[k] = posScale[k]; }
		unsigned long long* cnt = (ctx->statsMode & RB_STATS_COUNT) ? ctx->counters : nullptr;
		rb::LaunchShape shape = ctx->shape;
		shape.items = w.paths;
		cudaMemsetAsync(soa.counts, 0, sizeof(uint32_t) * rb::kCountSlots, st);
		timedStage(ctx, 0, st, [&] { rb::launchGenerate(sc, soa, w, shape, st); });
		for (int b = 0; b < bounces; ++b)
		{
			timedStage(ctx, 1, st, [&] { rb::launchExtend(sc, soa, b, shape, st, cnt); });
			timedStage(ctx, 2, st, [&] { rb::launchSurface(sc, soa, w, b, shape, st, cnt); });
			timedStage(ctx, 2, st, [&] { rb::launchEmission(sc, soa, b, shape, st); });
			timedStage(ctx, 5, st, [&] { rb::launchNee(sc, soa, w, b, shape, st); });
			ctx->launches[5] += 1;   // launchNee runs two light-sample kernels (tree and environment picks)
			timedStage(ctx, 6, st, [&] { rb::launchBsdf(sc, soa, w, b, shape, st); });
			ctx->launches[6] += 1;   // launchBsdf runs the light-sample evaluation and the BxDF sample kernels
			timedStage(ctx, 3, st, [&] { rb::launchShadow(sc, soa, b, shape, st, cnt); });
		}
		if (cached)
		{
			// answer the wave's cache queries, then train on its records
			timedStage(ctx, 7, st, [&] {
				rc = rb::nrc::applyQueries(ctx->cache, std::min(w.paths, soa.queueCap), soa.counts + rb::kCacheQueryCount, soa.cIn, soa.cPath,
					soa.L, soa.T, ctx->cacheCorr, st);
			});
			if (rc != RB_OK) return fail(ctx, rc, "rb_render: cache queries");
			if (!CP.frozen)
			{
				const uint64_t rows = static_cast<uint64_t>(CP.targets_per_sample) * planes;
				const uint32_t steps = static_cast<uint32_t>((rows + CP.batch - 1) / CP.batch);
				timedStage(ctx, 8, st, [&] {
					rb::launchTrainTargets(soa, w.keepFailed, ctx->shape.smCount, st);
					for (uint32_t k = 0; k < steps && rc == RB_OK; ++k)
					{
						rb::launchTrainGather(soa, w.keepFailed, CP.batch, static_cast<uint32_t>(ctx->cacheSteps++),
							ctx->batchIn, ctx->batchTarget, ctx->batchValid, st);
						rc = rb::nrc::trainRows(ctx->cache, CP.batch, ctx->batchValid, ctx->batchIn, ctx->batchTarget, st,
							true, ctx->cacheCorr);
					}
					rb::launchCacheCorrectionUpdate(ctx->cacheCorr, st);
				});
				if (rc != RB_OK) return fail(ctx, rc, "rb_render: cache training");
				// targets, per step the row gather and 9 network kernels (encode, forward, loss,
				// backward, weight gradients, grid backward, two Adam, transposed weights), corrections
				ctx->launches[8] += 10 * steps + 1;
			}
			rb::launchCacheTally(soa, ctx->cacheTally, st);
			++ctx->launches[8];
		}
		timedStage(ctx, 4, st, [&] { rb::launchResolve(sc, soa, w, ctx->accum, shape, st); });
		done += planes;
		ctx->pathsTraced += w.paths;
		++ctx->waves;
	}
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_render launch");
	return RB_OK;
}
} // namespace

extern "C" {

int rb_render(rb_ctx* ctx, uint32_t offset, uint32_t count, void* stream)
{
	const NvtxRange range("rb_render");
	if (!ctx) return RB_ERR_INVALID;
	int rc = renderReady(ctx);
	if (rc != RB_OK) return rc;
	if (count == 0) return RB_OK;
	rc = checkReferences(ctx);
	if (rc != RB_OK) return rc;
	cudaSetDevice(ctx->device);
	return renderWaves(ctx, offset, count, pick(ctx, stream), nullptr);
}

int rb_render_jobs(rb_ctx* const* jobs, uint32_t n, const uint32_t* offsets, const uint32_t* counts,
	const rb_jobs_options* options, void* stream)
{
	const NvtxRange range("rb_render_jobs");
	if (!jobs || n == 0 || !offsets || !counts || !jobs[0]) return RB_ERR_INVALID;
	rb_ctx* host = jobs[0];
	for (uint32_t j = 0; j < n; ++j)
	{
		rb_ctx* c = jobs[j];
		if (!c || c->device != host->device) return fail(host, RB_ERR_INVALID, "rb_render_jobs: jobs must share one device");
		int rc = renderReady(c);
		if (rc == RB_OK) rc = checkReferences(c);
		if (rc != RB_OK) return fail(host, rc, "rb_render_jobs: a job's scene is incomplete");
		if (c->cache) return fail(host, RB_ERR_UNSUPPORTED, "rb_render_jobs: jobs render the plain form");
		if (c->instanced) return fail(host, RB_ERR_UNSUPPORTED, "rb_render_jobs: jobs take flat geometry (RB_ACCEL_FLAT)");
		if (c->scene.launch.width > 65535 || c->scene.launch.height > 65535)
			return fail(host, RB_ERR_INVALID, "rb_render_jobs: film side above 65535");
		if (static_cast<uint64_t>(offsets[j]) + counts[j] > 0xFFFFFFFFull)
			return fail(host, RB_ERR_INVALID, "rb_render_jobs: sample range overflows");
	}
	cudaSetDevice(host->device);
	const cudaStream_t st = pick(host, stream);
	// wave capacity: at least the largest job's plane
	uint32_t maxPixels = 1;
	int bounces = 1;
	for (uint32_t j = 0; j < n; ++j)
	{
		const rb::DevLaunch& L = jobs[j]->scene.launch;
		maxPixels = std::max(maxPixels, L.width * L.height);
		bounces = std::max(bounces, static_cast<int>(std::min<uint32_t>(rb::kMaxBounces,
			std::max({ L.maxDepth, L.maxReflected, L.maxTransmitted }))));
	}
	const uint32_t want = options && options->max_paths_in_flight ? options->max_paths_in_flight
		: (host->requestedCapacity ? host->requestedCapacity : (16u << 20));
	const uint32_t cap = std::max(want, maxPixels);
	// the waves: jobs in order, whole sample planes, chunks of consecutive planes
	struct Wave { uint32_t firstChunk, chunks, paths, pixelSlots; };
	std::vector<uint32_t> lastWave(n, 0);
	std::vector<rb::WaveChunk> chunks;
	std::vector<Wave> waves;
	{
		Wave cur{ 0, 0, 0, 0 };
		for (uint32_t j = 0; j < n; ++j)
		{
			const rb::DevLaunch& L = jobs[j]->scene.launch;
			const uint32_t pixels = L.width * L.height;
			uint32_t done = 0;
			while (done < counts[j])
			{
				uint32_t fit = (cap - cur.paths) / pixels;
				if (fit == 0)
				{
					waves.push_back(cur);
					cur = Wave{ static_cast<uint32_t>(chunks.size()), 0, 0, 0 };
					continue;
				}
				const uint32_t planes = std::min(fit, counts[j] - done);
				rb::WaveChunk c{};
				c.job = j;
				c.slot = cur.paths;
				c.pixel = cur.pixelSlots;
				c.planes = planes;
				c.sample = offsets[j] + done;
				c.fresh = (offsets[j] == 0 && done == 0) ? 1u : 0u;
				c.pixels = pixels;
				c.width = L.width;
				c.height = L.height;
				chunks.push_back(c);
				lastWave[j] = static_cast<uint32_t>(waves.size());
				++cur.chunks;
				cur.paths += planes * pixels;
				cur.pixelSlots += pixels;
				done += planes;
			}
		}
		if (cur.chunks) waves.push_back(cur);
	}
	if (waves.empty()) return RB_OK;
	uint32_t wavePaths = 0;
	for (const Wave& w : waves) wavePaths = std::max(wavePaths, w.paths);
	const uint64_t allocs0 = host->allocCount;
	int rc = ensureWave(host, wavePaths);
	if (rc != RB_OK) return rc;
	// per-path job arrays, job and chunk tables (grown on demand)
	if (host->jobPathCap < host->capacity || host->jobTableCap < n || host->chunkCap < chunks.size())
	{
		cudaStreamSynchronize(host->stream);
		cudaStreamSynchronize(st);
		freeAll(host->jobBufs);
		host->jobPathCap = host->jobTableCap = host->chunkCap = 0;
		rc = upload(host, host->jobBufs, nullptr, sizeof(uint32_t) * host->capacity, host->jobIdx);
		if (rc == RB_OK) rc = upload(host, host->jobBufs, nullptr, sizeof(uint2) * host->capacity, host->jobKey);
		if (rc == RB_OK) rc = upload(host, host->jobBufs, nullptr, sizeof(rb::DevJob) * n, host->jobTable);
		if (rc == RB_OK) rc = upload(host, host->jobBufs, nullptr, sizeof(rb::WaveChunk) * chunks.size(), host->chunkTable);
		if (rc != RB_OK) { freeAll(host->jobBufs); return rc; }
		host->jobPathCap = host->capacity;
		host->jobTableCap = n;
		host->chunkCap = static_cast<uint32_t>(chunks.size());
	}
	rc = settleFills(host, allocs0, st);
	if (rc != RB_OK) return rc;
	std::vector<rb::DevJob> table(n);
	for (uint32_t j = 0; j < n; ++j)
	{
		table[j] = rb::DevJob{};
		table[j].scene = jobs[j]->scene;
		table[j].accum = jobs[j]->accum;
		table[j].keepFailed = jobs[j]->failedMode == RB_FAILED_KEEP ? 1u : 0u;
	}
	// the tables are copied from host memory that lives until the copies are done
	if (cudaMemcpyAsync(host->jobTable, table.data(), sizeof(rb::DevJob) * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
		cudaMemcpyAsync(host->chunkTable, chunks.data(), sizeof(rb::WaveChunk) * chunks.size(), cudaMemcpyHostToDevice, st)
			!= cudaSuccess)
		return fail(host, RB_ERR_CUDA, "rb_render_jobs: tables");
	rb::PathSoA soa = host->soa;
	soa.jobs = host->jobTable;
	soa.job = host->jobIdx;
	soa.key = host->jobKey;
	rb::LaunchShape shape = host->shape;
	const uint32_t pct = options && options->grid_percent ? options->grid_percent : 100u;
	for (int* b : { &shape.blocksGenerate, &shape.blocksExtend, &shape.blocksSurface, &shape.blocksEmission,
			&shape.blocksNee, &shape.blocksBsdf, &shape.blocksBsdfLight, &shape.blocksShadow,
			&shape.blocksResolve })
		*b = std::max(1, static_cast<int>(static_cast<uint64_t>(*b) * pct / 100u));
	const rb::DevScene& sc = host->scene;
	bool textured = false;
	for (uint32_t j = 0; j < n; ++j) textured = textured || jobs[j]->texturesNeeded != 0;
	for (uint32_t k = 0; k < waves.size(); ++k)
	{
		const Wave& wv = waves[k];
		rb::WaveParams w{};
		w.paths = wv.paths;
		w.pixels = 1;
		w.chunks = host->chunkTable + wv.firstChunk;
		w.nChunks = wv.chunks;
		w.pixelSlots = wv.pixelSlots;
		w.textured = textured ? 1u : 0u;
		shape.items = w.paths;
		cudaMemsetAsync(soa.counts, 0, sizeof(uint32_t) * rb::kCountSlots, st);
		rb::launchGenerate(sc, soa, w, shape, st);
		for (int b = 0; b < bounces; ++b)
		{
			rb::launchExtend(sc, soa, b, shape, st, nullptr);
			rb::launchSurface(sc, soa, w, b, shape, st, nullptr);
			rb::launchEmission(sc, soa, b, shape, st);
			rb::launchNee(sc, soa, w, b, shape, st);
			rb::launchBsdf(sc, soa, w, b, shape, st);
			rb::launchShadow(sc, soa, b, shape, st, nullptr);
		}
		rb::launchResolve(sc, soa, w, nullptr, shape, st);
		// kernels launched, by stage as rb_render counts them
		host->launches[0] += 1;
		host->launches[1] += bounces;
		host->launches[2] += 2 * bounces;
		host->launches[5] += 2 * bounces;
		host->launches[6] += 2 * bounces;
		host->launches[3] += bounces;
		host->launches[4] += 1;
		host->pathsTraced += w.paths;
		++host->waves;
		if (options && options->done_events)
			for (uint32_t j = 0; j < n; ++j)
				if (counts[j] && lastWave[j] == k && options->done_events[j])
					cudaEventRecord(static_cast<cudaEvent_t>(options->done_events[j]), st);
	}
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return cudaFail(host, e, "rb_render_jobs");
	return RB_OK;
}

int rb_render_graph(rb_ctx* ctx, uint32_t offset, uint32_t count, void* stream)
{
	const NvtxRange range("rb_render_graph");
	if (!ctx) return RB_ERR_INVALID;
	int rc = renderReady(ctx);
	if (rc != RB_OK) return rc;
	if (count == 0) return RB_OK;
	rc = checkReferences(ctx);
	if (rc != RB_OK) return rc;
	if (ctx->cache || ctx->statsMode) return rb_render(ctx, offset, count, stream);
	cudaSetDevice(ctx->device);
	const cudaStream_t st = pick(ctx, stream);
	// buffers first: the capture must not allocate
	const uint32_t pixels = ctx->scene.launch.width * ctx->scene.launch.height;
	const uint64_t allocs0 = ctx->allocCount;
	rc = ensureWave(ctx, planesPerWaveFor(ctx, count) * pixels);
	if (rc == RB_OK) rc = settleFills(ctx, allocs0, st);
	if (rc != RB_OK) return rc;
	rb_ctx::GraphKey key{};
	key.scene = ctx->scene;
	key.soa = ctx->soa;
	key.accum = ctx->accum;
	key.count = count;
	rb_ctx::Graph* g = nullptr;
	for (auto& c : ctx->graphs)
		if (std::memcmp(&c.key, &key, sizeof(key)) == 0) { g = &c; break; }
	if (!g)
	{
		// capture the wave sequence once for this call shape and scene state
		uint32_t launches[9];
		std::memcpy(launches, ctx->launches, sizeof(launches));
		const uint64_t paths0 = ctx->pathsTraced, waves0 = ctx->waves;
		// captured on the context's own stream (the caller's may be the legacy
		// default stream, which cannot be captured), launched on the caller's
		cudaGraph_t graph = nullptr;
		cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_render_graph: begin capture");
		rc = renderWaves(ctx, 0, count, ctx->stream, ctx->dyn);
		e = cudaStreamEndCapture(ctx->stream, &graph);
		if (rc != RB_OK || e != cudaSuccess)
		{
			if (graph) cudaGraphDestroy(graph);
			return rc != RB_OK ? rc : cudaFail(ctx, e, "rb_render_graph: capture");
		}
		rb_ctx::Graph ng{};
		ng.key = key;
		e = cudaGraphInstantiate(&ng.exec, graph, 0);
		cudaGraphDestroy(graph);
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_render_graph: instantiate");
		for (int k = 0; k < 9; ++k) ng.launches[k] = ctx->launches[k] - launches[k];
		ng.paths = ctx->pathsTraced - paths0;
		ng.waves = ctx->waves - waves0;
		std::memcpy(ctx->launches, launches, sizeof(launches));
		ctx->pathsTraced = paths0;
		ctx->waves = waves0;
		// graphs of an older scene state are not replayed again; up to 8
		// call shapes of the current one are kept
		std::vector<rb_ctx::Graph> keep;
		for (auto& c : ctx->graphs)
		{
			rb_ctx::GraphKey k = c.key;
			k.count = count;
			if (keep.size() < 7 && std::memcmp(&k, &key, sizeof(key)) == 0) keep.push_back(c);
			else cudaGraphExecDestroy(c.exec);
		}
		keep.push_back(ng);
		ctx->graphs.swap(keep);
		g = &ctx->graphs.back();
	}
	rb::launchSetWaveDyn(ctx->dyn, offset, offset == 0 ? 1u : 0u, st);
	const cudaError_t e = cudaGraphLaunch(g->exec, st);
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_render_graph: launch");
	for (int k = 0; k < 9; ++k) ctx->launches[k] += g->launches[k];
	ctx->pathsTraced += g->paths;
	ctx->waves += g->waves;
	return RB_OK;
}

int rb_read_accum(rb_ctx* ctx, double* out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	if (!ctx->accum) return fail(ctx, RB_ERR_NO_SCENE, "rb_read_accum: no accumulation buffer");
	cudaSetDevice(ctx->device);
	cudaError_t e = cudaStreamSynchronize(ctx->stream);
	if (e == cudaSuccess) e = cudaDeviceSynchronize();
	if (e == cudaSuccess) e = cudaMemcpy(out, ctx->accum, sizeof(double4) * ctx->accumPixels, cudaMemcpyDeviceToHost);
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_read_accum");
	return RB_OK;
}

int rb_write_accum(rb_ctx* ctx, const double* in)
{
	if (!ctx || !in) return RB_ERR_INVALID;
	if (!ctx->accum) return fail(ctx, RB_ERR_NO_SCENE, "rb_write_accum: no accumulation buffer");
	cudaSetDevice(ctx->device);
	cudaError_t e = cudaStreamSynchronize(ctx->stream);
	if (e == cudaSuccess) e = cudaDeviceSynchronize();
	if (e == cudaSuccess) e = cudaMemcpy(ctx->accum, in, sizeof(double4) * ctx->accumPixels, cudaMemcpyHostToDevice);
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_write_accum");
	return RB_OK;
}

int rb_accum_device_ptr(rb_ctx* ctx, void** out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	*out = ctx->accum;
	return ctx->accum ? RB_OK : fail(ctx, RB_ERR_NO_SCENE, "no accumulation buffer");
}

int rb_copy_accum_async(rb_ctx* ctx, void* dst, void* stream)
{
	if (!ctx || !dst) return RB_ERR_INVALID;
	if (!ctx->accum) return fail(ctx, RB_ERR_NO_SCENE, "rb_copy_accum_async: no accumulation buffer");
	cudaSetDevice(ctx->device);
	const cudaError_t e = cudaMemcpyAsync(dst, ctx->accum, sizeof(double4) * ctx->accumPixels, cudaMemcpyDefault,
		pick(ctx, stream));
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_copy_accum_async");
}

namespace
{
// updateSamplingState (src/core/rendering_interface.cpp:1859-1872): the
// sub-launch after (offset, count).
void advance(uint32_t total, int mode, uint32_t& offset, uint32_t& count)
{
	offset += count;
	int size = 1;
	if (mode == RB_MODE_GRADUAL)
		size = std::min(static_cast<int>(std::pow(std::max(3, static_cast<int>(count)), 1.5)), 64);
	const int left = std::max(0, static_cast<int>(total) - static_cast<int>(offset));
	count = static_cast<uint32_t>(std::min(left, size));
}
} // namespace

int rb_progressive_plan(uint32_t total, int mode, uint32_t* offsets, uint32_t* counts, uint32_t capacity)
{
	if ((mode != RB_MODE_IMMEDIATE && mode != RB_MODE_GRADUAL) || total > (1u << 30)) return RB_ERR_INVALID;
	if (capacity && (!offsets || !counts)) return RB_ERR_INVALID;
	uint32_t offset = 0, count = total ? 1u : 0u, n = 0;
	while (count)
	{
		if (n < capacity) { offsets[n] = offset; counts[n] = count; }
		++n;
		advance(total, mode, offset, count);
	}
	return static_cast<int>(n);
}

int rb_progressive_restart(rb_ctx* ctx, uint32_t total, int mode)
{
	if (!ctx) return RB_ERR_INVALID;
	if ((mode != RB_MODE_IMMEDIATE && mode != RB_MODE_GRADUAL) || total > (1u << 30))
		return fail(ctx, RB_ERR_INVALID, "rb_progressive_restart: bad mode or sample count");
	ctx->progOffset = 0;
	ctx->progCount = total ? 1u : 0u;
	ctx->progTotal = total;
	ctx->progMode = mode;
	return RB_OK;
}

int rb_progressive_step(rb_ctx* ctx, void* stream, rb_progress* out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	*out = rb_progress{};
	out->total = ctx->progTotal;
	out->processed = ctx->progOffset;
	if (ctx->progCount == 0)
	{
		out->finished = 1;
		return RB_OK;
	}
	const uint32_t offset = ctx->progOffset, count = ctx->progCount;
	const int rc = rb_render(ctx, offset, count, stream);
	if (rc != RB_OK) return rc;
	advance(ctx->progTotal, ctx->progMode, ctx->progOffset, ctx->progCount);
	out->launched_offset = offset;
	out->launched_count = count;
	out->finished = ctx->progCount == 0 ? 1u : 0u;
	return RB_OK;
}

int rb_resolve(rb_ctx* ctx, const float colorspace[9], float exposure_scale, void* stream)
{
	if (!ctx || !colorspace) return RB_ERR_INVALID;
	if (!ctx->accum || !ctx->haveLaunch) return fail(ctx, RB_ERR_NO_SCENE, "rb_resolve: nothing rendered");
	cudaSetDevice(ctx->device);
	const cudaStream_t st = pick(ctx, stream);
	if (ctx->imagePixels != ctx->accumPixels)
	{
		cudaStreamSynchronize(st);
		cudaStreamSynchronize(ctx->stream);
		if (ctx->image) cudaFree(ctx->image);
		ctx->image = nullptr;
		ctx->imagePixels = 0;
		const cudaError_t e = devMalloc(ctx, reinterpret_cast<void**>(&ctx->image), sizeof(uint32_t) * ctx->accumPixels);
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_resolve: image buffer");
		ctx->imagePixels = ctx->accumPixels;
	}
	rb::launchResolveImage(ctx->scene.launch.width, ctx->scene.launch.height, colorspace, exposure_scale, ctx->accum,
		ctx->image, ctx->shape.smCount, st);
	const cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_resolve");
}

int rb_read_image(rb_ctx* ctx, uint8_t* out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	if (!ctx->image) return fail(ctx, RB_ERR_NO_SCENE, "rb_read_image: nothing resolved");
	cudaSetDevice(ctx->device);
	cudaError_t e = cudaDeviceSynchronize();
	if (e == cudaSuccess) e = cudaMemcpy(out, ctx->image, sizeof(uint32_t) * ctx->imagePixels, cudaMemcpyDeviceToHost);
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_read_image");
}

int rb_image_device_ptr(rb_ctx* ctx, void** out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	*out = ctx->image;
	return ctx->image ? RB_OK : fail(ctx, RB_ERR_NO_SCENE, "no resolved image");
}

int rb_clear_accum(rb_ctx* ctx, void* stream)
{
	if (!ctx) return RB_ERR_INVALID;
	if (!ctx->accum) return fail(ctx, RB_ERR_NO_SCENE, "rb_clear_accum: no accumulation buffer");
	cudaSetDevice(ctx->device);
	const cudaError_t e = cudaMemsetAsync(ctx->accum, 0, sizeof(double4) * ctx->accumPixels, pick(ctx, stream));
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_clear_accum");
}

int rb_status(rb_ctx* ctx, rb_device_status* out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	uint32_t h[2] = { 0, 0 };
	cudaError_t e = cudaDeviceSynchronize();
	if (e == cudaSuccess) e = cudaMemcpy(h, ctx->status, sizeof(h), cudaMemcpyDeviceToHost);
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_status");
	out->flags = h[0];
	out->first_code_detail = h[1];
	out->paths_traced = ctx->pathsTraced;
	out->rays_traced = 0;
	return RB_OK;
}

int rb_clear_status(rb_ctx* ctx)
{
	if (!ctx) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	return cudaMemset(ctx->status, 0, 2 * sizeof(uint32_t)) == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}

int rb_synchronize(rb_ctx* ctx)
{
	if (!ctx) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	const cudaError_t e = cudaStreamSynchronize(ctx->stream);
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_synchronize");
}

int rb_set_stats(rb_ctx* ctx, uint32_t mode)
{
	if (!ctx || (mode & ~(RB_STATS_COUNT | RB_STATS_TIME))) return fail(ctx, RB_ERR_INVALID, "rb_set_stats: bad mode");
	cudaSetDevice(ctx->device);
	if ((mode & RB_STATS_COUNT) && !ctx->counters)
	{
		const cudaError_t e = devMalloc(ctx, reinterpret_cast<void**>(&ctx->counters), 7 * sizeof(unsigned long long));
		if (e != cudaSuccess) return cudaFail(ctx, e, "rb_set_stats");
		cudaMemset(ctx->counters, 0, 7 * sizeof(unsigned long long));
	}
	ctx->statsMode = mode;
	return RB_OK;
}

int rb_get_stats(rb_ctx* ctx, rb_render_stats* out)
{
	if (!ctx || !out) return RB_ERR_INVALID;
	cudaSetDevice(ctx->device);
	cudaError_t e = cudaStreamSynchronize(ctx->stream);
	if (e == cudaSuccess) e = cudaDeviceSynchronize();
	if (e != cudaSuccess) return cudaFail(ctx, e, "rb_get_stats");
	*out = rb_render_stats{};
	if (ctx->counters)
	{
		unsigned long long c[7] = {};
		cudaMemcpy(c, ctx->counters, sizeof(c), cudaMemcpyDeviceToHost);
		cudaMemset(ctx->counters, 0, sizeof(c));
		out->extend_rays = c[0]; out->extend_nodes = c[1]; out->extend_tris = c[2];
		out->shadow_rays = c[3]; out->shadow_nodes = c[4]; out->shadow_tris = c[5];
		out->surface_records = c[6];
	}
	drainTimed(ctx);
	const double* ms = ctx->stageMs;
	out->ms_generate = ms[0]; out->ms_extend = ms[1]; out->ms_shade = ms[2] + ms[5] + ms[6];
	out->ms_shadow = ms[3]; out->ms_resolve = ms[4];
	out->ms_surface = ms[2]; out->ms_nee = ms[5]; out->ms_bsdf = ms[6];
	out->launches_generate = ctx->launches[0]; out->launches_extend = ctx->launches[1];
	out->launches_shade = ctx->launches[2]; out->launches_shadow = ctx->launches[3]; out->launches_resolve = ctx->launches[4];
	out->launches_nee = ctx->launches[5]; out->launches_bsdf = ctx->launches[6];
	out->waves = ctx->waves;
	for (int k = 0; k < 7; ++k) { ctx->launches[k] = 0; ctx->stageMs[k] = 0.0; }
	ctx->waves = 0;
	return RB_OK;
}

// ---- per-function entry points ----------------------------------------
#define RB_K_CHECK(cond) do { if (!(cond)) return RB_ERR_INVALID; } while (0)
static int lastLaunch()
{
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}

int rb_k_sobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash, const uint32_t* bounce,
	const uint32_t* dim, float* out, void* stream)
{
	RB_K_CHECK(dims >= 1 && dims <= 3);
	if (n == 0) return RB_OK;
	RB_K_CHECK(sample && hash && bounce && dim && out);
	rb::launchSobol(n, dims, sample, hash, bounce, dim, out, static_cast<cudaStream_t>(stream));
	return lastLaunch();
}
int rb_k_pixel_hash(uint32_t n, const uint32_t* x, const uint32_t* y, uint32_t* out, void* stream)
{
	if (n == 0) return RB_OK;
	RB_K_CHECK(x && y && out);
	rb::launchPixelHash(n, x, y, out, static_cast<cudaStream_t>(stream));
	return lastLaunch();
}
int rb_k_wavelengths(uint32_t n, const float* u, float* lambda, float* pdf, void* stream)
{
	if (n == 0) return RB_OK;
	RB_K_CHECK(u && lambda && pdf);
	rb::launchWavelengths(n, u, lambda, pdf, static_cast<cudaStream_t>(stream));
	return lastLaunch();
}
int rb_k_camera_ray(rb_ctx* ctx, uint32_t n, const float* pixel, const float* fuv, const float* luv, float* out, void* stream)
{
	RB_K_CHECK(ctx && ctx->haveLaunch);
	if (n == 0) return RB_OK;
	RB_K_CHECK(pixel && fuv && luv && out);
	rb::launchCameraRay(ctx->scene, n, pixel, fuv, luv, out, pick(ctx, stream));
	return lastLaunch();
}
int rb_k_texture_sample(rb_ctx* ctx, uint32_t texture, uint32_t n, const float* uv, float* soft, float* hw,
	void* stream)
{
	RB_K_CHECK(ctx && texture < ctx->scene.textureCount);
	if (n == 0) return RB_OK;
	RB_K_CHECK(uv && soft && hw);
	cudaSetDevice(ctx->device);
	const cudaStream_t st = pick(ctx, stream);
	rb::DevTexture t{};
	if (cudaMemcpy(&t, ctx->scene.textures + texture, sizeof(t), cudaMemcpyDeviceToHost) != cudaSuccess)
		return fail(ctx, RB_ERR_CUDA, "rb_k_texture_sample: texture record");
	const cudaChannelFormatDesc fmt = t.channels == 1 ? cudaCreateChannelDesc<unsigned char>()
	                                                  : cudaCreateChannelDesc<uchar4>();
	cudaArray_t arr = nullptr;
	cudaTextureObject_t obj = 0;
	cudaError_t e = cudaMallocArray(&arr, &fmt, t.width, t.height);
	if (e == cudaSuccess)
		e = cudaMemcpy2DToArray(arr, 0, 0, t.data, static_cast<size_t>(t.width) * t.channels,
			static_cast<size_t>(t.width) * t.channels, t.height, cudaMemcpyDeviceToDevice);
	if (e == cudaSuccess)
	{
		cudaResourceDesc res{};
		res.resType = cudaResourceTypeArray;
		res.res.array.array = arr;
		auto mode = [](uint32_t m) {
			return m == RB_TEXADDR_WRAP ? cudaAddressModeWrap : (m == RB_TEXADDR_MIRROR ? cudaAddressModeMirror : cudaAddressModeClamp);
		};
		cudaTextureDesc td{};
		td.addressMode[0] = mode(t.addrU);
		td.addressMode[1] = mode(t.addrV);
		td.filterMode = t.filter == RB_TEXFILTER_LINEAR ? cudaFilterModeLinear : cudaFilterModePoint;
		td.readMode = cudaReadModeNormalizedFloat;
		td.normalizedCoords = 1;
		td.sRGB = t.srgb ? 1 : 0;
		e = cudaCreateTextureObject(&obj, &res, &td, nullptr);
	}
	if (e == cudaSuccess)
	{
		rb::launchTextureSample(ctx->scene, texture, obj, n, uv, soft, hw, st);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	if (obj) cudaDestroyTextureObject(obj);
	if (arr) cudaFreeArray(arr);
	return e == cudaSuccess ? RB_OK : cudaFail(ctx, e, "rb_k_texture_sample");
}
int rb_k_bxdf(rb_ctx* ctx, uint32_t n, rb_bxdf_case* cases, void* stream)
{
	RB_K_CHECK(ctx && ctx->scene.materials && ctx->scene.luts.conductor && ctx->scene.spectra.basis);
	if (n == 0) return RB_OK;
	RB_K_CHECK(cases);
	rb::launchBxdfCases(ctx->scene, n, cases, pick(ctx, stream));
	return lastLaunch();
}
int rb_k_light_tree(rb_ctx* ctx, uint32_t n, rb_light_case* cases, void* stream)
{
	RB_K_CHECK(ctx && (ctx->scene.lights.nodes || ctx->scene.env.enabled));
	if (n == 0) return RB_OK;
	RB_K_CHECK(cases);
	rb::launchLightCases(ctx->scene, n, cases, pick(ctx, stream));
	return lastLaunch();
}
int rb_k_resolve(uint32_t width, uint32_t height, const float* colorspace, float exposure_scale,
	const double* render_data, uint8_t* out_rgba, void* stream)
{
	if (width == 0 || height == 0) return RB_OK;
	RB_K_CHECK(colorspace && render_data && out_rgba);
	RB_K_CHECK(static_cast<uint64_t>(width) * height <= (1ull << 31));
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	rb::launchResolveImage(width, height, colorspace, exposure_scale, reinterpret_cast<const double4*>(render_data),
		reinterpret_cast<uint32_t*>(out_rgba), sms, static_cast<cudaStream_t>(stream));
	return lastLaunch();
}
int rb_k_offset_point(uint32_t n, const float* p, const float* nrm, float* out, void* stream)
{
	if (n == 0) return RB_OK;
	RB_K_CHECK(p && nrm && out);
	rb::launchOffsetPoint(n, p, nrm, out, static_cast<cudaStream_t>(stream));
	return lastLaunch();
}
int rb_k_oct_encode(uint32_t n, const float* v, uint32_t* out, void* stream)
{
	if (n == 0) return RB_OK;
	RB_K_CHECK(v && out);
	rb::launchOctEncode(n, v, out, static_cast<cudaStream_t>(stream));
	return lastLaunch();
}
int rb_k_oct_decode(uint32_t n, const uint32_t* code, float* out, void* stream)
{
	if (n == 0) return RB_OK;
	RB_K_CHECK(code && out);
	rb::launchOctDecode(n, code, out, static_cast<cudaStream_t>(stream));
	return lastLaunch();
}
int rb_k_trace(rb_ctx* ctx, uint32_t n, const float* rays, uint32_t* payload, float* t, int32_t* tri, void* stream)
{
	RB_K_CHECK(ctx && ctx->haveGeometry);
	if (checkReferences(ctx) != RB_OK) return RB_ERR_INVALID;
	if (n == 0) return RB_OK;
	RB_K_CHECK(rays && payload && t && tri);
	rb::launchTrace(ctx->scene, n, rays, payload, t, tri, pick(ctx, stream));
	return lastLaunch();
}
int rb_k_occluded(rb_ctx* ctx, uint32_t n, const float* rays, const float* tmax, uint32_t* out, void* stream)
{
	RB_K_CHECK(ctx && ctx->haveGeometry);
	if (n == 0) return RB_OK;
	RB_K_CHECK(rays && tmax && out);
	rb::launchOccluded(ctx->scene, n, rays, tmax, out, pick(ctx, stream));
	return lastLaunch();
}

} // extern "C"
