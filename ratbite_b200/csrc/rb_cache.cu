// Radiance-cache form of the wavefront: the training targets of a wave and
// the draw of training rows from them. The queries themselves are answered
// by the cache's fused inference kernel (rb_nrc.cu), and the vertices are
// queued by the shading kernels (rb_kernels.cu, cacheVertex).

#include <cstdint>

#include "rb_launch.cuh"
#include "rb_nrc_internal.h"
#include "rb_wavefront.h"
#include "ratbite_b200_nrc.h"

namespace rb
{
namespace
{
// Target of a record: the radiance the path gathered after the vertex
// (emission on arrival excluded), divided by the throughput at the vertex,
// per hero wavelength; non-finite or zero-throughput components give 0. A
// path that ends with the terminated flag is dropped whole at resolve
// (kResolve, unless keepFailed), so its targets are then 0.
__global__ void __launch_bounds__(kThreads) kTrainTargets(PathSoA s, uint32_t keepFailed)
{
	const uint32_t n = min(s.counts[kTrainRecordCount], s.trainCapacity);
	for (uint32_t r = gtid(); r < n; r += gstride())
	{
		const uint32_t p = s.tPath[r] & kRecordPathMask;
		if (!keepFailed && (s.fd[p].x & PF_PATH_TERMINATED))
		{
			s.tL[r] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			continue;
		}
		const float4 Lf = s.L[p], Lr = s.tL[r], T = s.tT[r];
		auto tgt = [](float lf, float lr, float t) {
			const float v = t > 0.0f ? (lf - lr) / t : 0.0f;
			return isfinite(v) ? v : 0.0f;
		};
		s.tL[r] = make_float4(tgt(Lf.x, Lr.x, T.x), tgt(Lf.y, Lr.y, T.y), tgt(Lf.z, Lr.z, T.z), tgt(Lf.w, Lr.w, T.w));
	}
}

// n training rows drawn uniformly (with replacement) from the wave's records:
// inputs, and targets as rows of 8 floats (radiance, drop: 1 if the path was
// dropped, drop-bias class of a record at the would-be query vertex: 1
// lit-prefix path, 2 other path, 0 not such a record; 2 unused).
__global__ void __launch_bounds__(kThreads) kTrainGather(PathSoA s, uint32_t keepFailed, uint32_t n, uint32_t step,
	float* __restrict__ in, float4* __restrict__ target, uint32_t* __restrict__ valid)
{
	const uint32_t count = min(s.counts[kTrainRecordCount], s.trainCapacity);
	const uint32_t salt = mix32(step * 0x9E3779B9u + 0x632BE5ABu);
	if (gtid() == 0) *valid = count ? n : 0u;
	for (uint32_t j = gtid(); j < n; j += gstride())
	{
		float* row = in + static_cast<size_t>(kNrcInputs) * j;
		if (count == 0)
		{
			for (int k = 0; k < kNrcInputs; ++k) row[k] = 0.0f;
			target[2 * j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			target[2 * j + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			continue;
		}
		const uint32_t r = mix32(j ^ salt) % count;
		const float* src = s.tIn + static_cast<size_t>(kNrcInputs) * r;
		for (int k = 0; k < kNrcInputs; ++k) row[k] = src[k];
		target[2 * j] = s.tL[r];
		const uint32_t tp = s.tPath[r];
		const float drop = !keepFailed && (s.fd[tp & kRecordPathMask].x & PF_PATH_TERMINATED) ? 1.0f : 0.0f;
		const float cls = (tp & kLitPrefixBit) ? 1.0f : ((tp & kQueryRecordBit) ? 2.0f : 0.0f);
		target[2 * j + 1] = make_float4(drop, cls, 0.0f, 0.0f);
	}
}

// Folds the wave's sums into the corrections (rb::nrc::kCorr* layout): the
// mean drop residual of each class, and the ratio of the radiance targets'
// sum to the clamped predictions' (kept within [0.5, 2]); a running mean
// over the first 33 waves, then an exponential average with weight 0.03.
// Cornell box at 1920 x 1080 (relative RMSE at 1024 spp, mean of five runs
// each): weight 0.1 0.108, 0.03 0.107, 0.01 0.110 (early estimates from a
// barely trained network weigh too long).
#ifndef RB_CORR_MIN_WEIGHT
#define RB_CORR_MIN_WEIGHT 0.03f
#endif
__global__ void kCacheCorrectionUpdate(float* state)
{
	for (int c = 0; c < 3; ++c)
	{
		float* st = state + 4 * c;
		if (st[1] > 0.0f)
		{
			const float v = c < 2 ? st[0] / st[1] : fminf(fmaxf(st[0] / st[1], 0.5f), 2.0f);
			const float a = fmaxf(1.0f / (st[3] + 1.0f), RB_CORR_MIN_WEIGHT);
			st[2] += a * (v - st[2]);
			st[3] += 1.0f;
		}
		st[0] = 0.0f;
		st[1] = 0.0f;
	}
}

__global__ void kCacheTally(PathSoA s, unsigned long long* tally)
{
	tally[0] += s.counts[kCacheQueryCount];
	tally[1] += min(s.counts[kTrainRecordCount], s.trainCapacity);
}
} // namespace

void launchCacheCorrectionUpdate(float* state, cudaStream_t st)
{
	kCacheCorrectionUpdate<<<1, 1, 0, st>>>(state);
}

void launchCacheTally(const PathSoA& s, unsigned long long* tally, cudaStream_t st)
{
	kCacheTally<<<1, 1, 0, st>>>(s, tally);
}

void launchTrainTargets(const PathSoA& s, uint32_t keepFailed, int smCount, cudaStream_t st)
{
	kTrainTargets<<<smCount * 8, kThreads, 0, st>>>(s, keepFailed);
}

void launchTrainGather(const PathSoA& s, uint32_t keepFailed, uint32_t n, uint32_t step, float* in, float* target,
	uint32_t* valid, cudaStream_t st)
{
	kTrainGather<<<gridFor(n), kThreads, 0, st>>>(s, keepFailed, n, step, in, reinterpret_cast<float4*>(target), valid);
}
} // namespace rb
