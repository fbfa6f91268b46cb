// Entry points of the radiance cache that the renderer calls with device-side
// row counts (no host synchronisation between the wave and the network).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ratbite_b200_nrc.h"

namespace rb
{
namespace nrc
{
// Correction state of the renderer's cached form (device floats), measured
// on the training rows drawn at the vertex where the cache would have ended
// a training path (its class: 1 the camera ray hit an emitter, 2 any other
// path) and applied to the queries:
//   kCorrDropLit, kCorrDropOther: sum and count of (drop target - predicted
//     drop probability) of the wave's rows of the class, the correction added
//     to the class's predicted drop probability, waves seen;
//   kCorrRadiance: sum of the radiance targets and of the clamped radiance
//     predictions over the wave's rows of both classes, the scale applied to
//     the queries' radiance, waves seen.
constexpr int kCorrDropLit = 0, kCorrDropOther = 4, kCorrRadiance = 8, kCorrFloats = 12;
// Evaluates min(*count, cap) query rows (kNrcInputs floats each) and sets
// L[p] = L[p] (1 - q) + T[p] s max(y, 0) for p = path[r] & 0x7FFFFFFF, with y
// the radiance outputs, q the drop probability (output 4) plus the drop
// correction of the path's class (path[r]'s high bit: the camera ray hit an
// emitter) and s the radiance scale, both from the correction state `corr`
// (null: none), stream-ordered.
int applyQueries(rb_nrc* h, uint32_t cap, const uint32_t* count, const float* inputs, const uint32_t* path, float4* L,
	const float4* T, const float* corr, cudaStream_t st);
// One optimisation step on n rows of which the first min(*valid, n) count
// (valid may be null: all n). Targets: rows of 4 radiance values, or with
// withDrop rows of 8 (radiance, drop probability, class, 2 unused); rows of
// class 1 or 2 add to the sums of the correction state `corr` (may be null).
int trainRows(rb_nrc* h, uint32_t n, const uint32_t* valid, const float* inputs, const float* targets, cudaStream_t st,
	bool withDrop, float* corr = nullptr);
// Device scalar with the mean loss of the latest step.
const float* lossDevice(const rb_nrc* h);
int deviceOf(const rb_nrc* h);
} // namespace nrc
} // namespace rb
