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
// Evaluates min(*count, cap) query rows (kNrcInputs floats each) and sets
// L[p] = L[p] (1 - q) + T[p] max(y, 0) for p = path[r] & 0x7FFFFFFF, with y
// the radiance outputs and q the drop probability (output 4) plus *dropBias
// where path[r]'s high bit is set (dropBias may be null), stream-ordered.
int applyQueries(rb_nrc* h, uint32_t cap, const uint32_t* count, const float* inputs, const uint32_t* path, float4* L,
	const float4* T, const float* dropBias, cudaStream_t st);
// One optimisation step on n rows of which the first min(*valid, n) count
// (valid may be null: all n). Targets: rows of 4 radiance values, or with
// withDrop rows of 8 (radiance, drop probability, flag, 2 unused); where the
// flag is set, (drop target - predicted drop) is added to dropResid[0] and
// 1 to dropResid[1] (dropResid may be null).
int trainRows(rb_nrc* h, uint32_t n, const uint32_t* valid, const float* inputs, const float* targets, cudaStream_t st,
	bool withDrop, float* dropResid = nullptr);
// Device scalar with the mean loss of the latest step.
const float* lossDevice(const rb_nrc* h);
int deviceOf(const rb_nrc* h);
} // namespace nrc
} // namespace rb
