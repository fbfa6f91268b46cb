// Environment-map CDF build (rb_envmap.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace rb
{
size_t envCdfScratchBytes(uint32_t w, uint32_t h);
int envCdfLaunch(uint32_t w, uint32_t h, const float* rgba, int mode, void* scratch, uint16_t* cond, uint16_t* marg,
	float* integral, cudaStream_t st);
} // namespace rb
