// Oracle test infrastructure (not product code).
//
// Runs the reference's own environment-map CDF kernels (src/kernels/cdf.cu),
// compiled device-only for sm_100a into oracle/_ref/cdf.cubin, through the
// CUDA driver API exactly as RenderingInterface does it
// (createCDFBuildProgram :437, loadEnvironmentMap :1339-1432): RGBA float
// texture in a CUDA array read through a surface object,
// buildCDFLatLongRGBUpTo{4k,8k,16k,32k} launched with cuLaunchKernel on grid
// (1, h) with the width-dependent block size, the integral divided by w*h on
// the host, then invertCDFToIndices on grid (h+1, ceil(max(w,h)/1024)) x 1024.
// It is the checker of the product's CDF kernel and the timed reference arm
// of the CDF row.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace
{
CUmodule g_module = nullptr;
CUfunction g_build[4] = {};
CUfunction g_invert = nullptr;

int ensureModule(const char* cubinPath)
{
	if (g_module) return 0;
	cudaFree(nullptr);   // initialise the runtime's primary context first
	if (cuModuleLoad(&g_module, cubinPath) != CUDA_SUCCESS) return -3;
	const char* names[4] = { "buildCDFLatLongRGBUpTo4k", "buildCDFLatLongRGBUpTo8k", "buildCDFLatLongRGBUpTo16k",
	                         "buildCDFLatLongRGBUpTo32k" };
	for (int i = 0; i < 4; ++i)
		if (cuModuleGetFunction(&g_build[i], g_module, names[i]) != CUDA_SUCCESS) return -3;
	if (cuModuleGetFunction(&g_invert, g_module, "invertCDFToIndices") != CUDA_SUCCESS) return -3;
	return 0;
}

struct RefCdfRun
{
	cudaArray_t array = nullptr;
	cudaSurfaceObject_t surface = 0;
	float* cdfX = nullptr;
	float* cdfY = nullptr;
	float* integral = nullptr;
	int* counter = nullptr;
	int w = 0, h = 0;

	int prepare(const float* dRgba, int width, int height)
	{
		w = width; h = height;
		cudaChannelFormatDesc desc = cudaCreateChannelDesc<float4>();
		if (cudaMallocArray(&array, &desc, w, h, cudaArraySurfaceLoadStore) != cudaSuccess) return -2;
		if (cudaMemcpy2DToArray(array, 0, 0, dRgba, sizeof(float4) * w, sizeof(float4) * w, h,
				cudaMemcpyDeviceToDevice) != cudaSuccess) return -2;
		cudaResourceDesc rd{};
		rd.resType = cudaResourceTypeArray;
		rd.res.array.array = array;
		if (cudaCreateSurfaceObject(&surface, &rd) != cudaSuccess) return -2;
		if (cudaMalloc(&cdfX, sizeof(float) * w * h) != cudaSuccess) return -2;
		if (cudaMalloc(&cdfY, sizeof(float) * h) != cudaSuccess) return -2;
		if (cudaMalloc(&integral, sizeof(float)) != cudaSuccess) return -2;
		if (cudaMalloc(&counter, sizeof(int)) != cudaSuccess) return -2;
		return 0;
	}
	int run(uint16_t* dCond, uint16_t* dMarg, float* hIntegral)
	{
		cudaMemset(counter, 0, sizeof(int));
		const int numElements = (w + 3) / 4;
		const int block = numElements <= 256 ? 256 : (numElements <= 512 ? 512 : 1024);
		const int blocksPerRow = (numElements + block - 1) / block;
		int fi;
		if (blocksPerRow == 1) fi = 0;
		else if (blocksPerRow == 2) fi = 1;
		else if (blocksPerRow <= 4) fi = 2;
		else if (blocksPerRow <= 8) fi = 3;
		else return -1;
		void* buildParams[] = { &w, &h, &surface, &cdfX, &cdfY, &integral, &counter };
		if (cuLaunchKernel(g_build[fi], 1, h, 1, block, 1, 1, block * sizeof(float), nullptr, buildParams, nullptr) != CUDA_SUCCESS)
			return -2;
		if (hIntegral)
		{
			float hi = 0.0f;
			if (cudaMemcpy(&hi, integral, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
			*hIntegral = hi / (static_cast<float>(w) * static_cast<float>(h));
		}
		void* invParams[] = { &w, &h, &cdfX, &cdfY, &dCond, &dMarg };
		const unsigned gy = static_cast<unsigned>(((w > h ? w : h) + 1023) / 1024);
		if (cuLaunchKernel(g_invert, h + 1, gy, 1, 1024, 1, 1, 0, nullptr, invParams, nullptr) != CUDA_SUCCESS)
			return -2;
		return 0;
	}
	void release()
	{
		if (surface) cudaDestroySurfaceObject(surface);
		if (array) cudaFreeArray(array);
		cudaFree(cdfX); cudaFree(cdfY); cudaFree(integral); cudaFree(counter);
	}
};
} // namespace

extern "C" int rbrefgpu_envmap_cdf(const char* cubinPath, int w, int h, const float* dRgba, uint16_t* dCond,
	uint16_t* dMarg, float* hIntegral)
{
	int rc = ensureModule(cubinPath);
	if (rc != 0) return rc;
	RefCdfRun r;
	rc = r.prepare(dRgba, w, h);
	if (rc == 0) rc = r.run(dCond, dMarg, hIntegral);
	if (cudaDeviceSynchronize() != cudaSuccess && rc == 0) rc = -2;
	r.release();
	return rc;
}

// Mean milliseconds per rebuild (build + invert) over `iters` rebuilds after
// `warmup`, each timed alone with CUDA events on the default stream. Before
// each timed rebuild `flushBytes` of `flush` (device memory larger than L2,
// or null) are overwritten so that the image is read from HBM, not L2.
extern "C" float rbrefgpu_envmap_cdf_time(const char* cubinPath, int w, int h, const float* dRgba, uint16_t* dCond,
	uint16_t* dMarg, int warmup, int iters, void* flush, size_t flushBytes)
{
	if (ensureModule(cubinPath) != 0 || iters <= 0) return -1.0f;
	RefCdfRun r;
	if (r.prepare(dRgba, w, h) != 0) { r.release(); return -1.0f; }
	for (int i = 0; i < warmup; ++i) r.run(dCond, dMarg, nullptr);
	cudaEvent_t a, b;
	cudaEventCreate(&a); cudaEventCreate(&b);
	float total = 0.0f;
	bool ok = true;
	for (int i = 0; i < iters && ok; ++i)
	{
		if (flush) cudaMemsetAsync(flush, i & 0xFF, flushBytes, 0);
		cudaEventRecord(a, 0);
		ok = r.run(dCond, dMarg, nullptr) == 0;
		cudaEventRecord(b, 0);
		cudaEventSynchronize(b);
		float ms = 0.0f;
		cudaEventElapsedTime(&ms, a, b);
		total += ms;
	}
	cudaEventDestroy(a); cudaEventDestroy(b);
	r.release();
	return ok ? total / static_cast<float>(iters) : -1.0f;
}
