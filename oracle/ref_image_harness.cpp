// Oracle test infrastructure (not product code).
//
// Runs the reference's own resolve kernel (renderResolve with the AgX
// tonemap, src/kernels/image.cu:16-121), compiled device-only for sm_100a
// into oracle/_ref/image.cubin, through the CUDA driver API as
// RenderingInterface::resolveRender does it (src/core/rendering_interface.cpp
// :1512-1532): 16x16 blocks, parameters (width, height, glm::mat3 colorspace
// transform by value, exposure scale, renderData), output through a surface
// object over a uchar4 CUDA array. The GL interop that the reference maps the
// array from is replaced by a plain CUDA array, and the result is copied to
// host memory. It is the checker of the product's resolve kernel.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace
{
CUmodule g_module = nullptr;
CUfunction g_resolve = nullptr;

int ensureModule(const char* cubinPath)
{
	if (g_module) return 0;
	cudaFree(nullptr);   // initialise the runtime's primary context first
	if (cuModuleLoad(&g_module, cubinPath) != CUDA_SUCCESS) return -3;
	if (cuModuleGetFunction(&g_resolve, g_module, "renderResolve") != CUDA_SUCCESS) return -3;
	return 0;
}

struct Mat3 { float m[9]; };   // glm::mat3, column-major
}

extern "C" {

// dRender: device pointer to w*h double4. colorspace: 9 floats, column-major.
// hOut: host buffer of w*h*4 bytes.
int rbrefgpu_resolve(const char* cubinPath, uint32_t w, uint32_t h, const float* colorspace, float exposureScale,
	const double* dRender, uint8_t* hOut)
{
	int rc = ensureModule(cubinPath);
	if (rc) return rc;
	cudaChannelFormatDesc desc = cudaCreateChannelDesc<uchar4>();
	cudaArray_t array = nullptr;
	cudaSurfaceObject_t surface = 0;
	if (cudaMallocArray(&array, &desc, w, h, cudaArraySurfaceLoadStore) != cudaSuccess) return -2;
	cudaResourceDesc rd{};
	rd.resType = cudaResourceTypeArray;
	rd.res.array.array = array;
	rc = cudaCreateSurfaceObject(&surface, &rd) == cudaSuccess ? 0 : -2;
	if (rc == 0)
	{
		Mat3 cs;
		for (int i = 0; i < 9; ++i) cs.m[i] = colorspace[i];
		uint32_t width = w, height = h;
		float exposure = exposureScale;
		const double* data = dRender;
		void* params[] = { &width, &height, &cs, &exposure, &data, &surface };
		if (cuLaunchKernel(g_resolve, (w + 15) / 16, (h + 15) / 16, 1, 16, 16, 1, 0, nullptr, params, nullptr)
				!= CUDA_SUCCESS)
			rc = -4;
		else if (cudaMemcpy2DFromArray(hOut, sizeof(uchar4) * w, array, 0, 0, sizeof(uchar4) * w, h,
					 cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = -2;
	}
	if (surface) cudaDestroySurfaceObject(surface);
	cudaFreeArray(array);
	return rc;
}

// Mean milliseconds per renderResolve launch over `iters` launches after
// `warmup`, each timed alone with CUDA events on the default stream (output
// stays in the CUDA array; nothing is copied back). Before each timed launch
// `flushBytes` of `flush` (device memory larger than L2, or null) are
// overwritten so that the accumulation is read from HBM, not L2.
float rbrefgpu_resolve_time(const char* cubinPath, uint32_t w, uint32_t h, const float* colorspace,
	float exposureScale, const double* dRender, int warmup, int iters, void* flush, size_t flushBytes)
{
	if (ensureModule(cubinPath) != 0 || iters <= 0) return -1.0f;
	cudaChannelFormatDesc desc = cudaCreateChannelDesc<uchar4>();
	cudaArray_t array = nullptr;
	cudaSurfaceObject_t surface = 0;
	if (cudaMallocArray(&array, &desc, w, h, cudaArraySurfaceLoadStore) != cudaSuccess) return -1.0f;
	cudaResourceDesc rd{};
	rd.resType = cudaResourceTypeArray;
	rd.res.array.array = array;
	float ms = -1.0f;
	if (cudaCreateSurfaceObject(&surface, &rd) == cudaSuccess)
	{
		Mat3 cs;
		for (int i = 0; i < 9; ++i) cs.m[i] = colorspace[i];
		uint32_t width = w, height = h;
		float exposure = exposureScale;
		const double* data = dRender;
		void* params[] = { &width, &height, &cs, &exposure, &data, &surface };
		bool ok = true;
		auto launch = [&]() {
			ok = ok && cuLaunchKernel(g_resolve, (w + 15) / 16, (h + 15) / 16, 1, 16, 16, 1, 0, nullptr, params,
				nullptr) == CUDA_SUCCESS;
		};
		for (int i = 0; i < warmup; ++i) launch();
		cudaEvent_t a, b;
		cudaEventCreate(&a); cudaEventCreate(&b);
		float total = 0.0f;
		for (int i = 0; i < iters && ok; ++i)
		{
			if (flush) cudaMemsetAsync(flush, i & 0xFF, flushBytes, 0);
			cudaEventRecord(a, 0);
			launch();
			cudaEventRecord(b, 0);
			cudaEventSynchronize(b);
			float t = 0.0f;
			cudaEventElapsedTime(&t, a, b);
			total += t;
		}
		if (ok) ms = total / static_cast<float>(iters);
		cudaEventDestroy(a); cudaEventDestroy(b);
		cudaDestroySurfaceObject(surface);
	}
	cudaFreeArray(array);
	return ms;
}

} // extern "C"
