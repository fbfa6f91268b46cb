// Environment-map 2D CDF construction and inversion (the reference's
// makeCdf2d_kernel + invertCDFToIndices, src/kernels/cdf.cu:332-535, driven
// by loadEnvironmentMap, src/core/rendering_interface.cpp:1339-1432).
//
// One fused kernel. Block y owns image row y: it reads the row's RGBA texels
// once, forms power = max(0, (r+g+b)/3) per texel, builds the inclusive row
// CDF, keeps the normalised CDF in shared memory and inverts it there by
// binary search into the uint16 conditional index table, so the float CDF
// never touches HBM. The row total goes to scratch; the last block to finish
// (atomic ticket) builds the marginal CDF over the sin-weighted row totals,
// inverts it and writes the integral. HBM traffic is the algorithmic minimum:
// w*h*16 B read, w*h*2 + h*2 B written, plus O(h) scratch.
//
// Two arithmetic modes:
//   0  float32 in exactly the reference's order (4 texels per thread,
//      block-wide Hillis-Steele scan over thread totals with the same block
//      size and chunking, same normalisation) -> index tables bit-identical
//      to the reference's kernels on the same input;
//   1  float64 sums (thread-serial, warp Kogge-Stone, warp-total scan), CDF
//      values rounded to float once, sin weights in double.

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "ratbite_b200_kernels.h"
#include "rb_envmap.h"

namespace rb
{
namespace
{

// Reference thread-block size for a row of n4 = w/4 float4 groups.
int blockSizeFor(uint32_t n4) { return n4 <= 256 ? 256 : (n4 <= 512 ? 512 : 1024); }

struct Scratch
{
	uint32_t* ticket;     // completion counter, reset to 0 by the last block
	double* rowTotal;     // h entries
	float* marginal;      // h entries (mode 0 stores the float scan here, mode 1 the normalised CDF)
};
__host__ __device__ inline size_t alignUp(size_t v, size_t a) { return (v + a - 1) / a * a; }
__host__ __device__ inline Scratch carve(void* base, uint32_t h)
{
	char* p = static_cast<char*>(base);
	Scratch s;
	s.ticket = reinterpret_cast<uint32_t*>(p);
	s.rowTotal = reinterpret_cast<double*>(p + 256);
	s.marginal = reinterpret_cast<float*>(p + 256 + alignUp(sizeof(double) * h, 256));
	return s;
}

__device__ __forceinline__ float texelPower(float4 t)
{
	return fmaxf(0.0f, (t.x + t.y + t.z) / 3.0f);
}

// Reference binary search (cdf.cu:520-531): first index in [1, n-1] whose CDF
// value is >= p, with an iteration bound instead of an open loop.
__device__ __forceinline__ uint16_t invertOne(const float* cdf, int n, float p)
{
	int low = 0, high = n - 1;
	int mid = (high - low) / 2;
	for (int it = 0; it < 64; ++it)
	{
		if (p > cdf[mid]) low = mid; else high = mid;
		mid = low + (high - low) / 2;
		if (low + 1 == high) break;
	}
	return static_cast<uint16_t>(high);
}

// Block-wide inclusive scan of float4 groups in the reference's order
// (PrefixSumBlock, cdf.cu:287-323). `total` is the running total in shared memory.
__device__ __forceinline__ void scanFloat4Reference(float4& v, float* sm, float* total)
{
	const int t = threadIdx.x;
	v.y += v.x; v.z += v.y; v.w += v.z;
	for (int i = 1; i < static_cast<int>(blockDim.x); i <<= 1)
	{
		sm[t] = v.w;
		__syncthreads();
		if (t >= i)
		{
			const float o = sm[t - i];
			v.x += o; v.y += o; v.z += o; v.w += o;
		}
		__syncthreads();
	}
	const float tot = *total;
	v.x += tot; v.y += tot; v.z += tot; v.w += tot;
	__syncthreads();
	if (t == static_cast<int>(blockDim.x) - 1) *total = v.w;
	__syncthreads();
}

// Float64 block scan: thread-serial prefix of its 4 values, warp Kogge-Stone
// over thread totals, scan of warp totals, plus the running total.
// c[] holds the thread's inclusive prefixes on return, offset by the block base.
__device__ __forceinline__ void scanDouble4(double c[4], double* smWarp, double* total)
{
	const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nw = blockDim.x >> 5;
	c[1] = c[0] + c[1]; c[2] = c[1] + c[2]; c[3] = c[2] + c[3];
	double s = c[3];
#pragma unroll
	for (int d = 1; d < 32; d <<= 1)
	{
		const double o = __shfl_up_sync(0xFFFFFFFFu, s, d);
		if (lane >= d) s = s + o;
	}
	double excl = __shfl_up_sync(0xFFFFFFFFu, s, 1);
	if (lane == 0) excl = 0.0;
	if (lane == 31) smWarp[warp] = s;
	__syncthreads();
	if (warp == 0)
	{
		double ws = lane < nw ? smWarp[lane] : 0.0;
#pragma unroll
		for (int d = 1; d < 32; d <<= 1)
		{
			const double o = __shfl_up_sync(0xFFFFFFFFu, ws, d);
			if (lane >= d) ws = ws + o;
		}
		if (lane < nw) smWarp[32 + lane] = ws;
	}
	__syncthreads();
	const double warpExcl = warp == 0 ? 0.0 : smWarp[32 + warp - 1];
	const double base = (*total + warpExcl) + excl;
	for (int k = 0; k < 4; ++k) c[k] = base + c[k];
	__syncthreads();
	if (t == static_cast<int>(blockDim.x) - 1) *total = c[3];
	__syncthreads();
}

template<int MODE>
__global__ void kEnvCdf(uint32_t w, uint32_t h, const float4* __restrict__ rgba, Scratch scr,
	uint16_t* __restrict__ condIdx, uint16_t* __restrict__ margIdx, float* __restrict__ integral)
{
	extern __shared__ __align__(16) unsigned char smraw[];
	float* cdf = reinterpret_cast<float*>(smraw);                           // w floats (row CDF, then reused)
	float* scanF = reinterpret_cast<float*>(smraw + sizeof(float) * (w > h ? w : h));
	double* scanD = reinterpret_cast<double*>(scanF);                       // 64 doubles
	__shared__ float totalF;
	__shared__ double totalD;
	__shared__ bool last;

	const uint32_t y = blockIdx.x;
	const int B = blockDim.x;
	const uint32_t n4 = w / 4;
	const uint32_t chunks = (n4 + B - 1) / B;
	if (threadIdx.x == 0) { totalF = 0.0f; totalD = 0.0; }
	__syncthreads();

	// ---- row scan -------------------------------------------------------
	const float4* row = rgba + static_cast<size_t>(y) * w;
	if (MODE == 0)
	{
		for (uint32_t k = 0; k < chunks; ++k)
		{
			const uint32_t g = threadIdx.x + B * k;
			float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			if (g < n4)
			{
				v.x = texelPower(__ldg(row + 4 * g + 0));
				v.y = texelPower(__ldg(row + 4 * g + 1));
				v.z = texelPower(__ldg(row + 4 * g + 2));
				v.w = texelPower(__ldg(row + 4 * g + 3));
			}
			scanFloat4Reference(v, scanF, &totalF);
			if (g < n4) reinterpret_cast<float4*>(cdf)[g] = v;
		}
		const float norm = totalF != 0.0f ? 1.0f / totalF : 0.0f;
		for (uint32_t g = threadIdx.x; g < n4; g += B)
		{
			float4 v = reinterpret_cast<float4*>(cdf)[g];
			v.x *= norm; v.y *= norm; v.z *= norm; v.w *= norm;
			reinterpret_cast<float4*>(cdf)[g] = v;
		}
		if (threadIdx.x == 0) scr.rowTotal[y] = static_cast<double>(totalF);
	}
	else
	{
		for (uint32_t k = 0; k < chunks; ++k)
		{
			const uint32_t g = threadIdx.x + B * k;
			double c[4] = { 0.0, 0.0, 0.0, 0.0 };
			if (g < n4)
				for (int q = 0; q < 4; ++q) c[q] = static_cast<double>(texelPower(__ldg(row + 4 * g + q)));
			scanDouble4(c, scanD, &totalD);
			// Prefixes are parked in shared memory rounded to float and
			// normalised by the double total once it is known: two roundings,
			// about 1e-7 relative, against ~1e-5 for float32 running sums.
			if (g < n4)
				for (int q = 0; q < 4; ++q) cdf[4 * g + q] = static_cast<float>(c[q]);
		}
		__syncthreads();
		const double tot = totalD;
		for (uint32_t i = threadIdx.x; i < w; i += B)
			cdf[i] = tot != 0.0 ? static_cast<float>(static_cast<double>(cdf[i]) / tot) : 0.0f;
		if (threadIdx.x == 0) scr.rowTotal[y] = totalD;
	}
	__syncthreads();

	// ---- conditional inversion (p = i / (w-1)) from shared memory ----------
	uint16_t* out = condIdx + static_cast<size_t>(y) * w;
	for (uint32_t i = threadIdx.x; i < w; i += B)
	{
		const float p = static_cast<float>(i) / static_cast<float>(static_cast<int>(w) - 1);
		out[i] = invertOne(cdf, static_cast<int>(w), p);
	}

	// ---- last block: marginal ----------------------------------------------
	__syncthreads();
	if (threadIdx.x == 0)
	{
		__threadfence();
		last = atomicAdd(scr.ticket, 1u) == h - 1;
	}
	__syncthreads();
	if (!last) return;
	__threadfence();
	const uint32_t m4 = h / 4;
	const uint32_t mChunks = (m4 + B - 1) / B;
	if (threadIdx.x == 0) { totalF = 0.0f; totalD = 0.0; }
	__syncthreads();
	if (MODE == 0)
	{
		// Reference order: float row totals x float sin weights (Cdf2dSphericalCoordsJacobian,
		// cdf.cu:105-133, with the group count as its h), scanned, then normalised in place.
		for (uint32_t k = 0; k < mChunks; ++k)
		{
			const uint32_t g = threadIdx.x + B * k;
			float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			if (g < m4)
			{
				const float pi = 3.14159265358979323846f;
				const volatile double* rt = scr.rowTotal;
				v.x = static_cast<float>(rt[4 * g + 0]);
				v.y = static_cast<float>(rt[4 * g + 1]);
				v.z = static_cast<float>(rt[4 * g + 2]);
				v.w = static_cast<float>(rt[4 * g + 3]);
				v.x *= sinf(pi * (static_cast<float>(g) + 0.125f) / static_cast<float>(m4));
				v.y *= sinf(pi * (static_cast<float>(g) + 0.375f) / static_cast<float>(m4));
				v.z *= sinf(pi * (static_cast<float>(g) + 0.625f) / static_cast<float>(m4));
				v.w *= sinf(pi * (static_cast<float>(g) + 0.875f) / static_cast<float>(m4));
			}
			scanFloat4Reference(v, scanF, &totalF);
			if (g < m4) reinterpret_cast<float4*>(cdf)[g] = v;
		}
		const float norm = totalF != 0.0f ? 1.0f / totalF : 0.0f;
		for (uint32_t g = threadIdx.x; g < m4; g += B)
		{
			float4 v = reinterpret_cast<float4*>(cdf)[g];
			v.x *= norm; v.y *= norm; v.z *= norm; v.w *= norm;
			reinterpret_cast<float4*>(cdf)[g] = v;
		}
		if (threadIdx.x == 0) *integral = totalF / (static_cast<float>(w) * static_cast<float>(h));
	}
	else
	{
		for (uint32_t k = 0; k < mChunks; ++k)
		{
			const uint32_t g = threadIdx.x + B * k;
			double c[4] = { 0.0, 0.0, 0.0, 0.0 };
			if (g < m4)
			{
				const volatile double* rt = scr.rowTotal;
				for (int q = 0; q < 4; ++q)
				{
					const double yy = static_cast<double>(4 * g + q) + 0.5;
					c[q] = rt[4 * g + q] * sin(3.141592653589793 * yy / static_cast<double>(h));
				}
			}
			scanDouble4(c, scanD, &totalD);
			if (g < m4)
				for (int q = 0; q < 4; ++q) scr.rowTotal[4 * g + q] = c[q];   // reuse: prefix sums in place
		}
		__syncthreads();
		__threadfence_block();
		const double tot = totalD;
		for (uint32_t i = threadIdx.x; i < h; i += B)
			cdf[i] = tot != 0.0 ? static_cast<float>(scr.rowTotal[i] / tot) : 0.0f;
		if (threadIdx.x == 0) *integral = static_cast<float>(tot / (static_cast<double>(w) * static_cast<double>(h)));
	}
	__syncthreads();
	for (uint32_t i = threadIdx.x; i < h; i += B)
	{
		const float p = static_cast<float>(i) / static_cast<float>(static_cast<int>(h) - 1);
		margIdx[i] = invertOne(cdf, static_cast<int>(h), p);
	}
	__syncthreads();
	if (threadIdx.x == 0) *scr.ticket = 0u;   // ready for the next build
}
} // namespace

size_t envCdfScratchBytes(uint32_t w, uint32_t h)
{
	(void)w;
	return 256 + alignUp(sizeof(double) * h, 256) + alignUp(sizeof(float) * h, 256);
}

namespace
{
constexpr int kMaxAttrDevices = 64;
// Largest dynamic shared-memory size already granted to each kernel variant
// on each device, so that cudaFuncSetAttribute runs once per device and size
// class instead of on every build.
std::atomic<int> g_smemGranted[2][kMaxAttrDevices];

int grantSharedMemory(int mode, int bytes)
{
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return RB_ERR_CUDA;
	std::atomic<int>* granted = (dev >= 0 && dev < kMaxAttrDevices) ? &g_smemGranted[mode][dev] : nullptr;
	if (granted && granted->load(std::memory_order_relaxed) >= bytes) return RB_OK;
	const cudaError_t e = mode == 0
		? cudaFuncSetAttribute(kEnvCdf<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)
		: cudaFuncSetAttribute(kEnvCdf<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
	if (e != cudaSuccess) return RB_ERR_CUDA;
	if (granted)
	{
		int cur = granted->load(std::memory_order_relaxed);
		while (cur < bytes && !granted->compare_exchange_weak(cur, bytes)) {}
	}
	return RB_OK;
}
} // namespace

int envCdfLaunch(uint32_t w, uint32_t h, const float* rgba, int mode, void* scratch, uint16_t* cond, uint16_t* marg,
	float* integral, cudaStream_t st)
{
	if (w < 4 || h < 4 || (w & 3u) || (h & 3u) || w > 32768 || h > 32768) return RB_ERR_INVALID;
	if (!rgba || !scratch || !cond || !marg || !integral || (mode != 0 && mode != 1)) return RB_ERR_INVALID;
	const int B = blockSizeFor(w / 4);
	const size_t smem = sizeof(float) * (w > h ? w : h) + sizeof(double) * 2 * 64 + sizeof(float) * 1024;
	const Scratch scr = carve(scratch, h);
	const int rc = grantSharedMemory(mode, static_cast<int>(smem));
	if (rc != RB_OK) return rc;
	// The completion ticket starts at zero whatever the caller's scratch
	// holds (the last block also resets it, but a fresh allocation is not
	// zeroed); the rest of the scratch is written before it is read.
	if (cudaMemsetAsync(scr.ticket, 0, sizeof(uint32_t), st) != cudaSuccess) return RB_ERR_CUDA;
	if (mode == 0)
		kEnvCdf<0><<<h, B, smem, st>>>(w, h, reinterpret_cast<const float4*>(rgba), scr, cond, marg, integral);
	else
		kEnvCdf<1><<<h, B, smem, st>>>(w, h, reinterpret_cast<const float4*>(rgba), scr, cond, marg, integral);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}
} // namespace rb

extern "C" size_t rb_envmap_cdf_scratch_bytes(uint32_t width, uint32_t height)
{
	return rb::envCdfScratchBytes(width, height);
}

// ---- no-allocation variant ---------------------------------------------
// The CDF build needs a small scratch area (completion ticket, per-row
// totals, marginal). For callers that may not allocate device memory it
// lives in a fixed file-scope device array sized for the largest supported
// image height; every GPU that loads this library holds it until exit.
namespace
{
constexpr uint32_t kNoAllocMaxHeight = 8192;
constexpr size_t kNoAllocScratchBytes = 256 + ((sizeof(double) * kNoAllocMaxHeight + 255) / 256) * 256
	+ ((sizeof(float) * kNoAllocMaxHeight + 255) / 256) * 256;
__device__ __align__(256) unsigned char g_envCdfScratch[kNoAllocScratchBytes];

// Device address of g_envCdfScratch in the current device's context. In
// host code the array's name is only a host-side handle, so the address has
// to come from cudaGetSymbolAddress; it is looked up on every call (a lookup
// allocates nothing), so a context that was torn down and created again
// never leaves a stale address behind.
int scratchAddress(void** out)
{
	void* p = nullptr;
	if (cudaGetSymbolAddress(&p, g_envCdfScratch) != cudaSuccess || !p) return RB_ERR_CUDA;
	*out = p;
	return RB_OK;
}
} // namespace

extern "C" int rb_envmap_cdf_noalloc(uint32_t width, uint32_t height, const float* rgba, int mode,
	uint16_t* conditional_idx, uint16_t* marginal_idx, float* integral, void* stream)
{
	if (height > kNoAllocMaxHeight) return RB_ERR_TOO_LARGE;
	void* scratch = nullptr;
	const int rc = scratchAddress(&scratch);
	if (rc != RB_OK) return rc;
	// envCdfLaunch zeroes the completion ticket on the stream before the build.
	return rb::envCdfLaunch(width, height, rgba, mode, scratch, conditional_idx, marginal_idx, integral,
		static_cast<cudaStream_t>(stream));
}

extern "C" int rb_envmap_cdf(uint32_t width, uint32_t height, const float* rgba, int mode, void* scratch,
	uint16_t* conditional_idx, uint16_t* marginal_idx, float* integral, void* stream)
{
	return rb::envCdfLaunch(width, height, rgba, mode, scratch, conditional_idx, marginal_idx, integral,
		static_cast<cudaStream_t>(stream));
}
