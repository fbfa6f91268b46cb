// Neural radiance cache: multiresolution hash-grid encoding and a 4 x 64
// MLP, trained online on radiance estimates the renderer produces.
//
// Encoding (Mueller et al. 2022): 16 levels, 2 features per level, 2^19
// entries per level (FP16 table, FP32 master copy for the optimiser);
// resolutions grow geometrically from 16 to 2048; a level whose dense grid
// fits the table is indexed densely, the others by the spatial hash
// x * 1 ^ y * 2654435761 ^ z * 805459861. Features are trilinear in the cell.
// Network input (64): 32 grid features, direction and normal mapped to
// [0, 1], the normalised hero wavelength, a constant 1, zero padding. Four
// hidden layers of 64 with ReLU, a linear output of 4 (radiance at the four
// hero wavelengths) plus a fifth, the probability that the plain estimator
// would drop the sample, which only the renderer's cached form trains. No
// biases except through the constant input.
//
// Tensor cores: the fused forward kernel keeps a 16-row tile of activations
// in registers as mma.sync m16n8k16 BF16 fragments (FP32 accumulation); an
// accumulator fragment of one layer is repacked in registers into the A
// fragment of the next. The fused backward kernel chains dX = dY W the same
// way with the transposed weights; the weight gradients dW = dY^T X over the
// batch are plain GEMMs (cuBLAS). Adam runs in FP32 on the master copies.

#include <cstdint>
#include <cstring>
#include <vector>

#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "rb_launch.cuh"
#include "ratbite_b200_nrc.h"
#include "rb_nrc_internal.h"

namespace rb
{
namespace nrc
{
constexpr int kLevels = 16, kFeat = 2, kLog2T = 19, kTable = 1 << kLog2T;
constexpr int kIn = 64, kH = 64, kOutPad = 16;
constexpr int kGridFeatures = kLevels * kFeat;          // 32
// offset of W_l in the packed weights: W0..W3 are 64 x 64, W4 is 16 x 64
__host__ __device__ constexpr int wOffset(int l) { return l < 5 ? l * kH * kH : 4 * kH * kH + kOutPad * kH; }
constexpr int kWTotal = wOffset(5);                     // 17408 weights
constexpr int kWStride = 72;                            // smem row stride (bf16), conflict-free fragment loads
constexpr int kTile = 16;                               // rows per warp tile
constexpr uint32_t kMaxTrainRows = 1u << 24;          // rows per training batch (encode kernels index rows x levels)
constexpr int kOutStride = 8;                           // forward outputs per row in the training scratch
constexpr int kDropOutput = 4;                          // output trained by the renderer: drop probability

struct Resolutions { float s[kLevels]; uint32_t dense[kLevels]; uint32_t side[kLevels]; };

RB_D uint32_t cellIndex(const Resolutions& R, int l, uint32_t x, uint32_t y, uint32_t z)
{
	if (R.dense[l]) return x + R.side[l] * (y + R.side[l] * z);
	return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (kTable - 1u);
}

// ---------------------------------------------------------------- encoding
// The two features of level l at a position in [0,1]^3: trilinear in the cell.
RB_D void levelFeatures(const Resolutions& R, const __half2* __restrict__ grid, int l, float px, float py, float pz,
	float& f0, float& f1)
{
	const float sx = px * R.s[l], sy = py * R.s[l], sz = pz * R.s[l];
	const float fx = floorf(sx), fy = floorf(sy), fz = floorf(sz);
	const float wx = sx - fx, wy = sy - fy, wz = sz - fz;
	const uint32_t cx = static_cast<uint32_t>(fx), cy = static_cast<uint32_t>(fy), cz = static_cast<uint32_t>(fz);
	f0 = 0.0f;
	f1 = 0.0f;
	for (int c = 0; c < 8; ++c)
	{
		const uint32_t dx = c & 1u, dy = (c >> 1) & 1u, dz = (c >> 2) & 1u;
		const float w = (dx ? wx : 1.0f - wx) * (dy ? wy : 1.0f - wy) * (dz ? wz : 1.0f - wz);
		const float2 e = __half22float2(grid[static_cast<size_t>(l) * kTable + cellIndex(R, l, cx + dx, cy + dy, cz + dz)]);
		f0 += w * e.x;
		f1 += w * e.y;
	}
}
RB_D float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }
// Columns 32..63 of an input row: direction and normal mapped to [0,1], the
// wavelength, a constant 1, zeros.
RB_D float restColumn(const float* v, int k)
{
	if (k < 6) return v[3 + k] * 0.5f + 0.5f;
	if (k == 6) return v[9];
	return k == 7 ? 1.0f : 0.0f;
}

// One thread per (row, level): the level's two features, and for levels
// 0..7 four of the 32 remaining columns of the row.
__global__ void kEncode(uint32_t n, const float* __restrict__ in, const __half2* __restrict__ grid, Resolutions R,
	__nv_bfloat16* __restrict__ X)
{
	for (uint32_t i = gtid(); i < n * kLevels; i += gstride())
	{
		const uint32_t r = i / kLevels, l = i % kLevels;
		const float* v = in + static_cast<size_t>(kNrcInputs) * r;
		__nv_bfloat16* row = X + static_cast<size_t>(kIn) * r;
		float f0, f1;
		levelFeatures(R, grid, static_cast<int>(l), clamp01(v[0]), clamp01(v[1]), clamp01(v[2]), f0, f1);
		row[2 * l] = __float2bfloat16_rn(f0);
		row[2 * l + 1] = __float2bfloat16_rn(f1);
		if (l < 8)
			for (int k = 4 * static_cast<int>(l); k < 4 * static_cast<int>(l) + 4; ++k)
				row[32 + k] = __float2bfloat16_rn(restColumn(v, k));
	}
}

// Scatters the gradient of the 32 grid features into the FP32 gradient
// table, one thread per (row, level).
__global__ void kEncodeBackward(uint32_t n, const float* __restrict__ in, const float* __restrict__ dX0, Resolutions R,
	float* __restrict__ gridGrad)
{
	for (uint32_t i = gtid(); i < n * kLevels; i += gstride())
	{
		const uint32_t r = i / kLevels, l = i % kLevels;
		const float g0 = dX0[static_cast<size_t>(kGridFeatures) * r + 2 * l];
		const float g1 = dX0[static_cast<size_t>(kGridFeatures) * r + 2 * l + 1];
		if (g0 == 0.0f && g1 == 0.0f) continue;
		const float* v = in + static_cast<size_t>(kNrcInputs) * r;
		const float sx = clamp01(v[0]) * R.s[l], sy = clamp01(v[1]) * R.s[l], sz = clamp01(v[2]) * R.s[l];
		const float fx = floorf(sx), fy = floorf(sy), fz = floorf(sz);
		const float wx = sx - fx, wy = sy - fy, wz = sz - fz;
		const uint32_t cx = static_cast<uint32_t>(fx), cy = static_cast<uint32_t>(fy), cz = static_cast<uint32_t>(fz);
		for (int c = 0; c < 8; ++c)
		{
			const uint32_t dx = c & 1u, dy = (c >> 1) & 1u, dz = (c >> 2) & 1u;
			const float w = (dx ? wx : 1.0f - wx) * (dy ? wy : 1.0f - wy) * (dz ? wz : 1.0f - wz);
			float2* e = reinterpret_cast<float2*>(gridGrad) + static_cast<size_t>(l) * kTable
				+ cellIndex(R, static_cast<int>(l), cx + dx, cy + dy, cz + dz);
			atomicAdd(e, make_float2(w * g0, w * g1));
		}
	}
}

// ---------------------------------------------------------------- MLP tiles
RB_D uint32_t pack2(float lo, float hi)
{
	const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
	return *reinterpret_cast<const uint32_t*>(&h);
}
RB_D float2 unpack2(uint32_t v)
{
	const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&v);
	return __bfloat1622float2(h);
}
RB_D void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
	asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
		"{%0,%1,%2,%3};\n"
		: "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
		: "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Four 8x8 b16 matrices from shared memory (ldmatrix.x4): lanes 8m..8m+7
// give the row addresses of matrix m; register m receives matrix m's
// fragment (row lane / 4, columns 2 (lane % 4), +1).
RB_D void ldsm4(uint32_t (&r)[4], const __nv_bfloat16* p)
{
	const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
	asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}

// One layer on a 16-row tile: C[16 x 8*NT] = A[16 x 64] x W^T, W in smem as
// [out][in] rows of kWStride bf16. A: 4 k-tiles of fragments. The B
// fragments of two k-tiles come from one ldmatrix.x4 (matrices at k offsets
// 0, 8, 16, 24 of the lane's weight row).
template<int NT>
RB_D void layer(const uint32_t (&A)[4][4], const __nv_bfloat16* W, float (&C)[NT][4])
{
	const uint32_t lane = threadIdx.x & 31u, r = lane & 7u, m = lane >> 3;
#pragma unroll
	for (int j = 0; j < NT; ++j)
	{
		C[j][0] = C[j][1] = C[j][2] = C[j][3] = 0.0f;
		const __nv_bfloat16* wr = W + (8 * j + r) * kWStride + 8 * m;
		uint32_t b[4];
		ldsm4(b, wr);
		mma16816(C[j], A[0], b[0], b[1]);
		mma16816(C[j], A[1], b[2], b[3]);
		ldsm4(b, wr + 32);
		mma16816(C[j], A[2], b[0], b[1]);
		mma16816(C[j], A[3], b[2], b[3]);
	}
}
// Accumulator fragments of 8 n-tiles -> A fragments of the next layer, with ReLU.
RB_D void toA(const float (&C)[8][4], uint32_t (&A)[4][4], bool relu)
{
#pragma unroll
	for (int t = 0; t < 4; ++t)
	{
		const float* a = C[2 * t];
		const float* b = C[2 * t + 1];
		auto r = [relu](float x) { return relu ? fmaxf(x, 0.0f) : x; };
		A[t][0] = pack2(r(a[0]), r(a[1]));
		A[t][1] = pack2(r(a[2]), r(a[3]));
		A[t][2] = pack2(r(b[0]), r(b[1]));
		A[t][3] = pack2(r(b[2]), r(b[3]));
	}
}
// A fragments of rows r0..r0+15 of a row-major [rows][64] bf16 array.
RB_D void loadA(const __nv_bfloat16* X, uint32_t r0, uint32_t rows, uint32_t (&A)[4][4])
{
	const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
	const uint32_t ra = r0 + g, rb = r0 + g + 8;
#pragma unroll
	for (int t = 0; t < 4; ++t)
	{
		const uint32_t k0 = 16 * t + 2 * c;
		A[t][0] = ra < rows ? *reinterpret_cast<const uint32_t*>(X + static_cast<size_t>(ra) * kIn + k0) : 0u;
		A[t][1] = rb < rows ? *reinterpret_cast<const uint32_t*>(X + static_cast<size_t>(rb) * kIn + k0) : 0u;
		A[t][2] = ra < rows ? *reinterpret_cast<const uint32_t*>(X + static_cast<size_t>(ra) * kIn + k0 + 8) : 0u;
		A[t][3] = rb < rows ? *reinterpret_cast<const uint32_t*>(X + static_cast<size_t>(rb) * kIn + k0 + 8) : 0u;
	}
}
RB_D void storeA(__nv_bfloat16* Y, uint32_t r0, uint32_t rows, const uint32_t (&A)[4][4])
{
	const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
	const uint32_t ra = r0 + g, rb = r0 + g + 8;
#pragma unroll
	for (int t = 0; t < 4; ++t)
	{
		const uint32_t k0 = 16 * t + 2 * c;
		if (ra < rows)
		{
			*reinterpret_cast<uint32_t*>(Y + static_cast<size_t>(ra) * kIn + k0) = A[t][0];
			*reinterpret_cast<uint32_t*>(Y + static_cast<size_t>(ra) * kIn + k0 + 8) = A[t][2];
		}
		if (rb < rows)
		{
			*reinterpret_cast<uint32_t*>(Y + static_cast<size_t>(rb) * kIn + k0) = A[t][1];
			*reinterpret_cast<uint32_t*>(Y + static_cast<size_t>(rb) * kIn + k0 + 8) = A[t][3];
		}
	}
}

// Copies the 5 weight matrices (global, [out][in] bf16, dense) into shared
// memory with the padded stride.
RB_D void stageWeights(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* sw)
{
	for (int i = threadIdx.x; i < kWTotal / 2; i += blockDim.x)
	{
		const int e = 2 * i, row = e / kH, col = e % kH;
		*reinterpret_cast<uint32_t*>(sw + row * kWStride + col) = *reinterpret_cast<const uint32_t*>(w + e);
	}
	__syncthreads();
}
constexpr int kWRowsTotal = kWTotal / kH;   // 272 rows of 64
constexpr size_t kSmemWeights = sizeof(__nv_bfloat16) * kWRowsTotal * kWStride;
// backward: W4^T as 64 rows (16 used columns) + W3^T..W0^T as 4 x 64 rows
constexpr int kWtRows = 64 + 4 * 64;
constexpr size_t kSmemBackward = sizeof(__nv_bfloat16) * kWtRows * kWStride;

// Forward: out[n][kOutStride] (FP32; outputs 0..3 radiance, 4 the drop
// probability the renderer trains, 5..7 unused). With acts, the post-ReLU hidden activations of
// layers 1..4 are stored ([4][n][64] bf16) for the backward pass.
__global__ void __launch_bounds__(128) kMlpForward(uint32_t n, const __nv_bfloat16* __restrict__ X,
	const __nv_bfloat16* __restrict__ w, float* __restrict__ out, __nv_bfloat16* __restrict__ acts)
{
	extern __shared__ __nv_bfloat16 sw[];
	stageWeights(w, sw);
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
	for (uint32_t r0 = warp * kTile; r0 < n; r0 += warps * kTile)
	{
		uint32_t A[4][4];
		loadA(X, r0, n, A);
		float C[8][4];
#pragma unroll
		for (int l = 0; l < 4; ++l)
		{
			layer<8>(A, sw + wOffset(l) / kH * kWStride, C);
			toA(C, A, true);
			if (acts) storeA(acts + static_cast<size_t>(l) * n * kIn, r0, n, A);
		}
		float O[1][4];
		layer<1>(A, sw + wOffset(4) / kH * kWStride, O);
		// O: rows g, g+8; cols 2c, 2c+1: the first 8 output rows of W4
		const uint32_t ra = r0 + g, rb = r0 + g + 8;
		if (ra < n) { out[kOutStride * ra + 2 * c] = O[0][0]; out[kOutStride * ra + 2 * c + 1] = O[0][1]; }
		if (rb < n) { out[kOutStride * rb + 2 * c] = O[0][2]; out[kOutStride * rb + 2 * c + 1] = O[0][3]; }
	}
}

// Inference with the encoding fused in: each warp encodes its 16-row tile
// into a shared-memory tile (lanes split the 16 rows x 16 levels of grid
// lookups, then the 32 remaining columns), reads the A fragments from it and
// runs the layers as kMlpForward. Rows: min(*count, cap) when count is given,
// else cap. Outputs 0..3 go to out[rows][4] and/or, with path, are applied
// as L[p] = L[p] (1 - q) + T[p] max(y, 0), p = path[r], q = output 4
// clamped to [0, 1] (radiance-cache queries).
// RB_INFER_THREADS threads share one copy of the weights; as many blocks per
// SM as fit (3 at 256 threads: 56 KB of shared memory each, registers capped
// for 3). Measured on the cached Cornell frame (1920x1080, 64 spp): 256
// threads 8.06 ms of inference, 384: 8.14, 512: 8.71 (spills at the
// 64-register cap).
#ifndef RB_INFER_THREADS
#define RB_INFER_THREADS 256
#endif
#ifndef RB_INFER_GATHER_UNROLL
#define RB_INFER_GATHER_UNROLL 2
#endif
constexpr int kInferThreads = RB_INFER_THREADS;
constexpr int kGatherUnroll = RB_INFER_GATHER_UNROLL;
#ifndef RB_INFER_MIN_BLOCKS
#define RB_INFER_MIN_BLOCKS 3
#endif
constexpr int kInferMinBlocks = RB_INFER_MIN_BLOCKS;
constexpr size_t kSmemInfer = kSmemWeights + sizeof(__nv_bfloat16) * (kInferThreads / 32) * kTile * kWStride;
__global__ void __launch_bounds__(kInferThreads, kInferMinBlocks) kMlpInfer(uint32_t cap, const uint32_t* __restrict__ count,
	const float* __restrict__ in, const __half2* __restrict__ grid, Resolutions R, const __nv_bfloat16* __restrict__ w,
	float* __restrict__ out, const uint32_t* __restrict__ path, float4* __restrict__ L, const float4* __restrict__ T,
	const float* __restrict__ corr)
{
	extern __shared__ __nv_bfloat16 sw[];
	stageWeights(w, sw);
	const uint32_t n = count ? min(*count, cap) : cap;
	__nv_bfloat16* tile = sw + kWRowsTotal * kWStride + (threadIdx.x >> 5) * kTile * kWStride;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
	for (uint32_t r0 = warp * kTile; r0 < n; r0 += warps * kTile)
	{
		// grid features: lane handles (row k / 16, level k % 16) for k = lane + 32 i
#pragma unroll kGatherUnroll
		for (uint32_t k = lane; k < kTile * kLevels; k += 32)
		{
			const uint32_t row = k >> 4, l = k & 15u, r = r0 + row;
			float f0 = 0.0f, f1 = 0.0f;
			if (r < n)
			{
				const float* v = in + static_cast<size_t>(kNrcInputs) * r;
				levelFeatures(R, grid, static_cast<int>(l), clamp01(v[0]), clamp01(v[1]), clamp01(v[2]), f0, f1);
			}
			*reinterpret_cast<uint32_t*>(tile + row * kWStride + 2 * l) = pack2(f0, f1);
		}
		// columns 32..63: lane handles 16 columns of row lane / 2
		{
			const uint32_t row = lane >> 1, r = r0 + row, k0 = 16 * (lane & 1u);
			const float* v = in + static_cast<size_t>(kNrcInputs) * r;
#pragma unroll
			for (uint32_t k = 0; k < 16; k += 2)
			{
				const float a = r < n ? restColumn(v, static_cast<int>(k0 + k)) : 0.0f;
				const float b = r < n ? restColumn(v, static_cast<int>(k0 + k + 1)) : 0.0f;
				*reinterpret_cast<uint32_t*>(tile + row * kWStride + 32 + k0 + k) = pack2(a, b);
			}
		}
		__syncwarp();
		// A fragments (ldmatrix.x4 per k-tile: rows 0-7 / 8-15 x columns 0-7 / 8-15 of the tile)
		uint32_t A[4][4];
		{
			const uint32_t m = lane >> 3, rr = (lane & 7u) + 8u * (m & 1u);
#pragma unroll
			for (int t = 0; t < 4; ++t) ldsm4(A[t], tile + rr * kWStride + 16 * t + 8 * (m >> 1));
		}
		__syncwarp();
		float C[8][4];
#pragma unroll
		for (int l = 0; l < 4; ++l)
		{
			layer<8>(A, sw + wOffset(l) / kH * kWStride, C);
			toA(C, A, true);
		}
		float O[1][4];
		layer<1>(A, sw + wOffset(4) / kH * kWStride, O);
		// lanes c = 0 hold outputs 0, 1, lanes c = 1 outputs 2, 3 and lanes
		// c = 2 output 4 (drop probability) of rows g and g + 8
		const float a2 = __shfl_down_sync(0xFFFFFFFFu, O[0][0], 1), a3 = __shfl_down_sync(0xFFFFFFFFu, O[0][1], 1);
		const float b2 = __shfl_down_sync(0xFFFFFFFFu, O[0][2], 1), b3 = __shfl_down_sync(0xFFFFFFFFu, O[0][3], 1);
		const float aq = __shfl_down_sync(0xFFFFFFFFu, O[0][0], 2), bq = __shfl_down_sync(0xFFFFFFFFu, O[0][2], 2);
		if (c == 0)
		{
			const uint32_t rows[2] = { r0 + g, r0 + g + 8 };
			const float4 y[2] = { make_float4(O[0][0], O[0][1], a2, a3), make_float4(O[0][2], O[0][3], b2, b3) };
			const float q[2] = { aq, bq };
#pragma unroll
			for (int h = 0; h < 2; ++h)
			{
				if (rows[h] >= n) continue;
				if (out) reinterpret_cast<float4*>(out)[rows[h]] = y[h];
				if (path)
				{
					// the plain estimator drops a whole sample whose later BxDF
					// sample fails: the prefix survives with 1 - q, q plus the
					// correction measured on the path's class (the path
					// index's high bit: the camera ray hit an emitter, whose
					// radiance dominates the prefix); the radiance is scaled
					// by the measured ratio of targets to predictions
					const uint32_t pr = path[rows[h]];
					const uint32_t p = pr & 0x7FFFFFFFu;
					const float4 t = T[p];
					const float qq = q[h] + (corr ? corr[((pr >> 31) ? kCorrDropLit : kCorrDropOther) + 2] : 0.0f);
					const float keep = fminf(fmaxf(1.0f - qq, 0.0f), 1.0f);
					const float sc = corr && corr[kCorrRadiance + 3] > 0.0f ? corr[kCorrRadiance + 2] : 1.0f;
					float4 l = L[p];
					l.x = l.x * keep + t.x * (sc * fmaxf(y[h].x, 0.0f));
					l.y = l.y * keep + t.y * (sc * fmaxf(y[h].y, 0.0f));
					l.z = l.z * keep + t.z * (sc * fmaxf(y[h].z, 0.0f));
					l.w = l.w * keep + t.w * (sc * fmaxf(y[h].w, 0.0f));
					L[p] = l;
				}
			}
		}
	}
}

// Relative L2 loss (Mueller et al. 2021): sum over the first `outs` outputs
// of (y - t)^2 / (sg(y)^2 + 0.01), averaged over the batch; targets are rows
// of tStride floats; dY is written as bf16 rows of 16 and the loss sum
// accumulated. With valid, only the first min(*valid, n) rows count (the
// others get a zero gradient).
__global__ void kLoss(uint32_t n, const float* __restrict__ y, const float* __restrict__ t,
	__nv_bfloat16* __restrict__ dY, float* __restrict__ lossSum, const uint32_t* __restrict__ valid, int outs,
	int tStride, float* __restrict__ corr)
{
	float local = 0.0f;
	// sums of the renderer's correction state over this thread's rows of a
	// class (1, 2): drop residual and count per class, radiance targets and
	// clamped predictions
	float cs[6] = { 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f };
	const uint32_t nv = valid ? min(*valid, n) : n;
	const float scale = nv ? 1.0f / static_cast<float>(nv) : 0.0f;
	for (uint32_t i = gtid(); i < n; i += gstride())
	{
		for (int k = 0; k < kOutPad; ++k)
		{
			float gk = 0.0f;
			if (k < outs && i < nv)
			{
				const float yy = y[kOutStride * i + k], tt = t[static_cast<size_t>(tStride) * i + k];
				const float den = yy * yy + 0.01f;
				const float d = yy - tt;
				local += d * d / den;
				gk = 2.0f * d / den * scale;
				const float cls = corr && outs > kDropOutput ? t[static_cast<size_t>(tStride) * i + kDropOutput + 1] : 0.0f;
				if (cls != 0.0f)
				{
					if (k == kDropOutput)
					{
						cs[cls == 1.0f ? 0 : 2] += tt - yy;
						cs[cls == 1.0f ? 1 : 3] += 1.0f;
					}
					else
					{
						cs[4] += tt;
						cs[5] += fmaxf(yy, 0.0f);
					}
				}
			}
			dY[static_cast<size_t>(kOutPad) * i + k] = __float2bfloat16_rn(gk);
		}
	}
	for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
	if ((threadIdx.x & 31u) == 0) atomicAdd(lossSum, local * scale);
	if (corr)
	{
		const int slot[6] = { kCorrDropLit, kCorrDropLit + 1, kCorrDropOther, kCorrDropOther + 1, kCorrRadiance,
			kCorrRadiance + 1 };
#pragma unroll
		for (int j = 0; j < 6; ++j)
		{
			float v = cs[j];
			for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
			if ((threadIdx.x & 31u) == 0 && v != 0.0f) atomicAdd(corr + slot[j], v);
		}
	}
}

// Backward through the layers on 16-row tiles: with the transposed weights
// wt ([in][out] per layer, the output layer padded to 16 columns), dH4 = dY W4
// masked by ReLU', ..., dX0 = dH1 W0. Writes the masked gradients of the
// hidden layers ([4][n][64] bf16, for the weight gradients) and the
// gradient of the 32 grid features (FP32).
__global__ void __launch_bounds__(128) kMlpBackward(uint32_t n, const __nv_bfloat16* __restrict__ dY,
	const __nv_bfloat16* __restrict__ wt, const __nv_bfloat16* __restrict__ acts, __nv_bfloat16* __restrict__ dH,
	float* __restrict__ dX0)
{
	extern __shared__ __nv_bfloat16 sw[];
	// wt layout: W4^T [64][16] first (as 64 rows of 16), then W3^T..W0^T [64][64]
	for (int i = threadIdx.x; i < (64 * 16) / 2; i += blockDim.x)
	{
		const int e = 2 * i, row = e / 16, col = e % 16;
		*reinterpret_cast<uint32_t*>(sw + row * kWStride + col) = *reinterpret_cast<const uint32_t*>(wt + e);
	}
	for (int i = threadIdx.x; i < (4 * 64 * 64) / 2; i += blockDim.x)
	{
		const int e = 2 * i, row = e / 64, col = e % 64;
		*reinterpret_cast<uint32_t*>(sw + (64 + row) * kWStride + col) = *reinterpret_cast<const uint32_t*>(wt + 64 * 16 + e);
	}
	__syncthreads();
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
	for (uint32_t r0 = warp * kTile; r0 < n; r0 += warps * kTile)
	{
		// dY tile as one k-tile (16 columns, 4 used)
		uint32_t A[4][4];
		const uint32_t ra = r0 + g, rb = r0 + g + 8;
		{
			const __nv_bfloat16* base = dY;
			A[0][0] = ra < n ? *reinterpret_cast<const uint32_t*>(base + static_cast<size_t>(ra) * kOutPad + 2 * c) : 0u;
			A[0][1] = rb < n ? *reinterpret_cast<const uint32_t*>(base + static_cast<size_t>(rb) * kOutPad + 2 * c) : 0u;
			A[0][2] = ra < n ? *reinterpret_cast<const uint32_t*>(base + static_cast<size_t>(ra) * kOutPad + 8 + 2 * c) : 0u;
			A[0][3] = rb < n ? *reinterpret_cast<const uint32_t*>(base + static_cast<size_t>(rb) * kOutPad + 8 + 2 * c) : 0u;
		}
		float C[8][4];
		// dH4 = dY[16 x 16] x W4 (B(k = out, n = in) = W4^T[in][out])
#pragma unroll
		for (int j = 0; j < 8; ++j)
		{
			C[j][0] = C[j][1] = C[j][2] = C[j][3] = 0.0f;
			const __nv_bfloat16* wr = sw + (8 * j + g) * kWStride;
			const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr + 2 * c);
			const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + 8 + 2 * c);
			mma16816(C[j], A[0], b0, b1);
		}
		for (int l = 3; l >= 0; --l)
		{
			// mask by ReLU' of the stored activation of layer l (post-ReLU > 0)
			uint32_t H[4][4];
			loadA(acts + static_cast<size_t>(l) * n * kIn, r0, n, H);
#pragma unroll
			for (int t = 0; t < 4; ++t)
			{
				const float2 h00 = unpack2(H[t][0]), h10 = unpack2(H[t][1]), h01 = unpack2(H[t][2]), h11 = unpack2(H[t][3]);
				float* a = C[2 * t];
				float* b = C[2 * t + 1];
				a[0] = h00.x > 0.0f ? a[0] : 0.0f; a[1] = h00.y > 0.0f ? a[1] : 0.0f;
				a[2] = h10.x > 0.0f ? a[2] : 0.0f; a[3] = h10.y > 0.0f ? a[3] : 0.0f;
				b[0] = h01.x > 0.0f ? b[0] : 0.0f; b[1] = h01.y > 0.0f ? b[1] : 0.0f;
				b[2] = h11.x > 0.0f ? b[2] : 0.0f; b[3] = h11.y > 0.0f ? b[3] : 0.0f;
			}
			toA(C, A, false);
			storeA(dH + static_cast<size_t>(l) * n * kIn, r0, n, A);
			// next: dH_{l} x W_l  (W_l^T at row block 64 + (3 - l) * 64)
			layer<8>(A, sw + (64 + (3 - l) * 64) * kWStride, C);
		}
		// C = dX0 (64 columns); the first 32 are the grid features
#pragma unroll
		for (int j = 0; j < 4; ++j)
		{
			if (ra < n) { dX0[32 * ra + 8 * j + 2 * c] = C[j][0]; dX0[32 * ra + 8 * j + 2 * c + 1] = C[j][1]; }
			if (rb < n) { dX0[32 * rb + 8 * j + 2 * c] = C[j][2]; dX0[32 * rb + 8 * j + 2 * c + 1] = C[j][3]; }
		}
	}
}

// ---------------------------------------------------------------- optimiser
// Adam on float4 groups (n must be a multiple of 4: both parameter tables
// are); the gradient is cleared, and the bf16 / fp16 copies refreshed.
RB_D void adam1(float& p, float g, float& m, float& v, float lr, float b1, float b2, float eps, float c1, float c2)
{
	m = b1 * m + (1.0f - b1) * g;
	v = b2 * v + (1.0f - b2) * g * g;
	p = p - lr * (m / c1) / (sqrtf(v / c2) + eps);
}
__global__ void kAdam(uint32_t n, float* __restrict__ p, float* __restrict__ grad, float* __restrict__ m,
	float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2, __nv_bfloat16* outBf16,
	__half* outF16)
{
	float4* P = reinterpret_cast<float4*>(p);
	float4* G = reinterpret_cast<float4*>(grad);
	float4* M = reinterpret_cast<float4*>(m);
	float4* V = reinterpret_cast<float4*>(v);
	for (uint32_t i = gtid(); i < n / 4; i += gstride())
	{
		float4 pp = P[i], mm = M[i], vv = V[i];
		const float4 gg = G[i];
		adam1(pp.x, gg.x, mm.x, vv.x, lr, b1, b2, eps, c1, c2);
		adam1(pp.y, gg.y, mm.y, vv.y, lr, b1, b2, eps, c1, c2);
		adam1(pp.z, gg.z, mm.z, vv.z, lr, b1, b2, eps, c1, c2);
		adam1(pp.w, gg.w, mm.w, vv.w, lr, b1, b2, eps, c1, c2);
		P[i] = pp;
		M[i] = mm;
		V[i] = vv;
		G[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		if (outBf16)
		{
			__nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(outBf16) + 2 * i;
			o[0] = __floats2bfloat162_rn(pp.x, pp.y);
			o[1] = __floats2bfloat162_rn(pp.z, pp.w);
		}
		if (outF16)
		{
			__half2* o = reinterpret_cast<__half2*>(outF16) + 2 * i;
			o[0] = __floats2half2_rn(pp.x, pp.y);
			o[1] = __floats2half2_rn(pp.z, pp.w);
		}
	}
}
static_assert(kWTotal % 4 == 0 && (kLevels * kTable * kFeat) % 4 == 0, "kAdam works on float4 groups");

// transposed bf16 copies of the weights for the backward kernel
__global__ void kTransposeWeights(const float* __restrict__ w, __nv_bfloat16* __restrict__ wt)
{
	for (uint32_t i = gtid(); i < static_cast<uint32_t>(kWTotal); i += gstride())
	{
		if (i < 64u * 16u)
		{
			const uint32_t in = i / 16, out = i % 16;                     // W4^T [64][16]
			wt[i] = __float2bfloat16_rn(w[wOffset(4) + out * kH + in]);
		}
		else
		{
			const uint32_t j = i - 64u * 16u, blk = j / 4096u, e = j % 4096u;   // blocks: W3^T, W2^T, W1^T, W0^T
			const uint32_t l = 3u - blk, in = e / 64u, out = e % 64u;
			wt[i] = __float2bfloat16_rn(w[wOffset(l) + out * kH + in]);
		}
	}
}
} // namespace nrc
} // namespace rb

// ------------------------------------------------------------------ C ABI
using namespace rb::nrc;
using rb::gridFor;
using rb::kThreads;

struct rb_nrc
{
	int device = 0;
	rb_nrc_config cfg{};
	Resolutions R{};
	float *gridF32 = nullptr, *gridGrad = nullptr, *gridM = nullptr, *gridV = nullptr;
	__half* grid = nullptr;
	float *wF32 = nullptr, *wGrad = nullptr, *wM = nullptr, *wV = nullptr;
	__nv_bfloat16 *w = nullptr, *wt = nullptr;
	// training scratch, grown on demand
	uint32_t cap = 0;
	__nv_bfloat16 *X = nullptr, *acts = nullptr, *dY = nullptr, *dH = nullptr;
	float *out = nullptr, *dX0 = nullptr, *loss = nullptr;
	cublasHandle_t blas = nullptr;
	uint32_t step = 0;
	int smCount = 148;
	uint32_t inferBlocksPerSm = 2;
};

namespace
{
int nrcFail(cudaError_t e) { return e == cudaErrorMemoryAllocation ? RB_ERR_OOM : RB_ERR_CUDA; }

// Deterministic uniform init (SplitMix64), as floats in [-a, a].
void initUniform(std::vector<float>& v, uint64_t seed, float a)
{
	uint64_t s = seed;
	for (float& x : v)
	{
		s += 0x9E3779B97F4A7C15ull;
		uint64_t z = s;
		z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
		z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
		z ^= z >> 31;
		x = (static_cast<float>(z >> 40) / 16777216.0f * 2.0f - 1.0f) * a;
	}
}

int growScratch(rb_nrc* h, uint32_t n)
{
	if (n <= h->cap) return RB_OK;
	cudaFree(h->X); cudaFree(h->acts); cudaFree(h->dY); cudaFree(h->dH); cudaFree(h->out); cudaFree(h->dX0);
	h->X = h->acts = h->dY = h->dH = nullptr;
	h->out = h->dX0 = nullptr;
	h->cap = 0;
	cudaError_t e = cudaMalloc(&h->X, sizeof(__nv_bfloat16) * kIn * n);
	if (e == cudaSuccess) e = cudaMalloc(&h->acts, sizeof(__nv_bfloat16) * 4 * kIn * n);
	if (e == cudaSuccess) e = cudaMalloc(&h->dY, sizeof(__nv_bfloat16) * kOutPad * n);
	if (e == cudaSuccess) e = cudaMalloc(&h->dH, sizeof(__nv_bfloat16) * 4 * kIn * n);
	if (e == cudaSuccess) e = cudaMalloc(&h->out, sizeof(float) * kOutStride * n);
	if (e == cudaSuccess) e = cudaMalloc(&h->dX0, sizeof(float) * kGridFeatures * n);
	if (e != cudaSuccess) return nrcFail(e);
	h->cap = n;
	return RB_OK;
}

int blocksFor(const rb_nrc* h, uint32_t rows)
{
	const uint32_t tiles = (rows + kTile - 1) / kTile, perBlock = 4;   // 4 warps, one tile each
	const uint32_t need = (tiles + perBlock - 1) / perBlock;
	const uint32_t cap = static_cast<uint32_t>(h->smCount) * 4;
	return static_cast<int>(need < 1 ? 1 : (need < cap ? need : cap));
}

int inferBlocks(const rb_nrc* h, uint32_t rows)
{
	const uint32_t tiles = (rows + kTile - 1) / kTile, perBlock = kInferThreads / 32;
	const uint32_t need = (tiles + perBlock - 1) / perBlock;
	const uint32_t cap = static_cast<uint32_t>(h->smCount) * h->inferBlocksPerSm;
	return static_cast<int>(need < 1 ? 1 : (need < cap ? need : cap));
}

int encodeBlocks(uint32_t rows)
{
	return gridFor(rows * static_cast<uint32_t>(kLevels));
}
} // namespace

extern "C" {

int rb_nrc_create(const rb_nrc_config* config, rb_nrc** out)
{
	if (!out) return RB_ERR_INVALID;
	*out = nullptr;
	rb_nrc* h = new (std::nothrow) rb_nrc();
	if (!h) return RB_ERR_OOM;
	h->cfg = config ? *config : rb_nrc_config{};
	if (h->cfg.learning_rate <= 0.0f) h->cfg.learning_rate = 1e-2f;
	if (h->cfg.beta1 <= 0.0f) h->cfg.beta1 = 0.9f;
	if (h->cfg.beta2 <= 0.0f) h->cfg.beta2 = 0.99f;
	if (h->cfg.epsilon <= 0.0f) h->cfg.epsilon = 1e-15f;
	h->device = h->cfg.device;
	cudaSetDevice(h->device);
	cudaDeviceGetAttribute(&h->smCount, cudaDevAttrMultiProcessorCount, h->device);
	// resolutions 16 .. 2048, geometric
	const double growth = std::exp((std::log(2048.0) - std::log(16.0)) / (kLevels - 1));
	for (int l = 0; l < kLevels; ++l)
	{
		const double res = std::floor(16.0 * std::pow(growth, l));
		h->R.s[l] = static_cast<float>(res);
		const double side = res + 2.0;
		h->R.dense[l] = side * side * side <= static_cast<double>(kTable) ? 1u : 0u;
		h->R.side[l] = static_cast<uint32_t>(side);
	}
	const size_t gridN = static_cast<size_t>(kLevels) * kTable * kFeat;
	cudaError_t e = cudaMalloc(&h->gridF32, sizeof(float) * gridN);
	if (e == cudaSuccess) e = cudaMalloc(&h->gridGrad, sizeof(float) * gridN);
	if (e == cudaSuccess) e = cudaMalloc(&h->gridM, sizeof(float) * gridN);
	if (e == cudaSuccess) e = cudaMalloc(&h->gridV, sizeof(float) * gridN);
	if (e == cudaSuccess) e = cudaMalloc(&h->grid, sizeof(__half) * gridN);
	if (e == cudaSuccess) e = cudaMalloc(&h->wF32, sizeof(float) * kWTotal);
	if (e == cudaSuccess) e = cudaMalloc(&h->wGrad, sizeof(float) * kWTotal);
	if (e == cudaSuccess) e = cudaMalloc(&h->wM, sizeof(float) * kWTotal);
	if (e == cudaSuccess) e = cudaMalloc(&h->wV, sizeof(float) * kWTotal);
	if (e == cudaSuccess) e = cudaMalloc(&h->w, sizeof(__nv_bfloat16) * kWTotal);
	if (e == cudaSuccess) e = cudaMalloc(&h->wt, sizeof(__nv_bfloat16) * kWTotal);
	if (e == cudaSuccess) e = cudaMalloc(&h->loss, sizeof(float));
	if (e != cudaSuccess) { rb_nrc_destroy(h); return nrcFail(e); }
	cudaMemset(h->gridGrad, 0, sizeof(float) * gridN);
	cudaMemset(h->gridM, 0, sizeof(float) * gridN);
	cudaMemset(h->gridV, 0, sizeof(float) * gridN);
	cudaMemset(h->wGrad, 0, sizeof(float) * kWTotal);
	cudaMemset(h->wM, 0, sizeof(float) * kWTotal);
	cudaMemset(h->wV, 0, sizeof(float) * kWTotal);
	// initial parameters: grid U(-1e-4, 1e-4), weights U(-sqrt(6/fan_in), ...); padded output rows zero
	std::vector<float> g(gridN), w(kWTotal, 0.0f);
	initUniform(g, h->cfg.seed * 2 + 1, 1e-4f);
	std::vector<float> wl(4096);
	for (int l = 0; l < 4; ++l)
	{
		initUniform(wl, h->cfg.seed * 2 + 2 + l, std::sqrt(6.0f / kIn));
		std::memcpy(w.data() + wOffset(l), wl.data(), sizeof(float) * 4096);
	}
	std::vector<float> wo(4 * kH);
	initUniform(wo, h->cfg.seed * 2 + 7, std::sqrt(6.0f / kH));
	std::memcpy(w.data() + wOffset(4), wo.data(), sizeof(float) * wo.size());
	const int rc = rb_nrc_set_parameters(h, g.data(), w.data());
	if (rc != RB_OK) { rb_nrc_destroy(h); return rc; }
	if (cublasCreate(&h->blas) != CUBLAS_STATUS_SUCCESS) { rb_nrc_destroy(h); return RB_ERR_CUDA; }
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kMlpForward), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kSmemWeights));
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kMlpBackward), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kSmemBackward));
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kMlpInfer), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kSmemInfer));
	int perSm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kMlpInfer, kInferThreads, kSmemInfer) == cudaSuccess && perSm > 0)
		h->inferBlocksPerSm = static_cast<uint32_t>(perSm);
	*out = h;
	return RB_OK;
}

int rb_nrc_destroy(rb_nrc* h)
{
	if (!h) return RB_ERR_INVALID;
	cudaSetDevice(h->device);
	cudaDeviceSynchronize();
	for (void* p : { (void*)h->gridF32, (void*)h->gridGrad, (void*)h->gridM, (void*)h->gridV, (void*)h->grid,
			(void*)h->wF32, (void*)h->wGrad, (void*)h->wM, (void*)h->wV, (void*)h->w, (void*)h->wt, (void*)h->X,
			(void*)h->acts, (void*)h->dY, (void*)h->dH, (void*)h->out, (void*)h->dX0, (void*)h->loss })
		if (p) cudaFree(p);
	if (h->blas) cublasDestroy(h->blas);
	delete h;
	return RB_OK;
}

size_t rb_nrc_grid_size(void) { return static_cast<size_t>(kLevels) * kTable * kFeat; }
size_t rb_nrc_weight_count(void) { return kWTotal; }

int rb_nrc_set_parameters(rb_nrc* h, const float* grid, const float* weights)
{
	if (!h || !grid || !weights) return RB_ERR_INVALID;
	cudaSetDevice(h->device);
	const size_t gridN = rb_nrc_grid_size();
	cudaError_t e = cudaMemcpy(h->gridF32, grid, sizeof(float) * gridN, cudaMemcpyHostToDevice);
	if (e == cudaSuccess) e = cudaMemcpy(h->wF32, weights, sizeof(float) * kWTotal, cudaMemcpyHostToDevice);
	if (e != cudaSuccess) return nrcFail(e);
	// refresh the low-precision copies with a zero-gradient, zero-rate Adam pass
	kAdam<<<4 * h->smCount, 256>>>(static_cast<uint32_t>(gridN), h->gridF32, h->gridGrad, h->gridM, h->gridV, 0.0f,
		0.0f, 0.0f, 1.0f, 1.0f, 1.0f, nullptr, h->grid);
	kAdam<<<64, 256>>>(kWTotal, h->wF32, h->wGrad, h->wM, h->wV, 0.0f, 0.0f, 0.0f, 1.0f, 1.0f, 1.0f, h->w, nullptr);
	kTransposeWeights<<<64, 256>>>(h->wF32, h->wt);
	e = cudaDeviceSynchronize();
	return e == cudaSuccess ? RB_OK : nrcFail(e);
}

int rb_nrc_get_parameters(rb_nrc* h, float* grid, float* weights)
{
	if (!h || !grid || !weights) return RB_ERR_INVALID;
	cudaSetDevice(h->device);
	cudaError_t e = cudaDeviceSynchronize();
	if (e == cudaSuccess) e = cudaMemcpy(grid, h->gridF32, sizeof(float) * rb_nrc_grid_size(), cudaMemcpyDeviceToHost);
	if (e == cudaSuccess) e = cudaMemcpy(weights, h->wF32, sizeof(float) * kWTotal, cudaMemcpyDeviceToHost);
	return e == cudaSuccess ? RB_OK : nrcFail(e);
}

int rb_nrc_infer(rb_nrc* h, uint32_t n, const float* inputs, float* outputs, void* stream)
{
	if (!h || (n && (!inputs || !outputs))) return RB_ERR_INVALID;
	if (reinterpret_cast<uintptr_t>(outputs) & 15u) return RB_ERR_INVALID;
	if (n == 0) return RB_OK;
	cudaSetDevice(h->device);
	const cudaStream_t st = static_cast<cudaStream_t>(stream);
	kMlpInfer<<<inferBlocks(h, n), kInferThreads, kSmemInfer, st>>>(n, nullptr, inputs, reinterpret_cast<const __half2*>(h->grid),
		h->R, h->w, outputs, nullptr, nullptr, nullptr, nullptr);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}

namespace
{
// Forward, loss, backward: accumulates the batch's gradients into wGrad and
// gridGrad (which the optimiser step or rb_nrc_gradients consume).
int computeGradients(rb_nrc* h, uint32_t n, const float* inputs, const float* targets, cudaStream_t st,
	const uint32_t* valid = nullptr, int outs = 4, int tStride = 4, float* corr = nullptr)
{
	int rc = growScratch(h, n);
	if (rc != RB_OK) return rc;
	cudaMemsetAsync(h->loss, 0, sizeof(float), st);
	kEncode<<<encodeBlocks(n), kThreads, 0, st>>>(n, inputs, reinterpret_cast<const __half2*>(h->grid), h->R, h->X);
	kMlpForward<<<blocksFor(h, n), 128, kSmemWeights, st>>>(n, h->X, h->w, h->out, h->acts);
	kLoss<<<gridFor(n), kThreads, 0, st>>>(n, h->out, targets, h->dY, h->loss, valid, outs, tStride, corr);
	kMlpBackward<<<blocksFor(h, n), 128, kSmemBackward, st>>>(n, h->dY, h->wt, h->acts, h->dH, h->dX0);
	// weight gradients: dW_l[out][in] = sum over rows dY_l[r][out] X_l[r][in]
	// (column-major view: dW^T = X^T dY with X [n][64] row-major = X^T column-major)
	cublasSetStream(h->blas, st);
	const float one = 1.0f;
	const __nv_bfloat16* inputsOf[5] = { h->X, h->acts, h->acts + static_cast<size_t>(n) * kIn,
		h->acts + 2 * static_cast<size_t>(n) * kIn, h->acts + 3 * static_cast<size_t>(n) * kIn };
	for (int l = 0; l < 5; ++l)
	{
		const int outDim = l < 4 ? kH : kOutPad;
		const __nv_bfloat16* dOut = l < 4 ? h->dH + static_cast<size_t>(l) * n * kIn : h->dY;
		const int ldd = l < 4 ? kIn : kOutPad;
		// C (col-major, in x out) = A (in x n) * B^T... written as C[in][out] += sum_r X[r][in] dOut[r][out]:
		// A = X viewed col-major (in x n, lda = 64), B = dOut viewed col-major (out x n, ldb = ldd), op(B) = T.
		if (cublasGemmEx(h->blas, CUBLAS_OP_N, CUBLAS_OP_T, kIn, outDim, static_cast<int>(n), &one, inputsOf[l],
				CUDA_R_16BF, kIn, dOut, CUDA_R_16BF, ldd, &one, h->wGrad + wOffset(l), CUDA_R_32F, kIn,
				CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT) != CUBLAS_STATUS_SUCCESS)
			return RB_ERR_CUDA;
	}
	kEncodeBackward<<<encodeBlocks(n), kThreads, 0, st>>>(n, inputs, h->dX0, h->R, h->gridGrad);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}
} // namespace

int rb_nrc_gradients(rb_nrc* h, uint32_t n, const float* inputs, const float* targets, float* grid_grad,
	float* weight_grad)
{
	if (!h || n == 0 || n > kMaxTrainRows || !inputs || !targets || !grid_grad || !weight_grad) return RB_ERR_INVALID;
	cudaSetDevice(h->device);
	int rc = computeGradients(h, n, inputs, targets, nullptr);
	if (rc != RB_OK) return rc;
	const size_t gridN = rb_nrc_grid_size();
	cudaError_t e = cudaDeviceSynchronize();
	if (e == cudaSuccess) e = cudaMemcpy(grid_grad, h->gridGrad, sizeof(float) * gridN, cudaMemcpyDeviceToHost);
	if (e == cudaSuccess) e = cudaMemcpy(weight_grad, h->wGrad, sizeof(float) * kWTotal, cudaMemcpyDeviceToHost);
	if (e == cudaSuccess) e = cudaMemset(h->gridGrad, 0, sizeof(float) * gridN);
	if (e == cudaSuccess) e = cudaMemset(h->wGrad, 0, sizeof(float) * kWTotal);
	return e == cudaSuccess ? RB_OK : nrcFail(e);
}

int rb_nrc_train(rb_nrc* h, uint32_t n, const float* inputs, const float* targets, float* loss_out, void* stream)
{
	if (!h || n == 0 || n > kMaxTrainRows || !inputs || !targets) return RB_ERR_INVALID;
	cudaSetDevice(h->device);
	const cudaStream_t st = static_cast<cudaStream_t>(stream);
	const int rc = rb::nrc::trainRows(h, n, nullptr, inputs, targets, st, false);
	if (rc != RB_OK) return rc;
	if (loss_out) cudaMemcpyAsync(loss_out, h->loss, sizeof(float), cudaMemcpyDefault, st);
	const cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}

} // extern "C"

namespace rb
{
namespace nrc
{
int applyQueries(rb_nrc* h, uint32_t cap, const uint32_t* count, const float* inputs, const uint32_t* path, float4* L,
	const float4* T, const float* corr, cudaStream_t st)
{
	if (cap == 0) return RB_OK;
	kMlpInfer<<<inferBlocks(h, cap), kInferThreads, kSmemInfer, st>>>(cap, count, inputs, reinterpret_cast<const __half2*>(h->grid),
		h->R, h->w, nullptr, path, L, T, corr);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}

const float* lossDevice(const rb_nrc* h) { return h->loss; }
int deviceOf(const rb_nrc* h) { return h->device; }

int trainRows(rb_nrc* h, uint32_t n, const uint32_t* valid, const float* inputs, const float* targets, cudaStream_t st,
	bool withDrop, float* corr)
{
	const int rc = withDrop ? computeGradients(h, n, inputs, targets, st, valid, kDropOutput + 1, 8, corr)
		: computeGradients(h, n, inputs, targets, st, valid);
	if (rc != RB_OK) return rc;
	++h->step;
	const float b1 = h->cfg.beta1, b2 = h->cfg.beta2;
	const float c1 = 1.0f - std::pow(b1, static_cast<float>(h->step)), c2 = 1.0f - std::pow(b2, static_cast<float>(h->step));
	kAdam<<<4 * h->smCount, 256, 0, st>>>(static_cast<uint32_t>(rb_nrc_grid_size()), h->gridF32, h->gridGrad, h->gridM,
		h->gridV, h->cfg.learning_rate, b1, b2, h->cfg.epsilon, c1, c2, nullptr, h->grid);
	kAdam<<<64, 256, 0, st>>>(kWTotal, h->wF32, h->wGrad, h->wM, h->wV, h->cfg.learning_rate, b1, b2, h->cfg.epsilon,
		c1, c2, h->w, nullptr);
	kTransposeWeights<<<64, 256, 0, st>>>(h->wF32, h->wt);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}
} // namespace nrc
} // namespace rb
