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
// Tensor cores: inference (with the encoding fused in), the training forward
// and the backward chain dX = dY W run on tcgen05 (rb_umma.cuh): 128-row
// tiles in swizzled shared memory, BF16 operands, FP32 accumulators in
// tensor memory, one thread per row for the epilogue (ReLU, repack to BF16
// in place as the next layer's input). The weight gradients dW = dY^T X of
// all five layers are one hand-written kernel (mma.sync over the batch,
// operands transposed by ldmatrix). Adam runs in FP32 on the master copies.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "rb_launch.cuh"
#include "ratbite_b200_nrc.h"
#include "rb_nrc_internal.h"
#include "rb_umma.cuh"

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
constexpr int kWStride = 72;                            // smem row stride (bf16) of kWeightGrad, conflict-free ldmatrix
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

// ------------------------------------------------- tcgen05 (Blackwell) tiles
// The MLP on the 5th-generation tensor cores (rb_umma.cuh): a CTA of 128
// threads owns a tile of 128 rows; thread t owns row t of the tile for the
// whole pass (it writes the row's inputs into the swizzled activation tile,
// reads the row's accumulator lane back from TMEM, applies ReLU, and writes
// the row of the next layer's input in place). One thread issues each
// layer's MMAs (M = 128, N = 64 or 16, four K steps of 16) and commits them
// to an mbarrier; the CTA waits on it (bounded; a wait that gives up sets
// RB_DEV_ITERATION_LIMIT in *status and the CTA stops). Several CTAs per SM
// (about 51 KB of shared memory and 64 TMEM columns each) overlap one
// tile's grid gathers with another's MMAs.
namespace t5
{
constexpr uint32_t kRows = 128;
constexpr uint32_t kWBytes = 8192;                       // one 64 x 64 layer
constexpr uint32_t kOffW4 = 4 * kWBytes;                 // output layer: 16 rows (2 KB)
constexpr uint32_t kOffAct = kOffW4 + 2048;              // 34816: activation tile, 16 KB
constexpr uint32_t kOffBar = kOffAct + kRows * 128;      // mbarrier (8 B) + TMEM slot (4 B)
constexpr uint32_t kSmem = kOffBar + 16 + 1024;          // + alignment slack of the dynamic base
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kWaitLimit = 1u << 22;
static_assert(kOffAct % 1024 == 0, "operand tiles start on 1024-byte boundaries");

RB_D unsigned char* alignBase(unsigned char* p)
{
	return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 1023u) & ~static_cast<uintptr_t>(1023u));
}
RB_D unsigned char* layerTile(unsigned char* base, int l) { return base + (l < 4 ? l * kWBytes : kOffW4); }

// Copies 272 rows of 64 bf16 ([out][in] per layer, or [in][out] for the
// transposed copy) into the swizzled tiles: rows 0..255 layers 0..3, rows
// 256..271 the 16-row output block.
RB_D void stageLayers(const __nv_bfloat16* __restrict__ w, unsigned char* base)
{
	for (uint32_t i = threadIdx.x; i < 272u * 8u; i += blockDim.x)
	{
		const uint32_t row = i >> 3, c = i & 7u;
		const int l = row < 256u ? static_cast<int>(row >> 6) : 4;
		const uint32_t r = row < 256u ? (row & 63u) : row - 256u;
		*reinterpret_cast<uint4*>(layerTile(base, l) + r * 128u + (((c ^ r) & 7u) << 4)) =
			*reinterpret_cast<const uint4*>(w + static_cast<size_t>(row) * 64u + 8u * c);
	}
}

struct Ctx
{
	unsigned char* base;
	unsigned char* act;
	uint64_t* bar;
	uint32_t tmem;
	uint32_t phase;
};

// Prologue shared by the tcgen05 kernels: barrier, TMEM, weights.
RB_D Ctx begin(unsigned char* smraw, const __nv_bfloat16* __restrict__ w)
{
	Ctx c;
	c.base = alignBase(smraw);
	c.act = c.base + kOffAct;
	c.bar = reinterpret_cast<uint64_t*>(c.base + kOffBar);
	uint32_t* slot = reinterpret_cast<uint32_t*>(c.base + kOffBar + 8);
	if (threadIdx.x == 0) umma::barrierInit(c.bar, 1);
	if ((threadIdx.x >> 5) == 0) umma::tmemAlloc(slot, kTmemCols);
	stageLayers(w, c.base);
	umma::fenceProxyAsync();
	umma::fenceBeforeSync();
	__syncthreads();
	umma::fenceAfterSync();
	c.tmem = *slot;
	c.phase = 0;
	return c;
}
RB_D void end(const Ctx& c)
{
	umma::fenceBeforeSync();
	__syncthreads();
	if ((threadIdx.x >> 5) == 0) umma::tmemFree(c.tmem, kTmemCols);
}

// D = act (128 x 64) x layer(l)^T with nK K steps, then the CTA waits for
// it. Every thread must have written its row of `act` (and fenced it for
// the tensor cores) before. Returns false (uniformly) when the wait gave up.
RB_D bool layerMma(Ctx& c, const unsigned char* bTile, uint32_t n, int nK, uint32_t* status)
{
	if (threadIdx.x == 0)
	{
		umma::fenceAfterSync();
		const uint32_t idesc = umma::idescBf16(kRows, n);
		for (int k = 0; k < nK; ++k)
			umma::mma(c.tmem, umma::descK(c.act, static_cast<uint32_t>(k)), umma::descK(bTile, static_cast<uint32_t>(k)),
				idesc, k > 0);
		umma::commit(c.bar);
	}
	const bool ok = __syncthreads_and(umma::barrierWait(c.bar, c.phase, kWaitLimit)) != 0;
	c.phase ^= 1u;
	if (!ok)
	{
		if (threadIdx.x == 0) atomicOr(status, RB_DEV_ITERATION_LIMIT);
		// give the MMAs in flight a second bounded wait before TMEM is freed
		umma::barrierWait(c.bar, c.phase ^ 1u, kWaitLimit);
		return false;
	}
	umma::fenceAfterSync();
	return true;
}

// This thread's 64 accumulator columns.
RB_D void readAcc64(const Ctx& c, float (&v)[64])
{
	uint32_t r[4][16];
#pragma unroll
	for (int q = 0; q < 4; ++q) umma::tmemLoad16(umma::laneAddr(c.tmem, 16u * q), r[q]);
	umma::tmemWaitLoad();
#pragma unroll
	for (int q = 0; q < 4; ++q)
#pragma unroll
		for (int j = 0; j < 16; ++j) v[16 * q + j] = __uint_as_float(r[q][j]);
}
RB_D void readAcc16(const Ctx& c, float (&v)[16])
{
	uint32_t r[16];
	umma::tmemLoad16(umma::laneAddr(c.tmem, 0), r);
	umma::tmemWaitLoad();
#pragma unroll
	for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}
// After this thread's TMEM reads and its write of its row of `act`: make both
// safe for the next MMA.
RB_D void rowWritten()
{
	umma::fenceBeforeSync();
	umma::fenceProxyAsync();
	__syncthreads();
}
// Named barrier among the 128 threads of one role (the ids are immediates,
// so the kernel reserves only the barriers it uses), and its AND-reduction.
template<int ID>
RB_D void namedSync() { asm volatile("bar.sync %0, 128;" :: "n"(ID) : "memory"); }
template<int ID>
RB_D bool namedAnd(bool p)
{
	uint32_t out;
	asm volatile(
		"{\n\t.reg .pred pi, po;\n\t"
		"setp.ne.u32 pi, %1, 0;\n\t"
		"bar.red.and.pred po, %2, 128, pi;\n\t"
		"selp.u32 %0, 1, 0, po;\n\t}\n"
		: "=r"(out) : "r"(p ? 1u : 0u), "n"(ID) : "memory");
	return out != 0;
}

RB_D void reluPack(const float (&v)[64], uint32_t (&row)[32])
{
#pragma unroll
	for (int j = 0; j < 32; ++j) row[j] = pack2(fmaxf(v[2 * j], 0.0f), fmaxf(v[2 * j + 1], 0.0f));
}
} // namespace t5

// Inference (the query path), warp-specialized: 8 encoder warps
// fill a ring of activation tiles with encoded rows (two threads per row,
// 8 grid levels each), 4 MLP warps run the five tcgen05 layers on each
// filled tile and apply the output. mbarriers pass the tiles (full: one
// arrival per encoder thread; empty: one arrival once the tile's last MMA
// has completed), so the encoders' grid gathers for the next tiles overlap
// the layers of the current one and no warp waits on a block-wide barrier.
// Every wait is bounded: one that gives up sets RB_DEV_ITERATION_LIMIT and
// its role stops; the other role's waits then give up too.
namespace ws
{
// Shape of the kernel, measured on B200 (cached Cornell frame 1920x1080x64,
// inference ms per frame). The grid gathers decide it: without the MLP the
// encoders alone took the whole time, and they depend on L1 hits (nearby
// queries share cells; loading the hashed levels without allocating in L1
// made it 41 ms). Shared memory the blocks take is carved out of the SM's
// 256 KB of L1, so the ring is short: 2 stages x 2 blocks 7.4 ms (164 KB
// carve-out config, about 90 KB of L1); 3 stages 8.3; 4 stages 14.5 (228 KB,
// about 28 KB of L1); one block of 16 encoder warps with 2 / 4 stages 8.2 /
// 8.4. At 4 stages, 12 or 16 encoder warps per block (64 / 48 registers) or
// 16-32 gathers issued together per thread were slower (16.3 - 20.5), and
// the encoder layout (one level per thread, half a row per thread, rows
// consecutive or strided per warp) moved it by less than 2 ms.
#ifndef RB_WS_ENC_WARPS
#define RB_WS_ENC_WARPS 8
#endif
constexpr uint32_t kEncWarps = RB_WS_ENC_WARPS, kMlpWarps = 4;
constexpr uint32_t kEncThreads = 32u * kEncWarps;
constexpr uint32_t kThreads = kEncThreads + 32u * kMlpWarps;
#ifndef RB_WS_STAGES
#define RB_WS_STAGES 2
#endif
constexpr uint32_t kStages = RB_WS_STAGES;
constexpr uint32_t kTileBytes = t5::kRows * 128u;
constexpr uint32_t kOffStages = t5::kOffAct;
constexpr uint32_t kOffBars = kOffStages + kStages * kTileBytes;  // full[kStages], empty[kStages], mma, TMEM slot
constexpr uint32_t kSmem = kOffBars + 8u * (2u * kStages + 1u) + 8u + 1024u;
// Blocks per SM the kernel is compiled and launched for. Shared memory the
// blocks do not take is L1, which the grid gathers depend on.
#ifndef RB_WS_CTAS
#define RB_WS_CTAS 2
#endif
constexpr int kMinBlocks = RB_WS_CTAS;
static_assert(kOffStages % 1024 == 0 && kTileBytes % 1024 == 0, "operand tiles start on 1024-byte boundaries");
static_assert(kEncThreads % 16u == 0 && kEncThreads >= 256u, "whole levels per thread; the remaining columns in one pass");
#ifndef RB_WS_ENCODE_UNROLL
#define RB_WS_ENCODE_UNROLL 8
#endif
constexpr int kWsEncodeUnroll = RB_WS_ENCODE_UNROLL;
// Rows of an encoder warp: 1, 16 consecutive rows per warp; 0, rows strided
// over the tile.
#ifndef RB_WS_ENCODE_MAP
#define RB_WS_ENCODE_MAP 1
#endif

// Encoder thread e keeps one grid level, l = e % 16, and encodes it for rows
// e / 16, e / 16 + kEncThreads / 16, ... of the tile, so a warp's gathers at
// one instruction cover 16 levels of 2 rows (the level's resolution and table
// are per-thread constants); then threads 0..255 write the 32 remaining
// columns, 16 for each of rows e / 2.
RB_D void encodeLevels(uint32_t t0, uint32_t n, const float* __restrict__ in, const __half2* __restrict__ grid,
	const Resolutions& R, unsigned char* tile)
{
	const uint32_t e = threadIdx.x, l = e & 15u;
#if RB_WS_ENCODE_MAP
	// warp w takes rows W w .. W w + W - 1, W = 128 / encoder warps
	// (consecutive queries, nearby pixels): lane k gathers level k % 16 of
	// rows W w + k / 16 + 2 i
	constexpr uint32_t kWarpRows = t5::kRows / kEncWarps;
	static_assert(t5::kRows % kEncWarps == 0 && kWarpRows % 2 == 0, "whole row pairs per encoder warp");
	const uint32_t base = kWarpRows * (e >> 5) + ((e >> 4) & 1u);
#pragma unroll kWsEncodeUnroll
	for (uint32_t i = 0; i < kWarpRows / 2; ++i)
	{
		const uint32_t rl = base + 2u * i, r = t0 + rl;
		float f0 = 0.0f, f1 = 0.0f;
		if (r < n)
		{
			const float* v = in + static_cast<size_t>(kNrcInputs) * r;
			levelFeatures(R, grid, static_cast<int>(l), clamp01(v[0]), clamp01(v[1]), clamp01(v[2]), f0, f1);
		}
		*reinterpret_cast<uint32_t*>(tile + umma::swzOffset(rl, 2u * l)) = pack2(f0, f1);
	}
#else
#pragma unroll kWsEncodeUnroll
	for (uint32_t rl = e >> 4; rl < t5::kRows; rl += kEncThreads / 16u)
	{
		const uint32_t r = t0 + rl;
		float f0 = 0.0f, f1 = 0.0f;
		if (r < n)
		{
			const float* v = in + static_cast<size_t>(kNrcInputs) * r;
			levelFeatures(R, grid, static_cast<int>(l), clamp01(v[0]), clamp01(v[1]), clamp01(v[2]), f0, f1);
		}
		*reinterpret_cast<uint32_t*>(tile + umma::swzOffset(rl, 2u * l)) = pack2(f0, f1);
	}
#endif
	if (e >= 2u * t5::kRows) return;
	const uint32_t rl = e >> 1, r = t0 + rl, k0 = 16u * (e & 1u);
	const float* v = in + static_cast<size_t>(kNrcInputs) * r;
	uint32_t w[8];
#pragma unroll
	for (int j = 0; j < 8; ++j)
		w[j] = r < n ? pack2(restColumn(v, static_cast<int>(k0) + 2 * j), restColumn(v, static_cast<int>(k0) + 2 * j + 1)) : 0u;
	const uint32_t c = 4u + (k0 >> 3);
	unsigned char* row = tile + rl * 128u;
	*reinterpret_cast<uint4*>(row + (((c ^ rl) & 7u) << 4)) = make_uint4(w[0], w[1], w[2], w[3]);
	*reinterpret_cast<uint4*>(row + ((((c + 1u) ^ rl) & 7u) << 4)) = make_uint4(w[4], w[5], w[6], w[7]);
}

// Hidden layer epilogue for row m, in two halves of 32 columns (so that the
// 64-register cap of 16 warps per block holds): TMEM -> ReLU -> BF16 ->
// chunks 4 h .. 4 h + 3 of the row, in place.
RB_D void reluRowHalves(uint32_t tmem, unsigned char* act, uint32_t m)
{
#pragma unroll
	for (uint32_t h = 0; h < 2; ++h)
	{
		uint32_t q0[16], q1[16];
		umma::tmemLoad16(umma::laneAddr(tmem, 32u * h), q0);
		umma::tmemLoad16(umma::laneAddr(tmem, 32u * h + 16u), q1);
		umma::tmemWaitLoad();
		uint32_t w[16];
#pragma unroll
		for (int j = 0; j < 8; ++j)
		{
			w[j] = pack2(fmaxf(__uint_as_float(q0[2 * j]), 0.0f), fmaxf(__uint_as_float(q0[2 * j + 1]), 0.0f));
			w[8 + j] = pack2(fmaxf(__uint_as_float(q1[2 * j]), 0.0f), fmaxf(__uint_as_float(q1[2 * j + 1]), 0.0f));
		}
		unsigned char* row = act + m * 128u;
#pragma unroll
		for (uint32_t c = 0; c < 4; ++c)
			*reinterpret_cast<uint4*>(row + ((((4u * h + c) ^ m) & 7u) << 4)) =
				make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
	}
}
} // namespace ws

__global__ void __launch_bounds__(ws::kThreads, ws::kMinBlocks) kMlpInferWS(uint32_t cap, const uint32_t* __restrict__ count,
	const float* __restrict__ in, const __half2* __restrict__ grid, Resolutions R, const __nv_bfloat16* __restrict__ w,
	float* __restrict__ out, const uint32_t* __restrict__ path, float4* __restrict__ L, const float4* __restrict__ T,
	const float* __restrict__ corr, uint32_t* __restrict__ status)
{
	extern __shared__ unsigned char smraw[];
	unsigned char* base = t5::alignBase(smraw);
	uint64_t* full = reinterpret_cast<uint64_t*>(base + ws::kOffBars);
	uint64_t* empty = full + ws::kStages;
	uint64_t* mmaBar = empty + ws::kStages;
	uint32_t* slot = reinterpret_cast<uint32_t*>(mmaBar + 1);
	const uint32_t warp = threadIdx.x >> 5;
	if (threadIdx.x == 0)
	{
		for (uint32_t s = 0; s < ws::kStages; ++s)
		{
			umma::barrierInit(full + s, 32u * ws::kEncWarps);
			umma::barrierInit(empty + s, 1);
		}
		umma::barrierInit(mmaBar, 1);
	}
	if (warp == 0) umma::tmemAlloc(slot, t5::kTmemCols);
	t5::stageLayers(w, base);
	umma::fenceProxyAsync();
	umma::fenceBeforeSync();
	__syncthreads();
	umma::fenceAfterSync();
	const uint32_t tmem = *slot;
	const uint32_t n = count ? min(*count, cap) : cap;
	const uint32_t tiles = (n + t5::kRows - 1) / t5::kRows;
	if (warp < ws::kEncWarps)
	{
		uint32_t k = 0;
		for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++k)
		{
			const uint32_t s = k % ws::kStages;
			if (k >= ws::kStages && !umma::barrierWait(empty + s, ((k / ws::kStages) + 1u) & 1u, t5::kWaitLimit))
			{
				atomicOr(status, RB_DEV_ITERATION_LIMIT);
				break;
			}
			unsigned char* tile = base + ws::kOffStages + s * ws::kTileBytes;
			ws::encodeLevels(t * t5::kRows, n, in, grid, R, tile);
			umma::fenceProxyAsync();
			umma::barrierArrive(full + s);
		}
	}
	else
	{
		// MLP: thread m owns row m of the tile and TMEM lane m
		const uint32_t m = threadIdx.x - 32u * ws::kEncWarps;
		uint32_t k = 0, mmaPhase = 0;
		bool ok = true;
		for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++k)
		{
			const uint32_t s = k % ws::kStages;
			unsigned char* act = base + ws::kOffStages + s * ws::kTileBytes;
			ok = t5::namedAnd<1>(umma::barrierWait(full + s, (k / ws::kStages) & 1u, t5::kWaitLimit));
			if (!ok)
			{
				if (m == 0) atomicOr(status, RB_DEV_ITERATION_LIMIT);
				break;
			}
			umma::fenceAfterSync();
			for (int l = 0; l < 5; ++l)
			{
				if (m == 0)
				{
					const uint32_t idesc = umma::idescBf16(t5::kRows, l < 4 ? 64u : 16u);
					const unsigned char* bTile = t5::layerTile(base, l);
					for (uint32_t kk = 0; kk < 4; ++kk)
						umma::mma(tmem, umma::descK(act, kk), umma::descK(bTile, kk), idesc, kk > 0);
					umma::commit(mmaBar);
				}
				ok = t5::namedAnd<1>(umma::barrierWait(mmaBar, mmaPhase, t5::kWaitLimit));
				mmaPhase ^= 1u;
				if (!ok) break;
				umma::fenceAfterSync();
				if (l == 4) break;
				ws::reluRowHalves(tmem, act, m);
				umma::fenceBeforeSync();
				umma::fenceProxyAsync();
				t5::namedSync<1>();
			}
			if (!ok)
			{
				if (m == 0) atomicOr(status, RB_DEV_ITERATION_LIMIT);
				umma::barrierWait(mmaBar, mmaPhase ^ 1u, t5::kWaitLimit);
				break;
			}
			uint32_t ro[16];
			umma::tmemLoad16(umma::laneAddr(tmem, 0), ro);
			umma::tmemWaitLoad();
			umma::fenceBeforeSync();
			t5::namedSync<1>();              // every lane read before the next tile's MMAs
			if (m == 0) umma::barrierArrive(empty + s);
			const uint32_t r = t * t5::kRows + m;
			if (r < n)
			{
				const float4 y = make_float4(__uint_as_float(ro[0]), __uint_as_float(ro[1]), __uint_as_float(ro[2]),
					__uint_as_float(ro[3]));
				if (out) reinterpret_cast<float4*>(out)[r] = y;
				if (path)
				{
					// the plain estimator drops a whole sample whose later BxDF
					// sample fails: the prefix survives with 1 - q, q plus the
					// correction measured on the path's class (the path index's
					// high bit: the camera ray hit an emitter); the radiance is
					// scaled by the measured ratio of targets to predictions
					const uint32_t pr = path[r];
					const uint32_t p = pr & 0x7FFFFFFFu;
					const float4 tt = T[p];
					const float qq = __uint_as_float(ro[4]) + (corr ? corr[((pr >> 31) ? kCorrDropLit : kCorrDropOther) + 2] : 0.0f);
					const float keep = fminf(fmaxf(1.0f - qq, 0.0f), 1.0f);
					const float sc = corr && corr[kCorrRadiance + 3] > 0.0f ? corr[kCorrRadiance + 2] : 1.0f;
					float4 l = L[p];
					l.x = l.x * keep + tt.x * (sc * fmaxf(y.x, 0.0f));
					l.y = l.y * keep + tt.y * (sc * fmaxf(y.y, 0.0f));
					l.z = l.z * keep + tt.z * (sc * fmaxf(y.z, 0.0f));
					l.w = l.w * keep + tt.w * (sc * fmaxf(y.w, 0.0f));
					L[p] = l;
				}
			}
		}
	}
	umma::fenceBeforeSync();
	__syncthreads();
	if (warp == 0) umma::tmemFree(tmem, t5::kTmemCols);
}

// Training forward on the encoded rows X [n][64] (kMlpForward's contract):
// out [n][kOutStride] f32 and the post-ReLU hidden rows acts [4][n][64] bf16.
__global__ void __launch_bounds__(128) kMlpForwardT(uint32_t n, const __nv_bfloat16* __restrict__ X,
	const __nv_bfloat16* __restrict__ w, float* __restrict__ out, __nv_bfloat16* __restrict__ acts,
	uint32_t* __restrict__ status)
{
	extern __shared__ unsigned char smraw[];
	t5::Ctx c = t5::begin(smraw, w);
	bool ok = true;
	for (uint32_t r0 = blockIdx.x * t5::kRows; r0 < n && ok; r0 += gridDim.x * t5::kRows)
	{
		const uint32_t r = r0 + threadIdx.x;
		{
			uint32_t row[32];
#pragma unroll
			for (int j = 0; j < 8; ++j)
			{
				const uint4 q = r < n ? *reinterpret_cast<const uint4*>(X + static_cast<size_t>(r) * kIn + 8 * j)
					: make_uint4(0u, 0u, 0u, 0u);
				row[4 * j] = q.x; row[4 * j + 1] = q.y; row[4 * j + 2] = q.z; row[4 * j + 3] = q.w;
			}
			umma::storeRow(c.act, threadIdx.x, row);
		}
		umma::fenceProxyAsync();
		__syncthreads();
		for (int l = 0; l < 4 && ok; ++l)
		{
			ok = t5::layerMma(c, t5::layerTile(c.base, l), 64, 4, status);
			if (!ok) break;
			float v[64];
			t5::readAcc64(c, v);
			uint32_t row[32];
			t5::reluPack(v, row);
			umma::storeRow(c.act, threadIdx.x, row);
			if (acts && r < n)
			{
				uint4* dst = reinterpret_cast<uint4*>(acts + (static_cast<size_t>(l) * n + r) * kIn);
#pragma unroll
				for (int j = 0; j < 8; ++j) dst[j] = make_uint4(row[4 * j], row[4 * j + 1], row[4 * j + 2], row[4 * j + 3]);
			}
			t5::rowWritten();
		}
		if (!ok) break;
		ok = t5::layerMma(c, t5::layerTile(c.base, 4), 16, 4, status);
		if (!ok) break;
		float o[16];
		t5::readAcc16(c, o);
		if (r < n)
		{
			float4* dst = reinterpret_cast<float4*>(out + static_cast<size_t>(kOutStride) * r);
			dst[0] = make_float4(o[0], o[1], o[2], o[3]);
			dst[1] = make_float4(o[4], o[5], o[6], o[7]);
		}
		umma::fenceBeforeSync();
		__syncthreads();
	}
	t5::end(c);
}

// Backward through the layers (kMlpBackward's contract) with the
// transposed weights wt (rows [in][out]: W4^T as 64 rows of 16 outputs, then
// W3^T..W0^T): g4 = dY W4 masked by ReLU'(h4), ..., dX = g1 W0. Writes the
// masked gradients dH [4][n][64] (layer l at block l: g_{l+1}) and the
// gradient of the 32 grid features dX0 [n][32] (f32).
__global__ void __launch_bounds__(128) kMlpBackwardT(uint32_t n, const __nv_bfloat16* __restrict__ dY,
	const __nv_bfloat16* __restrict__ wt, const __nv_bfloat16* __restrict__ acts, __nv_bfloat16* __restrict__ dH,
	float* __restrict__ dX0, uint32_t* __restrict__ status)
{
	extern __shared__ unsigned char smraw[];
	unsigned char* base = t5::alignBase(smraw);
	// transposed tiles: W4^T (64 rows of 16 outputs, zero-padded to 64
	// columns) at tile 0, then W3^T, W2^T, W1^T, W0^T at tiles 1..4 (all 64
	// rows; the output-layer slot of the forward layout is not used)
	{
		for (uint32_t i = threadIdx.x; i < 64u * 8u; i += blockDim.x)
		{
			const uint32_t r = i >> 3, ch = i & 7u;
			uint4 v = make_uint4(0u, 0u, 0u, 0u);
			if (ch < 2u) v = *reinterpret_cast<const uint4*>(wt + static_cast<size_t>(r) * 16u + 8u * ch);
			*reinterpret_cast<uint4*>(base + r * 128u + (((ch ^ r) & 7u) << 4)) = v;
		}
	}
	t5::Ctx c;
	c.base = base;
	c.act = base + 5 * t5::kWBytes;      // activation tile after the five 8 KB tiles
	c.bar = reinterpret_cast<uint64_t*>(c.act + t5::kRows * 128u);
	uint32_t* slot = reinterpret_cast<uint32_t*>(c.act + t5::kRows * 128u + 8u);
	if (threadIdx.x == 0) umma::barrierInit(c.bar, 1);
	if ((threadIdx.x >> 5) == 0) umma::tmemAlloc(slot, t5::kTmemCols);
	for (uint32_t i = threadIdx.x; i < 256u * 8u; i += blockDim.x)
	{
		const uint32_t row = i >> 3, ch = i & 7u, tile = 1u + (row >> 6), r = row & 63u;
		*reinterpret_cast<uint4*>(base + tile * t5::kWBytes + r * 128u + (((ch ^ r) & 7u) << 4)) =
			*reinterpret_cast<const uint4*>(wt + 64u * 16u + static_cast<size_t>(row) * 64u + 8u * ch);
	}
	umma::fenceProxyAsync();
	umma::fenceBeforeSync();
	__syncthreads();
	umma::fenceAfterSync();
	c.tmem = *slot;
	c.phase = 0;
	bool ok = true;
	for (uint32_t r0 = blockIdx.x * t5::kRows; r0 < n && ok; r0 += gridDim.x * t5::kRows)
	{
		const uint32_t r = r0 + threadIdx.x;
		{
			// dY row: 16 columns (4 used), zero-padded to 64
			uint32_t row[32];
#pragma unroll
			for (int j = 0; j < 32; ++j) row[j] = 0u;
			if (r < n)
			{
				const uint4 a = *reinterpret_cast<const uint4*>(dY + static_cast<size_t>(r) * kOutPad);
				const uint4 b = *reinterpret_cast<const uint4*>(dY + static_cast<size_t>(r) * kOutPad + 8);
				row[0] = a.x; row[1] = a.y; row[2] = a.z; row[3] = a.w;
				row[4] = b.x; row[5] = b.y; row[6] = b.z; row[7] = b.w;
			}
			umma::storeRow(c.act, threadIdx.x, row);
		}
		umma::fenceProxyAsync();
		__syncthreads();
		// tile 0: K = 16 (one step); tiles 1..4: K = 64
		for (int l = 3; l >= -1 && ok; --l)
		{
			const int tile = 3 - l;                  // W4^T, W3^T, ..., W0^T
			ok = t5::layerMma(c, base + tile * t5::kWBytes, 64, tile == 0 ? 1 : 4, status);
			if (!ok) break;
			float v[64];
			t5::readAcc64(c, v);
			if (l < 0)
			{
				// dX: the first 32 columns are the grid features
				if (r < n)
				{
					float4* dst = reinterpret_cast<float4*>(dX0 + static_cast<size_t>(kGridFeatures) * r);
#pragma unroll
					for (int j = 0; j < 8; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
				}
				umma::fenceBeforeSync();
				__syncthreads();
				break;
			}
			// mask by ReLU' of the layer's stored activation
			uint32_t row[32];
			if (r < n)
			{
				const uint4* hsrc = reinterpret_cast<const uint4*>(acts + (static_cast<size_t>(l) * n + r) * kIn);
#pragma unroll
				for (int j = 0; j < 8; ++j)
				{
					const uint4 h = hsrc[j];
					const uint32_t hw[4] = { h.x, h.y, h.z, h.w };
#pragma unroll
					for (int q = 0; q < 4; ++q)
					{
						const float2 hh = unpack2(hw[q]);
						const int k = 8 * j + 2 * q;
						row[4 * j + q] = pack2(hh.x > 0.0f ? v[k] : 0.0f, hh.y > 0.0f ? v[k + 1] : 0.0f);
					}
				}
				uint4* dst = reinterpret_cast<uint4*>(dH + (static_cast<size_t>(l) * n + r) * kIn);
#pragma unroll
				for (int j = 0; j < 8; ++j) dst[j] = make_uint4(row[4 * j], row[4 * j + 1], row[4 * j + 2], row[4 * j + 3]);
			}
			else
			{
#pragma unroll
				for (int j = 0; j < 32; ++j) row[j] = 0u;
			}
			umma::storeRow(c.act, threadIdx.x, row);
			t5::rowWritten();
		}
	}
	t5::end(c);
}
constexpr size_t kSmemBackwardT = 5 * t5::kWBytes + t5::kRows * 128 + 16 + 1024;

// Weight gradients dW_l[out][in] += sum over rows G_l[r][out] A_l[r][in]
// for all five layers in one launch (no library GEMM): G = dY (layer 4, 16
// columns) or dH block l, A = X (layer 0) or acts block l - 1. Block b takes
// layer b % 5 and a chunk of rows; its 4 warps each own 16 outputs x 64
// inputs (8 m16n8k16 tiles, FP32 accumulation), read through shared memory
// with ldmatrix.trans (both operands are row-major over the batch), and the
// partial sums are added to wGrad with one atomic per element.
constexpr uint32_t kWgRows = 1024;                      // rows per block
constexpr uint32_t kWgChunk = 64;                       // rows staged per step
RB_D void ldsm4t(uint32_t (&r)[4], const __nv_bfloat16* p)
{
	const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
	asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}
__global__ void __launch_bounds__(128) kWeightGrad(uint32_t n, const __nv_bfloat16* __restrict__ X,
	const __nv_bfloat16* __restrict__ acts, const __nv_bfloat16* __restrict__ dY, const __nv_bfloat16* __restrict__ dH,
	float* __restrict__ wGrad)
{
	__shared__ __align__(16) __nv_bfloat16 sG[kWgChunk][kWStride];
	__shared__ __align__(16) __nv_bfloat16 sA[kWgChunk][kWStride];
	const uint32_t layer = blockIdx.x % 5u, chunk = blockIdx.x / 5u;
	const uint32_t rBegin = chunk * kWgRows;
	if (rBegin >= n) return;
	const uint32_t rEnd = min(n, rBegin + kWgRows);
	const uint32_t outs = layer == 4u ? static_cast<uint32_t>(kOutPad) : 64u;
	const __nv_bfloat16* G = layer == 4u ? dY : dH + static_cast<size_t>(layer) * n * kIn;
	const uint32_t gStride = layer == 4u ? static_cast<uint32_t>(kOutPad) : static_cast<uint32_t>(kIn);
	const __nv_bfloat16* A = layer == 0u ? X : acts + static_cast<size_t>(layer - 1u) * n * kIn;
	const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
	const bool active = warp * 16u < outs;           // layer 4: one warp (16 outputs)
	float acc[8][4];
#pragma unroll
	for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
	for (uint32_t c0 = rBegin; c0 < rEnd; c0 += kWgChunk)
	{
		__syncthreads();
		// stage rows c0 .. c0+63 of G (outs columns) and A (64 columns), zero beyond rEnd
		for (uint32_t i = threadIdx.x; i < kWgChunk * 8u; i += blockDim.x)
		{
			const uint32_t rr = i >> 3, ch = i & 7u, r = c0 + rr;
			uint4 a = make_uint4(0u, 0u, 0u, 0u), g = a;
			if (r < rEnd)
			{
				a = *reinterpret_cast<const uint4*>(A + static_cast<size_t>(r) * kIn + 8u * ch);
				if (8u * ch < outs) g = *reinterpret_cast<const uint4*>(G + static_cast<size_t>(r) * gStride + 8u * ch);
			}
			*reinterpret_cast<uint4*>(&sA[rr][8u * ch]) = a;
			*reinterpret_cast<uint4*>(&sG[rr][8u * ch]) = g;
		}
		__syncthreads();
		if (!active) continue;
		// K steps of 16 rows: A fragment (16 outputs x 16 rows) = G^T, B (16 rows x 8 inputs) = A
#pragma unroll
		for (uint32_t k = 0; k < kWgChunk; k += 16)
		{
			// G^T fragment: matrices (rows k..k+7 | k+8..k+15) x (outputs o..o+7 | o+8..o+15), transposed
			uint32_t af[4];
			{
				const uint32_t m = lane >> 3, rr = lane & 7u;
				// a0: out 0-7 x rows 0-7; a1: out 8-15 x rows 0-7; a2: out 0-7 x rows 8-15; a3: out 8-15 x rows 8-15
				const uint32_t rowOff = (m & 2u) ? 8u : 0u, colOff = (m & 1u) ? 8u : 0u;
				ldsm4t(af, &sG[k + rowOff + rr][warp * 16u + colOff]);
			}
#pragma unroll
			for (int j = 0; j < 8; j += 2)
			{
				// B fragments of input tiles j, j+1: (rows k..k+15) x (inputs 8j..8j+7), col-major = A rows
				uint32_t bf[4];
				const uint32_t m = lane >> 3, rr = lane & 7u;
				// b0(j): rows 0-7, b1(j): rows 8-15, b0(j+1): rows 0-7, b1(j+1): rows 8-15
				const uint32_t rowOff = (m & 1u) ? 8u : 0u, col = 8u * (j + (m >> 1));
				ldsm4t(bf, &sA[k + rowOff + rr][col]);
				mma16816(acc[j], af, bf[0], bf[1]);
				mma16816(acc[j + 1], af, bf[2], bf[3]);
			}
		}
	}
	if (!active) return;
	// accumulator fragment: rows (outputs) g, g+8 of the warp's 16; columns 2c, 2c+1 of tile j
	const uint32_t g = lane >> 2, c = lane & 3u;
	float* dst = wGrad + wOffset(static_cast<int>(layer));
#pragma unroll
	for (int j = 0; j < 8; ++j)
	{
		const uint32_t o0 = warp * 16u + g, in0 = 8u * j + 2u * c;
		atomicAdd(dst + o0 * kH + in0, acc[j][0]);
		atomicAdd(dst + o0 * kH + in0 + 1, acc[j][1]);
		atomicAdd(dst + (o0 + 8u) * kH + in0, acc[j][2]);
		atomicAdd(dst + (o0 + 8u) * kH + in0 + 1, acc[j][3]);
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
	uint32_t* status = nullptr;            // RB_DEV_* bits of the network's kernels
	uint32_t step = 0;
	int smCount = 148;
	uint32_t wsBlocksPerSm = 1, forwardBlocksPerSm = 1, trainBlocksPerSm = 1;
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

// Resident blocks per SM of a tcgen05 kernel of `threads` threads that
// allocates `tmemCols` TMEM columns, from the SM's limits: shared memory
// (with the per-block reservation), registers (per warp in units of 256),
// threads, and tensor memory (512 columns). The kernels loop over tiles, so the grid is this many
// blocks per SM; a grid of one block per SM leaves the grid gathers with
// 4 warps per SM to hide their latency.
uint32_t residentTileBlocks(const void* fn, size_t dynSmem, int device, uint32_t threads, uint32_t tmemCols)
{
	int smemSm = 0, reserved = 0, regsSm = 0, threadsSm = 0;
	cudaDeviceGetAttribute(&smemSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
	cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
	cudaDeviceGetAttribute(&regsSm, cudaDevAttrMaxRegistersPerMultiprocessor, device);
	cudaDeviceGetAttribute(&threadsSm, cudaDevAttrMaxThreadsPerMultiProcessor, device);
	cudaFuncAttributes fa{};
	if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess || smemSm <= 0 || regsSm <= 0 || threadsSm <= 0) return 1;
	const size_t perBlockSmem = dynSmem + fa.sharedSizeBytes + static_cast<size_t>(reserved);
	const uint32_t bySmem = static_cast<uint32_t>(static_cast<size_t>(smemSm) / perBlockSmem);
	const uint32_t warpRegs = (static_cast<uint32_t>(fa.numRegs) * 32u + 255u) / 256u * 256u;
	const uint32_t byRegs = warpRegs ? static_cast<uint32_t>(regsSm) / ((threads / 32u) * warpRegs) : 32u;
	const uint32_t byThreads = static_cast<uint32_t>(threadsSm) / threads;
	const uint32_t byTmem = 512u / tmemCols;
	const uint32_t b = std::min({ bySmem, byRegs, byThreads, byTmem });
	return b < 1 ? 1u : b;
}

// Blocks of the tcgen05 kernels: one 128-row tile per block and step, at
// most perSm resident blocks per SM (the kernels loop over tiles).
int tileBlocks(const rb_nrc* h, uint32_t rows, uint32_t perSm)
{
	const uint32_t tiles = (rows + t5::kRows - 1) / t5::kRows;
	const uint32_t cap = static_cast<uint32_t>(h->smCount) * perSm;
	return static_cast<int>(tiles < 1 ? 1 : (tiles < cap ? tiles : cap));
}
// Queries [0, min(*count, cap)) (count null: cap rows): outputs to `out`
// and/or the cached-form update of L (path, T, corr).
void launchInfer(const rb_nrc* h, uint32_t cap, const uint32_t* count, const float* in, float* out, const uint32_t* path,
	float4* L, const float4* T, const float* corr, cudaStream_t st)
{
	const __half2* grid = reinterpret_cast<const __half2*>(h->grid);
	const uint32_t tiles = (cap + t5::kRows - 1) / t5::kRows;
	const uint32_t most = static_cast<uint32_t>(h->smCount) * h->wsBlocksPerSm;
	const int blocks = static_cast<int>(tiles < 1 ? 1 : (tiles < most ? tiles : most));
	kMlpInferWS<<<blocks, ws::kThreads, ws::kSmem, st>>>(cap, count, in, grid, h->R, h->w, out, path, L, T, corr,
		h->status);
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
	if (e == cudaSuccess) e = cudaMalloc(&h->status, sizeof(uint32_t));
	if (e == cudaSuccess) e = cudaMemset(h->status, 0, sizeof(uint32_t));
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
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kMlpForwardT), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(t5::kSmem));
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kMlpBackwardT), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kSmemBackwardT));
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kMlpInferWS), cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(ws::kSmem));
	h->wsBlocksPerSm = std::min<uint32_t>(static_cast<uint32_t>(ws::kMinBlocks),
		residentTileBlocks(reinterpret_cast<const void*>(kMlpInferWS), ws::kSmem, h->device, ws::kThreads, t5::kTmemCols));
	// shared memory for exactly that many blocks, the rest of the SM's 256 KB as L1
	cudaFuncSetAttribute(reinterpret_cast<const void*>(kMlpInferWS), cudaFuncAttributePreferredSharedMemoryCarveout,
		static_cast<int>(std::min<uint32_t>(100u, (h->wsBlocksPerSm * (ws::kSmem + 1024u) * 100u + 233471u) / 233472u)));
	h->forwardBlocksPerSm = residentTileBlocks(reinterpret_cast<const void*>(kMlpForwardT), t5::kSmem, h->device, 128u,
		t5::kTmemCols);
	h->trainBlocksPerSm = residentTileBlocks(reinterpret_cast<const void*>(kMlpBackwardT), kSmemBackwardT, h->device, 128u,
		t5::kTmemCols);
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
			(void*)h->acts, (void*)h->dY, (void*)h->dH, (void*)h->out, (void*)h->dX0, (void*)h->loss,
			(void*)h->status })
		if (p) cudaFree(p);
	delete h;
	return RB_OK;
}

size_t rb_nrc_grid_size(void) { return static_cast<size_t>(kLevels) * kTable * kFeat; }

int rb_nrc_status(rb_nrc* h, uint32_t* flags)
{
	if (!h || !flags) return RB_ERR_INVALID;
	cudaSetDevice(h->device);
	cudaError_t e = cudaDeviceSynchronize();
	if (e == cudaSuccess) e = cudaMemcpy(flags, h->status, sizeof(uint32_t), cudaMemcpyDeviceToHost);
	return e == cudaSuccess ? RB_OK : nrcFail(e);
}
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
	h->step = 0;              // the optimiser starts over with the new parameters
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
	launchInfer(h, n, nullptr, inputs, outputs, nullptr, nullptr, nullptr, nullptr, st);
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
	kMlpForwardT<<<tileBlocks(h, n, h->forwardBlocksPerSm), 128, t5::kSmem, st>>>(n, h->X, h->w, h->out, h->acts,
		h->status);
	kLoss<<<gridFor(n), kThreads, 0, st>>>(n, h->out, targets, h->dY, h->loss, valid, outs, tStride, corr);
	kMlpBackwardT<<<tileBlocks(h, n, h->trainBlocksPerSm), 128, kSmemBackwardT, st>>>(n, h->dY, h->wt, h->acts, h->dH,
		h->dX0, h->status);
	// weight gradients of the five layers, one launch
	kWeightGrad<<<5 * ((n + kWgRows - 1) / kWgRows), 128, 0, st>>>(n, h->X, h->acts, h->dY, h->dH, h->wGrad);
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
	launchInfer(h, cap, count, inputs, nullptr, path, L, T, corr, st);
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
