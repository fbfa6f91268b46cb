/* Oracle test infrastructure (not product code).
 *
 * C restatement of the environment-map CDF build and inversion.
 * mode 0 follows the reference kernels step for step (src/kernels/cdf.cu:
 * power = max(0, mean RGB) per texel :137-167; 4 texels per thread and a
 * block-wide Hillis-Steele scan of thread totals with the reference's block
 * size and chunking :287-323, :332-412; sin(pi*(4i+k+0.5)/h) row weights
 * :105-133 applied to the float row totals; in-place normalisation; binary
 * search inversion :493-535). The CUDA block is emulated sequentially, one
 * scan step at a time over all threads, so every float addition happens in
 * the same order as on the GPU. Only sinf may differ (libm versus CUDA) in
 * the last ulp, so mode-0 marginals are compared with that in mind.
 * mode 1 restates the project's float64 variant in the kernel's exact order
 * (thread-serial prefix, warp Kogge-Stone, warp-total scan, running total). */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_restate.h"

static int block_size(uint32_t n4) { return n4 <= 256 ? 256 : (n4 <= 512 ? 512 : 1024); }

static float power_of(const float* t) { float p = (t[0] + t[1] + t[2]) / 3.0f; return p > 0.0f ? p : 0.0f; }

/* Reference-order scan of groups of 4 floats (in: n4*4 values), writes the
 * inclusive unnormalised prefix to out and returns the total. */
static float scan_reference(const float* in, uint32_t n4, int B, float* out)
{
	float total = 0.0f;
	const uint32_t chunks = (n4 + B - 1) / B;
	float (*v)[4] = malloc(sizeof(float) * 4 * B);
	float* sm = malloc(sizeof(float) * B);
	for (uint32_t k = 0; k < chunks; ++k)
	{
		for (int t = 0; t < B; ++t)
		{
			const uint32_t g = t + B * k;
			for (int q = 0; q < 4; ++q) v[t][q] = g < n4 ? in[4 * g + q] : 0.0f;
			v[t][1] += v[t][0]; v[t][2] += v[t][1]; v[t][3] += v[t][2];
		}
		for (int i = 1; i < B; i <<= 1)
		{
			for (int t = 0; t < B; ++t) sm[t] = v[t][3];
			for (int t = i; t < B; ++t)
			{
				const float o = sm[t - i];
				v[t][0] += o; v[t][1] += o; v[t][2] += o; v[t][3] += o;
			}
		}
		for (int t = 0; t < B; ++t)
			for (int q = 0; q < 4; ++q) v[t][q] += total;
		total = v[B - 1][3];
		for (int t = 0; t < B; ++t)
		{
			const uint32_t g = t + B * k;
			if (g < n4) for (int q = 0; q < 4; ++q) out[4 * g + q] = v[t][q];
		}
	}
	free(v);
	free(sm);
	return total;
}

/* The float64 kernel order (rb_envmap.cu scanDouble4). */
static double scan_double(const double* in, uint32_t n4, int B, double* out)
{
	double total = 0.0;
	const uint32_t chunks = (n4 + B - 1) / B;
	const int nw = B / 32;
	double (*c)[4] = malloc(sizeof(double) * 4 * B);
	double* s = malloc(sizeof(double) * B);
	double* sn = malloc(sizeof(double) * B);
	double* excl = malloc(sizeof(double) * B);
	double ws[32], wsn[32];
	for (uint32_t k = 0; k < chunks; ++k)
	{
		for (int t = 0; t < B; ++t)
		{
			const uint32_t g = t + B * k;
			for (int q = 0; q < 4; ++q) c[t][q] = g < n4 ? in[4 * g + q] : 0.0;
			c[t][1] = c[t][0] + c[t][1]; c[t][2] = c[t][1] + c[t][2]; c[t][3] = c[t][2] + c[t][3];
			s[t] = c[t][3];
		}
		for (int d = 1; d < 32; d <<= 1)
		{
			for (int t = 0; t < B; ++t) sn[t] = ((t & 31) >= d) ? s[t] + s[t - d] : s[t];
			memcpy(s, sn, sizeof(double) * B);
		}
		for (int t = 0; t < B; ++t) excl[t] = (t & 31) == 0 ? 0.0 : s[t - 1];
		for (int w = 0; w < 32; ++w) ws[w] = w < nw ? s[32 * w + 31] : 0.0;
		for (int d = 1; d < 32; d <<= 1)
		{
			for (int w = 0; w < 32; ++w) wsn[w] = w >= d ? ws[w] + ws[w - d] : ws[w];
			memcpy(ws, wsn, sizeof(ws));
		}
		for (int t = 0; t < B; ++t)
		{
			const int w = t >> 5;
			const double warpExcl = w == 0 ? 0.0 : ws[w - 1];
			const double base = (total + warpExcl) + excl[t];
			for (int q = 0; q < 4; ++q) c[t][q] = base + c[t][q];
		}
		total = c[B - 1][3];
		for (int t = 0; t < B; ++t)
		{
			const uint32_t g = t + B * k;
			if (g < n4) for (int q = 0; q < 4; ++q) out[4 * g + q] = c[t][q];
		}
	}
	free(c); free(s); free(sn); free(excl);
	return total;
}

static uint16_t invert_one(const float* cdf, int n, float p)
{
	int low = 0, high = n - 1, mid = (high - low) / 2;
	for (int it = 0; it < 64; ++it)
	{
		if (p > cdf[mid]) low = mid; else high = mid;
		mid = low + (high - low) / 2;
		if (low + 1 == high) break;
	}
	return (uint16_t)high;
}

int orc_envmap_cdf(uint32_t w, uint32_t h, const float* rgba, int mode, uint16_t* cond, uint16_t* marg, float* integral)
{
	if (w < 4 || h < 4 || (w & 3u) || (h & 3u) || w > 32768 || h > 32768) return -1;
	const int B = block_size(w / 4);
	float* rowF = malloc(sizeof(float) * w);
	float* cdf = malloc(sizeof(float) * (w > h ? w : h));
	double* rowD = malloc(sizeof(double) * (w > h ? w : h));
	double* outD = malloc(sizeof(double) * (w > h ? w : h));
	double* totals = malloc(sizeof(double) * h);
	for (uint32_t y = 0; y < h; ++y)
	{
		const float* row = rgba + (size_t)y * w * 4;
		if (mode == 0)
		{
			for (uint32_t i = 0; i < w; ++i) rowF[i] = power_of(row + 4 * i);
			const float total = scan_reference(rowF, w / 4, B, cdf);
			const float norm = total != 0.0f ? 1.0f / total : 0.0f;
			for (uint32_t i = 0; i < w; ++i) cdf[i] *= norm;
			totals[y] = (double)total;
		}
		else
		{
			for (uint32_t i = 0; i < w; ++i) rowD[i] = (double)power_of(row + 4 * i);
			const double total = scan_double(rowD, w / 4, B, outD);
			for (uint32_t i = 0; i < w; ++i)
			{
				const float parked = (float)outD[i];
				cdf[i] = total != 0.0 ? (float)((double)parked / total) : 0.0f;
			}
			totals[y] = total;
		}
		for (uint32_t i = 0; i < w; ++i)
			cond[(size_t)y * w + i] = invert_one(cdf, (int)w, (float)i / (float)((int)w - 1));
	}
	const uint32_t m4 = h / 4;
	if (mode == 0)
	{
		const float pi = 3.14159265358979323846f;
		for (uint32_t g = 0; g < m4; ++g)
		{
			const float off[4] = { 0.125f, 0.375f, 0.625f, 0.875f };
			for (int q = 0; q < 4; ++q)
				rowF[4 * g + q] = (float)totals[4 * g + q] * sinf(pi * ((float)g + off[q]) / (float)m4);
		}
		const float total = scan_reference(rowF, m4, B, cdf);
		const float norm = total != 0.0f ? 1.0f / total : 0.0f;
		for (uint32_t i = 0; i < h; ++i) cdf[i] *= norm;
		*integral = total / ((float)w * (float)h);
	}
	else
	{
		for (uint32_t i = 0; i < h; ++i)
			rowD[i] = totals[i] * sin(3.141592653589793 * ((double)i + 0.5) / (double)h);
		const double total = scan_double(rowD, m4, B, outD);
		for (uint32_t i = 0; i < h; ++i) cdf[i] = total != 0.0 ? (float)(outD[i] / total) : 0.0f;
		*integral = (float)(total / ((double)w * (double)h));
	}
	for (uint32_t i = 0; i < h; ++i) marg[i] = invert_one(cdf, (int)h, (float)i / (float)((int)h - 1));
	free(rowF); free(cdf); free(rowD); free(outD); free(totals);
	return 0;
}
