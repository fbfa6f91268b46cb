// Monte Carlo regeneration of the multiple-scattering compensation tables
// that the BxDFs read (the reference ships them as data, bin/*.bin, with no
// generator). Each texel is the directional albedo of one microfacet lobe,
// integrated with the lobe formulas of rb_bxdf.cuh, on the axes the BxDFs
// look it up with (bxdfComplexSurface), sampled at i / 31 for i = 0..31 (the
// reference's tables are generated on these end-inclusive grids, although its
// texture lookup puts texel i at (i + 0.5) / 32; matching them showed it):
//   x: |cos theta_o| = i / 31 (at least kMinCos), y: roughness r = j / 31 (at
//   least 0.001, as the BxDFs clamp it), alpha = r^2 (isotropic GGX), z (3D
//   tables): w = k / 31 = sqrt(|f0Sr|) with f0Sr = (1 - eta) / (1 + eta), so
//   eta = (1 + w^2) / (1 - w^2) for the outer tables (eta > 1) and
//   (1 - w^2) / (1 + w^2) for the inner ones.
// Tables (definitions found by matching the reference's data, see below):
//   conductor  = albedo of GGX reflection with F = 1;
//   dielectric = albedo of reflection plus transmission, Schlick Fresnel
//                with total internal reflection (F = 1 where no refracted
//                direction exists), transmitted energy not scaled by eta^2;
//   reflective = albedo of the Schlick-Fresnel reflection alone, Schlick
//                without the total-internal-reflection override, divided by
//                the dielectric albedo (the share of the compensated
//                specular layer, which the BxDF scales by 1 / dielectric);
//   at w = 0 (eta = 1, no interface) dielectric = 1 and reflective = 0.
// Against the reference's bin/*.bin, away from the |cos| = 0 column that it
// fills in its own way, the regenerated conductor, dielectric and reflective
// tables agree to a few 1e-4 (Monte Carlo noise). Microfacet normals are drawn from the visible-normal
// distribution (spherical-cap sampling, the BxDFs' own sampler), so each
// sample weighs G2 / G1 times the lobe's Fresnel factor; a Hammersley point
// set with a per-texel rotation gives the (u, v) pairs.

#include <cstdint>

#include "rb_bxdf.cuh"
#include "rb_launch.cuh"
#include "ratbite_b200_kernels.h"

namespace rb
{
namespace
{
constexpr uint32_t kLut2 = kLutN * kLutN, kLut3 = kLutN * kLutN * kLutN;
constexpr float kMinCos = 1e-4f;
RB_D float lutAxis(uint32_t i) { return static_cast<float>(i) / static_cast<float>(kLutN - 1); }

struct LutOut
{
	float* conductor;
	float* dielOuter;
	float* dielInner;
	float* reflOuter;
	float* reflInner;
};

// texel t: [0, kLut2) conductor, then 2 x kLut3 (outer, inner) for the
// dielectric and reflective tables (one pass computes both).
__global__ void __launch_bounds__(kThreads) kGenerateLuts(LutOut o, uint32_t samples)
{
	for (uint32_t t = gtid(); t < kLut2 + 2 * kLut3; t += gstride())
	{
		const bool cond = t < kLut2;
		const uint32_t u3 = cond ? t : (t - kLut2) % kLut3;
		const bool inner = !cond && (t - kLut2) >= kLut3;
		const uint32_t ix = u3 % kLutN, iy = (u3 / kLutN) % kLutN, iz = u3 / kLut2;
		const float mu = fmaxf(lutAxis(ix), kMinCos);
		const float r = fmaxf(lutAxis(iy), 0.001f);
		const float alpha = r * r;
		const f3 wo = mk(sqrtf(fmaxf(0.0f, 1.0f - mu * mu)), 0.0f, mu);
		const CtxDir co = ctxDir(wo);
		const float g1 = G1(co, alpha, alpha);
		float eta = 1.0f, f0 = 0.0f;
		if (!cond)
		{
			const float w = lutAxis(iz), w2 = w * w;
			eta = inner ? (1.0f - w2) / (1.0f + w2) : (1.0f + w2) / (1.0f - w2);
			f0 = w2 * w2;
		}
		const uint32_t h = mix32(t * 0x9E3779B9u + 0x85EBCA6Bu);
		const float ru = static_cast<float>(h >> 8) * (1.0f / 16777216.0f);
		const float rv = static_cast<float>(mix32(h) >> 8) * (1.0f / 16777216.0f);
		double accR = 0.0, accT = 0.0, accS = 0.0;   // reflection (with TIR), transmission, Schlick reflection
		for (uint32_t s = 0; s < samples; ++s)
		{
			float u = (static_cast<float>(s) + 0.5f) / static_cast<float>(samples) + ru;
			float v = static_cast<float>(__brev(s) >> 8) * (1.0f / 16777216.0f) + rv;
			u -= floorf(u);
			v -= floorf(v);
			const f3 m = vndfSampleCap(wo, alpha, alpha, u, v);
			const float ad = fabsf(dot(wo, m));
			float F = 1.0f, Fs = 1.0f;
			if (!cond)
			{
				Fs = fresnelSchlick(f0, ad);
				const float s2t = fmaxf(0.0f, 1.0f - ad * ad) / (eta * eta);
				F = s2t >= 1.0f ? 1.0f : Fs;
			}
			const f3 wi = normalize(reflectAbout(wo, m));
			if (wi.z > 0.0f)
			{
				const float g = G2(ctxDir(wi), co, alpha, alpha) / g1;
				accR += static_cast<double>(F * g);
				accS += static_cast<double>(Fs * g);
			}
			if (!cond && F < 1.0f)
			{
				const f3 wt = refractSimple(wo, m, eta);
				if (wt.z < 0.0f) accT += static_cast<double>((1.0f - F) * G2(ctxDir(wt), co, alpha, alpha) / g1);
			}
		}
		if (cond)
		{
			o.conductor[u3] = static_cast<float>(accR / samples);
		}
		else
		{
			const double diel = (accR + accT) / samples;
			const bool noInterface = iz == 0;
			(inner ? o.dielInner : o.dielOuter)[u3] = noInterface ? 1.0f : static_cast<float>(diel);
			(inner ? o.reflInner : o.reflOuter)[u3] =
				noInterface || diel <= 0.0 ? 0.0f : static_cast<float>(accS / samples / diel);
		}
	}
}
// ---------------------------------------------------------------------------
// Sheen LTC table (the reference's bin/sheenLUT.bin: per texel the LTC
// coefficients A, B and the albedo R that microflake::LTC reads,
// src/device/surface.h:38-89; the lobe is Zeltner, Burley and Chiang 2022,
// "Practical Multiple-Scattering Sheen Using Linearly Transformed Cosines").
// Ground truth: a slab of optical thickness 1 (unit thickness, unit density
// per unit projected area) of specular SGGX microflakes with a fiber-like
// distribution along the normal, S = diag(1, 1, sigma^2) with sigma =
// alpha^2 (Heitz, Dupuy, Crassin and Dachsbacher 2015, "The SGGX Microflake
// Distribution": projected area sqrt(w^T S w), visible-normal sampling,
// specular phase function), flake albedo 1, nothing below the slab. Light
// enters the top along -wo; R is the fraction of paths that leave through
// the top, and their exit directions wi (in the frame where wo has phi = 0)
// are binned (sqrt(cos theta) x phi, 64 x 32) for a maximum-likelihood fit
// of the LTC lobe D(wi) = A^2 z / (pi |(A x + B z, A y, z)|^4) by Newton's
// method on (ln A, B). Axes: x = cos theta_o = i / 31 (at least 0.01),
// y = alpha = j / 31; the alpha = 0 row is zero (flakes of a vertical fiber
// keep the vertical component of a direction, so no path returns).
constexpr int kSheenU = 64, kSheenPhi = 32, kSheenBins = kSheenU * kSheenPhi;
constexpr int kSheenThreads = 256;
constexpr float kSheenMinCos = 0.01f;
constexpr int kSheenMaxEvents = 100000;

struct Pcg
{
	uint64_t s;
	RB_D uint32_t next()
	{
		s = s * 6364136223846793005ull + 1442695040888963407ull;
		const uint32_t x = static_cast<uint32_t>(((s >> 18u) ^ s) >> 27u);
		const uint32_t r = static_cast<uint32_t>(s >> 59u);
		return (x >> r) | (x << ((32u - r) & 31u));
	}
	RB_D float uniform() { return (static_cast<float>(next() >> 8) + 0.5f) * (1.0f / 16777216.0f); }
};

// S = diag(1, 1, szz): the projected area sqrt(w^T S w)
RB_D float sggxSigma(f3 w, float szz) { return sqrtf(fmaxf(w.x * w.x + w.y * w.y + szz * w.z * w.z, 0.0f)); }
RB_D float sggxQ(f3 a, f3 b, float szz) { return a.x * b.x + a.y * b.y + szz * a.z * b.z; }

// A microflake normal drawn from the visible normals seen from wi (unit,
// pointing away from the flake): the published SGGX visible-normal sampler.
RB_D f3 sggxSampleVisible(f3 wi, float szz, float u1, float u2)
{
	const float sg = wi.z >= 0.0f ? 1.0f : -1.0f;
	const float ia = -1.0f / (sg + wi.z), bb = wi.x * wi.y * ia;
	const f3 wk = mk(1.0f + sg * wi.x * wi.x * ia, sg * bb, -sg * wi.x);
	const f3 wj = mk(bb, sg + wi.y * wi.y * ia, -wi.y);
	const float skk = sggxQ(wk, wk, szz), sjj = sggxQ(wj, wj, szz), sii = sggxQ(wi, wi, szz);
	const float skj = sggxQ(wk, wj, szz), ski = sggxQ(wk, wi, szz), sji = sggxQ(wj, wi, szz);
	(void)skk;
	const float sqrtDet = sqrtf(szz);
	const float invSii = rsqrtf(sii);
	const float tmp = sqrtf(fmaxf(sjj * sii - sji * sji, 1e-30f));
	const f3 mkv = mk(sqrtDet / tmp, 0.0f, 0.0f);
	const f3 mjv = mk(-invSii * (ski * sji - skj * sii) / tmp, invSii * tmp, 0.0f);
	const f3 miv = mk(invSii * ski, invSii * sji, invSii * sii);
	const float r = sqrtf(u1), ph = 6.283185307179586f * u2;
	float sp, cp;
	sincosf(ph, &sp, &cp);
	const float x = r * cp, y = r * sp, z = sqrtf(fmaxf(0.0f, 1.0f - u1));
	const f3 m = normalize(x * mkv + y * mjv + z * miv);
	return normalize(m.x * wk + m.y * wj + m.z * wi);
}

// One random walk from the top of the slab; true with the exit direction
// when the path leaves through the top.
RB_D bool sheenWalk(f3 wo, float szz, Pcg& rng, f3& out)
{
	f3 d = -wo;
	float z = 1.0f;
	for (int e = 0; e < kSheenMaxEvents; ++e)
	{
		const float t = -__logf(rng.uniform()) / sggxSigma(d, szz);
		const float z2 = z + t * d.z;
		if (z2 <= 0.0f) return false;
		if (z2 >= 1.0f) { out = d; return true; }
		z = z2;
		const f3 w = -d;
		const float u1 = rng.uniform(), u2 = rng.uniform();
		const f3 m = sggxSampleVisible(w, szz, u1, u2);
		d = normalize(2.0f * dot(w, m) * m - w);
	}
	return false;
}

// Block-wide sums over the histogram at (a, b) (bin centres stand for their
// samples), in the parameters (s = ln a, b):
//   ML:  v = [log-likelihood, gradient (2), Hessian (ss, sb, bb)];
//   L2:  v = [E, J^T r (2), J^T J (ss, sb, bb)] for E = sum over bins of
//        solid angle x (density - R D)^2, residuals r = sqrt(solid angle)
//        (density - R D), J = dr / d(s, b).
template<bool ML>
RB_D void sheenSums(const uint32_t* hist, float total, float paths, float a, float b, double* v, double* red)
{
	double acc[6] = { 0.0, 0.0, 0.0, 0.0, 0.0, 0.0 };
	const double A = a, B = b, R = total / paths;
	for (int k = threadIdx.x; k < kSheenBins; k += blockDim.x)
	{
		const uint32_t c = hist[k];
		if (ML && !c) continue;
		const double u = (static_cast<double>(k / kSheenPhi) + 0.5) / kSheenU;
		const double ph = (static_cast<double>(k % kSheenPhi) + 0.5) * (3.141592653589793 / kSheenPhi);
		const double Z = u * u, S = sqrt(fmax(0.0, 1.0 - Z * Z));
		const double X = S * cos(ph), Y = S * sin(ph);
		const double q = A * X + B * Z;
		const double l2 = q * q + A * A * Y * Y + Z * Z;
		const double la = 2.0 * q * X + 2.0 * A * Y * Y, lb = 2.0 * q * Z;   // d l2 / da, d l2 / db
		if (ML)
		{
			const double w = c / static_cast<double>(total);
			const double laa = 2.0 * X * X + 2.0 * Y * Y, lab = 2.0 * X * Z, lbb = 2.0 * Z * Z;
			// L = 2 ln a - 2 ln l2 per sample; derivatives in a, converted to s below
			acc[0] += w * (2.0 * log(A) - 2.0 * log(l2));
			acc[1] += w * (2.0 / A - 2.0 * la / l2);
			acc[2] += w * (-2.0 * lb / l2);
			acc[3] += w * (-2.0 / (A * A) - 2.0 * (laa / l2 - la * la / (l2 * l2)));
			acc[4] += w * (-2.0 * (lab / l2 - la * lb / (l2 * l2)));
			acc[5] += w * (-2.0 * (lbb / l2 - lb * lb / (l2 * l2)));
		}
		else
		{
			const double omega = 2.0 * (2.0 * u / kSheenU) * (3.141592653589793 / kSheenPhi);
			const double dens = c / (static_cast<double>(paths) * omega);
			const double D = A * A * Z / (3.141592653589793 * l2 * l2);
			const double dDs = D * (2.0 - 2.0 * A * la / l2), dDb = D * (-2.0 * lb / l2);
			const double so = sqrt(omega);
			const double r = so * (dens - R * D), js = -so * R * dDs, jb = -so * R * dDb;
			acc[0] += r * r;
			acc[1] += js * r;
			acc[2] += jb * r;
			acc[3] += js * js;
			acc[4] += js * jb;
			acc[5] += jb * jb;
		}
	}
	for (int i = 0; i < 6; ++i)
	{
		double x = acc[i];
		for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
		if ((threadIdx.x & 31) == 0) red[(threadIdx.x >> 5) * 6 + i] = x;
	}
	__syncthreads();
	if (threadIdx.x < 6)
	{
		double x = 0.0;
		for (int wv = 0; wv < static_cast<int>(blockDim.x >> 5); ++wv) x += red[wv * 6 + threadIdx.x];
		v[threadIdx.x] = x;
	}
	__syncthreads();
	if (ML && threadIdx.x == 0)
	{
		// chain rule a -> s = ln a: dL/ds = a dL/da, d2L/ds2 = a^2 d2L/da2 + a dL/da
		const double g = v[1];
		v[1] = A * g;
		v[3] = A * A * v[3] + A * g;
		v[4] = A * v[4];
	}
	__syncthreads();
}

// One block per texel: the walks fill the block's histogram, then the block
// fits the lobe: Newton's method on the log-likelihood (concave near its
// maximum, started from a = 0.5, b = 0), then Levenberg-Marquardt on the
// L2 distance between the binned density and R D from there. (The L2 fit
// follows the reference's table more closely than the likelihood alone:
// over table entries with alpha >= 6/31 and R >= 0.05, A within about 2 %
// against up to 5 %.)
__global__ void __launch_bounds__(kSheenThreads) kSheenLut(float4* out, uint32_t paths)
{
	__shared__ uint32_t hist[kSheenBins];
	__shared__ uint32_t exits;
	__shared__ double red[(kSheenThreads / 32) * 6];
	__shared__ double v[6];
	__shared__ double ds, db;
	__shared__ float sa, sb;
	const uint32_t texel = blockIdx.x;
	const uint32_t ix = texel % kLutN, iy = texel / kLutN;
	if (iy == 0)
	{
		if (threadIdx.x == 0) out[texel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		return;
	}
	for (int k = threadIdx.x; k < kSheenBins; k += blockDim.x) hist[k] = 0u;
	if (threadIdx.x == 0) exits = 0u;
	__syncthreads();
	const float mu = fmaxf(lutAxis(ix), kSheenMinCos);
	const float alpha = lutAxis(iy);
	const float sigma = alpha * alpha, szz = sigma * sigma;
	const f3 wo = mk(sqrtf(fmaxf(0.0f, 1.0f - mu * mu)), 0.0f, mu);
	Pcg rng{ (static_cast<uint64_t>(texel) << 32) ^ (0x9E3779B97F4A7C15ull * (threadIdx.x + 1)) };
	rng.next();
	uint32_t mine = 0;
	for (uint32_t pth = threadIdx.x; pth < paths; pth += blockDim.x)
	{
		f3 d;
		if (!sheenWalk(wo, szz, rng, d)) continue;
		++mine;
		const float u = sqrtf(fminf(fmaxf(d.z, 0.0f), 1.0f));
		const float ph = atan2f(fabsf(d.y), d.x);
		const int bu = min(kSheenU - 1, static_cast<int>(u * kSheenU));
		const int bp = min(kSheenPhi - 1, max(0, static_cast<int>(ph * (kSheenPhi / 3.14159265358979f))));
		atomicAdd(&hist[bu * kSheenPhi + bp], 1u);
	}
	atomicAdd(&exits, mine);
	__syncthreads();
	const float total = static_cast<float>(exits), fp = static_cast<float>(paths);
	const float R = total / fp;
	if (exits < 32u)
	{
		if (threadIdx.x == 0) out[texel] = make_float4(1.0f, 0.0f, R, 0.0f);
		return;
	}
	if (threadIdx.x == 0) { sa = 0.5f; sb = 0.0f; }
	__syncthreads();
	// 1. maximum likelihood (Newton, backtracking; gradient steps where the
	// Hessian is not negative definite)
	sheenSums<true>(hist, total, fp, sa, sb, v, red);
	double cur = v[0];
	for (int it = 0; it < 60; ++it)
	{
		if (threadIdx.x == 0)
		{
			const double g0 = v[1], g1 = v[2], h00 = v[3], h01 = v[4], h11 = v[5];
			const double det = h00 * h11 - h01 * h01;
			if (h00 < 0.0 && det > 0.0) { ds = -(h11 * g0 - h01 * g1) / det; db = -(-h01 * g0 + h00 * g1) / det; }
			else { ds = 0.1 * g0; db = 0.1 * g1; }
			const double n = sqrt(ds * ds + db * db);
			if (n > 1.0) { ds /= n; db /= n; }
		}
		__syncthreads();
		const float a0 = sa, b0 = sb;
		const double dS = ds, dB = db;
		double step = 1.0;
		bool better = false;
		for (int h = 0; h < 30 && !better; ++h)
		{
			const float a1 = static_cast<float>(a0 * exp(step * dS)), b1 = static_cast<float>(b0 + step * dB);
			sheenSums<true>(hist, total, fp, a1, b1, v, red);
			if (v[0] >= cur) { better = true; if (threadIdx.x == 0) { sa = a1; sb = b1; } }
			else step *= 0.5;
			__syncthreads();
		}
		if (!better) break;
		const double gain = v[0] - cur;
		cur = v[0];
		if (gain < 1e-12 && step * sqrt(dS * dS + dB * dB) < 1e-7) break;
	}
	// 2. least squares on the density (Levenberg-Marquardt)
	sheenSums<false>(hist, total, fp, sa, sb, v, red);
	double err = v[0], lambda = 1e-3;
	for (int it = 0; it < 60; ++it)
	{
		const double g0 = v[1], g1 = v[2], h00 = v[3], h01 = v[4], h11 = v[5];
		const float a0 = sa, b0 = sb;
		bool better = false;
		for (int h = 0; h < 20 && !better; ++h)
		{
			const double m00 = h00 * (1.0 + lambda), m11 = h11 * (1.0 + lambda);
			const double det = m00 * m11 - h01 * h01;
			double dS = 0.0, dB = 0.0;
			if (det > 0.0) { dS = -(m11 * g0 - h01 * g1) / det; dB = -(-h01 * g0 + m00 * g1) / det; }
			const double n = sqrt(dS * dS + dB * dB);
			if (n > 0.5) { dS *= 0.5 / n; dB *= 0.5 / n; }
			const float a1 = static_cast<float>(a0 * exp(dS)), b1 = static_cast<float>(b0 + dB);
			sheenSums<false>(hist, total, fp, a1, b1, v, red);
			if (v[0] < err) { better = true; if (threadIdx.x == 0) { sa = a1; sb = b1; } }
			else lambda *= 4.0;
			__syncthreads();
		}
		if (!better) break;
		const double gain = err - v[0];
		err = v[0];
		lambda = fmax(lambda / 3.0, 1e-7);
		if (gain < 1e-10 * err) break;
	}
	__syncthreads();
	if (threadIdx.x == 0) out[texel] = make_float4(sa, sb, R, 0.0f);
}
} // namespace
} // namespace rb

extern "C" int rb_k_generate_sheen_lut(uint32_t paths, float* sheen, void* stream)
{
	if (paths == 0 || !sheen) return RB_ERR_INVALID;
	rb::kSheenLut<<<rb::kLut2, rb::kSheenThreads, 0, static_cast<cudaStream_t>(stream)>>>(
		reinterpret_cast<float4*>(sheen), paths);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}

extern "C" int rb_k_generate_luts(uint32_t samples, float* conductor, float* dielectric_outer, float* dielectric_inner,
	float* reflective_outer, float* reflective_inner, void* stream)
{
	if (samples == 0 || !conductor || !dielectric_outer || !dielectric_inner || !reflective_outer || !reflective_inner)
		return RB_ERR_INVALID;
	rb::LutOut o{ conductor, dielectric_outer, dielectric_inner, reflective_outer, reflective_inner };
	const uint32_t texels = rb::kLut2 + 2 * rb::kLut3;
	rb::kGenerateLuts<<<rb::gridFor(texels), rb::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(o, samples);
	return cudaGetLastError() == cudaSuccess ? RB_OK : RB_ERR_CUDA;
}
