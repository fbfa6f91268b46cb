/* Oracle test infrastructure (not product code).
 * C restatement of the reference's Owen-scrambled Sobol sampler
 * (src/device/quasi_random.h): pixel hash (:30-37), dimension hash (:102-111),
 * reversed-bit Owen scramble (:119-127), Burley's Sobol (:132-204) and the
 * 1D/2D/3D samplers (:76-99) with their scramble constants. */
#include "oracle_restate.h"

static const uint32_t kDirections[3][32] = {
	{ 0x00000001u, 0x00000003u, 0x00000005u, 0x0000000fu, 0x00000011u, 0x00000033u, 0x00000055u, 0x000000ffu,
	  0x00000101u, 0x00000303u, 0x00000505u, 0x00000f0fu, 0x00001111u, 0x00003333u, 0x00005555u, 0x0000ffffu,
	  0x00010001u, 0x00030003u, 0x00050005u, 0x000f000fu, 0x00110011u, 0x00330033u, 0x00550055u, 0x00ff00ffu,
	  0x01010101u, 0x03030303u, 0x05050505u, 0x0f0f0f0fu, 0x11111111u, 0x33333333u, 0x55555555u, 0xffffffffu },
	{ 0x00000001u, 0x00000003u, 0x00000006u, 0x00000009u, 0x00000017u, 0x0000003au, 0x00000071u, 0x000000a3u,
	  0x00000116u, 0x00000339u, 0x00000677u, 0x000009aau, 0x00001601u, 0x00003903u, 0x00007706u, 0x0000aa09u,
	  0x00010117u, 0x0003033au, 0x00060671u, 0x000909a3u, 0x00171616u, 0x003a3939u, 0x00717777u, 0x00a3aaaau,
	  0x01170001u, 0x033a0003u, 0x06710006u, 0x09a30009u, 0x16160017u, 0x3939003au, 0x77770071u, 0xaaaa00a3u },
	{ 0x00000001u, 0x00000003u, 0x00000004u, 0x0000000au, 0x0000001fu, 0x0000002eu, 0x00000045u, 0x000000c9u,
	  0x0000011bu, 0x000002a4u, 0x0000079au, 0x00000b67u, 0x0000101eu, 0x0000302du, 0x00004041u, 0x0000a0c3u,
	  0x0001f104u, 0x0002e28au, 0x000457dfu, 0x000c9baeu, 0x0011a105u, 0x002a7289u, 0x0079e7dbu, 0x00b6dba4u,
	  0x0100011au, 0x030002a7u, 0x0400079eu, 0x0a000b6du, 0x1f001001u, 0x2e003003u, 0x45004004u, 0xc900a00au },
};

static uint32_t brev(uint32_t x)
{
	uint32_t r = 0;
	for (int i = 0; i < 32; ++i) { r = (r << 1) | (x & 1u); x >>= 1; }
	return r;
}
static uint32_t clz32(uint32_t x) { return x == 0 ? 32u : (uint32_t)__builtin_clz(x); }

uint32_t orc_pixel_hash(uint32_t x, uint32_t y)
{
	const uint32_t qx = 1103515245u * ((x >> 1u) ^ y);
	const uint32_t qy = 1103515245u * ((y >> 1u) ^ x);
	return 1103515245u * (qx ^ (qy >> 3u));
}
static uint32_t dim_hash(uint32_t i)
{
	i ^= i >> 16; i *= 0x21f0aaadu; i ^= i >> 15; i *= 0xd35a2d97u; i ^= i >> 15;
	return i ^ 0xe6fe3bebu;
}
static uint32_t owen(uint32_t n, uint32_t seed)
{
	n ^= n * 0x3d20adeau; n += seed; n *= (seed >> 16) | 1u; n ^= n * 0x05526c56u; n ^= n * 0x53a22864u;
	return n;
}
static float burley(uint32_t rev, uint32_t dim, uint32_t scramble)
{
	uint32_t result = 0;
	if (dim == 0)
		result = brev(rev);
	else
	{
		uint32_t i = 0;
		while (rev != 0)
		{
			const uint32_t j = clz32(rev);
			result ^= kDirections[dim - 1][i + j];
			i += j + 1;
			rev <<= j;
			rev <<= 1;
		}
	}
	return (float)brev(owen(result, scramble)) * (1.0f / 4294967808.0f);
}

void orc_sobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash,
               const uint32_t* bounce, const uint32_t* dim, float* out)
{
	for (uint32_t k = 0; k < n; ++k)
	{
		const uint32_t offset = 16u * (bounce[k] + 1u) + dim[k];
		const uint32_t seed = hash[k] ^ dim_hash(offset);
		if (dims == 1)
		{
			const uint32_t idx = owen(brev(sample[k]), seed ^ 0xbff95bfeu);
			out[k] = burley(idx, 0, seed ^ 0x635c77bdu);
		}
		else if (dims == 2)
		{
			const uint32_t idx = owen(brev(sample[k]), seed ^ 0xf8ade99au);
			out[2 * k] = burley(idx, 0, seed ^ 0xe0aaaf76u);
			out[2 * k + 1] = burley(idx, 1, seed ^ 0x94964d4eu);
		}
		else
		{
			const uint32_t idx = owen(brev(sample[k]), seed ^ 0xcaa726acu);
			out[3 * k] = burley(idx, 0, seed ^ 0x9e78e391u);
			out[3 * k + 1] = burley(idx, 1, seed ^ 0x67c33241u);
			out[3 * k + 2] = burley(idx, 2, seed ^ 0x78c395c5u);
		}
	}
}
