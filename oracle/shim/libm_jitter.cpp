// Oracle test infrastructure (not product code).
//
// Optional perturbation of the single-precision libm results that the
// reference's device code gets when the oracle runs it on the CPU. The
// oracle library is linked with `-Wl,--wrap=<fn>` for every float libm
// function the reference calls (the list below is what `nm -D` shows it
// imports), so each call comes here first. With jitter off (the default)
// the glibc result is returned unchanged. With jitter on, the result is
// moved by a random whole number of ulps in [-b, b], where b is the maximum
// error that NVIDIA's CUDA Math API documentation states for the function
// in single precision, plus one ulp for glibc's own error.
//
// The parity tests use it to measure how far the reference's own outputs
// move when its libm results move by as much as CUDA's and glibc's may
// differ: an output of the GPU path that differs from the oracle by more
// than 1e-5 relative must still lie within that spread.

#include <cmath>
#include <cstdint>

extern "C" {
float __real_acosf(float);
float __real_atan2f(float, float);
float __real_atanhf(float);
float __real_cosf(float);
float __real_coshf(float);
float __real_exp2f(float);
float __real_expf(float);
float __real_expm1f(float);
float __real_hypotf(float, float);
float __real_logf(float);
float __real_powf(float, float);
float __real_sinf(float);
void __real_sincosf(float, float*, float*);
}

namespace
{
bool g_on = false;
thread_local uint64_t t_state = 0x9E3779B97F4A7C15ull;
uint64_t g_seed = 1;
thread_local uint64_t t_seed_used = 0;

uint32_t next()
{
	if (t_seed_used != g_seed) { t_state = g_seed * 0x9E3779B97F4A7C15ull + 1; t_seed_used = g_seed; }
	// xorshift64*
	t_state ^= t_state >> 12;
	t_state ^= t_state << 25;
	t_state ^= t_state >> 27;
	return static_cast<uint32_t>((t_state * 0x2545F4914F6CDD1Dull) >> 32);
}

float jitter(float v, int bound)
{
	if (!g_on || !std::isfinite(v) || v == 0.0f) return v;
	const int k = static_cast<int>(next() % static_cast<uint32_t>(2 * bound + 1)) - bound;
	const float toward = k > 0 ? INFINITY : -INFINITY;
	for (int i = 0; i < (k > 0 ? k : -k); ++i) v = std::nextafter(v, toward);
	return v;
}
} // namespace

extern "C" {
// Stated CUDA single-precision maximum ulp errors (+1 for glibc).
float __wrap_acosf(float x) { return jitter(__real_acosf(x), 2 + 1); }
float __wrap_atan2f(float y, float x) { return jitter(__real_atan2f(y, x), 3 + 1); }
float __wrap_atanhf(float x) { return jitter(__real_atanhf(x), 3 + 1); }
float __wrap_cosf(float x) { return jitter(__real_cosf(x), 2 + 1); }
float __wrap_coshf(float x) { return jitter(__real_coshf(x), 2 + 1); }
float __wrap_exp2f(float x) { return jitter(__real_exp2f(x), 2 + 1); }
float __wrap_expf(float x) { return jitter(__real_expf(x), 2 + 1); }
float __wrap_expm1f(float x) { return jitter(__real_expm1f(x), 1 + 1); }
float __wrap_hypotf(float x, float y) { return jitter(__real_hypotf(x, y), 3 + 1); }
float __wrap_logf(float x) { return jitter(__real_logf(x), 1 + 1); }
float __wrap_powf(float x, float y) { return jitter(__real_powf(x, y), 4 + 1); }
float __wrap_sinf(float x) { return jitter(__real_sinf(x), 2 + 1); }
void __wrap_sincosf(float x, float* s, float* c)
{
	__real_sincosf(x, s, c);
	*s = jitter(*s, 2 + 1);
	*c = jitter(*c, 2 + 1);
}

// on != 0 turns the perturbation on with the given seed; 0 turns it off.
void rbref_set_libm_jitter(int on, uint64_t seed)
{
	g_on = on != 0;
	g_seed = seed ? seed : 1;
}
}
