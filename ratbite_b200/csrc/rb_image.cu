// Resolve of the FP64 accumulation to a headless 8-bit RGBA image
// (renderResolve with the AgX tonemap, src/kernels/image.cu:16-121).
//
// The reference writes through a surface object into a GL-mapped array; here
// the image is a plain row-major buffer of width*height RGBA8 words in device
// memory. The arithmetic is the reference's, written in the same expression
// order (glm's component-wise vector operations, column-major mat3 * vec3,
// min/max as `y < x ? y : x` / `x < y ? y : x`, so NaN propagates as in glm),
// and this translation unit keeps the compiler's default multiply-add
// contraction, as the reference's own device build does, so the bytes match.
// One pixel reads 32 B and writes 4 B: the kernel is bound by HBM bandwidth.

#include <cstdint>

#include "rb_launch.cuh"
#include "rb_wavefront.h"

namespace rb
{
namespace
{
struct Mat3
{
	float m[9];   // column-major, as glm::mat3
};

RB_D float glmMax(float x, float y) { return (x < y) ? y : x; }
RB_D float glmMin(float x, float y) { return (y < x) ? y : x; }
RB_D float glmClamp(float x, float lo, float hi) { return glmMin(glmMax(x, lo), hi); }

// Polynomial fit of the AgX contrast curve (image.cu:42-55).
RB_D float agxContrast(float x)
{
	const float x2 = x * x;
	const float x4 = x2 * x2;
	return - 17.86f * x4 * x2 * x
		   + 78.01f * x4 * x2
		   - 126.7f * x4 * x
		   + 92.06f * x4
		   - 28.72f * x2 * x
		   + 4.361f * x2
		   - 0.1718f * x
		   + 0.002857f;
}

// AgX (image.cu:26-62): inset matrix, log2 encoding on [-12.47393, 4.026069]
// EV, contrast polynomial, outset matrix, clamp to [0, 1].
RB_D void agx(float& r, float& g, float& b)
{
	const float a0 = 0.842479062253094f, a1 = 0.0423282422610123f, a2 = 0.0423756549057051f,
		a3 = 0.0784335999999992f, a4 = 0.878468636469772f, a5 = 0.0784336f,
		a6 = 0.0792237451477643f, a7 = 0.0791661274605434f, a8 = 0.879142973793104f;
	constexpr float minEv = -12.47393f;
	constexpr float maxEv = 4.026069f;
	float x = a0 * r + a3 * g + a6 * b;
	float y = a1 * r + a4 * g + a7 * b;
	float z = a2 * r + a5 * g + a8 * b;
	x = glmClamp(log2f(x), minEv, maxEv);
	y = glmClamp(log2f(y), minEv, maxEv);
	z = glmClamp(log2f(z), minEv, maxEv);
	x = (x - minEv) / (maxEv - minEv);
	y = (y - minEv) / (maxEv - minEv);
	z = (z - minEv) / (maxEv - minEv);
	x = agxContrast(x);
	y = agxContrast(y);
	z = agxContrast(z);
	const float i0 = 1.1968790051201738155f, i1 = -0.052896851757456180321f, i2 = -0.052971635514443794537f,
		i3 = -0.098020881140136776078f, i4 = 1.1519031299041727435f, i5 = -0.098043450117124120312f,
		i6 = -0.099029744079720471434f, i7 = -0.098961176844843346553f, i8 = 1.1510736726411610622f;
	r = glmClamp(i0 * x + i3 * y + i6 * z, 0.0f, 1.0f);
	g = glmClamp(i1 * x + i4 * y + i7 * z, 0.0f, 1.0f);
	b = glmClamp(i2 * x + i5 * y + i8 * z, 0.0f, 1.0f);
}

__global__ void __launch_bounds__(256) kResolveImage(uint32_t pixels, Mat3 cs, float exposureScale,
	const double4* __restrict__ data, uint32_t* __restrict__ out)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += gridDim.x * blockDim.x)
	{
		const double4 d = data[i];
		const double normval = 1.0 / d.w;
		const float nx = static_cast<float>(d.x * normval);
		const float ny = static_cast<float>(d.y * normval);
		const float nz = static_cast<float>(d.z * normval);
		const float cx = glmMax(nx, 0.0f) * exposureScale;
		const float cy = glmMax(ny, 0.0f) * exposureScale;
		const float cz = glmMax(nz, 0.0f) * exposureScale;
		float r = cs.m[0] * cx + cs.m[3] * cy + cs.m[6] * cz;
		float g = cs.m[1] * cx + cs.m[4] * cy + cs.m[7] * cz;
		float b = cs.m[2] * cx + cs.m[5] * cy + cs.m[8] * cz;
		agx(r, g, b);
		const uint32_t R = static_cast<uint8_t>(r * 255.99999f);
		const uint32_t G = static_cast<uint8_t>(g * 255.99999f);
		const uint32_t B = static_cast<uint8_t>(b * 255.99999f);
		out[i] = R | (G << 8) | (B << 16) | (255u << 24);
	}
}
} // namespace

void launchResolveImage(uint32_t width, uint32_t height, const float* colorspace, float exposureScale,
	const double4* data, uint32_t* out, int smCount, cudaStream_t st)
{
	Mat3 cs;
	for (int k = 0; k < 9; ++k) cs.m[k] = colorspace[k];
	const uint32_t pixels = width * height;
	const uint32_t need = (pixels + 255u) / 256u;
	const uint32_t cap = static_cast<uint32_t>(smCount > 0 ? smCount : 148) * 8u;
	kResolveImage<<<need < cap ? (need ? need : 1u) : cap, 256, 0, st>>>(pixels, cs, exposureScale, data, out);
}
} // namespace rb
