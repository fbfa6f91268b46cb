// Small float3 toolkit for the device code. Operation order follows the
// expressions of the reference's glm-based code (dot = (x*x + y*y) + z*z,
// normalize = v * (1 / sqrt(dot(v, v)))) so results stay within a few ulps
// of the reference on identical inputs.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define RB_HD __host__ __device__ __forceinline__
#define RB_D __device__ __forceinline__

namespace rb
{
constexpr float kPi = 3.14159265358979323846f;

struct f3
{
	float x, y, z;
};

RB_HD f3 mk(float x, float y, float z) { return f3{ x, y, z }; }
RB_HD f3 mk(float s) { return f3{ s, s, s }; }
RB_HD f3 operator+(f3 a, f3 b) { return f3{ a.x + b.x, a.y + b.y, a.z + b.z }; }
RB_HD f3 operator-(f3 a, f3 b) { return f3{ a.x - b.x, a.y - b.y, a.z - b.z }; }
RB_HD f3 operator-(f3 a) { return f3{ -a.x, -a.y, -a.z }; }
RB_HD f3 operator*(f3 a, f3 b) { return f3{ a.x * b.x, a.y * b.y, a.z * b.z }; }
RB_HD f3 operator*(f3 a, float s) { return f3{ a.x * s, a.y * s, a.z * s }; }
RB_HD f3 operator*(float s, f3 a) { return f3{ a.x * s, a.y * s, a.z * s }; }
RB_HD f3 operator/(f3 a, float s) { return f3{ a.x / s, a.y / s, a.z / s }; }
RB_HD f3& operator+=(f3& a, f3 b) { a = a + b; return a; }
RB_HD f3& operator-=(f3& a, f3 b) { a = a - b; return a; }
RB_HD f3& operator*=(f3& a, float s) { a = a * s; return a; }
RB_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// Dot product with every operation rounded separately (no FMA contraction),
// for the few places where cancellation makes the last bit matter.
RB_D float dotRn(f3 a, f3 b)
{
	return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
RB_HD f3 cross(f3 a, f3 b)
{
	return f3{ a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y };
}
RB_HD float length(f3 a) { return sqrtf(dot(a, a)); }
RB_HD f3 normalize(f3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
RB_HD float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
// glm::mix form: x * (1 - a) + y * a.
RB_HD float mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }
RB_HD f3 f3_of(float4 v) { return f3{ v.x, v.y, v.z }; }
RB_HD float4 f4_of(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
// The w word of a float4 in memory, read alone (a 4-byte load).
RB_HD float lastWord(const float4* v) { return reinterpret_cast<const float*>(v)[3]; }

// Four-wavelength spectrum sample (SampledSpectrum, src/device/spectral.h:14-194).
struct S4
{
	float v[4];
};
RB_HD S4 s4(float s) { return S4{ { s, s, s, s } }; }
RB_HD S4 s4(float4 a) { return S4{ { a.x, a.y, a.z, a.w } }; }
RB_HD float4 f4(const S4& a) { return make_float4(a.v[0], a.v[1], a.v[2], a.v[3]); }
RB_HD S4 operator+(const S4& a, const S4& b) { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] + b.v[i]; return r; }
RB_HD S4 operator*(const S4& a, const S4& b) { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] * b.v[i]; return r; }
RB_HD S4 operator*(const S4& a, float s) { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] * s; return r; }
RB_HD S4 operator*(float s, const S4& a) { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] * s; return r; }
RB_HD S4 operator/(const S4& a, float s) { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] / s; return r; }
RB_HD S4& operator+=(S4& a, const S4& b) { for (int i = 0; i < 4; ++i) a.v[i] += b.v[i]; return a; }
RB_HD S4& operator*=(S4& a, const S4& b) { for (int i = 0; i < 4; ++i) a.v[i] *= b.v[i]; return a; }
RB_HD S4& operator*=(S4& a, float s) { for (int i = 0; i < 4; ++i) a.v[i] *= s; return a; }
RB_HD S4& operator/=(S4& a, float s) { for (int i = 0; i < 4; ++i) a.v[i] /= s; return a; }
RB_HD float s4max(const S4& a)
{
	float t = a.v[0];
	for (int i = 1; i < 4; ++i) if (a.v[i] > t) t = a.v[i];
	return t;
}
} // namespace rb
