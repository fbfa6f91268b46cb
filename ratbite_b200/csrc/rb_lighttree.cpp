// Host light-tree construction over emissive triangles: a restatement of
// ratbite's LightTree::Builder (src/core/light_tree.cpp:47-418) driven as
// RenderingInterface::buildLightTree drives it
// (src/core/rendering_interface.cpp:1065-1167, 1433-1503), producing the
// reference's byte layouts (PackedNode, LightPointer, 64-bit path masks,
// EmissiveTriangleLightData) so the output is node-for-node what the
// reference uploads.
//
// The algorithm has to be the reference's step for step for the tree to be
// identical: binned SAOH split search over 32 bins and 3 axes with its
// orientation-cone bookkeeping (including bins whose empty bounds start at
// the origin), the split point placed with std::nth_element on box centres,
// leaves of at most 8 lights, leaf attributes from triangle mean / variance /
// normal, bottom-up merging of spherical-Gaussian attributes, and octahedral
// packing of the average direction (leaf directions re-read through the
// reference's unpack, :396-418). Float expressions keep the reference's
// operand order; the file is compiled with -ffp-contract=off.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "ratbite_b200.h"
#include "rb_light.cuh"

namespace
{
constexpr uint32_t kMaxLeafLights = 8;
constexpr uint32_t kBins = 32;
constexpr float kEntireCone = -1.0f;
constexpr float kPiF = 3.14159265358979323846f;

struct Box
{
	float min[3] = { 0.0f, 0.0f, 0.0f };
	float max[3] = { 0.0f, 0.0f, 0.0f };
	static Box empty()
	{
		Box b;
		for (int k = 0; k < 3; ++k) { b.min[k] = INFINITY; b.max[k] = -INFINITY; }
		return b;
	}
	void center(float c[3]) const
	{
		for (int k = 0; k < 3; ++k) c[k] = min[k] + (max[k] - min[k]) * 0.5f;
	}
	void dims(float d[3]) const
	{
		for (int k = 0; k < 3; ++k) d[k] = max[k] - min[k];
	}
	float area() const
	{
		float d[3];
		dims(d);
		return d[0] * d[1] * 2.0f + d[0] * d[2] * 2.0f + d[1] * d[2] * 2.0f;
	}
	bool valid() const { return min[0] <= max[0] && min[1] <= max[1] && min[2] <= max[2]; }
};
Box unite(const Box& a, const Box& b)
{
	Box r;
	for (int k = 0; k < 3; ++k) { r.min[k] = std::min(a.min[k], b.min[k]); r.max[k] = std::max(a.max[k], b.max[k]); }
	return r;
}

struct Light
{
	Box bounds;
	float cone[3];
	float cosCone;
	float flux;
	uint32_t index;
};

struct Attr
{
	float mean[3];
	float variance;
	float flux;
	float dir[3];
	float sharpness;
};

// Banerjee et al. 2005 vMF sharpness from mean-vector length, and its inverse
// by the cubic of Xu & Wang 2015 (src/core/math_util.h:566-588).
float axisLengthToSharpness(float l) { return l * (3.0f - l * l) / (1.0f - l * l); }
float sharpnessToAxisLength(float s)
{
	const float a = s / 3.0f;
	const float b = a * a * a;
	const float c = std::sqrt(1.0f + 3.0f * (a * a) * (1.0f + a * a));
	const float theta = std::atan2(c, b) / 3.0f;
	const float sqrt3 = 1.7320508075688772935274463415059f;
	const float d = std::sin(theta) * sqrt3 - std::cos(theta);
	return (s > 0x1.0p25) ? 1.0f : std::sqrt(1.0f + a * a) * d + a;
}

// NodeAttributes::add (src/core/light_tree_types.h:65-100).
Attr add(const Attr& A, const Attr& B)
{
	Attr r{};
	const float wa = A.flux / (A.flux + B.flux);
	const float wb = B.flux / (A.flux + B.flux);
	const float la = sharpnessToAxisLength(A.sharpness);
	const float lb = sharpnessToAxisLength(B.sharpness);
	float d[3] = { wa * la * A.dir[0] + wb * lb * B.dir[0], wa * la * A.dir[1] + wb * lb * B.dir[1],
	               wa * la * A.dir[2] + wb * lb * B.dir[2] };
	const float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
	for (int k = 0; k < 3; ++k) d[k] = len > 0.0001f ? d[k] / len : 0.0f;
	const float dm[3] = { B.mean[0] - A.mean[0], B.mean[1] - A.mean[1], B.mean[2] - A.mean[2] };
	const float dm2 = dm[0] * dm[0] + dm[1] * dm[1] + dm[2] * dm[2];
	for (int k = 0; k < 3; ++k) r.mean[k] = wa * A.mean[k] + wb * B.mean[k];
	r.variance = wa * A.variance + wb * B.variance + wa * wb * dm2;
	for (int k = 0; k < 3; ++k) r.dir[k] = d[k];
	r.flux = A.flux + B.flux;
	r.sharpness = axisLengthToSharpness(len);
	return r;
}

// Normalised cross product in glm's operand order.
void normalizedCross(const float a[3], const float b[3], float out[3])
{
	const float c[3] = { a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1] };
	const float inv = 1.0f / std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
	for (int k = 0; k < 3; ++k) out[k] = c[k] * inv;
}

class Builder
{
public:
	Builder(const float* world, const float* flux, uint32_t n) : m_world(world), m_flux(flux), m_n(n) {}
	std::vector<rb::PackedNode> nodes;
	std::vector<uint32_t> pointers;
	std::vector<uint64_t> masks;

	void build(std::vector<Light>& lights)
	{
		nodes.reserve(2 * m_n);
		pointers.assign(m_n, 0u);
		masks.assign(m_n, ~0ull);
		hierarchy(0ull, 0u, lights, 0u, m_n);
		fillBranch(0);
	}

private:
	const float* m_world;
	const float* m_flux;
	uint32_t m_n;

	// generateLightNodeAttributes (src/core/light_tree.cpp:14-45), world space.
	Attr leafAttributes(const Light& l) const
	{
		const float* v = m_world + 9 * l.index;
		const float e1[3] = { v[3] - v[0], v[4] - v[1], v[5] - v[2] };
		const float e2[3] = { v[6] - v[0], v[7] - v[1], v[8] - v[2] };
		Attr a{};
		normalizedCross(e1, e2, a.dir);
		for (int k = 0; k < 3; ++k) a.mean[k] = (v[k] + v[3 + k] + v[6 + k]) / 3.0f;
		a.variance = ((e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]) + (e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2])
			- (e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2])) / 18.0f;
		a.sharpness = axisLengthToSharpness(0.5f);
		a.flux = l.flux;
		return a;
	}

	static void packAttributes(rb::PackedNode& p, const Attr& a)
	{
		for (int k = 0; k < 3; ++k) p.mean[k] = a.mean[k];
		p.variance = a.variance;
		p.direction = rb::octEncodeU32(rb::mk(a.dir[0], a.dir[1], a.dir[2]));
		p.sharpness = a.sharpness;
		p.flux = a.flux;
	}

	struct Split
	{
		uint32_t axis = UINT32_MAX, index = UINT32_MAX;
		bool valid() const { return axis != UINT32_MAX && index != UINT32_MAX; }
	};

	struct Bin
	{
		Box bounds;                 // zero-initialised, as in the reference
		uint32_t count = 0;
		float flux = 0.0f;
		float cone[3] = { 0.0f, 0.0f, 0.0f };
		float cosCone = 1.0f;
		void merge(const Box& b, uint32_t c, float f, const float* cd)
		{
			bounds = unite(bounds, b);
			count += c;
			flux += f;
			for (int k = 0; k < 3; ++k) cone[k] += cd[k];
		}
	};

	static float combineCones(const float* dirA, float cosA, const float* dirB, float cosB)
	{
		float res = kEntireCone;
		if (cosA != kEntireCone && cosB != kEntireCone)
		{
			const float cd = dirA[0] * dirB[0] + dirA[1] * dirB[1] + dirA[2] * dirB[2];
			const float sd = std::sqrt(1.0f - cd * cd);
			const float sb = std::sqrt(1.0f - cosB * cosB);
			const float ct = cosB * cd - sb * sd;
			const float st = sb * cd + cosB * sd;
			if (st > 0.0f) res = std::min(cosB, ct);
		}
		return res;
	}
	static float saoh(const Box& b, float flux, float cosTheta)
	{
		const float pi = kPiF;
		const float aabb = b.valid() ? b.area() : 0.0f;
		const float thetaO = cosTheta != kEntireCone ? std::acos(std::max(std::min(cosTheta, 1.0f), -1.0f)) : pi;
		const float thetaW = std::min(thetaO + pi / 2.0f, pi);
		const float so = std::sin(thetaO);
		const float co = std::cos(thetaO);
		const float orient = 2.0f * pi * (1.0f - co)
			+ pi / 2.0f * (2.0f * thetaW * so - std::cos(thetaO - 2.0f * thetaW) - 2.0f * thetaO * so + co);
		return flux * aabb * orient;
	}

	// splitFunction (src/core/light_tree.cpp:162-394).
	Split splitFunction(const std::vector<Light>& L, uint32_t begin, uint32_t end, const Box& bounds) const
	{
		float splitCost = std::numeric_limits<float>::max();
		Split split;
		float dims[3];
		bounds.dims(dims);
		const uint32_t largest = dims[0] > dims[1] && dims[0] > dims[2] ? 0u : (dims[1] > dims[2] ? 1u : 2u);
		const uint32_t nCosts = kBins - 1;
		Bin bins[kBins];
		float costs[kBins - 1];
		for (uint32_t dim = 0; dim < 3; ++dim)
		{
			auto binId = [&](const Light& l) {
				const float bmin = bounds.min[dim], bmax = bounds.max[dim];
				const float w = bmax - bmin;
				const float scale = w > std::numeric_limits<float>::min() ? static_cast<float>(kBins) / w : 0.0f;
				float c[3];
				l.bounds.center(c);
				return std::min(static_cast<uint32_t>((c[dim] - bmin) * scale), kBins - 1);
			};
			for (uint32_t i = 0; i < kBins; ++i) bins[i] = Bin{};
			for (uint32_t i = begin; i < end; ++i)
			{
				Bin& b = bins[binId(L[i])];
				// Bin(sd) |= : a one-light bin from the record, merged in.
				Bin one;
				one.bounds = L[i].bounds; one.count = 1; one.flux = L[i].flux;
				for (int k = 0; k < 3; ++k) one.cone[k] = L[i].cone[k];
				one.cosCone = L[i].cosCone;
				b.merge(one.bounds, one.count, one.flux, one.cone);
			}
			for (uint32_t i = 0; i < kBins; ++i)
			{
				Bin& b = bins[i];
				const float l = std::sqrt(b.cone[0] * b.cone[0] + b.cone[1] * b.cone[1] + b.cone[2] * b.cone[2]);
				if (l < std::numeric_limits<float>::min())
					b.cosCone = kEntireCone;
				else
				{
					b.cosCone = 1.0f;
					for (int k = 0; k < 3; ++k) b.cone[k] /= l;
				}
			}
			for (uint32_t i = begin; i < end; ++i)
			{
				Bin& b = bins[binId(L[i])];
				b.cosCone = combineCones(b.cone, b.cosCone, L[i].cone, L[i].cosCone);
			}
			auto coneOf = [&](const Bin& total, uint32_t j0, uint32_t j1) {
				float cosTheta = kEntireCone;
				const float l = std::sqrt(total.cone[0] * total.cone[0] + total.cone[1] * total.cone[1] + total.cone[2] * total.cone[2]);
				if (l > std::numeric_limits<float>::min())
				{
					cosTheta = 1.0f;
					const float cd[3] = { total.cone[0] / l, total.cone[1] / l, total.cone[2] / l };
					for (uint32_t j = j0; j <= j1; ++j) cosTheta = combineCones(cd, cosTheta, bins[j].cone, bins[j].cosCone);
				}
				return cosTheta;
			};
			Bin total;
			for (uint32_t i = 0; i < nCosts; ++i)
			{
				total.merge(bins[i].bounds, bins[i].count, bins[i].flux, bins[i].cone);
				costs[i] = saoh(total.bounds, total.flux, coneOf(total, 0, i));
			}
			total = Bin{};
			for (uint32_t i = nCosts; i > 0; --i)
			{
				total.merge(bins[i].bounds, bins[i].count, bins[i].flux, bins[i].cone);
				costs[i - 1] += saoh(total.bounds, total.flux, coneOf(total, i, nCosts));
			}
			float axisCost = std::numeric_limits<float>::max();
			Split axisSplit{ dim, 0u };
			for (uint32_t i = 0, li = begin; i < nCosts; ++i)
			{
				li += bins[i].count;
				if (costs[i] < axisCost) { axisCost = costs[i]; axisSplit = Split{ dim, li }; }
			}
			axisCost *= dims[largest] / dims[dim];
			if (axisSplit.index == begin || axisSplit.index == end) continue;
			if (axisCost < splitCost) { splitCost = axisCost; split = axisSplit; }
		}
		if (!split.valid())
		{
			if (end - begin <= kMaxLeafLights) return Split{};
			return Split{ largest, (begin + end) / 2 };
		}
		return split;
	}

	// buildNodeHierarchy (src/core/light_tree.cpp:80-160).
	uint32_t hierarchy(uint64_t mask, uint32_t depth, std::vector<Light>& L, uint32_t begin, uint32_t end)
	{
		Box bounds = Box::empty();
		for (uint32_t i = begin; i < end; ++i) bounds = unite(bounds, L[i].bounds);
		const Split split = end - begin > kMaxLeafLights ? splitFunction(L, begin, end, bounds) : Split{};
		if (split.valid())
		{
			const uint32_t axis = split.axis;
			std::nth_element(L.begin() + begin, L.begin() + split.index, L.begin() + end,
				[axis](const Light& a, const Light& b) {
					float ca[3], cb[3];
					a.bounds.center(ca);
					b.bounds.center(cb);
					return ca[axis] < cb[axis];
				});
			const uint32_t me = static_cast<uint32_t>(nodes.size());
			nodes.emplace_back();
			hierarchy(mask | (0ull << depth), depth + 1, L, begin, split.index);
			const uint32_t right = hierarchy(mask | (1ull << depth), depth + 1, L, split.index, end);
			rb::PackedNode br{};
			br.core = ((1u << 31) - 1u) & right;
			nodes[me] = br;
			return me;
		}
		const uint32_t me = static_cast<uint32_t>(nodes.size());
		nodes.emplace_back();
		Attr a = leafAttributes(L[begin]);
		for (uint32_t i = begin + 1; i < end; ++i) a = add(a, leafAttributes(L[i]));
		rb::PackedNode leaf{};
		packAttributes(leaf, a);
		const uint32_t count = end - begin;
		leaf.core = (1u << 31) | ((count & 0xFu) << 27) | (begin & ((1u << 27) - 1u));
		nodes[me] = leaf;
		for (uint32_t i = begin; i < end; ++i)
		{
			pointers[i] = (rb::kLightTypeTriangle << 30) | (L[i].index & ((1u << 30) - 1u));
			masks[L[i].index] = mask;
		}
		return me;
	}

	// fillBranchNodeAttributes (src/core/light_tree.cpp:396-418): leaf
	// attributes re-read through the packed form (unpackNode).
	Attr fillBranch(uint32_t i)
	{
		const rb::PackedNode& p = nodes[i];
		if (p.core >> 31)
		{
			Attr a{};
			for (int k = 0; k < 3; ++k) a.mean[k] = p.mean[k];
			a.variance = p.variance;
			a.flux = p.flux;
			a.sharpness = p.sharpness;
			const rb::f3 d = rb::octDecode(static_cast<float>(p.direction & 0xFFFFu) / 65535.0f,
				static_cast<float>(p.direction >> 16) / 65535.0f);
			a.dir[0] = d.x; a.dir[1] = d.y; a.dir[2] = d.z;
			return a;
		}
		const uint32_t right = p.core;
		const Attr l = fillBranch(i + 1);
		const Attr r = fillBranch(right);
		const Attr m = add(l, r);
		packAttributes(nodes[i], m);
		return m;
	}
};
} // namespace

extern "C" int rb_build_light_tree(uint32_t n, const float* world, const float* flux, const uint32_t* material,
	const uint32_t* primitive, const double* cam, void* outTriangles, void* outNodes, uint32_t* outPointers,
	uint64_t* outBitmasks, uint32_t* outNodeCount)
{
	if (!outNodeCount) return RB_ERR_INVALID;
	*outNodeCount = 0;
	if (n == 0) return RB_OK;
	if (!world || !flux || !material || !primitive || !cam || !outTriangles || !outNodes || !outPointers || !outBitmasks)
		return RB_ERR_INVALID;
	if (n > (1u << 27) - 1u + kMaxLeafLights) return RB_ERR_INVALID;
	for (uint32_t k = 0; k < 9 * n; ++k)
		if (!std::isfinite(world[k])) return RB_ERR_INVALID;
	for (uint32_t k = 0; k < n; ++k)
		if (!(flux[k] > 0.0f) || !std::isfinite(flux[k])) return RB_ERR_INVALID;   // zero-flux emitters are culled upstream
	std::vector<Light> lights(n);
	auto* tris = static_cast<rb::EmissiveTri*>(outTriangles);
	for (uint32_t k = 0; k < n; ++k)
	{
		const float* v = world + 9 * k;
		float t[3][3];
		for (int j = 0; j < 3; ++j)
			for (int a = 0; a < 3; ++a)
				t[j][a] = static_cast<float>(static_cast<double>(v[3 * j + a]) - cam[a]);
		Light& l = lights[k];
		l.index = k;
		const float e1[3] = { t[1][0] - t[0][0], t[1][1] - t[0][1], t[1][2] - t[0][2] };
		const float e2[3] = { t[2][0] - t[0][0], t[2][1] - t[0][1], t[2][2] - t[0][2] };
		normalizedCross(e1, e2, l.cone);
		for (int a = 0; a < 3; ++a)
		{
			l.bounds.min[a] = std::min(t[0][a], std::min(t[1][a], t[2][a]));
			l.bounds.max[a] = std::max(t[0][a], std::max(t[1][a], t[2][a]));
			if (l.bounds.max[a] <= l.bounds.min[a])
			{
				l.bounds.min[a] = l.bounds.max[a] - std::numeric_limits<float>::epsilon();
				l.bounds.max[a] = l.bounds.max[a] + std::numeric_limits<float>::epsilon();
			}
		}
		l.cosCone = 1.0f;
		l.flux = flux[k];
		rb::EmissiveTri& et = tris[k];
		for (int q = 0; q < 9; ++q) et.v[q] = static_cast<float>(static_cast<double>(v[q]) - cam[q % 3]);
		for (int q = 0; q < 6; ++q) et.uv[q] = 0.0f;
		et.material = material[k];
		et.prim = primitive[k];
	}
	Builder b(world, flux, n);
	b.build(lights);
	auto* nodes = static_cast<rb::PackedNode*>(outNodes);
	for (size_t i = 0; i < b.nodes.size(); ++i)
	{
		nodes[i] = b.nodes[i];
		for (int a = 0; a < 3; ++a) nodes[i].mean[a] = static_cast<float>(static_cast<double>(nodes[i].mean[a]) - cam[a]);
	}
	std::memcpy(outPointers, b.pointers.data(), sizeof(uint32_t) * n);
	std::memcpy(outBitmasks, b.masks.data(), sizeof(uint64_t) * n);
	*outNodeCount = static_cast<uint32_t>(b.nodes.size());
	return RB_OK;
}
