// Oracle test infrastructure (not product code).
//
// CPU stand-in for OptiX's closed traversal (the reference calls it through
// optixTrace / optixTraverse, src/kernels/pathtrace.cu:1162,1708). It is a
// binned-SAH binary BVH over world-space triangles with the watertight
// ray/triangle test of Woop, Benthin and Wald (JCGT 2013), evaluated in strict
// IEEE float (the oracle is compiled with -ffp-contract=off). Triangles are
// two-sided (the reference disables face culling,
// src/core/rendering_interface.cpp:797). Closest-hit ties on t are broken
// towards the smaller triangle id so the result does not depend on traversal
// order.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace oracle_bvh
{
	struct V3 { float x, y, z; };
	inline float comp(const V3& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

	struct Ray
	{
		V3 o, d;
		int kx, ky, kz;
		float sx, sy, sz;
		V3 inv;
	};
	inline Ray makeRay(V3 o, V3 d)
	{
		Ray r{ o, d };
		float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
		r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
		r.kx = (r.kz + 1) % 3;
		r.ky = (r.kx + 1) % 3;
		if (comp(d, r.kz) < 0.0f) std::swap(r.kx, r.ky);
		r.sx = comp(d, r.kx) / comp(d, r.kz);
		r.sy = comp(d, r.ky) / comp(d, r.kz);
		r.sz = 1.0f / comp(d, r.kz);
		r.inv = V3{ 1.0f / d.x, 1.0f / d.y, 1.0f / d.z };
		return r;
	}

	// Watertight test. On a hit inside (tmin, tmax) returns true with t and the
	// barycentrics (b1, b2) of vertices 1 and 2.
	inline bool intersect(const Ray& r, const V3& v0, const V3& v1, const V3& v2,
		float tmin, float tmax, float& t, float& b1, float& b2)
	{
		const V3 A{ v0.x - r.o.x, v0.y - r.o.y, v0.z - r.o.z };
		const V3 B{ v1.x - r.o.x, v1.y - r.o.y, v1.z - r.o.z };
		const V3 C{ v2.x - r.o.x, v2.y - r.o.y, v2.z - r.o.z };
		const float Ax = comp(A, r.kx) - r.sx * comp(A, r.kz);
		const float Ay = comp(A, r.ky) - r.sy * comp(A, r.kz);
		const float Bx = comp(B, r.kx) - r.sx * comp(B, r.kz);
		const float By = comp(B, r.ky) - r.sy * comp(B, r.kz);
		const float Cx = comp(C, r.kx) - r.sx * comp(C, r.kz);
		const float Cy = comp(C, r.ky) - r.sy * comp(C, r.kz);
		float U = Cx * By - Cy * Bx;
		float V = Ax * Cy - Ay * Cx;
		float W = Bx * Ay - By * Ax;
		if (U == 0.0f || V == 0.0f || W == 0.0f)
		{
			// Edge case of the paper: redo the 2D edge functions in double.
			U = static_cast<float>(static_cast<double>(Cx) * By - static_cast<double>(Cy) * Bx);
			V = static_cast<float>(static_cast<double>(Ax) * Cy - static_cast<double>(Ay) * Cx);
			W = static_cast<float>(static_cast<double>(Bx) * Ay - static_cast<double>(By) * Ax);
		}
		if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f))
			return false;
		const float det = U + V + W;
		if (det == 0.0f)
			return false;
		const float Az = r.sz * comp(A, r.kz);
		const float Bz = r.sz * comp(B, r.kz);
		const float Cz = r.sz * comp(C, r.kz);
		const float T = U * Az + V * Bz + W * Cz;
		const float rcp = 1.0f / det;
		const float tt = T * rcp;
		if (!(tt > tmin && tt < tmax))
			return false;
		t = tt;
		b1 = V * rcp;
		b2 = W * rcp;
		return true;
	}

	struct Node
	{
		float lo[3], hi[3];
		int left;   // interior: index of first child (second is left+1); leaf: first triangle
		int count;  // 0 for interior nodes
	};

	class BVH
	{
	public:
		std::vector<V3> v;          // 3 vertices per triangle, world space
		std::vector<int> order;     // leaf slot -> triangle id
		std::vector<Node> nodes;

		void build(const float* worldVerts, int triCount)
		{
			v.resize(static_cast<size_t>(triCount) * 3);
			for (int i = 0; i < triCount * 3; ++i)
				v[i] = V3{ worldVerts[i * 3 + 0], worldVerts[i * 3 + 1], worldVerts[i * 3 + 2] };
			order.resize(triCount);
			for (int i = 0; i < triCount; ++i) order[i] = i;
			nodes.clear();
			if (triCount == 0) return;
			nodes.reserve(static_cast<size_t>(triCount) * 2);
			nodes.push_back(Node{});
			buildRange(0, 0, triCount);
		}

		// Closest hit: returns triangle id or -1.
		int closest(V3 o, V3 d, float tmin, float tmax, float& t, float& b1, float& b2) const
		{
			if (nodes.empty()) return -1;
			const Ray r = makeRay(o, d);
			int best = -1;
			float bestT = tmax;
			int stack[128];
			int sp = 0;
			stack[sp++] = 0;
			while (sp > 0)
			{
				const Node& n = nodes[stack[--sp]];
				if (!slab(r, n, tmin, bestT)) continue;
				if (n.count > 0)
				{
					for (int i = n.left; i < n.left + n.count; ++i)
					{
						const int id = order[i];
						float tt, u, w;
						// Accept equal t only for a smaller id (order independence).
						if (intersect(r, v[id * 3], v[id * 3 + 1], v[id * 3 + 2], tmin,
								best < 0 ? bestT : std::nextafter(bestT, INFINITY), tt, u, w))
						{
							if (tt < bestT || (tt == bestT && id < best) || best < 0)
							{
								best = id; bestT = tt; b1 = u; b2 = w;
							}
						}
					}
				}
				else
				{
					stack[sp++] = n.left + 1;
					stack[sp++] = n.left;
				}
			}
			t = bestT;
			return best;
		}

		bool any(V3 o, V3 d, float tmin, float tmax) const
		{
			if (nodes.empty()) return false;
			const Ray r = makeRay(o, d);
			int stack[128];
			int sp = 0;
			stack[sp++] = 0;
			while (sp > 0)
			{
				const Node& n = nodes[stack[--sp]];
				if (!slab(r, n, tmin, tmax)) continue;
				if (n.count > 0)
				{
					for (int i = n.left; i < n.left + n.count; ++i)
					{
						const int id = order[i];
						float tt, u, w;
						if (intersect(r, v[id * 3], v[id * 3 + 1], v[id * 3 + 2], tmin, tmax, tt, u, w))
							return true;
					}
				}
				else
				{
					stack[sp++] = n.left + 1;
					stack[sp++] = n.left;
				}
			}
			return false;
		}

	private:
		// Conservative slab test: interval widened by a few ulps so that no
		// triangle the exact test would hit is culled by box rounding.
		static bool slab(const Ray& r, const Node& n, float tmin, float tmax)
		{
			float t0 = tmin, t1 = tmax;
			const float o[3] = { r.o.x, r.o.y, r.o.z };
			const float inv[3] = { r.inv.x, r.inv.y, r.inv.z };
			for (int k = 0; k < 3; ++k)
			{
				float a = (n.lo[k] - o[k]) * inv[k];
				float b = (n.hi[k] - o[k]) * inv[k];
				if (std::isnan(a) || std::isnan(b)) continue; // ray in the slab plane
				if (a > b) std::swap(a, b);
				b *= 1.0000004f;
				t0 = a > t0 ? a : t0;
				t1 = b < t1 ? b : t1;
			}
			return t0 <= t1;
		}

		void bounds(int first, int count, float lo[3], float hi[3], float clo[3], float chi[3]) const
		{
			for (int k = 0; k < 3; ++k) { lo[k] = clo[k] = INFINITY; hi[k] = chi[k] = -INFINITY; }
			for (int i = first; i < first + count; ++i)
			{
				const int id = order[i];
				for (int j = 0; j < 3; ++j)
				{
					const V3& p = v[id * 3 + j];
					const float c[3] = { p.x, p.y, p.z };
					for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], c[k]); hi[k] = std::max(hi[k], c[k]); }
				}
				for (int k = 0; k < 3; ++k)
				{
					const float c = centroid(id, k);
					clo[k] = std::min(clo[k], c); chi[k] = std::max(chi[k], c);
				}
			}
		}
		float centroid(int id, int k) const
		{
			return (comp(v[id * 3], k) + comp(v[id * 3 + 1], k) + comp(v[id * 3 + 2], k)) * (1.0f / 3.0f);
		}
		static float area(const float lo[3], const float hi[3])
		{
			const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
			return dx * dy + dy * dz + dz * dx;
		}

		void buildRange(int nodeIndex, int first, int count)
		{
			float lo[3], hi[3], clo[3], chi[3];
			bounds(first, count, lo, hi, clo, chi);
			for (int k = 0; k < 3; ++k) { nodes[nodeIndex].lo[k] = lo[k]; nodes[nodeIndex].hi[k] = hi[k]; }
			if (count <= 2)
			{
				nodes[nodeIndex].left = first; nodes[nodeIndex].count = count;
				return;
			}
			constexpr int kBins = 16;
			int bestAxis = -1, bestSplit = -1;
			float bestCost = INFINITY;
			for (int k = 0; k < 3; ++k)
			{
				const float ext = chi[k] - clo[k];
				if (!(ext > 0.0f)) continue;
				int cnt[kBins] = {};
				float blo[kBins][3], bhi[kBins][3];
				for (int b = 0; b < kBins; ++b)
					for (int j = 0; j < 3; ++j) { blo[b][j] = INFINITY; bhi[b][j] = -INFINITY; }
				for (int i = first; i < first + count; ++i)
				{
					const int id = order[i];
					int b = static_cast<int>((centroid(id, k) - clo[k]) / ext * kBins);
					b = std::min(std::max(b, 0), kBins - 1);
					++cnt[b];
					for (int j = 0; j < 3; ++j)
						for (int q = 0; q < 3; ++q)
						{
							const float c = comp(v[id * 3 + j], q);
							blo[b][q] = std::min(blo[b][q], c); bhi[b][q] = std::max(bhi[b][q], c);
						}
				}
				for (int s = 1; s < kBins; ++s)
				{
					float l0[3] = { INFINITY, INFINITY, INFINITY }, l1[3] = { -INFINITY, -INFINITY, -INFINITY };
					float r0[3] = { INFINITY, INFINITY, INFINITY }, r1[3] = { -INFINITY, -INFINITY, -INFINITY };
					int nl = 0, nr = 0;
					for (int b = 0; b < kBins; ++b)
					{
						if (cnt[b] == 0) continue;
						float* a0 = b < s ? l0 : r0;
						float* a1 = b < s ? l1 : r1;
						(b < s ? nl : nr) += cnt[b];
						for (int q = 0; q < 3; ++q) { a0[q] = std::min(a0[q], blo[b][q]); a1[q] = std::max(a1[q], bhi[b][q]); }
					}
					if (nl == 0 || nr == 0) continue;
					const float cost = nl * area(l0, l1) + nr * area(r0, r1);
					if (cost < bestCost) { bestCost = cost; bestAxis = k; bestSplit = s; }
				}
			}
			int mid;
			if (bestAxis < 0)
			{
				mid = first + count / 2;
			}
			else
			{
				const float ext = chi[bestAxis] - clo[bestAxis];
				auto it = std::partition(order.begin() + first, order.begin() + first + count, [&](int id) {
					int b = static_cast<int>((centroid(id, bestAxis) - clo[bestAxis]) / ext * kBins);
					b = std::min(std::max(b, 0), kBins - 1);
					return b < bestSplit;
				});
				mid = static_cast<int>(it - order.begin());
				if (mid == first || mid == first + count) mid = first + count / 2;
			}
			const int left = static_cast<int>(nodes.size());
			nodes.push_back(Node{});
			nodes.push_back(Node{});
			nodes[nodeIndex].left = left;
			nodes[nodeIndex].count = 0;
			buildRange(left, first, mid - first);
			buildRange(left + 1, mid, first + count - mid);
		}
	};
}
