// Host construction of the 8-wide BVH traversed by rb_bvh.cuh.
//
// 1. Binned SAH binary BVH (32 bins per axis on centroid bounds, leaves of at
//    most kLeafMaxTris triangles, SAH leaf/split decision).
// 2. Collapse to 8-wide: each wide node takes its binary node's children and
//    repeatedly opens the interior child with the largest surface area until
//    it has 8 children (the greedy collapse of Wald et al. 2008 / Ylitie et
//    al. 2017).
// 3. Place each wide node's children in its 8 slots by direction octant
//    (Ylitie, Karras and Laine 2017, sec. 3.2), so that traversal can visit
//    them roughly near to far without sorting: see assignSlots.
// 4. Quantize child boxes to 8 bits per plane against a node origin and a
//    power-of-two scale per axis. The scale is at least two float ulps of the
//    node's coordinates and the origin is a multiple of it, so every decoded
//    plane origin + q*scale is exact in float; boxes are rounded outward and
//    padded by one step, so the quantized box always contains the exact one.
#include "rb_bvh_build.h"
#include "rb_bvh_quant.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace rb
{
namespace
{
struct Box
{
	double lo[3] = { INFINITY, INFINITY, INFINITY };
	double hi[3] = { -INFINITY, -INFINITY, -INFINITY };
	void grow(const Box& b)
	{
		for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
	}
	void grow(double x, double y, double z)
	{
		lo[0] = std::min(lo[0], x); lo[1] = std::min(lo[1], y); lo[2] = std::min(lo[2], z);
		hi[0] = std::max(hi[0], x); hi[1] = std::max(hi[1], y); hi[2] = std::max(hi[2], z);
	}
	double area() const
	{
		if (!(hi[0] >= lo[0])) return 0.0;
		const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
		return 2.0 * (dx * dy + dy * dz + dz * dx);
	}
};

struct BinNode
{
	Box box;
	int left = -1, right = -1;   // children (interior)
	int first = 0, count = 0;    // triangle range (leaf)
};

class BinaryBuilder
{
public:
	BinaryBuilder(const std::vector<Box>& boxes, const std::vector<float>& cx, const std::vector<float>& cy,
		const std::vector<float>& cz, int maxLeaf)
		: m_boxes(boxes), m_maxLeaf(maxLeaf)
	{
		m_c[0] = &cx; m_c[1] = &cy; m_c[2] = &cz;
		m_order.resize(boxes.size());
		for (size_t i = 0; i < boxes.size(); ++i) m_order[i] = static_cast<uint32_t>(i);
	}
	std::vector<BinNode> nodes;
	std::vector<uint32_t> m_order;

	void build()
	{
		nodes.reserve(m_boxes.size() * 2);
		nodes.emplace_back();
		buildNode(0, 0, static_cast<int>(m_boxes.size()));
	}

private:
	const std::vector<Box>& m_boxes;
	const int m_maxLeaf;
	const std::vector<float>* m_c[3];

	void buildNode(int ni, int first, int count)
	{
		Box box, cbox;
		for (int i = first; i < first + count; ++i)
		{
			const uint32_t t = m_order[i];
			box.grow(m_boxes[t]);
			cbox.grow((*m_c[0])[t], (*m_c[1])[t], (*m_c[2])[t]);
		}
		nodes[ni].box = box;
		nodes[ni].first = first;
		nodes[ni].count = count;
		if (count <= 1) return;

		constexpr int kBins = 32;
		int bestAxis = -1, bestSplit = -1;
		double bestCost = INFINITY;
		for (int a = 0; a < 3; ++a)
		{
			const double ext = cbox.hi[a] - cbox.lo[a];
			if (!(ext > 0.0)) continue;
			const double scale = kBins / ext;
			Box bb[kBins];
			int bc[kBins] = {};
			for (int i = first; i < first + count; ++i)
			{
				const uint32_t t = m_order[i];
				int b = static_cast<int>(((*m_c[a])[t] - cbox.lo[a]) * scale);
				b = std::min(std::max(b, 0), kBins - 1);
				bb[b].grow(m_boxes[t]);
				++bc[b];
			}
			double rightArea[kBins];
			int rightCount[kBins];
			Box acc;
			int n = 0;
			for (int b = kBins - 1; b > 0; --b)
			{
				acc.grow(bb[b]); n += bc[b];
				rightArea[b] = acc.area(); rightCount[b] = n;
			}
			acc = Box{}; n = 0;
			for (int b = 0; b < kBins - 1; ++b)
			{
				acc.grow(bb[b]); n += bc[b];
				if (n == 0 || rightCount[b + 1] == 0) continue;
				const double cost = acc.area() * n + rightArea[b + 1] * rightCount[b + 1];
				if (cost < bestCost) { bestCost = cost; bestAxis = a; bestSplit = b + 1; }
			}
		}
		// SAH leaf test: traversal cost 1, triangle cost 1, relative to the parent area.
		const double leafCost = static_cast<double>(count);
		const double parentArea = box.area();
		const double splitCost = parentArea > 0.0 ? 1.0 + bestCost / parentArea : INFINITY;
		if (count <= m_maxLeaf && (bestAxis < 0 || leafCost <= splitCost)) return;

		int mid;
		if (bestAxis < 0)
		{
			// All centroids coincide: split the range in half.
			mid = first + count / 2;
		}
		else
		{
			const double ext = cbox.hi[bestAxis] - cbox.lo[bestAxis];
			const double scale = kBins / ext;
			const std::vector<float>& c = *m_c[bestAxis];
			const double lo = cbox.lo[bestAxis];
			auto it = std::partition(m_order.begin() + first, m_order.begin() + first + count, [&](uint32_t t) {
				int b = static_cast<int>((c[t] - lo) * scale);
				b = std::min(std::max(b, 0), kBins - 1);
				return b < bestSplit;
			});
			mid = static_cast<int>(it - m_order.begin());
			if (mid == first || mid == first + count) mid = first + count / 2;
		}
		const int l = static_cast<int>(nodes.size());
		nodes.emplace_back();
		nodes.emplace_back();
		nodes[ni].left = l;
		nodes[ni].right = l + 1;
		nodes[ni].count = 0;
		buildNode(l, first, mid - first);
		buildNode(l + 1, mid, first + count - mid);
	}
};

bool isLeaf(const BinNode& n) { return n.left < 0; }

class WideBuilder
{
public:
	WideBuilder(const std::vector<BinNode>& bin) : m_bin(bin) {}
	std::vector<BvhNode> nodes;
	std::vector<uint32_t> leafRanges;   // pairs: binary leaf first, count in emission order

	// Emits the wide node for binary node `bi`; returns its index.
	uint32_t emit(int bi, std::vector<uint32_t>& triOrderOut, const std::vector<uint32_t>& binOrder)
	{
		// Gather up to 8 children.
		int kids[8];
		int n = 0;
		kids[n++] = m_bin[bi].left;
		kids[n++] = m_bin[bi].right;
		while (n < 8)
		{
			int best = -1;
			double bestArea = -1.0;
			for (int i = 0; i < n; ++i)
			{
				if (isLeaf(m_bin[kids[i]])) continue;
				const double a = m_bin[kids[i]].box.area();
				if (a > bestArea) { bestArea = a; best = i; }
			}
			if (best < 0) break;
			const int open = kids[best];
			kids[best] = m_bin[open].left;
			kids[n++] = m_bin[open].right;
		}
		int slotOf[8];
		assignSlots(bi, kids, n, slotOf);
		const uint32_t me = static_cast<uint32_t>(nodes.size());
		nodes.emplace_back();
		BvhNode node{};
		double lo[8][3], hi[8][3];
		uint32_t slots = 0;
		for (int c = 0; c < n; ++c)
		{
			const int s = slotOf[c];
			slots |= 1u << s;
			for (int a = 0; a < 3; ++a) { lo[s][a] = m_bin[kids[c]].box.lo[a]; hi[s][a] = m_bin[kids[c]].box.hi[a]; }
		}
		quantizeChildren(slots, lo, hi, node);
		for (int c = 0; c < 8; ++c) node.child[c] = kEmptyChild;
		// Children: leaves reference their (re-emitted) triangle range, interior
		// nodes recurse.
		for (int c = 0; c < n; ++c)
		{
			const BinNode& k = m_bin[kids[c]];
			if (isLeaf(k))
			{
				const uint32_t first = static_cast<uint32_t>(triOrderOut.size());
				for (int i = k.first; i < k.first + k.count; ++i) triOrderOut.push_back(binOrder[i]);
				node.child[slotOf[c]] = kLeafBit | (static_cast<uint32_t>(k.count - 1) << 28) | first;
			}
		}
		nodes[me] = node;
		for (int c = 0; c < n; ++c)
		{
			if (!isLeaf(m_bin[kids[c]]))
			{
				const uint32_t ci = emit(kids[c], triOrderOut, binOrder);
				nodes[me].child[slotOf[c]] = ci;
			}
		}
		return me;
	}

private:
	const std::vector<BinNode>& m_bin;

	// Slot s (bit 0: x, bit 1: y, bit 2: z) holds the child that a ray whose
	// direction has those negative components meets first: the child whose
	// centre lies farthest back along that direction. The cost of child c in
	// slot s is dot(centre_c - centre_parent, d_s) with d_s = (+-1, +-1, +-1)
	// the octant's diagonal; pairs are taken greedily, cheapest first.
	void assignSlots(int bi, const int* kids, int n, int* slotOf) const
	{
		const Box& pb = m_bin[bi].box;
		double pc[3];
		for (int a = 0; a < 3; ++a) pc[a] = 0.5 * (pb.lo[a] + pb.hi[a]);
		double cost[8][8];
		for (int c = 0; c < n; ++c)
		{
			const Box& b = m_bin[kids[c]].box;
			double d[3];
			for (int a = 0; a < 3; ++a) d[a] = 0.5 * (b.lo[a] + b.hi[a]) - pc[a];
			for (int s = 0; s < 8; ++s)
				cost[c][s] = ((s & 1) ? -d[0] : d[0]) + ((s & 2) ? -d[1] : d[1]) + ((s & 4) ? -d[2] : d[2]);
		}
		bool childDone[8] = {}, slotUsed[8] = {};
		for (int k = 0; k < n; ++k)
		{
			int bc = -1, bs = -1;
			double best = INFINITY;
			for (int c = 0; c < n; ++c)
			{
				if (childDone[c]) continue;
				for (int s = 0; s < 8; ++s)
					if (!slotUsed[s] && (bc < 0 || cost[c][s] < best)) { best = cost[c][s]; bc = c; bs = s; }
			}
			childDone[bc] = true;
			slotUsed[bs] = true;
			slotOf[bc] = bs;
		}
	}
};
} // namespace

WideBvh buildWideBvh(const std::vector<float>& worldVerts, int maxLeaf)
{
	WideBvh out;
	const size_t n = worldVerts.size() / 9;
	if (n == 0) return out;
	std::vector<Box> boxes(n);
	std::vector<float> cx(n), cy(n), cz(n);
	for (size_t t = 0; t < n; ++t)
	{
		const float* v = worldVerts.data() + 9 * t;
		for (int k = 0; k < 3; ++k) boxes[t].grow(v[3 * k], v[3 * k + 1], v[3 * k + 2]);
		cx[t] = (v[0] + v[3] + v[6]) / 3.0f;
		cy[t] = (v[1] + v[4] + v[7]) / 3.0f;
		cz[t] = (v[2] + v[5] + v[8]) / 3.0f;
	}
	BinaryBuilder bb(boxes, cx, cy, cz, std::min(std::max(maxLeaf, 1), kLeafMaxTris));
	bb.build();
	if (isLeaf(bb.nodes[0]))
	{
		out.rootIsLeaf = true;
		out.triOrder.assign(bb.m_order.begin(), bb.m_order.end());
		return out;
	}
	WideBuilder wb(bb.nodes);
	wb.emit(0, out.triOrder, bb.m_order);
	out.nodes = std::move(wb.nodes);
	// Refit order: nodes grouped by depth, deepest level first.
	std::vector<uint32_t> depth(out.nodes.size(), 0);
	uint32_t maxDepth = 0;
	for (uint32_t i = 0; i < out.nodes.size(); ++i)          // pre-order: parents come first
		for (int c = 0; c < 8; ++c)
		{
			const uint32_t ref = out.nodes[i].child[c];
			if (ref != kEmptyChild && !(ref & kLeafBit))
			{
				depth[ref] = depth[i] + 1;
				maxDepth = std::max(maxDepth, depth[ref]);
			}
		}
	out.maxDepth = maxDepth;
	out.levelStart.assign(1, 0);
	for (int d = static_cast<int>(maxDepth); d >= 0; --d)
	{
		for (uint32_t i = 0; i < out.nodes.size(); ++i)
			if (depth[i] == static_cast<uint32_t>(d)) out.refitOrder.push_back(i);
		out.levelStart.push_back(static_cast<uint32_t>(out.refitOrder.size()));
	}
	return out;
}
} // namespace rb
