// Host construction of the wide BVH (see rb_bvh_build.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "rb_scene.h"

namespace rb
{
struct WideBvh
{
	std::vector<BvhNode> nodes;      // node 0 is the root unless rootIsLeaf
	std::vector<uint32_t> triOrder;  // leaf order -> input triangle index
	bool rootIsLeaf = false;         // <= kLeafMaxTris triangles: the root is one leaf
	// Bottom-up refit schedule: node indices grouped by depth, deepest first;
	// level k is refitOrder[levelStart[k] .. levelStart[k+1]).
	std::vector<uint32_t> refitOrder;
	std::vector<uint32_t> levelStart;
	uint32_t maxDepth = 0;           // wide levels below the root
};

// worldVerts: 9 floats per triangle. Degenerate triangles must already be
// removed. Leaves hold at most maxLeaf (1..kLeafMaxTris) triangles.
WideBvh buildWideBvh(const std::vector<float>& worldVerts, int maxLeaf = kLeafMaxTris);
} // namespace rb
