// Host-side builder of the compressed 8-wide BVH traversed by the GPU kernels.
//
// Replaces the reference's TLAS construction, TBvhBuilder<2> with bucketed SAH and one item per
// leaf (Engine/Source/Math/Algorithm/BVH/TBvhBuilder.ipp:36,516; BvhParams.h:23-35) followed by
// TLinearDepthFirstBinaryBvh::build. The hit a ray finds does not depend on the tree: both trees
// bound every triangle conservatively, and the closest hit is decided by the watertight triangle
// test alone (ties between triangles at identical t are resolved by the smaller primitive index).
#pragma once

#include "pg_common.cuh"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace pg
{

struct BvhBuildInput
{
	const float*    tris;          // [num_tris][3][3] world-space vertices
	const uint32_t* materials;     // [num_tris] material index (may be null = 0)
	const uint32_t* emitters;      // [num_tris] emitter index + 1, 0 = none (may be null)
	std::size_t     num_tris;
	// Largest coordinate magnitude any ray origin will have (camera included); used to size the
	// conservative padding of child boxes so that FP32 slab-test rounding never loses a hit.
	float           max_origin_abs;
	// Binned-SAH builder: a node with at most this many triangles becomes a leaf (1..3, the node
	// layout's limit). Fewer triangles per leaf: more nodes, fewer triangle tests per ray.
	uint32_t        max_leaf_tris = 3;
};

struct BvhBuildStats
{
	std::size_t num_nodes = 0;
	std::size_t num_leaf_tris = 0;
	int         max_depth = 0;        // wide-tree depth (root = 1)
	int         binary_max_depth = 0;
	double      build_seconds = 0.0;
	float       box_padding = 0.0f;
};

struct WideBvh
{
	std::vector<WideNode> nodes;     // node 0 is the root
	std::vector<LeafTri>  tris;      // leaf order
	BvhBuildStats         stats;
};

// Builds the wide BVH. Degenerate triangles are kept (the traversal test rejects them), so the
// leaf triangle count always equals num_tris. Throws std::runtime_error on invalid input.
WideBvh build_wide_bvh(const BvhBuildInput& in);

}// end namespace pg
