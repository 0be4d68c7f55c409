// Internal layout of a u26_lbvh (one tree over vertices, edges or faces).
// Mirrors LbvhData (lbvh.h:77-150) with device-sorted Morton keys instead of the host copy.
#pragma once
#include "u26_internal.h"

struct u26_lbvh
{
	u26_ctx* ctx = nullptr;
	int type = U26_TREE_FACE;
	uint32_t n = 0; // leaves
	u26::DevBuf morton_sorted;		 // uint64[n]
	u26::DevBuf sorted_get_original; // uint32[n]
	u26::DevBuf parent;				 // uint32[2n-1]
	u26::DevBuf children;			 // uint32[2n-1][2]
	u26::DevBuf object_idx;			 // uint32[2n-1]
	u26::DevBuf node_aabb;			 // NodeBox[2n-1]
	u26::DevBuf block_aabb;			 // float[ceil(n/256)][6]
	u26::DevBuf global_aabb;		 // float[6]
	u26::DevBuf refit_flags;		 // uint32[max(n-1,1)]: arrival counters, even between refits
	u26::DevBuf node_range;			 // uint32[max(n-1,1)]: inner node i covers leaves [min(i, r), max(i, r)], r = node_range[i]
	u26::DevBuf health;				 // uint32[1]: 1 healthy
	u26::RadixSorter sorter;
	// inputs of the last reduce_aabb (construct_tree reads them, as the reference
	// keeps sa_leaf_center from the reduce pass)
	const float* last_x = nullptr;
	const uint32_t* last_prims = nullptr;
	// 0: the reference's second-pass block count ceil(num_verts/256) (parity mode);
	// 1: all leaf blocks (the true global AABB, better Morton spread)
	int full_global_aabb = 0;
	uint32_t last_num_verts = 0;
	bool built = false; // construct_tree has run (parent / children / node_range are valid)

	uint32_t num_inner() const { return n > 0 ? n - 1 : 0; }
	uint32_t num_nodes() const { return n > 0 ? 2 * n - 1 : 0; }
};

namespace u26
{
	// Traversal view handed to the query kernels.
	struct TreeView
	{
		const NodeBox* __restrict__ boxes;
		const uint2* __restrict__ children;
		const uint32_t* __restrict__ object_idx;
		const uint32_t* __restrict__ health;
		uint32_t n;
	};
	inline TreeView tree_view(const u26_lbvh* t)
	{
		return TreeView{ t->node_aabb.as<NodeBox>(), t->children.as<uint2>(), t->object_idx.as<uint32_t>(),
			t->health.as<uint32_t>(), t->n };
	}
} // namespace u26
