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
	u26::DevBuf refit_flags;		 // uint32[max(n-1,1)]: arrival counters of the height pass (construction)
	u26::DevBuf node_range;			 // uint32[max(n-1,1)]: inner node i covers leaves [min(i, r), max(i, r)], r = node_range[i]
	// refit plan, prepared by construct_tree (one per topology)
	u26::DevBuf height;			 // uint8[max(n-1,1)]: inner node height (leaves 0)
	u26::DevBuf chunk_lo;		 // uint32[nchunks + 1]: first leaf of each refit chunk, then n
	u26::DevBuf top_nodes;		 // uint32[m]: nodes of more than 1024 leaves, by height
	u26::DevBuf top_links;		 // uint2[m]: their children as compact ids (top j, or 0x80000000 | treelet b)
	u26::DevBuf height_end;		 // uint32[65]: end of each height's run in top_nodes (0: none)
	u26::DevBuf roots;			 // uint32[nt]: treelet roots (maximal subtrees of <= 1024 leaves) in leaf order
	u26::DevBuf chunk_tb;		 // uint32[nchunks + 1]: first treelet of each chunk, then nt
	u26::DevBuf top_height;		 // uint8[m]: heights of top_nodes
	u26::DevBuf root_box;		 // float[nt][6]: the treelet roots' boxes of the last refit, compact
	u26::DevBuf plan_scratch;	 // construction scratch (list keys, counts, compact map), freed when the plan is made
	uint32_t nchunks = 0, ntop = 0, ntreelets = 0;
	bool top_in_shared = false;
	u26::DevBuf leaf_prims;			 // uint32[n][K]: the primitive table in leaf order (edge / face trees)
	const uint32_t* leaf_prims_src = nullptr; // the table leaf_prims was permuted from
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
