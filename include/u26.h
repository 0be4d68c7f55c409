/*
 * libu26 — C ABI of the B200-native Untangling26 collision-and-untangling hot path.
 *
 * Every entry point takes plain pointers and sizes. Unless a parameter says "host",
 * array pointers are DEVICE pointers (cudaMalloc'd or torch tensors' data_ptr()) that
 * the caller owns and that are borrowed for the duration of the call. Work is enqueued
 * on the stream of the context; calls return after enqueue unless they say they
 * synchronise. Sizes are explicit. No entry point aborts: failures come back as a
 * u26_status and a message from u26_ctx_last_error().
 *
 * Layouts (the reference's, Solver/SimulationCore and Solver/CollisionDetector):
 *   positions      float[3*V]       xyz per vertex (AoS, 12 B), float3 in the reference
 *   edges          uint32[2*E]      sorted unique (v0 < v1), mesh_reader.cpp:270-340
 *   faces          uint32[3*F]
 *   vert_property  uint32[V]        VertexProperty::attribute_info (simulation_data.h:36-66):
 *                                   bit0 fixed, bit1 rigid body, bits 16-30 object id
 *   EF pair        48 bytes         {uint32 idx[5]; float bary[3]; float grad[3]; float stiff}
 *                                   = CollisionPair::EfPair (collision_data.h:150-220)
 *   tree node box  float[8]         (min.x, min.y, min.z, flag, max.x, max.y, max.z, flag)
 *                                   = CompressedAABB (lbvh.h:35)
 */
#ifndef U26_H
#define U26_H

#include <stdint.h>

#ifdef __cplusplus
#define U26_API extern "C" __attribute__((visibility("default")))
#else
#define U26_API __attribute__((visibility("default")))
#endif

typedef enum u26_status
{
	U26_OK = 0,
	U26_ERR_CAPACITY = 1,		/* an output list was too small; its count holds the size needed */
	U26_ERR_UNHEALTHY_TREE = 2, /* tree failed its construction/refit check (LbvhData::sa_is_healthy) */
	U26_ERR_ITERATION_CAP = 3,	/* a bounded device loop gave up */
	U26_ERR_INVALID_INPUT = 4,
	U26_ERR_CUDA = 5,
	U26_ERR_NO_DEVICE = 6
} u26_status;

typedef enum u26_tree_type
{
	U26_TREE_VERT = 0, /* LBVHTreeTypeVert */
	U26_TREE_FACE = 1, /* LBVHTreeTypeFace */
	U26_TREE_EDGE = 2  /* LBVHTreeTypeEdge */
} u26_tree_type;

typedef enum u26_query_mode
{
	U26_QUERY_VERTS = 0,		  /* broad_phase_query_from_verts, lbvh.cpp:780-813 */
	U26_QUERY_EDGES = 1,		  /* broad_phase_query_from_edges (keeps eid < adj_eid), lbvh.cpp:815-852 */
	U26_QUERY_EDGES_UNCULLED = 2 /* broad_phase_query_from_edges_unculled, lbvh.cpp:854-894 */
} u26_query_mode;

typedef struct u26_ctx u26_ctx;
typedef struct u26_lbvh u26_lbvh;

/* ---- context -------------------------------------------------------------------
 * One context per CUDA stream; calls on one context are serialised by the caller.
 * Distinct contexts are independent. (Replaces the luisa::compute::Device/Stream pair
 * every reference entry point takes, e.g. lbvh.h:181-229.) */
U26_API u26_status u26_ctx_create(int device, void* cuda_stream, u26_ctx** out);
U26_API void u26_ctx_destroy(u26_ctx* ctx);
U26_API u26_status u26_ctx_set_stream(u26_ctx* ctx, void* cuda_stream);
U26_API u26_status u26_ctx_synchronize(u26_ctx* ctx);
U26_API const char* u26_ctx_last_error(const u26_ctx* ctx);
/* OR of the device-side error flags (1 unhealthy tree, 2 iteration cap, 4 traversal
 * stack overflow) raised since the last reset. Synchronises. */
U26_API u26_status u26_ctx_device_errors(u26_ctx* ctx, uint32_t* flags, int reset);
/* Number of kernels this context has launched since creation (instrumentation). */
U26_API uint64_t u26_ctx_launch_count(const u26_ctx* ctx);
U26_API const char* u26_version(void);

/* ---- LBVH (replaces lcs::LBVH, lbvh.h:164-325) -----------------------------------
 * Node layout as LbvhData (lbvh.h:77-150): inner nodes [0, n-2], leaves [n-1, 2n-2],
 * object_idx = ~0 for inner nodes, parent[0] = ~0. */
/* LbvhData::allocate (lbvh.h:99-140) */
U26_API u26_status u26_lbvh_create(u26_ctx* ctx, int tree_type, uint32_t num_leaves, u26_lbvh** out);
U26_API void u26_lbvh_destroy(u26_lbvh* tree);
/* LBVH::reduce_{vert,edge,face}_tree_aabb (lbvh.cpp:988-1021): global AABB of the
 * primitives at `x`. prims = edges (edge tree), faces (face tree) or NULL (vert tree).
 * num_verts sets the reference's second-pass block count (ceil(num_verts/256)). */
U26_API u26_status u26_lbvh_reduce_aabb(u26_lbvh* tree, const float* x, uint32_t num_verts, const uint32_t* prims);
/* LBVH::construct_tree (lbvh.cpp:1023-1047): Morton keys, device radix sort,
 * Karras emission, construction check. Uses the positions/prims of the last reduce. */
U26_API u26_status u26_lbvh_construct_tree(u26_lbvh* tree);
/* LBVH::update_{vert,edge,face}_tree_leave_aabb (lbvh.cpp:1050-1085): leaf AABB =
 * AABB(x_start U x_end) +- thickness[first vertex]. */
U26_API u26_status u26_lbvh_update_leaves(u26_lbvh* tree, const float* thickness, const float* x_start,
	const float* x_end, const uint32_t* prims);
/* LBVH::refit (lbvh.cpp:1087-1092): bottom-up union of the leaf AABBs. */
U26_API u26_status u26_lbvh_refit(u26_lbvh* tree);
/* Fused leaf update + refit in one launch (same result as the two calls above). */
U26_API u26_status u26_lbvh_update_and_refit(u26_lbvh* tree, const float* thickness, const float* x_start,
	const float* x_end, const uint32_t* prims);
/* LBVH::broad_phase_query_from_{verts,edges,edges_unculled} (lbvh.cpp:1193-1262).
 * Appends (query id, leaf object id) pairs to pairs[2*max_pairs] through the device
 * counter *count (not reset here; the caller zeroes it, as reset_broadphase_count does).
 * *count may end above max_pairs: the pairs past it are dropped, as in the reference. */
U26_API u26_status u26_lbvh_query(u26_lbvh* tree, int mode, const float* x_begin, const float* x_end,
	const uint32_t* edges, uint32_t num_queries, const float* d_hat, const float* thickness, uint32_t* count,
	uint32_t* pairs, uint32_t max_pairs);
/* LBVH::check_health (lbvh.cpp:1081-1085). Synchronises. *healthy = 1 or 0. */
/* Tree options (no reference counterpart; defaults reproduce the reference):
 *   U26_LBVH_OPT_FULL_GLOBAL_AABB = 1: normalise Morton codes by the AABB of ALL leaves
 *   instead of the reference's first ceil(num_verts/256) blocks (lbvh.cpp:999-1021).
 *   Query and EF results are unchanged (they do not depend on the topology unless a
 *   traversal stack overflows); the tree is better balanced in space. */
#define U26_LBVH_OPT_FULL_GLOBAL_AABB 1
U26_API u26_status u26_lbvh_set_option(u26_lbvh* tree, int option, int value);
U26_API u26_status u26_lbvh_check_health(u26_lbvh* tree, int* healthy);

typedef struct u26_lbvh_arrays
{
	uint32_t num_leaves;
	uint32_t num_nodes;
	const uint64_t* morton_sorted;		  /* [n]     sa_morton_sorted */
	const uint32_t* sorted_get_original;  /* [n]     sa_sorted_get_original */
	const uint32_t* parent;				  /* [2n-1]  sa_parrent */
	const uint32_t* children;			  /* [2n-1][2] sa_children */
	const uint32_t* object_idx;			  /* [2n-1]  sa_object_idx */
	const float* node_aabb;				  /* [2n-1][8] sa_node_aabb_v2 */
	const float* global_aabb;			  /* [6]     sa_block_aabb[0] */
} u26_lbvh_arrays;
/* Device pointers to the tree arrays (valid until the tree is destroyed). */
U26_API u26_status u26_lbvh_arrays_get(const u26_lbvh* tree, u26_lbvh_arrays* out);

/* ---- EF detection (replaces IntersectionResolver::ef_dcd_intersection_query,
 * intersection_resolver.h:41-52 / intersection_resolver.cpp:365-423) ---------------
 * Narrow phase over broad-phase (eid, fid) pairs: segment-triangle test with the
 * reference's grazing filters (intersection_resolver.cpp:86-197). The number of broad
 * pairs is read on the device from *broad_count (clamped to max_broad). EF pairs are
 * appended through *ef_count (caller zeroes it); ef_pairs is 48 B per pair and
 * ef_indices is uint32[2] per pair. vert_property may be NULL (all zero). */
U26_API u26_status u26_ef_narrow_phase(u26_ctx* ctx, const uint32_t* broad_pairs, const uint32_t* broad_count,
	uint32_t max_broad, const float* x, const uint32_t* edges, const uint32_t* faces, const uint32_t* vert_property,
	const float* d_hat, uint32_t* ef_count, void* ef_pairs, uint32_t* ef_indices, uint32_t max_ef);

/* Fused EF detection: edges of the mesh against a refit face tree, segment-triangle
 * test at each overlapping leaf, no broad-phase list in between. Same EF pair set as
 * u26_lbvh_query(U26_QUERY_EDGES_UNCULLED) + u26_ef_narrow_phase whenever the broad
 * list would not have overflowed. edge_order (optional, uint32[num_edges]) is the order
 * in which threads take the edges, e.g. an edge tree's sorted_get_original so that a
 * warp walks spatially close edges; NULL means edge id order. stats (optional,
 * uint64[2]) accumulates node boxes tested and leaf triangles tested. */
U26_API u26_status u26_ef_detect(u26_lbvh* face_tree, const float* x, const uint32_t* edges, uint32_t num_edges,
	const uint32_t* faces, const uint32_t* vert_property, const float* d_hat, const float* thickness,
	const uint32_t* edge_order, uint32_t* ef_count, void* ef_pairs, uint32_t* ef_indices, uint32_t max_ef,
	uint64_t* stats);

/* Canonical EF order on the device: sort by (eid, fid) — the order
 * host_preprocess_ef_pairs establishes (intersection_resolver.cpp:693-726). count is a
 * host value; num_edges/num_faces bound the key. Pairs and indices are permuted in place. */
U26_API u26_status u26_ef_canonicalize(u26_ctx* ctx, uint32_t count, void* ef_pairs, uint32_t* ef_indices,
	uint32_t num_edges, uint32_t num_faces);

#endif /* U26_H */
