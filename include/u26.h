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
/* Device and pinned host allocations the library has made in this process so far (every
 * context); a diagnostic: entry points documented as allocation-free leave it unchanged. No
 * reference counterpart. */
U26_API uint64_t u26_alloc_count(void);
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
/* Fused leaf update + refit (same result as the two calls above): a launch over chunks of at
 * most 1024 leaves (whole subtrees; leaf boxes and the chunk's inner nodes united height by
 * height in shared memory) and a one-block launch for the nodes above them (construct_tree
 * prepares both, once per topology). When prims is the table the tree was
 * constructed from (the pointer given to the last reduce_aabb before construct_tree), the
 * leaf boxes read the tree's copy of it in leaf order; the topology is assumed unchanged
 * since that construction. Another table is read through the leaf order. */
U26_API u26_status u26_lbvh_update_and_refit(u26_lbvh* tree, const float* thickness, const float* x_start,
	const float* x_end, const uint32_t* prims);
/* LBVH::broad_phase_query_from_{verts,edges,edges_unculled} (lbvh.cpp:1193-1262).
 * Appends (query id, leaf object id) pairs to pairs[2*max_pairs] through the device
 * counter *count (not reset here; the caller zeroes it, as reset_broadphase_count does).
 * *count may end above max_pairs: the pairs past it are dropped, as in the reference. */
U26_API u26_status u26_lbvh_query(u26_lbvh* tree, int mode, const float* x_begin, const float* x_end,
	const uint32_t* edges, uint32_t num_queries, const float* d_hat, const float* thickness, uint32_t* count,
	uint32_t* pairs, uint32_t max_pairs);
/* Tree options (no reference counterpart; defaults reproduce the reference):
 *   U26_LBVH_OPT_FULL_GLOBAL_AABB = 1: normalise Morton codes by the AABB of ALL leaves
 *   instead of the reference's first ceil(num_verts/256) blocks (lbvh.cpp:999-1021).
 *   Query and EF results are unchanged (they do not depend on the topology unless a
 *   traversal stack overflows); the tree is better balanced in space. */
#define U26_LBVH_OPT_FULL_GLOBAL_AABB 1
U26_API u26_status u26_lbvh_set_option(u26_lbvh* tree, int option, int value);
/* LBVH::check_health (lbvh.cpp:1081-1085). Synchronises. *healthy = 1 or 0. */
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
 * uint64[4]) accumulates node boxes tested, leaf triangles tested, and (given stats) the
 * FP64 recheck of every EF test whose FP32 decision lies inside its static error band:
 * [2] the tests rechecked, [3] those whose FP64 decision differs. The EF set keeps the
 * FP32 decisions either way. */
U26_API u26_status u26_ef_detect(u26_lbvh* face_tree, const float* x, const uint32_t* edges, uint32_t num_edges,
	const uint32_t* faces, const uint32_t* vert_property, const float* d_hat, const float* thickness,
	const uint32_t* edge_order, uint32_t* ef_count, void* ef_pairs, uint32_t* ef_indices, uint32_t max_ef,
	uint64_t* stats);

/* Canonical EF order on the device: sort by (eid, fid), equal keys by memcmp of the 48-byte
 * records — the order host_preprocess_ef_pairs establishes (intersection_resolver.cpp:693-726).
 * count is a host value; num_edges/num_faces bound the key. Pairs and indices are permuted in place. */
U26_API u26_status u26_ef_canonicalize(u26_ctx* ctx, uint32_t count, void* ef_pairs, uint32_t* ef_indices,
	uint32_t num_edges, uint32_t num_faces);

/* Allocation-free variant of u26_ef_canonicalize (no counterpart in the reference, which
 * sorts on the host). For callers that cannot let the library allocate device memory: a
 * solver that owns all GPU memory in its own arena, or a loop that must not run
 * cudaMalloc / cudaFree because they can synchronise the device. Same result as
 * u26_ef_canonicalize. Its scratch is a fixed array of U26_NOALLOC_SCRATCH_BYTES in
 * the library's static device memory, held on every GPU that loads the library until the
 * process exits; count above U26_NOALLOC_MAX_EF_PAIRS returns U26_ERR_CAPACITY. The
 * first call on each context looks up the array's device address on the context's device
 * and keeps it on the context (make that first call before any stream capture; a context
 * created after a device reset looks the address up again). All calls share the one array:
 * calls that overlap on the GPU (other streams or contexts) race and must be ordered by
 * the caller. */
#define U26_NOALLOC_MAX_EF_PAIRS 32768u
#define U26_NOALLOC_SCRATCH_BYTES 2637824u
U26_API u26_status u26_ef_canonicalize_noalloc(u26_ctx* ctx, uint32_t count, void* ef_pairs, uint32_t* ef_indices,
	uint32_t num_edges, uint32_t num_faces);

/* ---- PRP contour evaluation ---------------------------------------------------------
 * The reference's IntersectionResolver::host_resolve with the PRP method
 * (intersection_resolver.cpp:2131-2218 -> host_resolve_intersections_PRP,
 * intersection_resolver2.cpp:2750-4072, or device_resolve_intersections_PRP,
 * intersection_resolver_gpu.cpp:2792-4460): EF preprocessing and contours, per-contour
 * runtime (hop/geodesic distances, candidate directions), adaptive k-ring evaluation of
 * every (contour, direction) with VF/EE/FV ray casting, product-complex cluster culling
 * and J(r), selection, cross-contour suppression.
 *
 * Mesh tables are HOST pointers in the reference's conventions (MeshData, built once per
 * scene by its initialiser, init_mesh_data.cpp:294-835); u26_scene_create uploads them. */
typedef struct u26_mesh_desc
{
	uint32_t num_verts, num_edges, num_faces, num_objects;
	const float* x;				  /* [V][3] current positions (used only by host-side stages) */
	const float* rest_x;		  /* [V][3] rest positions (geodesic distances) */
	const uint32_t* edges;		  /* [E][2] sorted unique, grouped by object */
	const uint32_t* faces;		  /* [F][3] grouped by object */
	const uint32_t* face_adj_edges; /* [F][3] edge of (face[j], face[j+1]) */
	const uint32_t *vert_adj_verts_offsets, *vert_adj_verts; /* CSR, edge-id order */
	const uint32_t *vert_adj_edges_offsets, *vert_adj_edges; /* CSR, ascending */
	const uint32_t *vert_adj_faces_offsets, *vert_adj_faces; /* CSR, ascending */
	const uint32_t *edge_adj_faces_offsets, *edge_adj_faces; /* CSR, edge_adj_faces_ext */
	const uint32_t *edge_adj_edges_offsets, *edge_adj_edges; /* CSR, edge_adj_edges_ext */
	const uint32_t *prefix_num_verts, *prefix_num_edges, *prefix_num_faces; /* [objects+1] */
	const uint32_t* vert_object;	/* sa_vert_mesh_id */
	const uint32_t* vert_component; /* vert_topology_component_id */
	const float *rest_vert_area, *rest_edge_area, *rest_face_area, *vert_mass;
	const uint32_t* mesh_orientation; /* [objects] 0: normals along the triangle winding */
	const uint32_t* object_scene;	  /* [objects] independent scene of each object, or NULL (one scene): several
									   * simulations evaluated in one batch keep their own global centroid
									   * (the radial seed direction of get_raycasting_direction) */
	const uint32_t* object_solid;	  /* [objects] 1 for rigid / tetrahedral material (sa_vert_mesh_type), or NULL:
									   * no solid objects (the solid-interior hit links never apply) */
} u26_mesh_desc;

typedef struct u26_scene u26_scene;
U26_API u26_status u26_scene_create(u26_ctx* ctx, const u26_mesh_desc* mesh, u26_scene** out);
U26_API void u26_scene_destroy(u26_scene* scene);

/* SceneParams fields of the PRP path (scene_params.h:65-81). */
typedef struct u26_prp_params
{
	uint32_t max_contours;		/* untangling_process_contours_count (256) */
	uint32_t direction_mode;	/* 0: the reference's seed directions (resolver2.cpp:1488-1569); 1: 26 lattice directions */
	uint32_t use_ccr;			/* PRP_use_intrinsic_contour_side_candidates (1) */
	float ccr_tau;				/* PRP_intrinsic_tau (0.25) */
	uint32_t ccr_use_rest;		/* PRP_use_rest_geodesic_distance_for_intrinsic_candidates (1) */
	uint32_t ccr_use_current;	/* PRP_use_deformed_boundary_distance_for_intrinsic_candidates (1) */
	uint32_t batch_size;		/* PRP_cpu_contour_batch_size (32): a contour's merge partners are limited to its own or earlier batches */
	uint32_t opt_iterations;	/* PRP_direction_optimization_iterations (0 = off): projected Newton / Cauchy steps of the
								 * selected direction on S^2 (intersection_resolver2.cpp:1232-1486) */
	uint32_t ccr_blend;			/* PRP_use_blended_intrinsic_coordinates (0): one blended ownership coordinate */
	float ccr_blend_weight;		/* PRP_intrinsic_blend_weight (0.5): rest-coordinate weight of the blend */
	uint32_t form;				/* ray casting form: 0 batched packet traversal clipped to the candidate boxes (default),
								 * 1 the plain form (one thread per request from the root, one launch per contour);
								 * both decide the same pairs and return the same results */
	uint32_t solid_interior;	/* PRP_solid_interior_adjacency (1): link hits through solid interiors */
	uint32_t solid_all;			/* PRP_solid_interior_adjacency_all_meshes (0): treat every mesh as solid */
	float solid_eps_n;			/* PRP_solid_interior_adjacency_normal_eps (1e-4) */
	float solid_eps_d;			/* PRP_solid_interior_adjacency_dist_eps (1e-5) */
	uint32_t ignore_near_zero_dist_pairs; /* ignore_near_zero_dist_pairs (1, scene_params.h:55; the CLI sets 0):
										   * 0 drops degenerate EF pairs (a barycentric coordinate < 1e-4) that
										   * have no non-degenerate adjacent pair (intersection_resolver.cpp:841-896) */
	uint32_t fp64_recheck;		/* 1 (default): every VF / FV / EE leaf test of the batched form whose FP32 decision lies
								 * inside its static forward-error band is re-evaluated in FP64 and counted
								 * (u26_prp_output_view.fp64_rechecks / fp64_flips); the hit sets keep the FP32
								 * decisions. Also evaluates the selected supports' metrics in FP64 (fp64_*_rel_err). */
	uint32_t autotune;			/* 1: the scene's first pass times every ray-casting configuration (subtree parts x blocks
								 * per SM x grid form) on each of its launches and the scene keeps the fastest;
								 * 0: 8 parts, 7 blocks, a warp per work item */
	uint32_t raycast_config;	/* 0: the default or autotuned configuration; k in 1..18: use configuration k - 1 of the
								 * table in u26_prp_output_view.tune_ms (every configuration returns the same results) */
} u26_prp_params;

/* Per-contour result (PRPMinContourHitInfo, intersection_resolver2.h:508-550). flags:
 * 1 response_eligible, 2 no_response_terminal, 4 suppressed, 8 full_mesh_evaluated,
 * 16 processed (contour index < max_contours). combo_idx = ~0 when there is no response. */
typedef struct u26_prp_result
{
	uint32_t contour_idx, contour_type, num_pairs, combo_idx;
	uint32_t num_dirs, hit_count, unculled_hit_count, covered_anchor_count;
	uint32_t boundary_anchor_count, eval_k_src, eval_k_dst, max_frontier_hop_src;
	uint32_t max_frontier_hop_dst, expansion_level_count, flags, object_id0;
	uint32_t object_id1, init_k_src, init_k_dst, diam_src;
	uint32_t diam_dst, num_boundary_src, num_boundary_dst, opt_attempted;
	float dir[3];
	float depth, volume, objective, area, displacement_cost, coverage, normalized_objective, pre_finalize_area;
	uint32_t opt_accepted; /* direction refinement: trial steps taken / accepted (direction_optimization_*_count) */
} u26_prp_result;

/* One hit of a selected support S(r) (RayCasting::HitInfo, intersection_resolver_helper.h:260-449,
 * without the group and direction fields). type 0 VF, 1 EE, 2 FV; unused vertex slots ~0. */
typedef struct u26_prp_hit
{
	uint32_t type, src_id, dst_id, src_verts[3], dst_verts[3];
	float bary[2], dist;
} u26_prp_hit;

typedef struct u26_prp_output u26_prp_output;
typedef struct u26_prp_output_view
{
	uint32_t num_pairs, num_orig_pairs, num_contours, num_hits;
	const void* pairs;				 /* [num_pairs] 48-B EF pairs, loop-vertex pairs appended */
	const uint32_t* pair_indices;	 /* [num_pairs][2] (eid, fid) */
	const uint32_t* mesh_index;		 /* [num_pairs] ef_pair_mesh_index */
	const uint32_t* contour_index;	 /* [num_pairs] ef_pair_contour_index */
	const float* pair_length;		 /* [num_pairs] ef_pair_length */
	const uint32_t* contour_offsets; /* [num_contours+1] into contour_pairs */
	const uint32_t* contour_pairs;	 /* pair ids of each contour in flood-fill order */
	const u26_prp_result* results;	 /* [num_contours] */
	const uint32_t* hit_offsets;	 /* [num_contours+1] into hits */
	const u26_prp_hit* hits;		 /* selected supports, canonical (type, src, dst) order */
	const float* directions;		 /* [num_contours][26][3] candidate directions (num_dirs used) */
	uint64_t ray_tests;				 /* leaf primitive tests of all ray casts */
	uint64_t ray_requests;			 /* VF + EE + FV ray requests */
	uint64_t ray_pairs;				 /* (request, candidate target) pairs decided: the
									  * implementation-independent ray-primitive test count */
	uint32_t levels;				 /* k-ring levels evaluated (max over batches) */
	uint32_t device_error_flags;
	double stage_ms[8];				 /* host wall time per stage: preprocess, runtime, candidates, raycast, cull, control, finalize, total */
	uint64_t ray_nodes;				 /* ray / node box tests of the ray casts (per ray) */
	uint64_t ray_edge_tests;		 /* leaf tests of the EE (edge-edge) casts, included in ray_tests */
	double gpu_ms[6];				 /* GPU time (CUDA events): ray casting, hit sort, union-find, support entries, selection + metrics, download */
	uint64_t ray_node_fetches;		 /* BVH node records brought in by the ray casts (one per warp packet visit) */
	uint64_t ray_tri_fetches;		 /* triangle leaf records brought in (one per packet leaf visit) */
	uint64_t ray_edge_fetches;		 /* edge leaf records brought in */
	uint64_t ray_visits;			 /* BVH node tests each ray alone would make (the per-ray traversal work) */
	uint64_t ray_candidate_tests;	 /* leaf tests whose primitive is a candidate target of the request's task */
	uint64_t fp64_rechecks;			 /* with fp64_recheck: leaf tests inside their FP32 error band, re-evaluated in FP64 */
	uint64_t fp64_flips;			 /* ... of which the FP64 decision differs from the FP32 one (the hit sets keep FP32) */
	uint64_t dc_tie_rechecks;		 /* selected supports whose largest and second largest depth lie within the depth's
									  * error band (the argmax that sets D_C is uncertain), re-evaluated in FP64 */
	uint64_t dc_tie_flips;			 /* ... of which the FP64 argmax is another hit */
	double fp64_delta_rel_err;		 /* max over the selected hits of |delta_32 - delta_64| / delta_64 */
	double fp64_dc_rel_err;			 /* max over processed contours of |D_C,32 - D_C,64| / D_C,64 (depth) */
	double fp64_j_rel_err;			 /* max over processed contours of |J_32 - J_64| / J_64 (objective) */
	double tune_ms[18];				 /* autotune pass: ray-casting time (ms, summed over the pass's launches) of each
									  * configuration (subtree parts, blocks per SM, grid form): (4,6) (4,7) (4,8) (8,6)
									  * (8,7) (8,8) (16,6) (16,7) (16,8) with a warp per work item, then the same nine
									  * with a persistent grid whose warps take work items from a queue */
	uint32_t raycast_parts;			 /* configuration the scene's ray casts use from now on: subtree parts per request */
	uint32_t raycast_blocks_per_sm;	 /* ... resident 128-thread blocks per SM */
	uint32_t tuned;					 /* 1 when this pass ran the autotuner (its choice holds for the scene's later passes) */
	uint32_t raycast_queue;			 /* ... and 1 for the persistent work-queue grid */
} u26_prp_output_view;

/* One PRP pass. face_tree / edge_tree: the scene's face and edge LBVHs refit at x (any
 * thickness >= 0; ray casting only needs boxes that contain the primitives). x: DEVICE
 * positions [V][3]; ef_pairs / ef_indices: DEVICE canonical EF list (u26_ef_canonicalize)
 * of num_pairs entries. Synchronises; *out owns the host-side results until
 * u26_prp_output_destroy. */
U26_API u26_status u26_prp_resolve(u26_scene* scene, u26_lbvh* face_tree, u26_lbvh* edge_tree, const float* x,
	const void* ef_pairs, const uint32_t* ef_indices, uint32_t num_pairs, const u26_prp_params* params,
	u26_prp_output** out);
U26_API u26_status u26_prp_output_view_get(const u26_prp_output* out, u26_prp_output_view* view);
U26_API void u26_prp_output_destroy(u26_prp_output* out);

/* ---- response assembly ------------------------------------------------------------
 * The selected supports of a pass as collision pair templates for the Newton system
 * (make_response_from_min_hitinfo, intersection_resolver2.cpp:2105-2221), optionally
 * appended to a narrow-phase list after its penalty pairs (upload_response_pairs_to_gpu,
 * 2223-2294), and the contour-region lists of every vertex, edge and face
 * (host_apply_untangling_constraint, 2296-2427). */
typedef struct u26_prp_response_params
{
	float depth_threshold; /* untangling_response_depth (3e-3): C = max(-depth - 3e-3, -depth_threshold) */
	float stiffness;	   /* stiffness_untangling (1e8): k1 = area stiffness C, k2 = area stiffness */
} u26_prp_response_params;

/* CollisionPair::CollisionPairTemplate (collision_data.h:48-140), 64 B. VF (and FV, which
 * enters as the VF pair of its target vertex with the normal reversed): indices v f0 f1 f2,
 * bit 31 of indices[2] set, vec2 = k1 k2 face-bary0 face-bary1. EE: indices a0 a1 b0 b1, bit 31
 * of indices[3] set, vec2 = k1 k2 edge1-t edge2-t. vec1 = normal xyz, area; vec3 = 0. */
typedef struct u26_collision_pair
{
	uint32_t indices[4];
	float vec1[4], vec2[4], vec3[4];
} u26_collision_pair;

/* DEVICE arrays owned by the scene, valid until its next u26_prp_make_response. Region CSRs
 * use upload_2d_csr_from's layout (buffer_allocator.h:26-59): one array of [n + 1] absolute
 * offsets followed by the data; region ids 2 contour + mesh role, ascending per row. */
typedef struct u26_prp_response_view
{
	uint32_t num_pairs;
	const u26_collision_pair* pairs; /* [num_pairs]: contours in order, each contour's hits in order */
	const uint32_t* pair_info;		 /* [num_pairs][4]: src id, dst id (VF / FV: vertex, face; EE: edge1, edge2),
									  * packed region 2 (256 contour + solution key) + source role, type (0 VF, 1 FV, 2 EE) */
	const uint32_t* vert_regions;	 /* [vert_regions_len] */
	const uint32_t* edge_regions;	 /* [edge_regions_len]: union of the endpoints' regions */
	const uint32_t* face_regions;	 /* [face_regions_len]: union of the corners' regions */
	uint32_t vert_regions_len, edge_regions_len, face_regions_len;
} u26_prp_response_view;

/* out: a finished u26_prp_resolve of this scene (its normals are the scene's current ones).
 * narrow_list / narrow_indices: optional DEVICE narrow-phase list ([capacity] templates,
 * [capacity][2] indices) receiving the pairs at [first, first + num_pairs); when
 * first + num_pairs > capacity nothing is written, view->num_pairs holds the count and
 * U26_ERR_CAPACITY is returned. Synchronises. */
U26_API u26_status u26_prp_make_response(u26_scene* scene, const u26_prp_output* out, const u26_prp_response_params* params,
	u26_collision_pair* narrow_list, uint32_t* narrow_indices, uint32_t first, uint32_t capacity, u26_prp_response_view* view);

/* A fixed step along an assembled response (the position update of the scale form's passes and
 * of the untangling26 repair loop, in place of the Newton solve that consumes the same pairs,
 * newton_solver.cpp:2254-2326). Each DEVICE response pair asks its sides apart along its normal
 * by Delta = -k1 / k2 (= min(depth + 3e-3, depth_threshold)): the pair's first primitive (the
 * VF template's vertex, the EE template's first edge) by +Delta / 2, the second by -Delta / 2,
 * split among its vertices by the template's barycentric weights. Every vertex that a pair
 * touches moves by scale x the weighted mean of its requests. DEVICE x [num_verts][3] is
 * updated in place; scratch: DEVICE int64[4 * num_verts], all zero before the first call (each
 * call leaves it zero again); moved (optional, DEVICE uint64) receives the count of moved
 * vertices. Deterministic: the sums are taken in fixed point. No reference counterpart. */
U26_API u26_status u26_response_step(u26_ctx* ctx, const u26_collision_pair* pairs, uint32_t num_pairs, float* x, uint32_t num_verts,
	float scale, long long* scratch, unsigned long long* moved);

/* Near-zero-distance proximity pairs as EF pairs (fn_add_ef_from_proximity_pairs,
 * intersection_resolver.cpp:199-363; run by ef_dcd_intersection_query when
 * ignore_near_zero_dist_pairs is off, 404-422). Over the proximity pairs [0, min(*narrow_count,
 * max_proximity)) of the DEVICE narrow-phase list (count read on the device), a VF or EE pair
 * with |sum_k w_k x_k|^2 < 1e-10 appends zero-stiffness EF pairs through *ef_count: VF (v, f)
 * gives (e, f) for every edge e at v; EE (e1, e2) gives (e1, g) for each face g at e2 holding
 * e2 and no vertex of e1, and (e2, g) for each face at e1 likewise. vert_adj_edges_csr /
 * edge_adj_faces_csr: DEVICE adjacency in upload_2d_csr_from's one-array layout
 * (sa_vert_adj_edges_csr, edge_adj_faces_csr). Canonicalise the EF list afterwards. */
U26_API u26_status u26_ef_add_from_proximity(u26_ctx* ctx, const u26_collision_pair* narrow_list, const uint32_t* narrow_indices,
	const uint32_t* narrow_count, uint32_t max_proximity, const float* x, const uint32_t* edges, const uint32_t* faces,
	const uint32_t* vert_adj_edges_csr, const uint32_t* edge_adj_faces_csr, uint32_t* ef_count, void* ef_pairs, uint32_t* ef_indices,
	uint32_t max_ef);

/* ---- region-based pair filtering ----------------------------------------------------
 * The contour regions of a pass (u26_prp_response_view's CSRs) applied to the solver's contact
 * pairs. Region match of two primitives (fn_is_matched_invalid_region, intersection_resolver.cpp:
 * 2232-2337): 1 when a region of the first is the opposite side (id ^ 1) of a region of the
 * second; VF pairs compare the vertex row with the face row, EE pairs the two edge rows.
 *
 * IntersectionResolver::filter_invalid_pairs (intersection_resolver.cpp:2635-2676): over the
 * proximity pairs [0, num_proximity_pairs) of the DEVICE narrow-phase list, a pair with
 * |sum_k w_k x_k|^2 < (vert_offset[i0] + vert_offset[i2])^2 + 1e-10 sets vert_is_invalid on its
 * vertices; then every pair touching an invalid vertex, or (region arrays given: the reference's
 * use_untangling with a non-empty region list) whose region match is 1, gets k1 = k2 = 0.
 * Does nothing when num_ef == 0. vert_is_invalid [num_verts] is the caller's (zeroed at EF
 * detection, intersection_resolver.cpp:384); template slots with an index >= num_verts (the ~0
 * placeholder of VV / VE pairs) are skipped. */
U26_API u26_status u26_filter_invalid_pairs(u26_ctx* ctx, u26_collision_pair* narrow_list, const uint32_t* narrow_indices,
	uint32_t num_proximity_pairs, uint32_t num_ef, const float* x, const float* vert_offset, uint32_t num_verts, uint32_t* vert_is_invalid,
	const uint32_t* vert_regions, const uint32_t* edge_regions, const uint32_t* face_regions);

/* IntersectionResolver::filter_broad_phase_pairs (intersection_resolver.cpp:2586-2633): the CCD
 * broad-phase lists (DEVICE [n][2]: VF (vid, fid), EE (eid1, eid2)) get bit 31 on both ids when
 * the pair's region match is 1 and bit 30 when one of its four vertices is invalid. Does nothing
 * when num_ef == 0 or there are no regions (vert_regions NULL). */
U26_API u26_status u26_filter_broad_phase_pairs(u26_ctx* ctx, uint32_t* vf_list, uint32_t num_vf, uint32_t* ee_list, uint32_t num_ee,
	uint32_t num_ef, const uint32_t* vert_is_invalid, const uint32_t* vert_regions, const uint32_t* edge_regions,
	const uint32_t* face_regions, const uint32_t* faces, const uint32_t* edges);

/* Differentiation over fixed supports (the torch.autograd binding of the objective; the
 * reference computes dE/dr inside its direction refinement, intersection_resolver2.cpp:
 * 1268-1320, and has no standalone entry point). For each contour c, with support
 * hits[hit_offsets[c], hit_offsets[c+1]) and direction dirs[c]: the hit distances are
 * recomputed from x and r as delta = (w . n) / (r . n); J[c] = (sum of the hits' rest source
 * areas) * max(delta)^2 and E[c] = sum (delta + 3e-3)^2 / kappa (the displacement cost). With
 * grad_J / grad_E (upstream gradients, either may be NULL) it also writes grad_dirs[c] =
 * grad_J dJ/dr + grad_E dE/dr and ADDS grad_J dJ/dx + grad_E dE/dx into grad_x (zero it
 * first). J's subgradient runs through the first maximal hit in key order. All pointers are
 * device memory: x [V][3], hits as u26_prp_resolve returns them, hit_offsets [C+1], dirs,
 * grad_dirs [C][3], the per-vertex / edge / face rest areas and vertex masses of the mesh;
 * J, E may be NULL. Runs on ctx's stream. */
U26_API u26_status u26_prp_adjoint(u26_ctx* ctx, const float* x, const u26_prp_hit* hits, const uint32_t* hit_offsets,
	uint32_t num_contours, const float* dirs, const float* vert_area, const float* edge_area, const float* face_area,
	const float* vert_mass, float* J, float* E, const float* grad_J, const float* grad_E, float* grad_dirs, float* grad_x);

#endif /* U26_H */
