// Test infrastructure (oracle): CPU restatement of the reference's PRP contour evaluation
// (host_resolve_intersections_PRP, the CPU batched path), from the canonical EF list to
// the selected per-contour responses. Loaded only by tests/ and bench.py's CPU legs.
//
// Followed, stage by stage (all in Solver/CollisionDetector/):
//   EF preprocessing      intersection_resolver.cpp:431-558, 683-1096 (ignore_near_zero_dist_pairs = true)
//   contours              intersection_resolver2.cpp:254-309, intersection_resolver_helper.cpp:518-575
//   classification        intersection_resolver2.cpp:311-375, 2811-2845
//   boundary flags        intersection_resolver2.cpp:2646-2680, hit attachment 378-412
//   normals               intersection_resolver2.cpp:2605-2644
//   runtime               intersection_resolver2.cpp:2428-2585, hop/geodesic 618-722, directions 1488-1569
//   candidates + CCR      intersection_resolver2.cpp:1571-1804, intersection_resolver2.h:405-506
//   ray casting           cached_bvh.cpp:131-555, cached_bvh.hpp:6-46 (median split, leaf 8)
//   hit adjacency         intersection_resolver_helper.cpp:771-902
//   cluster culling       intersection_resolver2.cpp:3003-3771
//   metrics / J           intersection_resolver2.cpp:1806-1954, helper.cpp:611-645
//   adaptive k-ring       intersection_resolver2.cpp:1058-1230, intersection_resolver2.h:1177-1187
//   selection             intersection_resolver2.h:807-912, intersection_resolver2.cpp:996-1057
//   merge / suppression   intersection_resolver2.cpp:413-592, finalize 1956-2103
//   response + regions    intersection_resolver2.cpp:37-121, 2105-2221, 2296-2427
//
// Deviations, all shared with the CUDA path and stated once here:
//  * The 3x3 symmetric eigen solver (the reference calls Eigen::SelfAdjointEigenSolver::
//    computeDirect, not in this checkout) is cyclic Jacobi in double with eigenvalues
//    ascending and each eigenvector's largest-magnitude component made positive.
//  * Sums over a hit list (J, volume, area, displacement cost) run over the hits in
//    canonical order (type, source id, target id) with a fixed 32-lane strided partial
//    sum and xor-butterfly combine, the reduction order of the CUDA metrics kernel.
//    The reference reduces in its own (BVH-dependent) hit order with its block reduce
//    (reference_block_sum below); its sets are what parity pins, and oracle_prp_order_spread
//    measures how far the two orders' FP32 sums lie apart on a given support.
//  * Solid-interior hit links (intersection_resolver2.cpp:3298-3464) apply only to rigid
//    or tetrahedral meshes; the scenes here are cloth, so they never fire and are not
//    restated.
#include <map>
#include <memory>
#include <mutex>
#include <queue>
#include <random>
#include <set>
#include <string>

#include "oracle_common.h"
#include "oracle_fp64.h"

namespace u26o
{
	bool line_intersection(V3 p0, V3 p1, V3 A, V3 B, V3 C, V3& out_bary, float& out_time);
}

using namespace u26o;

namespace
{
	constexpr uint kInf = 0xFFFFFFFFu;
	constexpr float kGeoInf = std::numeric_limits<float>::max();

	struct MeshIn
	{
		uint num_verts, num_edges, num_faces, num_objects;
		const float* x;
		const float* rest_x;
		const uint* edges;
		const uint* faces;
		const uint* face_adj_edges;
		const uint *vav_off, *vav;
		const uint *vae_off, *vae;
		const uint *vaf_off, *vaf;
		const uint *eaf_off, *eaf;
		const uint *eae_off, *eae;
		const uint *prefix_verts, *prefix_edges, *prefix_faces;
		const uint* vert_object;
		const uint* vert_component;
		const float *rest_vert_area, *rest_edge_area, *rest_face_area, *vert_mass;
		const uint* mesh_orientation;
		const uint* object_scene; // [objects] or null: one scene
		const uint* object_solid; // [objects] 1: rigid / tetrahedral material (sa_vert_mesh_type), or null: none
	};

	struct Params
	{
		uint max_contours;
		uint direction_mode; // 0: reference seeds, 1: 26 lattice directions
		uint use_ccr;
		float ccr_tau;
		uint ccr_use_rest;
		uint ccr_use_current;
		uint batch_size;
		uint brute_force_raycast;
		uint contour_stride; // sampling option for timing: evaluate contours c with c % stride == 0 (0 or 1: all)
		uint opt_iterations; // PRP_direction_optimization_iterations (scene_params.h:65), 0 = off
		uint ccr_blend;		 // PRP_use_blended_intrinsic_coordinates (scene_params.h:72)
		float ccr_blend_weight; // PRP_intrinsic_blend_weight (scene_params.h:73)
		uint solid_interior;	// PRP_solid_interior_adjacency (scene_params.h:77)
		uint solid_all;			// PRP_solid_interior_adjacency_all_meshes (scene_params.h:78)
		float solid_eps_n;		// PRP_solid_interior_adjacency_normal_eps (1e-4)
		float solid_eps_d;		// PRP_solid_interior_adjacency_dist_eps (1e-5)
		uint ignore_near_zero_dist_pairs; // scene_params.h:55 (1; the CLI sets 0)
		uint contour_offset; // with contour_stride: evaluate contours c with c % stride == offset % stride
		uint fp64_recheck;	 // count the FP64 rechecks of the leaf tests inside their FP32 error band
	};

	struct EfPair
	{
		uint idx[5];
		float bary[3];
		float grad[3];
		float stiff;
		bool is_loop() const { return idx[0] == idx[1]; }
	};
	static_assert(sizeof(EfPair) == 48, "EfPair");

	struct Span
	{
		const uint* p;
		uint n;
		const uint* begin() const { return p; }
		const uint* end() const { return p + n; }
		uint size() const { return n; }
	};
	inline Span row(const uint* off, const uint* data, uint i) { return Span{ data + off[i], off[i + 1] - off[i] }; }

	enum HitType : uint
	{
		VF = 0,
		EE = 1,
		FV = 2
	};

	struct Hit
	{
		uint type, src_id, dst_id;
		uint sv[3], dv[3];
		float bary[2];
		float dist;
		uint64_t key() const
		{
			return (uint64_t(type) << 62) | (uint64_t(src_id & 0x3fffffffu) << 31) | uint64_t(dst_id & 0x7fffffffu);
		}
		uint vid() const { return type == VF ? src_id : dst_id; }
		uint fid() const { return type == VF ? dst_id : src_id; }
	};

	struct ComboInfo
	{
		bool present = false;
		uint combo_idx = 0;
		V3 dir = v3(0.0f);
		float depth = 0, volume = 0, objective = 0, area = 0, cost = 0;
		uint hit_count = 0, unculled = 0;
		uint covered = 0, anchors = 0;
		float coverage = 0;
		uint max_front_src = 0, max_front_dst = 0;
		uint eval_k_src = kInf, eval_k_dst = kInf;
		uint levels = 0;
		bool eligible = false, full_mesh = false;
		uint opt_attempted = 0, opt_accepted = 0; // direction_optimization_{iteration,accepted}_count
		std::vector<Hit> hits;
	};

	inline bool finitef(float v) { return std::isfinite(v); }

	// intersection_resolver2.h:807-850
	inline bool has_usable(const ComboInfo& c)
	{
		return !c.hits.empty() && c.covered > 0 && finitef(c.objective) && finitef(c.coverage) && c.coverage > 0.0f;
	}
	inline bool has_valid(const ComboInfo& c) { return c.eligible && has_usable(c); }
	inline float objective_div_cov2(float obj, float cov)
	{
		if (!finitef(obj) || !finitef(cov) || cov <= 0.0f)
			return std::numeric_limits<float>::infinity();
		const double o = double(obj) / (double(cov) * double(cov));
		return (std::isfinite(o) && o <= double(std::numeric_limits<float>::max())) ? float(o) : std::numeric_limits<float>::infinity();
	}
	inline float response_objective(const ComboInfo& c) { return objective_div_cov2(c.objective, c.coverage); }

	// prp_response_is_better (intersection_resolver2.h:852-884)
	inline int scalar_cmp(float lhs, float rhs)
	{
		const bool lf = finitef(lhs), rf = finitef(rhs);
		if (lf != rf)
			return lf ? -1 : 1;
		if (!lf)
			return 0;
		const float tol = 1e-7f + 1e-5f * std::fmax(std::fabs(lhs), std::fabs(rhs));
		if (lhs + tol < rhs)
			return -1;
		if (rhs + tol < lhs)
			return 1;
		return 0;
	}
	inline bool response_is_better(const ComboInfo& a, const ComboInfo& b)
	{
		int c = scalar_cmp(response_objective(a), response_objective(b));
		if (c != 0)
			return c < 0;
		c = scalar_cmp(a.depth, b.depth);
		if (c != 0)
			return c < 0;
		c = scalar_cmp(a.cost, b.cost);
		if (c != 0)
			return c < 0;
		if (a.hit_count != b.hit_count)
			return a.hit_count < b.hit_count;
		return a.combo_idx < b.combo_idx;
	}

	// ---- 3x3 symmetric eigen decomposition (cyclic Jacobi, double)
	void jacobi3(const double A_in[3][3], double evals[3], double evecs[3][3])
	{
		double A[3][3], V[3][3] = { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
		for (int i = 0; i < 3; i++)
			for (int j = 0; j < 3; j++)
				A[i][j] = A_in[i][j];
		for (int sweep = 0; sweep < 64; sweep++)
		{
			const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
			const double diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
			if (off <= 1e-30 * diag || off == 0.0)
				break;
			const int P[3] = { 0, 0, 1 }, Q[3] = { 1, 2, 2 };
			for (int k = 0; k < 3; k++)
			{
				const int p = P[k], q = Q[k];
				if (A[p][q] == 0.0)
					continue;
				const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
				const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
				const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
				for (int r = 0; r < 3; r++)
				{
					const double arp = A[r][p], arq = A[r][q];
					A[r][p] = c * arp - s * arq;
					A[r][q] = s * arp + c * arq;
				}
				for (int r = 0; r < 3; r++)
				{
					const double apr = A[p][r], aqr = A[q][r];
					A[p][r] = c * apr - s * aqr;
					A[q][r] = s * apr + c * aqr;
				}
				for (int r = 0; r < 3; r++)
				{
					const double vrp = V[r][p], vrq = V[r][q];
					V[r][p] = c * vrp - s * vrq;
					V[r][q] = s * vrp + c * vrq;
				}
			}
		}
		int order[3] = { 0, 1, 2 };
		std::stable_sort(order, order + 3, [&](int a, int b)
			{ return A[a][a] < A[b][b]; });
		for (int k = 0; k < 3; k++)
		{
			const int c = order[k];
			evals[k] = A[c][c];
			int big = 0;
			for (int r = 1; r < 3; r++)
				if (std::fabs(V[r][c]) > std::fabs(V[big][c]))
					big = r;
			const double sgn = V[big][c] < 0 ? -1.0 : 1.0;
			for (int r = 0; r < 3; r++)
				evecs[r][k] = sgn * V[r][c];
		}
	}

	struct Mat3
	{
		V3 c[3]; // columns
	};
	inline Mat3 mat_zero() { return Mat3{ { v3(0.0f), v3(0.0f), v3(0.0f) } }; }
	inline Mat3 outer(V3 a, V3 b) { return Mat3{ { a * b.x, a * b.y, a * b.z } }; }
	inline Mat3 mscale(float s, const Mat3& m) { return Mat3{ { m.c[0] * s, m.c[1] * s, m.c[2] * s } }; }
	inline Mat3 madd(const Mat3& a, const Mat3& b) { return Mat3{ { a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2] } }; }

	inline bool valid_dir(V3 v) { return finitef(v.x) && finitef(v.y) && finitef(v.z) && length_sq(v) > 1e-12f; }

	// compute_all_eigenvectors (intersection_resolver_helper.cpp:679-714)
	void all_eigenvectors(const Mat3& S, V3 out[3])
	{
		const V3 def[3] = { v3(0, 1, 0), v3(1, 0, 0), v3(0, 0, 1) };
		for (int i = 0; i < 3; i++)
			out[i] = def[i];
		for (int c = 0; c < 3; c++)
			if (!finitef(S.c[c].x) || !finitef(S.c[c].y) || !finitef(S.c[c].z))
				return;
		const float trace = S.c[0].x + S.c[1].y + S.c[2].z;
		if (trace < 1e-10f)
			return;
		float frob = 0.0f;
		for (int c = 0; c < 3; c++)
			frob += dot(S.c[c], S.c[c]);
		if (frob < 1e-20f)
			return;
		double A[3][3], ev[3], V[3][3];
		for (int r = 0; r < 3; r++)
		{
			A[r][0] = S.c[0].x * (r == 0) + S.c[0].y * (r == 1) + S.c[0].z * (r == 2);
			A[r][1] = S.c[1].x * (r == 0) + S.c[1].y * (r == 1) + S.c[1].z * (r == 2);
			A[r][2] = S.c[2].x * (r == 0) + S.c[2].y * (r == 1) + S.c[2].z * (r == 2);
		}
		jacobi3(A, ev, V);
		for (int k = 0; k < 3; k++)
		{
			const V3 v = v3(float(V[0][k]), float(V[1][k]), float(V[2][k]));
			out[k] = length_sq(v) > 1e-12f ? normalize(v) : def[k];
		}
	}

	// ---- CachedBVH restatement (cached_bvh.hpp / cached_bvh.cpp)
	struct BvhNode
	{
		V3 bmin, bmax;
		int left = -1, right = -1, start = -1, count = 0;
	};
	struct CachedBVH
	{
		std::vector<BvhNode> nodes;
		std::vector<uint> order;
		bool faces = true;

		template <typename Bounds>
		int build_node(int start, int end, std::vector<V3>& centroids, Bounds& bounds)
		{
			BvhNode node;
			bounds(start, end, node.bmin, node.bmax);
			const int idx = int(nodes.size());
			nodes.push_back(node);
			const int count = end - start;
			if (count <= 8)
			{
				nodes[idx].start = start;
				nodes[idx].count = count;
				return idx;
			}
			const V3 ext = node.bmax - node.bmin;
			int axis = 0;
			if (ext.y > ext.x && ext.y >= ext.z)
				axis = 1;
			else if (ext.z > ext.x && ext.z > ext.y)
				axis = 2;
			const int mid = (start + end) / 2;
			std::nth_element(order.begin() + start, order.begin() + mid, order.begin() + end, [&](uint a, uint b)
				{
					if (axis == 0) return centroids[a].x < centroids[b].x;
					if (axis == 1) return centroids[a].y < centroids[b].y;
					return centroids[a].z < centroids[b].z; });
			const int l = build_node(start, mid, centroids, bounds);
			const int r = build_node(mid, end, centroids, bounds);
			nodes[idx].left = l;
			nodes[idx].right = r;
			return idx;
		}

		void build(const std::vector<uint>& ids, const MeshIn& m, bool is_faces)
		{
			faces = is_faces;
			order = ids;
			nodes.clear();
			if (order.empty())
				return;
			uint mx = 0;
			for (uint id : order)
				mx = std::max(mx, id);
			std::vector<V3> centroids(mx + 1);
			for (uint id : order)
			{
				if (faces)
				{
					const V3 a = load3(m.x, m.faces[3 * id]), b = load3(m.x, m.faces[3 * id + 1]), c = load3(m.x, m.faces[3 * id + 2]);
					centroids[id] = ((a + b) + c) / 3.0f;
				}
				else
				{
					const V3 a = load3(m.x, m.edges[2 * id]), b = load3(m.x, m.edges[2 * id + 1]);
					centroids[id] = (a + b) * 0.5f;
				}
			}
			auto bounds = [&](int s, int e, V3& mn, V3& mxv)
			{
				bool first = true;
				for (int i = s; i < e; i++)
				{
					const uint id = order[i];
					V3 lo, hi;
					if (faces)
					{
						const V3 a = load3(m.x, m.faces[3 * id]), b = load3(m.x, m.faces[3 * id + 1]), c = load3(m.x, m.faces[3 * id + 2]);
						lo = vmin(a, vmin(b, c));
						hi = vmax(a, vmax(b, c));
					}
					else
					{
						const V3 a = load3(m.x, m.edges[2 * id]), b = load3(m.x, m.edges[2 * id + 1]);
						lo = vmin(a, b);
						hi = vmax(a, b);
					}
					if (first)
					{
						mn = lo;
						mxv = hi;
						first = false;
					}
					else
					{
						mn = vmin(mn, lo);
						mxv = vmax(mxv, hi);
					}
				}
			};
			build_node(0, int(order.size()), centroids, bounds);
		}
	};

	struct VertRequest
	{
		uint vid;
		V3 dir;
		bool fv;
		uint target_lo, target_cnt; // dense span
		const std::vector<uint>* targets;
		const std::vector<uint>* hop;
		uint max_hop;
	};
	struct EdgeRequest
	{
		uint eid;
		V3 dir;
		float max_dist;
		float target_proj_min;
		uint target_lo, target_cnt;
		const std::vector<uint>* targets;
		const std::vector<uint>* hop;
		uint max_hop;
	};

	inline bool in_span(uint id, uint lo, uint cnt)
	{
		if (cnt == 0)
			return false;
		if (cnt != kInf && (id < lo || id >= lo + cnt))
			return false;
		return true;
	}

	// VF (ray from vertex along dir) / FV (ray from vertex along -dir) primitive test
	// (cached_bvh.cpp:258-289).
	inline bool vert_face_test(const MeshIn& m, uint vid, V3 orig, V3 end, uint fid, Hit& h, bool fv, float ray_max)
	{
		const uint f0 = m.faces[3 * fid], f1 = m.faces[3 * fid + 1], f2 = m.faces[3 * fid + 2];
		if (vid == f0 || vid == f1 || vid == f2)
			return false;
		V3 bary;
		float t;
		if (!line_intersection(orig, end, load3(m.x, f0), load3(m.x, f1), load3(m.x, f2), bary, t) || !(t >= 0.0f && t <= 1.0f))
			return false;
		h.type = fv ? FV : VF;
		h.src_id = fv ? fid : vid;
		h.dst_id = fv ? vid : fid;
		if (fv)
		{
			h.sv[0] = f0; h.sv[1] = f1; h.sv[2] = f2;
			h.dv[0] = vid; h.dv[1] = kInf; h.dv[2] = kInf;
		}
		else
		{
			h.sv[0] = vid; h.sv[1] = kInf; h.sv[2] = kInf;
			h.dv[0] = f0; h.dv[1] = f1; h.dv[2] = f2;
		}
		h.bary[0] = bary.x;
		h.bary[1] = bary.y;
		h.dist = t * ray_max;
		return true;
	}

	// EE swept-edge test (cached_bvh.cpp:377-473, primitive part).
	struct EdgeRay
	{
		V3 p0, p1, e1, dir;
		bool plane;
		V3 pn;
		float pd;
		float max_dist;
	};
	inline EdgeRay make_edge_ray(const MeshIn& m, uint eid, V3 dir, float max_dist)
	{
		EdgeRay r;
		r.p0 = load3(m.x, m.edges[2 * eid]);
		r.p1 = load3(m.x, m.edges[2 * eid + 1]);
		r.e1 = r.p1 - r.p0;
		r.dir = dir;
		r.max_dist = max_dist;
		r.pn = cross(r.e1, dir);
		const float nl = length(r.pn);
		r.plane = nl >= 1e-10f;
		r.pd = 0.0f;
		if (r.plane)
		{
			r.pn = r.pn / nl;
			r.pd = dot(r.pn, r.p0);
		}
		return r;
	}
	inline bool edge_edge_test(const MeshIn& m, const EdgeRay& r, uint eid1, uint eid2, Hit& h)
	{
		const uint a0 = m.edges[2 * eid1], a1 = m.edges[2 * eid1 + 1];
		const uint b0 = m.edges[2 * eid2], b1 = m.edges[2 * eid2 + 1];
		if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1)
			return false;
		const V3 q0 = load3(m.x, b0), q1 = load3(m.x, b1);
		if (r.plane)
		{
			const float d0 = dot(r.pn, q0) - r.pd;
			const float d1 = dot(r.pn, q1) - r.pd;
			if ((d0 > 1e-6f && d1 > 1e-6f) || (d0 < -1e-6f && d1 < -1e-6f))
				return false;
		}
		const V3 e2 = q1 - q0;
		const V3 rr = q0 - r.p0;
		const V3 n = cross(r.e1, e2);
		const float det = -dot(r.dir, n);
		if (std::fabs(det) < 1e-10f)
			return false;
		const float inv = 1.0f / det;
		const float d_r_e1_e2 = dot(rr, cross(r.e1, e2));
		const float d_dir_r_e2 = dot(r.dir, cross(rr, e2));
		const float d_dir_e1_r = dot(r.dir, cross(r.e1, rr));
		const float s = -d_r_e1_e2 * inv;
		const float t1 = -d_dir_r_e2 * inv;
		const float t2 = d_dir_e1_r * inv;
		if (!(s >= 0.0f && s <= r.max_dist && t1 >= 0.0f && t1 <= 1.0f && t2 >= 0.0f && t2 <= 1.0f))
			return false;
		h.type = EE;
		h.src_id = eid1;
		h.dst_id = eid2;
		h.sv[0] = a0; h.sv[1] = a1; h.sv[2] = kInf;
		h.dv[0] = b0; h.dv[1] = b1; h.dv[2] = kInf;
		h.bary[0] = 1.0f - t1;
		h.bary[1] = 1.0f - t2;
		h.dist = s;
		return true;
	}

	inline bool hop_ok(const std::vector<uint>* hop, uint max_hop, std::initializer_list<uint> vs)
	{
		if (hop == nullptr || max_hop == kInf)
			return true;
		for (uint v : vs)
			if ((*hop)[v] > max_hop)
				return false;
		return true;
	}

	// FP64 recheck counts of the ray casts: leaf tests rechecked, FP32 / FP64 flips. Counted
	// over the leaf tests the CUDA path's batched form makes: those whose primitive box, grown
	// by its conservative margin 1e-5 (1 + |coordinate|) per axis, the ray (swept edge) meets.
	struct Recheck
	{
		uint64_t n = 0, flips = 0;
		void add(uint rc)
		{
			n += rc & 1u;
			flips += rc >> 1;
		}
	};

	// the ray [0, 1] of orig + t cast against the face's grown box (the slab test with one
	// fused multiply-add per plane, as the batched ray casts evaluate it)
	inline bool face_gate(V3 orig, V3 cast, V3 A, V3 B, V3 C)
	{
		const V3 mn = vmin(vmin(A, vmin(B, C)), vmin(A, vmin(B, C))), mx = vmax(vmax(A, vmax(B, C)), vmax(A, vmax(B, C)));
		const float lo[3] = { mn.x, mn.y, mn.z }, hi[3] = { mx.x, mx.y, mx.z };
		const float o[3] = { orig.x, orig.y, orig.z }, d[3] = { cast.x, cast.y, cast.z };
		float tmin = 0.0f, tmax = 1.0f;
		float a[3], b[3];
		for (int k = 0; k < 3; k++)
		{
			const float e = 1e-5f * (1.0f + std::fmax(std::fabs(lo[k]), std::fabs(hi[k])));
			const float inv = std::fabs(d[k]) < 1e-30f ? std::copysign(1e30f, d[k]) : 1.0f / d[k];
			const float oinv = o[k] * inv;
			a[k] = std::fma(lo[k] - e, inv, -oinv);
			b[k] = std::fma(hi[k] + e, inv, -oinv);
		}
		tmin = std::fmax(std::fmax(tmin, std::fmin(a[0], b[0])), std::fmax(std::fmin(a[1], b[1]), std::fmin(a[2], b[2])));
		tmax = std::fmin(std::fmin(tmax, std::fmax(a[0], b[0])), std::fmin(std::fmax(a[1], b[1]), std::fmax(a[2], b[2])));
		return tmin <= tmax;
	}
	// the batched form's leaf test of a target edge against a swept edge: the edge's grown box
	// (one margin for all axes) against the swept box, the swept edge's extent along dir
	// [proj_lo, proj_hi] and, with a plane, the slab |dot(pn, q) - pd| <= 1e-6
	inline bool edge_gate(V3 smin, V3 smax, float proj_lo, float proj_hi, V3 dir, bool plane, V3 pn, float pd, V3 q0, V3 q1)
	{
		const V3 mn = vmin(q0, q1), mx = vmax(q0, q1);
		const float e = 1e-5f * (1.0f + std::fmax(std::fmax(std::fmax(std::fabs(mn.x), std::fabs(mx.x)), std::fmax(std::fabs(mn.y), std::fabs(mx.y))),
			std::fmax(std::fabs(mn.z), std::fabs(mx.z))));
		const V3 gl = v3(mn.x - e, mn.y - e, mn.z - e), gh = v3(mx.x + e, mx.y + e, mx.z + e);
		if (!(smin.x <= gh.x && smax.x >= gl.x && smin.y <= gh.y && smax.y >= gl.y && smin.z <= gh.z && smax.z >= gl.z))
			return false;
		const V3 c = v3(0.5f * (gl.x + gh.x), 0.5f * (gl.y + gh.y), 0.5f * (gl.z + gh.z));
		const V3 h = v3(0.5f * (gh.x - gl.x), 0.5f * (gh.y - gl.y), 0.5f * (gh.z - gl.z));
		const float cp = dot(c, dir);
		const float pr = (h.x * std::fabs(dir.x) + h.y * std::fabs(dir.y)) + h.z * std::fabs(dir.z);
		if (cp + pr < proj_lo || cp - pr > proj_hi)
			return false;
		if (!plane)
			return true;
		const float rad = (h.x * std::fabs(pn.x) + h.y * std::fabs(pn.y)) + h.z * std::fabs(pn.z);
		return std::fabs(dot(pn, c) - pd) <= rad + 1e-6f;
	}

	// ray_cast_from_verts_batched for one request (BVH or brute force over the targets)
	void cast_vert(const MeshIn& m, const CachedBVH* bvh, const VertRequest& q, std::vector<Hit>& out, uint64_t& tested, Recheck* rc)
	{
		const float ray_max = 1.0f;
		if (q.target_cnt == 0)
			return;
		const V3 cast = q.fv ? -q.dir : q.dir;
		const V3 orig = load3(m.x, q.vid);
		const V3 end = orig + cast * ray_max;
		auto leaf = [&](uint fid)
		{
			tested++;
			if (!in_span(fid, q.target_lo, q.target_cnt))
				return;
			if (q.targets && !std::binary_search(q.targets->begin(), q.targets->end(), fid))
				return;
			if (!hop_ok(q.hop, q.max_hop, { m.faces[3 * fid], m.faces[3 * fid + 1], m.faces[3 * fid + 2] }))
				return;
			Hit h;
			if (vert_face_test(m, q.vid, orig, end, fid, h, q.fv, ray_max))
				out.push_back(h);
		};
		// the FP64 recheck count: the candidate faces (not incident to the ray's vertex) whose
		// grown box the ray meets, found by a second walk over node boxes grown by twice that
		// margin (so that rounding in the node test never drops one)
		auto count_leaf = [&](uint fid)
		{
			if (!in_span(fid, q.target_lo, q.target_cnt) || (q.targets && !std::binary_search(q.targets->begin(), q.targets->end(), fid)))
				return;
			const uint f0 = m.faces[3 * fid], f1 = m.faces[3 * fid + 1], f2 = m.faces[3 * fid + 2];
			if (!hop_ok(q.hop, q.max_hop, { f0, f1, f2 }) || q.vid == f0 || q.vid == f1 || q.vid == f2)
				return;
			const V3 A = load3(m.x, f0), B = load3(m.x, f1), C = load3(m.x, f2);
			if (!face_gate(orig, cast, A, B, C))
				return;
			Hit h;
			rc->add(recheck_vert_face(orig, end, A, B, C, vert_face_test(m, q.vid, orig, end, fid, h, q.fv, ray_max)));
		};
		if (bvh == nullptr)
		{
			for (uint fid : *q.targets)
			{
				leaf(fid);
				if (rc)
					count_leaf(fid);
			}
			return;
		}
		if (bvh->nodes.empty())
			return;
		if (rc)
		{
			auto grown = [&](const BvhNode& n)
			{
				const float lo[3] = { n.bmin.x, n.bmin.y, n.bmin.z }, hi[3] = { n.bmax.x, n.bmax.y, n.bmax.z };
				const float o[3] = { orig.x, orig.y, orig.z }, d[3] = { cast.x, cast.y, cast.z };
				float tmin = 0.0f, tmax = ray_max;
				for (int k = 0; k < 3; k++)
				{
					const float e = 2e-5f * (1.0f + std::fmax(std::fabs(lo[k]), std::fabs(hi[k])));
					const float l = lo[k] - e, hh = hi[k] + e;
					if (std::fabs(d[k]) < 1e-30f)
					{
						if (o[k] < l || o[k] > hh)
							return false;
						continue;
					}
					float t0 = (l - o[k]) / d[k], t1 = (hh - o[k]) / d[k];
					if (t0 > t1)
						std::swap(t0, t1);
					tmin = std::fmax(tmin, t0);
					tmax = std::fmin(tmax, t1);
				}
				return tmin <= tmax;
			};
			std::vector<int> st2{ 0 };
			while (!st2.empty())
			{
				const int nid = st2.back();
				st2.pop_back();
				const BvhNode& n = bvh->nodes[nid];
				if (!grown(n))
					continue;
				if (n.left == -1 && n.right == -1)
					for (int i = n.start; i < n.start + n.count; i++)
						count_leaf(bvh->order[i]);
				else
				{
					if (n.left != -1)
						st2.push_back(n.left);
					if (n.right != -1)
						st2.push_back(n.right);
				}
			}
		}
		const V3 inv = v3(1.0f / cast.x, 1.0f / cast.y, 1.0f / cast.z);
		auto slab = [&](const BvhNode& n)
		{
			float t1 = (n.bmin.x - orig.x) * inv.x, t2 = (n.bmax.x - orig.x) * inv.x;
			float tmin = std::fmin(t1, t2), tmax = std::fmax(t1, t2);
			t1 = (n.bmin.y - orig.y) * inv.y;
			t2 = (n.bmax.y - orig.y) * inv.y;
			tmin = std::fmax(tmin, std::fmin(t1, t2));
			tmax = std::fmin(tmax, std::fmax(t1, t2));
			t1 = (n.bmin.z - orig.z) * inv.z;
			t2 = (n.bmax.z - orig.z) * inv.z;
			tmin = std::fmax(tmin, std::fmin(t1, t2));
			tmax = std::fmin(tmax, std::fmax(t1, t2));
			return tmax >= std::fmax(tmin, 0.0f) && tmin <= ray_max;
		};
		std::vector<int> stack{ 0 };
		while (!stack.empty())
		{
			const int nid = stack.back();
			stack.pop_back();
			const BvhNode& n = bvh->nodes[nid];
			if (!slab(n))
				continue;
			if (n.left == -1 && n.right == -1)
			{
				for (int i = n.start; i < n.start + n.count; i++)
					leaf(bvh->order[i]);
			}
			else
			{
				if (n.left != -1)
					stack.push_back(n.left);
				if (n.right != -1)
					stack.push_back(n.right);
			}
		}
	}

	void cast_edge(const MeshIn& m, const CachedBVH* bvh, const EdgeRequest& q, std::vector<Hit>& out, uint64_t& tested, Recheck* rc)
	{
		const float ray_max = std::fmin(std::fmax(q.max_dist, 0.0f), 1.0f);
		if (ray_max <= 0.0f || q.target_cnt == 0)
			return;
		const EdgeRay r = make_edge_ray(m, q.eid, q.dir, ray_max);
		const V3 sw_lo = vmin(vmin(r.p0, r.p1), vmin(r.p0 + q.dir * ray_max, r.p1 + q.dir * ray_max));
		const V3 sw_hi = vmax(vmax(r.p0, r.p1), vmax(r.p0 + q.dir * ray_max, r.p1 + q.dir * ray_max));
		const float g_ep0 = dot(r.p0, q.dir), g_ep1 = dot(r.p1, q.dir);
		const float g_lo = std::fmax(std::fmin(g_ep0, g_ep1), q.target_proj_min - 1e-5f) - 1e-6f;
		const float g_hi = (std::fmax(g_ep0, g_ep1) + ray_max * dot(q.dir, q.dir)) + 1e-6f;
		auto leaf = [&](uint eid2)
		{
			tested++;
			if (!in_span(eid2, q.target_lo, q.target_cnt))
				return;
			if (q.targets && !std::binary_search(q.targets->begin(), q.targets->end(), eid2))
				return;
			if (!hop_ok(q.hop, q.max_hop, { m.edges[2 * eid2], m.edges[2 * eid2 + 1] }))
				return;
			Hit h;
			if (edge_edge_test(m, r, q.eid, eid2, h))
				out.push_back(h);
		};
		// the FP64 recheck count: the candidate edges (sharing no vertex with the swept edge)
		// whose grown box the swept edge's box meets, found by a second walk over node boxes
		// grown by twice that margin
		auto count_leaf = [&](uint eid2)
		{
			if (!in_span(eid2, q.target_lo, q.target_cnt) || (q.targets && !std::binary_search(q.targets->begin(), q.targets->end(), eid2)))
				return;
			const uint a0 = m.edges[2 * q.eid], a1 = m.edges[2 * q.eid + 1], b0 = m.edges[2 * eid2], b1 = m.edges[2 * eid2 + 1];
			if (!hop_ok(q.hop, q.max_hop, { b0, b1 }) || a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1)
				return;
			const V3 q0 = load3(m.x, b0), q1 = load3(m.x, b1);
			if (!edge_gate(sw_lo, sw_hi, g_lo, g_hi, q.dir, r.plane, r.pn, r.pd, q0, q1))
				return;
			Hit h;
			rc->add(recheck_edge_edge(r.p0, r.p1, q.dir, ray_max, r.plane, r.pn, r.pd, q0, q1, edge_edge_test(m, r, q.eid, eid2, h)));
		};
		if (rc && bvh != nullptr && !bvh->nodes.empty())
		{
			std::vector<int> st2{ 0 };
			while (!st2.empty())
			{
				const int nid = st2.back();
				st2.pop_back();
				const BvhNode& n = bvh->nodes[nid];
				const float e = 2e-5f * (1.0f + std::fmax(std::fmax(std::fmax(std::fabs(n.bmin.x), std::fabs(n.bmax.x)),
														std::fmax(std::fabs(n.bmin.y), std::fabs(n.bmax.y))),
												  std::fmax(std::fabs(n.bmin.z), std::fabs(n.bmax.z))));
				if (!(sw_lo.x <= n.bmax.x + e && sw_hi.x >= n.bmin.x - e && sw_lo.y <= n.bmax.y + e && sw_hi.y >= n.bmin.y - e &&
						sw_lo.z <= n.bmax.z + e && sw_hi.z >= n.bmin.z - e))
					continue;
				if (n.left == -1 && n.right == -1)
					for (int i = n.start; i < n.start + n.count; i++)
						count_leaf(bvh->order[i]);
				else
				{
					if (n.left != -1)
						st2.push_back(n.left);
					if (n.right != -1)
						st2.push_back(n.right);
				}
			}
		}
		if (bvh == nullptr)
		{
			for (uint e : *q.targets)
			{
				leaf(e);
				if (rc)
					count_leaf(e);
			}
			return;
		}
		if (bvh->nodes.empty())
			return;
		const V3 a_end = r.p0 + q.dir * ray_max, b_end = r.p1 + q.dir * ray_max;
		const V3 smin = vmin(vmin(r.p0, r.p1), vmin(a_end, b_end));
		const V3 smax = vmax(vmax(r.p0, r.p1), vmax(a_end, b_end));
		const float ep0 = dot(r.p0, q.dir), ep1 = dot(r.p1, q.dir);
		const float dl2 = dot(q.dir, q.dir);
		const float proj_min = std::fmax(std::fmin(ep0, ep1), q.target_proj_min - 1e-5f);
		const float proj_max = std::fmax(ep0, ep1) + ray_max * dl2;
		auto node_ok = [&](const BvhNode& n)
		{
			if (!((smin.x <= n.bmax.x && smax.x >= n.bmin.x) && (smin.y <= n.bmax.y && smax.y >= n.bmin.y) && (smin.z <= n.bmax.z && smax.z >= n.bmin.z)))
				return false;
			const V3 c = (n.bmin + n.bmax) * 0.5f;
			const V3 e = (n.bmax - n.bmin) * 0.5f;
			const float cp = dot(c, q.dir);
			const float pr = (e.x * std::fabs(q.dir.x) + e.y * std::fabs(q.dir.y)) + e.z * std::fabs(q.dir.z);
			if (cp + pr < proj_min - 1e-6f || cp - pr > proj_max + 1e-6f)
				return false;
			if (!r.plane)
				return true;
			const float cd = dot(r.pn, c) - r.pd;
			const float rad = (e.x * std::fabs(r.pn.x) + e.y * std::fabs(r.pn.y)) + e.z * std::fabs(r.pn.z);
			return std::fabs(cd) <= rad + 1e-6f;
		};
		std::vector<int> stack{ 0 };
		while (!stack.empty())
		{
			const int nid = stack.back();
			stack.pop_back();
			const BvhNode& n = bvh->nodes[nid];
			if (!node_ok(n))
				continue;
			if (n.left == -1 && n.right == -1)
			{
				for (int i = n.start; i < n.start + n.count; i++)
					leaf(bvh->order[i]);
			}
			else
			{
				if (n.left != -1)
					stack.push_back(n.left);
				if (n.right != -1)
					stack.push_back(n.right);
			}
		}
	}

	// ---- the evaluation state of one contour (PrpStandardContourRuntime)
	struct Runtime
	{
		uint contour_idx = 0;
		bool inited = false; // runtime identity built (its batch has started)
		std::vector<uint> contour;
		uint object_ids[2] = { 0, 0 };
		uint comp_ids[2] = { kInf, kInf };
		std::vector<uint> boundary[2];
		std::vector<uint> hop[2];
		std::vector<float> geo[2];
		uint diam[2] = { 0, 0 };
		std::vector<V3> dirs;
		std::vector<ComboInfo> results;
		std::vector<uint8_t> converged, pruned, present;
		std::vector<uint8_t> active; // active_combos as a mask (all directions, or the one under refinement)
		uint init_k[2] = { 0, 0 }, k[2] = { 0, 0 };
		bool finished = false, no_response = false;
		std::vector<uint> cand_v[2], cand_e[2], cand_f[2];
		std::map<uint, float> cur_dist[2];
	};

	struct Scene
	{
		MeshIn m;
		Params p;
		// EF data (augmented with loop-vertex pairs)
		std::vector<EfPair> ef;
		std::vector<uint> ef_e, ef_f;
		uint num_orig_pairs = 0;
		std::vector<std::vector<uint>> adj;
		std::vector<V3> pos3;
		std::vector<float> length;
		std::vector<std::vector<uint>> contours;
		std::vector<uint> mesh_index, contour_index;
		std::vector<uint> contour_type;
		std::vector<std::vector<uint>> vflags;
		std::vector<V3> fn, en, vn;
		std::vector<Runtime> rt;
		std::vector<ComboInfo> selected;
		std::vector<uint8_t> processed, suppressed;
		std::vector<float> pre_area;
		std::vector<std::vector<uint>> merge_adj;
		uint64_t tested = 0, requests = 0, pairs = 0, rechecks = 0, flips = 0;
		// per-object BVHs (faces, edges)
		std::vector<std::unique_ptr<CachedBVH>> face_bvh, edge_bvh;
		std::mutex mtx;
	};

	inline uint edge_of(const MeshIn& m, uint eid, int k) { return m.edges[2 * eid + k]; }
	inline uint face_of(const MeshIn& m, uint fid, int k) { return m.faces[3 * fid + k]; }
	inline bool contains(Span s, uint v) { return std::find(s.begin(), s.end(), v) != s.end(); }

	// ---- EF preprocessing (intersection_resolver.cpp:431-558, 683-1096)
	void preprocess(Scene& S)
	{
		const MeshIn& m = S.m;
		uint n = uint(S.ef.size());
		S.num_orig_pairs = n;
		auto build_adj = [&](uint count)
		{
			std::vector<std::vector<uint>> edge_pairs(m.num_edges), face_pairs(m.num_faces), adj(count);
			for (uint p = 0; p < count; p++)
				edge_pairs[S.ef_e[p]].push_back(p);
			for (uint f = 0; f < m.num_faces; f++)
				for (int j = 0; j < 3; j++)
				{
					const auto& ep = edge_pairs[m.face_adj_edges[3 * f + j]];
					face_pairs[f].insert(face_pairs[f].end(), ep.begin(), ep.end());
				}
			for (uint p = 0; p < count; p++)
			{
				const uint eid = S.ef_e[p], fid = S.ef_f[p];
				auto& out = adj[p];
				for (uint ae : row(m.eae_off, m.eae, eid))
					for (uint q : edge_pairs[ae])
						if (S.ef_f[q] == fid && q != p)
							out.push_back(q);
				const Span af = row(m.eaf_off, m.eaf, eid);
				for (uint q : face_pairs[fid])
					if (q != p)
						for (uint a : af)
							if (S.ef_f[q] == a && S.ef_e[q] != eid && q != p)
								out.push_back(q);
			}
			return adj;
		};
		S.adj = build_adj(n);
		// degenerate filter (intersection_resolver.cpp:841-896): with near-zero-distance pairs in
		// play, a pair with a barycentric coordinate below 1e-4 stays only when one of its
		// adjacent pairs is not degenerate; if that would remove every pair, all stay
		if (!S.p.ignore_near_zero_dist_pairs && n > 0)
		{
			auto degenerate = [](const EfPair& e)
			{
				const float eb0 = e.bary[0], eb1 = 1.0f - e.bary[0];
				const float f0 = e.bary[1], f1 = e.bary[2], f2 = 1.0f - e.bary[1] - e.bary[2];
				return std::min(eb0, eb1) < 1e-4f || std::min(std::min(f0, f1), f2) < 1e-4f;
			};
			std::vector<uint8_t> deg(n);
			uint ndeg = 0;
			for (uint p = 0; p < n; p++)
				ndeg += (deg[p] = degenerate(S.ef[p]) ? 1 : 0);
			if (ndeg)
			{
				std::vector<uint> keep;
				for (uint p = 0; p < n; p++)
				{
					bool k = !deg[p];
					for (uint q : S.adj[p])
						k = k || !deg[q];
					if (k)
						keep.push_back(p);
				}
				if (!keep.empty() && keep.size() < n)
				{
					std::vector<EfPair> ef;
					std::vector<uint> ee, ff;
					for (uint p : keep)
					{
						ef.push_back(S.ef[p]);
						ee.push_back(S.ef_e[p]);
						ff.push_back(S.ef_f[p]);
					}
					S.ef = std::move(ef);
					S.ef_e = std::move(ee);
					S.ef_f = std::move(ff);
					n = uint(keep.size());
					S.num_orig_pairs = n;
					S.adj = build_adj(n);
				}
			}
		}
		// loop vertices (find_loop_vertex, non-GIA path)
		std::vector<uint> loop_vid, loop_pair, loop_e, loop_f;
		for (uint p = 0; p < n; p++)
		{
			const uint eid = S.ef_e[p], fid = S.ef_f[p];
			const uint ex = edge_of(m, eid, 0), ey = edge_of(m, eid, 1);
			for (uint af : row(m.eaf_off, m.eaf, eid))
			{
				const uint av = face_of(m, af, 0) + face_of(m, af, 1) + face_of(m, af, 2) - ex - ey;
				if (av == face_of(m, fid, 0) || av == face_of(m, fid, 1) || av == face_of(m, fid, 2))
				{
					const uint* fa = m.face_adj_edges + 3 * af;
					auto has = [&](uint e, uint v)
					{ return edge_of(m, e, 0) == v || edge_of(m, e, 1) == v; };
					uint le;
					if (eid == fa[0])
						le = has(fa[1], av) ? fa[1] : fa[2];
					else if (eid == fa[1])
						le = has(fa[0], av) ? fa[0] : fa[2];
					else
						le = has(fa[0], av) ? fa[0] : fa[1];
					loop_vid.push_back(av);
					loop_pair.push_back(p);
					loop_e.push_back(le);
					loop_f.push_back(fid);
				}
			}
		}
		for (size_t l = 0; l < loop_vid.size(); l++)
		{
			const uint v = loop_vid[l];
			EfPair lp{};
			lp.idx[0] = lp.idx[1] = lp.idx[2] = lp.idx[3] = lp.idx[4] = v;
			lp.bary[0] = 1.0f;
			lp.bary[1] = 1.0f;
			lp.bary[2] = 0.0f;
			const uint np = uint(S.ef.size());
			S.ef.push_back(lp);
			S.ef_e.push_back(loop_e[l]);
			S.ef_f.push_back(loop_f[l]);
			S.adj.push_back({ loop_pair[l] });
			S.adj[loop_pair[l]].push_back(np);
		}
		const uint na = uint(S.ef.size());
		S.pos3.resize(na);
		S.length.resize(na);
		for (uint p = 0; p < na; p++)
		{
			const EfPair& e = S.ef[p];
			const float b0 = e.bary[0], b1 = 1.0f - e.bary[0];
			S.pos3[p] = load3(m.x, e.idx[0]) * b0 + load3(m.x, e.idx[1]) * b1;
		}
		for (uint p = 0; p < na; p++)
		{
			float sum = 0.0f;
			for (uint q : S.adj[p])
				sum += length(S.pos3[q] - S.pos3[p]);
			S.length[p] = 0.5f * sum;
		}
	}

	// ---- contours + classification
	// classify_contour_type (intersection_resolver2.cpp:311-375) over one contour's pairs in
	// flood-fill order: loop-vertex pairs, boundary-edge pairs, EF-adjacency degree, mesh side.
	// ContourType (intersection_resolver2.h:27-37): 0 Undefined, 1 Closed, 2 Eight, 3 LL,
	// 4 BLI, 5 Cross, 6 BIBI (boundary pairs on both sides), 7 BBII (both on one side)
	uint classify_contour(uint n, const uint8_t* is_loop, const uint8_t* is_bnd, const uint* adj_deg, const uint* mesh_index)
	{
		std::vector<uint> bnd, loops;
		bool closed = true;
		for (uint i = 0; i < n; i++)
		{
			if (is_loop[i])
				loops.push_back(i);
			if (is_bnd[i])
			{
				bnd.push_back(i);
				closed = false;
			}
			if (!is_loop[i] && adj_deg[i] == 1)
				closed = false;
		}
		uint t = 0;
		if (bnd.empty())
		{
			if (loops.empty() && closed)
				t = 1;
			else if (loops.size() == 1 && closed)
				t = 2;
			else if (loops.size() == 2 && closed)
				t = 3;
		}
		else if (loops.empty())
		{
			if (bnd.size() == 2)
				t = mesh_index[bnd.front()] == mesh_index[bnd.back()] ? 7 : 6;
		}
		else if (loops.size() == 1)
		{
			if (bnd.size() == 1)
				t = 4;
			else if (bnd.size() == 2)
				t = 5;
		}
		return t;
	}

	// Connected components of an undirected graph with a 0/1 flip weight per adjacency entry,
	// and a parity per node (the contour flood fill and mesh parity of
	// intersection_contour_construction_from_ext_adjacent): seeds in increasing node order, each
	// component filled depth first from its seed (parity 0); a node's parity is the sum of the
	// weights along its discovery path, mod 2. Components list their nodes in discovery order.
	// Returns whether some edge joins two nodes of a component whose parities differ by other
	// than its weight (an odd cycle of flips: that component's parities depend on the walk).
	bool flood_components(uint n, const std::vector<std::vector<uint>>& adj, const std::vector<std::vector<uint>>& w,
		std::vector<uint>& parity, std::vector<std::vector<uint>>& comps)
	{
		std::vector<uint8_t> visited(n, 0);
		parity.assign(n, kInf);
		for (uint seed = 0; seed < n; seed++)
		{
			if (visited[seed])
				continue;
			std::vector<std::pair<uint, uint>> group{ { seed, 0 } }, todo{ { seed, 0 } };
			visited[seed] = 1;
			while (!todo.empty())
			{
				const auto [pi, ps] = todo.back();
				todo.pop_back();
				for (size_t j = 0; j < adj[pi].size(); j++)
				{
					const uint q = adj[pi][j];
					if (!visited[q])
					{
						visited[q] = 1;
						todo.push_back({ q, ps + w[pi][j] });
						group.push_back({ q, ps + w[pi][j] });
					}
				}
			}
			std::vector<uint> c;
			for (auto& [pi, ps] : group)
			{
				c.push_back(pi);
				parity[pi] = ps % 2;
			}
			comps.push_back(c);
		}
		bool inconsistent = false;
		for (uint p = 0; p < n && !inconsistent; p++)
			for (size_t j = 0; j < adj[p].size(); j++)
				if ((parity[p] ^ parity[adj[p][j]]) != (w[p][j] & 1u))
				{
					inconsistent = true;
					break;
				}
		return inconsistent;
	}

	void contours(Scene& S)
	{
		const uint n = uint(S.ef.size());
		std::vector<std::vector<uint>> w(n);
		for (uint p = 0; p < n; p++)
		{
			for (uint q : S.adj[p])
			{
				const bool same = S.ef[p].idx[2] == S.ef[q].idx[2] && S.ef[p].idx[3] == S.ef[q].idx[3] && S.ef[p].idx[4] == S.ef[q].idx[4];
				w[p].push_back(same ? 0u : 1u);
			}
		}
		flood_components(n, S.adj, w, S.mesh_index, S.contours);
		S.contour_index.assign(n, kInf);
		for (uint c = 0; c < S.contours.size(); c++)
			for (uint p : S.contours[c])
				S.contour_index[p] = c;
		// classify_contour_type
		const MeshIn& m = S.m;
		S.contour_type.resize(S.contours.size());
		for (uint c = 0; c < S.contours.size(); c++)
		{
			const auto& C = S.contours[c];
			std::vector<uint8_t> is_loop(C.size()), is_bnd(C.size());
			std::vector<uint> deg(C.size()), mi(C.size());
			for (size_t i = 0; i < C.size(); i++)
			{
				const uint p = C[i];
				is_loop[i] = S.ef[p].is_loop() ? 1 : 0;
				is_bnd[i] = (m.eaf_off[S.ef_e[p] + 1] - m.eaf_off[S.ef_e[p]]) <= 1 ? 1 : 0;
				deg[i] = uint(S.adj[p].size());
				mi[i] = S.mesh_index[p];
			}
			S.contour_type[c] = classify_contour(uint(C.size()), is_loop.data(), is_bnd.data(), deg.data(), mi.data());
		}
		// vertex boundary flags
		S.vflags.assign(m.num_verts, {});
		for (uint p = 0; p < n; p++)
		{
			if (S.ef[p].is_loop())
				continue;
			const uint ef_flag = 2 * S.contour_index[p] + S.mesh_index[p];
			const uint ff = ef_flag ^ 1u;
			S.vflags[S.ef[p].idx[0]].push_back(ef_flag);
			S.vflags[S.ef[p].idx[1]].push_back(ef_flag);
			S.vflags[S.ef[p].idx[2]].push_back(ff);
			S.vflags[S.ef[p].idx[3]].push_back(ff);
			S.vflags[S.ef[p].idx[4]].push_back(ff);
		}
		for (auto& r : S.vflags)
		{
			std::sort(r.begin(), r.end());
			r.erase(std::unique(r.begin(), r.end()), r.end());
		}
	}

	void normals(Scene& S)
	{
		const MeshIn& m = S.m;
		auto safe_n = [](V3 n)
		{
			const float l2 = dot(n, n);
			return l2 > 1e-20f ? n / std::sqrt(l2) : v3(0.0f);
		};
		S.fn.resize(m.num_faces);
		S.en.resize(m.num_edges);
		S.vn.resize(m.num_verts);
		for (uint f = 0; f < m.num_faces; f++)
		{
			const V3 a = load3(m.x, face_of(m, f, 0)), b = load3(m.x, face_of(m, f, 1)), c = load3(m.x, face_of(m, f, 2));
			const V3 n = safe_n(cross(b - a, c - a));
			const uint obj = m.vert_object[face_of(m, f, 0)];
			S.fn[f] = (m.mesh_orientation == nullptr || m.mesh_orientation[obj] == 0 ? 1.0f : -1.0f) * n;
		}
		for (uint e = 0; e < m.num_edges; e++)
		{
			V3 s = v3(0.0f);
			for (uint f : row(m.eaf_off, m.eaf, e))
				s = s + m.rest_face_area[f] * S.fn[f];
			S.en[e] = safe_n(s);
		}
		for (uint v = 0; v < m.num_verts; v++)
		{
			V3 s = v3(0.0f);
			for (uint f : row(m.vaf_off, m.vaf, v))
				s = s + m.rest_face_area[f] * S.fn[f];
			S.vn[v] = safe_n(s);
		}
	}

	// ---- runtime initialisation
	void hop_geo(const Scene& S, Runtime& r)
	{
		const MeshIn& m = S.m;
		for (int side = 0; side < 2; side++)
		{
			const uint lo = m.prefix_verts[r.object_ids[side]], hi = m.prefix_verts[r.object_ids[side] + 1];
			auto& hop = r.hop[side];
			auto& geo = r.geo[side];
			hop.assign(m.num_verts, kInf);
			geo.assign(m.num_verts, kGeoInf);
			std::priority_queue<std::pair<uint, uint>, std::vector<std::pair<uint, uint>>, std::greater<>> hq;
			std::priority_queue<std::pair<float, uint>, std::vector<std::pair<float, uint>>, std::greater<>> gq;
			for (uint v : r.boundary[side])
			{
				hop[v] = 0;
				geo[v] = 0.0f;
				hq.emplace(0u, v);
				gq.emplace(0.0f, v);
			}
			while (!hq.empty())
			{
				auto [d, v] = hq.top();
				hq.pop();
				if (d > hop[v])
					continue;
				for (uint a : row(m.vav_off, m.vav, v))
				{
					if (a < lo || a >= hi)
						continue;
					if (d + 1 < hop[a])
					{
						hop[a] = d + 1;
						hq.emplace(d + 1, a);
					}
				}
			}
			while (!gq.empty())
			{
				auto [d, v] = gq.top();
				gq.pop();
				if (d > geo[v])
					continue;
				for (uint a : row(m.vav_off, m.vav, v))
				{
					if (a < lo || a >= hi)
						continue;
					const float nd = d + length(load3(m.rest_x, v) - load3(m.rest_x, a));
					if (nd < geo[a])
					{
						geo[a] = nd;
						gq.emplace(nd, a);
					}
				}
			}
			uint mx = 0;
			for (uint v = lo; v < hi; v++)
				if (hop[v] != kInf)
					mx = std::max(mx, hop[v]);
			r.diam[side] = mx;
		}
	}

	// get_raycasting_direction (intersection_resolver2.cpp:1488-1569): +-e0, +-e1, +-e2 of the
	// area-weighted scatter of both sides' anchors about the weighted contour centre
	// (ascending eigenvalues), centre - side centroid for each side (fallback e1 / e2),
	// +-(centre - global area-weighted centroid); mode 1: the 26 lattice directions
	std::vector<V3> seed_directions(uint direction_mode, const std::vector<V3>& pts, const std::vector<float>& pw,
		const std::vector<uint>* boundary, const float* x, const float* vert_area, uint num_verts,
		const std::function<bool(uint)>& in_scene = nullptr)
	{
		std::vector<V3> dirs;
		if (direction_mode == 1)
		{
			for (int dx = -1; dx <= 1; dx++)
				for (int dy = -1; dy <= 1; dy++)
					for (int dz = -1; dz <= 1; dz++)
						if (dx || dy || dz)
							dirs.push_back(normalize(v3(float(dx), float(dy), float(dz))));
			return dirs;
		}
		auto add_seed = [&](V3 d)
		{
			if (!valid_dir(d))
				return;
			dirs.push_back(normalize(d));
		};
		auto add_signed = [&](V3 d)
		{
			add_seed(d);
			add_seed(-d);
		};
		// weighted mean of the contour points (helper.h:199-228)
		V3 ws = v3(0.0f), us = v3(0.0f);
		float sw = 0.0f;
		for (size_t i = 0; i < pts.size(); i++)
		{
			const float w = pw[i];
			us = us + pts[i];
			ws = ws + pts[i] * w;
			sw += w;
		}
		const V3 center = sw == 0.0f ? us / float(pts.size()) : ws / sw;
		V3 mc[2] = { v3(0.0f), v3(0.0f) };
		Mat3 Sw = mat_zero();
		for (int side = 0; side < 2; side++)
		{
			float wsum = 0.0f;
			std::vector<float> wts;
			for (uint v : boundary[side])
			{
				const V3 xv = load3(x, v);
				const float w = std::fmax(vert_area[v], 1e-8f);
				wts.push_back(w);
				mc[side] = mc[side] + xv * w;
				const V3 c = xv - center;
				Sw = madd(Sw, mscale(w, outer(c, c)));
			}
			for (float w : wts)
				wsum += w;
			mc[side] = wsum > 1e-8f ? mc[side] / wsum : center;
		}
		V3 ev[3];
		all_eigenvectors(Sw, ev);
		for (int k = 0; k < 3; k++)
			add_signed(ev[k]);
		for (int side = 0; side < 2; side++)
		{
			V3 d = center - mc[side];
			if (!valid_dir(d))
				d = ev[side + 1];
			add_seed(d);
		}
		V3 gc = v3(0.0f);
		float tm = 0.0f;
		for (uint v = 0; v < num_verts; v++)
		{
			if (in_scene && !in_scene(v))
				continue;
			const float w = std::fmax(vert_area[v], 1e-8f);
			gc = gc + load3(x, v) * w;
			tm += w;
		}
		if (tm > 1e-8f)
		{
			gc = gc / tm;
			const V3 rad = center - gc;
			if (valid_dir(rad))
				add_signed(rad);
		}
		if (dirs.empty())
			add_signed(v3(0, 1, 0));
		return dirs;
	}

	std::vector<V3> ray_directions(const Scene& S, const Runtime& r)
	{
		std::vector<V3> pts;
		std::vector<float> pw;
		for (uint p : r.contour)
		{
			pts.push_back(S.pos3[p]);
			pw.push_back(S.length[p]);
		}
		const MeshIn& m = S.m;
		if (!m.object_scene)
			return seed_directions(S.p.direction_mode, pts, pw, r.boundary, m.x, m.rest_vert_area, m.num_verts);
		// independent scenes in one batch: the global centroid of the contour's own scene
		const uint sc = m.object_scene[r.object_ids[0]];
		return seed_directions(S.p.direction_mode, pts, pw, r.boundary, m.x, m.rest_vert_area, m.num_verts,
			[&](uint v)
			{ return m.object_scene[m.vert_object[v]] == sc; });
	}

	inline uint kring_init(uint boundary_count, uint diam)
	{
		const uint k0 = 3;
		if (diam == 0)
			return k0;
		const uint ka = uint(std::ceil(std::sqrt(float(boundary_count))));
		return std::max(k0, std::min(ka, diam));
	}

	void init_runtime(const Scene& S, Runtime& r, uint c)
	{
		const MeshIn& m = S.m;
		r.contour_idx = c;
		r.inited = true;
		r.contour = S.contours[c];
		const uint first = r.contour.front();
		const EfPair& fp = S.ef[first];
		const uint es = S.mesh_index[first];
		r.object_ids[es] = m.vert_object[fp.idx[0]];
		r.comp_ids[es] = m.vert_component ? m.vert_component[fp.idx[0]] : 0;
		r.object_ids[es ^ 1] = m.vert_object[fp.idx[2]];
		r.comp_ids[es ^ 1] = m.vert_component ? m.vert_component[fp.idx[2]] : 0;
		std::set<uint> bs[2];
		for (uint p : r.contour)
		{
			const uint mi = S.mesh_index[p];
			bs[mi].insert(S.ef[p].idx[0]);
			bs[mi].insert(S.ef[p].idx[1]);
			bs[mi ^ 1].insert(S.ef[p].idx[2]);
			bs[mi ^ 1].insert(S.ef[p].idx[3]);
			bs[mi ^ 1].insert(S.ef[p].idx[4]);
		}
		for (int s = 0; s < 2; s++)
			r.boundary[s].assign(bs[s].begin(), bs[s].end());
		hop_geo(S, r);
		r.dirs = ray_directions(S, r);
		const size_t nd = r.dirs.size();
		r.results.assign(nd, ComboInfo{});
		r.converged.assign(nd, 0);
		r.pruned.assign(nd, 0);
		r.present.assign(nd, 0);
		r.active.assign(nd, 1);
		for (int s = 0; s < 2; s++)
		{
			r.init_k[s] = kring_init(uint(r.boundary[s].size()), r.diam[s]);
			r.k[s] = r.init_k[s];
		}
	}

	// ---- candidates at level k with contour-side restriction (CCR, intersection_resolver2.h:405-506)
	inline bool reachable(float d) { return finitef(d) && d < std::numeric_limits<float>::max() * 0.5f; }

	// compute_normalized_phi
	inline float normalized_phi(float own, float opp, float eps = 1e-6f)
	{
		const bool g0 = reachable(own), g1 = reachable(opp);
		if (!g0 && !g1)
			return 0.0f;
		if (!g0)
			return 1.0f;
		if (!g1)
			return -1.0f;
		return (own - opp) / (own + opp + eps);
	}

	// prp_intrinsic_contour_side_owns_vertex
	inline bool owns_1(float own, float opp, float tau)
	{
		if (!reachable(own))
			return false;
		if (!reachable(opp))
			return true;
		return normalized_phi(own, opp) <= tau;
	}

	// prp_dual_metric_contour_side_owns_vertex: each enabled metric passes on its own
	inline bool owns_dual(float ro, float rp, float co, float cp, float tau, bool use_rest, bool use_cur)
	{
		return (!use_rest || owns_1(ro, rp, tau)) && (!use_cur || owns_1(co, cp, tau));
	}

	// prp_intrinsic_contour_side_blended_phi / _owns_vertex_blended
	inline float blended_phi(float ro, float rp, float co, float cp, float w, float eps = 1e-6f)
	{
		if (!finitef(w) || (!reachable(ro) && !reachable(co)))
			return std::numeric_limits<float>::infinity();
		const float pr = normalized_phi(ro, rp, eps), pc = normalized_phi(co, cp, eps);
		if (!(reachable(ro) && reachable(rp)))
			return pc;
		if (!(reachable(co) && reachable(cp)))
			return pr;
		const float wc = std::fmin(std::fmax(w, 0.0f), 1.0f);
		return wc * pr + (1.0f - wc) * pc;
	}
	inline bool owns_blended(float ro, float rp, float co, float cp, float tau, float w) { return blended_phi(ro, rp, co, cp, w) <= tau; }

	// prp_contour_roles_share_topology / prp_intrinsic_contour_side_restriction_applies
	inline bool roles_share_topology(const uint obj[2], const uint comp[2])
	{
		return obj[0] == obj[1] && comp[0] != kInf && comp[0] == comp[1];
	}
	inline bool ccr_applies(bool enabled, const uint obj[2], const uint comp[2], bool use_deformed)
	{
		if (!enabled)
			return false;
		if (use_deformed)
			return obj[0] != kInf && obj[1] != kInf;
		return roles_share_topology(obj, comp);
	}

	// the owner test of one vertex for a role (resolver2.cpp:1750-1772)
	inline bool owns_vertex(const Params& p, float ro, float rp, float co, float cp)
	{
		const bool rest = p.ccr_use_rest != 0, cur = p.ccr_use_current != 0;
		if (p.ccr_blend && rest && cur)
			return owns_blended(ro, rp, co, cp, p.ccr_tau, p.ccr_blend_weight);
		if (rest && !owns_1(ro, rp, p.ccr_tau))
			return false;
		if (!cur)
			return true;
		return owns_dual(ro, rp, co, cp, p.ccr_tau, rest, true);
	}

	void build_candidates(const Scene& S, Runtime& r)
	{
		const MeshIn& m = S.m;
		for (int s = 0; s < 2; s++)
		{
			const uint obj = r.object_ids[s];
			const uint k = r.k[s];
			const auto& d = r.hop[s];
			auto& cv = r.cand_v[s];
			auto& ce = r.cand_e[s];
			auto& cf = r.cand_f[s];
			cv.clear();
			ce.clear();
			cf.clear();
			for (uint v = m.prefix_verts[obj]; v < m.prefix_verts[obj + 1]; v++)
				if (d[v] <= k)
					cv.push_back(v);
			for (uint e = m.prefix_edges[obj]; e < m.prefix_edges[obj + 1]; e++)
				if (d[edge_of(m, e, 0)] <= k && d[edge_of(m, e, 1)] <= k)
					ce.push_back(e);
			for (uint f = m.prefix_faces[obj]; f < m.prefix_faces[obj + 1]; f++)
				if (d[face_of(m, f, 0)] <= k && d[face_of(m, f, 1)] <= k && d[face_of(m, f, 2)] <= k)
					cf.push_back(f);
		}
		if (!ccr_applies(S.p.use_ccr && (S.p.ccr_use_rest || S.p.ccr_use_current), r.object_ids, r.comp_ids, S.p.ccr_use_current != 0))
			return;
		auto cur = [&](int role, uint v)
		{
			auto it = r.cur_dist[role].find(v);
			if (it != r.cur_dist[role].end())
				return it->second;
			const V3 x = load3(m.x, v);
			float md = std::numeric_limits<float>::max();
			for (uint b : r.boundary[role])
				md = std::fmin(md, length(x - load3(m.x, b)));
			r.cur_dist[role].emplace(v, md);
			return md;
		};
		for (int role = 0; role < 2; role++)
		{
			auto owns = [&](uint v)
			{
				const float ro = r.geo[role][v], rp = r.geo[role ^ 1][v];
				const bool rest = S.p.ccr_use_rest != 0, cur_on = S.p.ccr_use_current != 0;
				// the current-space distances are only computed where the rule reads them
				if (!(S.p.ccr_blend && rest && cur_on) && rest && !owns_1(ro, rp, S.p.ccr_tau))
					return false;
				if (!cur_on)
					return true;
				return owns_vertex(S.p, ro, rp, cur(role, v), cur(role ^ 1, v));
			};
			auto& cv = r.cand_v[role];
			cv.erase(std::remove_if(cv.begin(), cv.end(), [&](uint v)
						 { return !owns(v); }),
				cv.end());
			auto& ce = r.cand_e[role];
			ce.erase(std::remove_if(ce.begin(), ce.end(), [&](uint e)
						 { return !owns(edge_of(m, e, 0)) && !owns(edge_of(m, e, 1)); }),
				ce.end());
			auto& cf = r.cand_f[role];
			cf.erase(std::remove_if(cf.begin(), cf.end(), [&](uint f)
						 { return !owns(face_of(m, f, 0)) && !owns(face_of(m, f, 1)) && !owns(face_of(m, f, 2)); }),
				cf.end());
		}
	}

	// ---- hit adjacency (find_adjacent_hits), as exact-key lookups in the sorted hit list
	struct HitIndex
	{
		std::vector<uint64_t> keys;
		std::vector<uint> idx;
		void build(const std::vector<Hit>& hits)
		{
			std::vector<std::pair<uint64_t, uint>> kv;
			for (uint i = 0; i < hits.size(); i++)
				kv.push_back({ hits[i].key(), i });
			std::sort(kv.begin(), kv.end());
			keys.clear();
			idx.clear();
			for (auto& [k, i] : kv)
			{
				keys.push_back(k);
				idx.push_back(i);
			}
		}
		template <typename F>
		void find(uint type, uint src, uint dst, F&& f) const
		{
			const uint64_t k = (uint64_t(type) << 62) | (uint64_t(src & 0x3fffffffu) << 31) | uint64_t(dst & 0x7fffffffu);
			auto it = std::lower_bound(keys.begin(), keys.end(), k);
			for (; it != keys.end() && *it == k; ++it)
				f(idx[it - keys.begin()]);
		}
	};

	// neighbours of hit i (intersection_resolver_helper.cpp:771-902), each rule restated as the
	// exact (type, source, target) keys its bucket scan would accept.
	void hit_neighbours(const MeshIn& m, const std::vector<Hit>& H, const HitIndex& ix, uint i, std::vector<uint>& out)
	{
		const Hit& h = H[i];
		auto add = [&](uint j)
		{
			if (j != i)
				out.push_back(j);
		};
		if (h.type == VF)
		{
			const uint v = h.src_id, f = h.dst_id;
			for (uint av : row(m.vav_off, m.vav, v))
				ix.find(VF, av, f, add);
			for (uint af : row(m.vaf_off, m.vaf, v))
				for (int k = 0; k < 3; k++)
					ix.find(FV, af, face_of(m, f, k), add);
			for (uint ae : row(m.vae_off, m.vae, v))
				for (int k = 0; k < 3; k++)
					ix.find(EE, ae, m.face_adj_edges[3 * f + k], add);
		}
		else if (h.type == FV)
		{
			const uint f = h.src_id, w = h.dst_id;
			for (int k = 0; k < 3; k++)
				for (uint af : row(m.vaf_off, m.vaf, w))
					ix.find(VF, face_of(m, f, k), af, add);
			for (uint aw : row(m.vav_off, m.vav, w))
				ix.find(FV, f, aw, add);
			for (int k = 0; k < 3; k++)
				for (uint ae : row(m.vae_off, m.vae, w))
					ix.find(EE, m.face_adj_edges[3 * f + k], ae, add);
		}
		else
		{
			const uint e1 = h.src_id, e2 = h.dst_id;
			for (int k = 0; k < 2; k++)
				for (uint af : row(m.eaf_off, m.eaf, e2))
					ix.find(VF, edge_of(m, e1, k), af, add);
			for (uint af : row(m.eaf_off, m.eaf, e1))
				for (int k = 0; k < 2; k++)
					ix.find(FV, af, edge_of(m, e2, k), add);
			for (uint ae2 : row(m.eae_off, m.eae, e2))
				ix.find(EE, e1, ae2, add);
			for (uint ae1 : row(m.eae_off, m.eae, e1))
				ix.find(EE, ae1, e2, add);
		}
	}

	// Solid-interior links (intersection_resolver2.cpp:3298-3464): hits that share a source
	// vertex (VF), a target vertex (FV) or a source edge (EE), ordered by distance, link each
	// hit to the next one when both targets belong to one solid (rigid / tetrahedral) mesh,
	// the distance grows by more than eps_d and the ray enters the first target and leaves
	// through the second (normal signs beyond eps_n). Equal distances are ordered by hit key.
	void solid_links(const Scene& S, const std::vector<Hit>& H, V3 r, std::vector<std::vector<uint>>& out)
	{
		const MeshIn& m = S.m;
		auto solid_v = [&](uint v)
		{ return S.p.solid_all || (m.object_solid && m.object_solid[m.vert_object[v]]); };
		std::map<std::pair<uint, uint>, std::vector<uint>> groups;
		for (uint i = 0; i < H.size(); i++)
		{
			const Hit& h = H[i];
			groups[{ h.type, h.type == FV ? h.dst_id : h.src_id }].push_back(i);
		}
		const float en = S.p.solid_eps_n, ed = S.p.solid_eps_d;
		for (auto& [g, idx] : groups)
		{
			if (idx.size() < 2)
				continue;
			std::sort(idx.begin(), idx.end(), [&](uint a, uint b)
				{
					if (H[a].dist != H[b].dist) return H[a].dist < H[b].dist;
					return H[a].key() < H[b].key(); });
			for (size_t q = 0; q + 1 < idx.size(); q++)
			{
				const Hit &A = H[idx[q]], &B = H[idx[q + 1]];
				bool link = false;
				if (g.first == EE)
				{
					const uint va = edge_of(m, A.dst_id, 0), vb = edge_of(m, B.dst_id, 0);
					if (m.vert_object[va] == m.vert_object[vb] && solid_v(va) && B.dist - A.dist > ed)
					{
						const float da = dot(S.en[A.dst_id], r), db = dot(S.en[B.dst_id], r);
						link = da < -en && db > en;
					}
				}
				else
				{
					const uint fa = A.fid(), fb = B.fid();
					const uint va = face_of(m, fa, 0), vb = face_of(m, fb, 0);
					if (m.vert_object[va] == m.vert_object[vb] && solid_v(va) && B.dist - A.dist > ed)
					{
						const float da = dot(S.fn[fa], r), db = dot(S.fn[fb], r);
						link = g.first == VF ? (da < -en && db > en) : (da > en && db < -en);
					}
				}
				if (link)
				{
					out[idx[q]].push_back(idx[q + 1]);
					out[idx[q + 1]].push_back(idx[q]);
				}
			}
		}
	}

	// Canonical 32-lane strided sum + xor butterfly (the CUDA metrics kernel's order).
	template <typename F>
	float lane_sum(uint n, F&& val)
	{
		float s[32];
		for (int l = 0; l < 32; l++)
			s[l] = 0.0f;
		for (uint i = 0; i < n; i++)
			s[i & 31] = s[i & 31] + val(i);
		for (int off = 16; off >= 1; off >>= 1)
		{
			float t[32];
			for (int l = 0; l < 32; l++)
				t[l] = s[l] + s[l ^ off];
			for (int l = 0; l < 32; l++)
				s[l] = t[l];
		}
		return s[0];
	}

	// The metrics' canonical sum: the lane sum over lists of up to 8192 terms; a longer list is
	// cut into chunks of 8192 from its start, each chunk lane-summed, and the chunk sums
	// lane-summed (the CUDA metrics kernels sum the chunks of a large support in parallel).
	constexpr uint kSumChunk = 8192;
	template <typename F>
	float chunked_sum(uint n, F&& val)
	{
		if (n <= kSumChunk)
			return lane_sum(n, val);
		const uint nc = (n + kSumChunk - 1) / kSumChunk;
		std::vector<float> cs(nc);
		for (uint c = 0; c < nc; c++)
		{
			const uint b = c * kSumChunk, m = std::min(kSumChunk, n - b);
			cs[c] = lane_sum(m, [&](uint i)
				{ return val(b + i); });
		}
		return lane_sum(nc, [&](uint i)
			{ return cs[i]; });
	}

	// The reference's deterministic parallel reduce (CpuParallel::parallel_for_and_reduce,
	// Solver/Utils/cpu_parallel.h:505-538, fiber backend) as a sum: blocks of 256 terms in index
	// order, each summed sequentially from zero, then the block sums combined by std::reduce,
	// restated with the GNU C++ library's order for random-access ranges (two pair sums folded
	// into the running value four blocks at a time, the remaining blocks one by one).
	template <typename F>
	float reference_block_sum(uint n, F&& val)
	{
		const uint nb = (n + 255u) / 256u;
		std::vector<float> b(nb, 0.0f);
		for (uint k = 0; k < nb; k++)
		{
			float v = 0.0f;
			for (uint i = 256u * k; i < std::min(n, 256u * k + 256u); i++)
				v = v + val(i);
			b[k] = v;
		}
		float acc = 0.0f;
		uint i = 0;
		for (; i + 4 <= nb; i += 4)
		{
			const float v1 = b[i] + b[i + 1], v2 = b[i + 2] + b[i + 3];
			acc = acc + (v1 + v2);
		}
		for (; i < nb; i++)
			acc = acc + b[i];
		return acc;
	}

	struct PenMetrics
	{
		float depth = 0, volume = 0, area = 0, objective = 0, cost = 0;
	};

	// prp_eval_penetration_v2 (intersection_resolver2.cpp:1883-1954) over hits in key order:
	// A = rest area of the source primitive, alpha = |n_src . r|, delta = dist; depth = max
	// delta, volume = sum A alpha delta, J = (sum A) depth^2, displacement cost = sum
	// (delta + 3e-3)^2 / kappa_h. Sums in the canonical 32-lane strided order.
	// reference_order: the sums in the reference's block-reduce order over the hits as given
	PenMetrics penetration_metrics(const MeshIn& m, const V3* vn, const V3* en, const V3* fn, V3 dir, const std::vector<Hit>& hits,
		bool reference_order = false)
	{
		struct HitsRef
		{
			V3 dir;
			const std::vector<Hit>& hits;
		} c{ dir, hits };
		const uint n = uint(hits.size());
		auto inv_mass = [&](uint v)
		{ return 1.0f / std::fmax(m.vert_mass[v], 1e-8f); };
		auto area_alpha = [&](const Hit& h, float& area, float& alpha)
		{
			const V3 d = c.dir;
			if (h.type == VF)
			{
				area = m.rest_vert_area[h.src_id];
				alpha = std::fabs(dot(vn[h.src_id], d));
			}
			else if (h.type == EE)
			{
				area = m.rest_edge_area[h.src_id];
				alpha = std::fabs(dot(en[h.src_id], d));
			}
			else
			{
				area = m.rest_face_area[h.src_id];
				alpha = std::fabs(dot(fn[h.src_id], d));
			}
		};
		auto eff_inv = [&](const Hit& h)
		{
			if (h.type == VF)
			{
				const float bx = h.bary[0], by = h.bary[1], bz = 1.0f - h.bary[0] - h.bary[1];
				return ((inv_mass(h.sv[0]) + bx * bx * inv_mass(h.dv[0])) + by * by * inv_mass(h.dv[1])) + bz * bz * inv_mass(h.dv[2]);
			}
			if (h.type == FV)
			{
				const float bx = h.bary[0], by = h.bary[1], bz = 1.0f - h.bary[0] - h.bary[1];
				return ((bx * bx * inv_mass(h.sv[0]) + by * by * inv_mass(h.sv[1])) + bz * bz * inv_mass(h.sv[2])) + inv_mass(h.dv[0]);
			}
			const float a0 = h.bary[0], a1 = 1.0f - h.bary[0], b0 = h.bary[1], b1 = 1.0f - h.bary[1];
			return ((a0 * a0 * inv_mass(h.sv[0]) + a1 * a1 * inv_mass(h.sv[1])) + b0 * b0 * inv_mass(h.dv[0])) + b1 * b1 * inv_mass(h.dv[1]);
		};
		float depth = 0.0f;
		for (const Hit& h : c.hits)
			depth = std::fmax(depth, h.dist);
		auto sum = [&](auto&& term)
		{ return reference_order ? reference_block_sum(n, term) : chunked_sum(n, term); };
		const float area = sum([&](uint i)
			{ float a, al; area_alpha(c.hits[i], a, al); return a; });
		const float volume = sum([&](uint i)
			{ float a, al; area_alpha(c.hits[i], a, al); return (a * al) * c.hits[i].dist; });
		const float kappa = sum([&](uint i)
			{
				const float sd = c.hits[i].dist + 3e-3f;
				const float e = eff_inv(c.hits[i]);
				return e > 1e-8f ? (sd * sd) / e : 0.0f; });
		PenMetrics pm;
		pm.depth = depth;
		pm.volume = volume;
		pm.area = area;
		pm.objective = (area * depth) * depth;
		pm.cost = kappa;
		return pm;
	}

	// prp_eval_penetration_v2 + prp_fill_combo_eval_info over hits in canonical order
	void fill_metrics(const Scene& S, const Runtime& r, ComboInfo& c)
	{
		std::sort(c.hits.begin(), c.hits.end(), [](const Hit& a, const Hit& b)
			{ return a.key() < b.key(); });
		const PenMetrics pm = penetration_metrics(S.m, S.vn.data(), S.en.data(), S.fn.data(), c.dir, c.hits);
		c.depth = pm.depth;
		c.volume = pm.volume;
		c.area = pm.area;
		c.objective = pm.objective;
		c.cost = pm.cost;
		c.hit_count = uint(c.hits.size());
		// EF-anchor coverage
		std::set<uint> sup[2];
		for (const Hit& h : c.hits)
		{
			for (int k = 0; k < 3; k++)
				if (h.sv[k] != kInf)
					sup[0].insert(h.sv[k]);
			for (int k = 0; k < 3; k++)
				if (h.dv[k] != kInf)
					sup[1].insert(h.dv[k]);
		}
		uint cov = 0;
		for (uint p : r.contour)
		{
			const uint mi = S.mesh_index[p];
			const EfPair& e = S.ef[p];
			const bool eo = sup[mi].count(e.idx[0]) || sup[mi].count(e.idx[1]);
			const bool fo = sup[mi ^ 1].count(e.idx[2]) || sup[mi ^ 1].count(e.idx[3]) || sup[mi ^ 1].count(e.idx[4]);
			cov += (eo && fo) ? 1 : 0;
		}
		c.anchors = uint(r.contour.size());
		c.covered = cov;
		c.coverage = c.anchors > 0 ? float(cov) / float(c.anchors) : 0.0f;
		// frontier hops
		uint mfs = 0, mfd = 0;
		for (const Hit& h : c.hits)
		{
			for (int k = 0; k < 3; k++)
				if (h.sv[k] != kInf && r.hop[0][h.sv[k]] != kInf)
					mfs = std::max(mfs, r.hop[0][h.sv[k]]);
			for (int k = 0; k < 3; k++)
				if (h.dv[k] != kInf && r.hop[1][h.dv[k]] != kInf)
					mfd = std::max(mfd, r.hop[1][h.dv[k]]);
		}
		c.max_front_src = mfs;
		c.max_front_dst = mfd;
	}

	// One (contour, combo) evaluation at the current k-ring (evaluate_batched_contours_of_single_combo).
	ComboInfo eval_combo(Scene& S, Runtime& r, uint combo)
	{
		const MeshIn& m = S.m;
		ComboInfo info;
		info.present = true;
		info.combo_idx = combo;
		info.dir = r.dirs[combo];
		info.eval_k_src = r.k[0];
		info.eval_k_dst = r.k[1];
		const V3 dir = r.dirs[combo];
		const float dl2 = dot(dir, dir);
		auto span = [](const std::vector<uint>& ids, uint& lo, uint& cnt)
		{
			if (ids.empty())
			{
				lo = 0;
				cnt = 0;
				return;
			}
			uint mn = kInf, mx = 0;
			for (uint id : ids)
			{
				mn = std::min(mn, id);
				mx = std::max(mx, id);
			}
			lo = mn;
			cnt = mx - mn + 1;
		};
		std::vector<Hit> hits;
		uint64_t tested = 0, requests = 0, pairs = 0;
		Recheck rcl;
		Recheck* rc = S.p.fp64_recheck ? &rcl : nullptr;
		const bool brute = S.p.brute_force_raycast != 0;
		const CachedBVH* fb_dst = brute ? nullptr : S.face_bvh[r.object_ids[1]].get();
		const CachedBVH* eb_dst = brute ? nullptr : S.edge_bvh[r.object_ids[1]].get();
		const CachedBVH* fb_src = brute ? nullptr : S.face_bvh[r.object_ids[0]].get();
		// VF
		if (!r.cand_f[1].empty())
		{
			VertRequest q{};
			span(r.cand_f[1], q.target_lo, q.target_cnt);
			q.dir = dir;
			q.fv = false;
			q.targets = &r.cand_f[1];
			q.hop = &r.hop[1];
			q.max_hop = r.k[1];
			for (uint v : r.cand_v[0])
			{
				q.vid = v;
				cast_vert(m, fb_dst, q, hits, tested, rc);
				requests++;
				pairs += r.cand_f[1].size();
			}
		}
		// EE
		if (!r.cand_e[1].empty())
		{
			float pmin = std::numeric_limits<float>::max(), pmax = -std::numeric_limits<float>::max();
			for (uint e : r.cand_e[1])
			{
				const float a = dot(load3(m.x, edge_of(m, e, 0)), dir), b = dot(load3(m.x, edge_of(m, e, 1)), dir);
				pmin = std::fmin(pmin, std::fmin(a, b));
				pmax = std::fmax(pmax, std::fmax(a, b));
			}
			EdgeRequest q{};
			span(r.cand_e[1], q.target_lo, q.target_cnt);
			q.dir = dir;
			q.targets = &r.cand_e[1];
			q.hop = &r.hop[1];
			q.max_hop = r.k[1];
			q.target_proj_min = pmin;
			for (uint e : r.cand_e[0])
			{
				q.eid = e;
				if (dl2 <= 1e-12f)
					q.max_dist = 1.0f;
				else
				{
					const float smin = std::fmin(dot(load3(m.x, edge_of(m, e, 0)), dir), dot(load3(m.x, edge_of(m, e, 1)), dir));
					q.max_dist = std::fmin(std::fmax((pmax - smin) / dl2 + 1e-5f, 0.0f), 1.0f);
				}
				cast_edge(m, eb_dst, q, hits, tested, rc);
				requests++;
				pairs += r.cand_e[1].size();
			}
		}
		// FV
		if (!r.cand_f[0].empty())
		{
			VertRequest q{};
			span(r.cand_f[0], q.target_lo, q.target_cnt);
			q.dir = dir;
			q.fv = true;
			q.targets = &r.cand_f[0];
			q.hop = &r.hop[0];
			q.max_hop = r.k[0];
			for (uint v : r.cand_v[1])
			{
				q.vid = v;
				cast_vert(m, fb_src, q, hits, tested, rc);
				requests++;
				pairs += r.cand_f[0].size();
			}
		}
		{
			std::lock_guard<std::mutex> lock(S.mtx);
			S.tested += tested;
			S.requests += requests;
			S.pairs += pairs;
			S.rechecks += rcl.n;
			S.flips += rcl.flips;
		}
		info.unculled = uint(hits.size());
		if (hits.empty())
			return info;
		// boundary attachment (is_hit_adj_contour), src mesh role 0
		const uint c = r.contour_idx;
		auto flag = [&](uint v, uint mi)
		{
			const auto& f = S.vflags[v];
			return std::binary_search(f.begin(), f.end(), 2 * c + mi);
		};
		std::vector<uint8_t> attached(hits.size());
		for (size_t i = 0; i < hits.size(); i++)
		{
			const Hit& h = hits[i];
			bool ok = true;
			for (int k = 0; k < 3; k++)
				if (h.sv[k] != kInf)
					ok = ok && flag(h.sv[k], 0);
			for (int k = 0; k < 3; k++)
				if (h.dv[k] != kInf)
					ok = ok && flag(h.dv[k], 1);
			attached[i] = ok;
		}
		// components
		HitIndex ix;
		ix.build(hits);
		std::vector<std::vector<uint>> solid(hits.size());
		if (S.p.solid_interior && (S.p.solid_all || m.object_solid))
			solid_links(S, hits, dir, solid);
		std::vector<uint8_t> vis(hits.size(), 0);
		std::vector<uint> nb;
		uint best_cov = 0, best_n = 0;
		uint64_t best_key = ~0ull;
		bool found = false;
		std::vector<uint> best_comp;
		for (uint seed = 0; seed < hits.size(); seed++)
		{
			if (vis[seed])
				continue;
			std::vector<uint> comp, todo{ seed };
			vis[seed] = 1;
			bool att = false;
			while (!todo.empty())
			{
				const uint i = todo.back();
				todo.pop_back();
				comp.push_back(i);
				att = att || attached[i];
				nb.clear();
				hit_neighbours(m, hits, ix, i, nb);
				nb.insert(nb.end(), solid[i].begin(), solid[i].end());
				for (uint j : nb)
					if (!vis[j])
					{
						vis[j] = 1;
						todo.push_back(j);
					}
			}
			if (!att)
				continue;
			// coverage of this component
			std::set<uint> sup[2];
			uint64_t key = ~0ull;
			for (uint i : comp)
			{
				const Hit& h = hits[i];
				key = std::min(key, h.key());
				for (int k = 0; k < 3; k++)
					if (h.sv[k] != kInf)
						sup[0].insert(h.sv[k]);
				for (int k = 0; k < 3; k++)
					if (h.dv[k] != kInf)
						sup[1].insert(h.dv[k]);
			}
			uint cov = 0;
			for (uint p : r.contour)
			{
				const uint mi = S.mesh_index[p];
				const EfPair& e = S.ef[p];
				const bool eo = sup[mi].count(e.idx[0]) || sup[mi].count(e.idx[1]);
				const bool fo = sup[mi ^ 1].count(e.idx[2]) || sup[mi ^ 1].count(e.idx[3]) || sup[mi ^ 1].count(e.idx[4]);
				cov += (eo && fo) ? 1 : 0;
			}
			const uint nh = uint(comp.size());
			const bool better = !found || cov > best_cov || (cov == best_cov && nh > best_n) || (cov == best_cov && nh == best_n && key < best_key);
			if (better)
			{
				found = true;
				best_cov = cov;
				best_n = nh;
				best_key = key;
				best_comp = comp;
			}
		}
		if (!found)
			return info;
		for (uint i : best_comp)
			info.hits.push_back(hits[i]);
		fill_metrics(S, r, info);
		return info;
	}

	// evaluate_current_runtime_directions_template (intersection_resolver2.cpp:1058-1230)
	// evaluate_current_runtime_directions_template (intersection_resolver2.cpp:1058-1230) over
	// the listed runtimes: k from the initial level, the active directions reset; per level
	// build(remaining) prepares the candidates and eval(runtime, combo) evaluates one active,
	// unconverged, unpruned direction at the runtime's current k. A response is eligible
	// when usable and detached (frontier hop below k, or k at the diameter, on both roles);
	// directions whose objective is not below the best valid one are pruned; only the roles
	// that touch the frontier grow (k <- min(2k, diameter)).
	template <typename Build, typename Eval>
	void kring_levels(const std::vector<Runtime*>& batch, Build&& build, Eval&& eval, bool parallel)
	{
		uint max_combo = 0;
		for (Runtime* rp : batch)
		{
			Runtime& r = *rp;
			r.k[0] = r.init_k[0];
			r.k[1] = r.init_k[1];
			r.finished = false;
			r.no_response = false;
			max_combo = std::max(max_combo, uint(r.dirs.size()));
			for (size_t ci = 0; ci < r.dirs.size(); ci++)
				if (r.active[ci])
				{
					r.converged[ci] = 0;
					r.pruned[ci] = 0;
					r.present[ci] = 0;
					r.results[ci] = ComboInfo{};
				}
		}
		auto grow = [](uint cur, uint diam) -> uint
		{
			if (cur >= diam)
				return cur;
			return uint(std::min<uint64_t>(diam, std::max<uint64_t>(1u, uint64_t(cur) * 2u)));
		};
		std::vector<Runtime*> remaining = batch;
		for (uint level = 0; !remaining.empty() && level < 65; level++)
		{
			build(remaining);
			for (uint combo = 0; combo < max_combo; combo++)
			{
				std::vector<Runtime*> active;
				for (Runtime* rp : remaining)
				{
					const Runtime& r = *rp;
					if (combo < r.dirs.size() && r.active[combo] && !r.converged[combo] && !r.pruned[combo])
						active.push_back(rp);
				}
				auto one = [&](uint i)
				{
					Runtime& r = *active[i];
					ComboInfo info = eval(r, combo);
					info.levels = level + 1;
					info.full_mesh = r.k[0] >= r.diam[0] && r.k[1] >= r.diam[1];
					const bool usable = has_usable(info);
					const bool src_ok = info.max_front_src < r.k[0] || r.k[0] >= r.diam[0];
					const bool dst_ok = info.max_front_dst < r.k[1] || r.k[1] >= r.diam[1];
					info.eligible = usable && src_ok && dst_ok;
					r.converged[combo] = (info.eligible || info.full_mesh) ? 1 : 0;
					r.present[combo] = 1;
					r.results[combo] = std::move(info);
				};
				if (parallel)
					parallel_for(uint(active.size()), one, 1);
				else
					for (uint i = 0; i < active.size(); i++)
						one(i);
			}
			std::vector<Runtime*> next;
			for (Runtime* rp : remaining)
			{
				Runtime& r = *rp;
				bool has = false;
				float best = std::numeric_limits<float>::infinity();
				for (size_t ci = 0; ci < r.dirs.size(); ci++)
					if (r.active[ci] && has_valid(r.results[ci]))
					{
						has = true;
						best = std::fmin(best, response_objective(r.results[ci]));
					}
				if (has)
					for (size_t ci = 0; ci < r.dirs.size(); ci++)
						if (r.active[ci] && !r.converged[ci] && r.present[ci] && response_objective(r.results[ci]) >= best)
							r.pruned[ci] = 1;
				bool pending = false, gs = false, gd = false;
				for (size_t ci = 0; ci < r.dirs.size(); ci++)
				{
					if (!r.active[ci] || r.converged[ci] || r.pruned[ci])
						continue;
					pending = true;
					const ComboInfo& info = r.results[ci];
					gs = gs || (r.k[0] < r.diam[0] && (!has_usable(info) || info.max_front_src >= r.k[0]));
					gd = gd || (r.k[1] < r.diam[1] && (!has_usable(info) || info.max_front_dst >= r.k[1]));
				}
				if (!pending)
				{
					r.finished = true;
					r.no_response = !has;
					continue;
				}
				const uint ns = gs ? grow(r.k[0], r.diam[0]) : r.k[0];
				const uint nd = gd ? grow(r.k[1], r.diam[1]) : r.k[1];
				if (ns <= r.k[0] && nd <= r.k[1])
				{
					r.finished = true; // stalled: cannot happen when a role still grows
					continue;
				}
				r.k[0] = ns;
				r.k[1] = nd;
				next.push_back(rp);
			}
			remaining.swap(next);
		}
	}

	void evaluate_directions(Scene& S, const std::vector<uint>& batch)
	{
		std::vector<Runtime*> rts;
		for (uint c : batch)
			rts.push_back(&S.rt[c]);
		kring_levels(
			rts, [&](const std::vector<Runtime*>& rem)
			{ parallel_for(uint(rem.size()), [&](uint i)
				  { build_candidates(S, *rem[i]); }, 1); },
			[&](Runtime& r, uint combo)
			{ return eval_combo(S, r, combo); },
			true);
	}

	// ---- S^2 direction refinement (prp_optimize_runtime_directions, resolver2.cpp:1232-1486)

	// compute_effective_inverse_mass_weight (intersection_resolver_helper.cpp:611-645)
	float eff_inv_mass(const MeshIn& m, const Hit& h)
	{
		auto inv_mass = [&](uint v)
		{ return 1.0f / std::fmax(m.vert_mass[v], 1e-8f); };
		if (h.type == VF)
		{
			const float bx = h.bary[0], by = h.bary[1], bz = 1.0f - h.bary[0] - h.bary[1];
			return ((inv_mass(h.sv[0]) + bx * bx * inv_mass(h.dv[0])) + by * by * inv_mass(h.dv[1])) + bz * bz * inv_mass(h.dv[2]);
		}
		if (h.type == FV)
		{
			const float bx = h.bary[0], by = h.bary[1], bz = 1.0f - h.bary[0] - h.bary[1];
			return ((bx * bx * inv_mass(h.sv[0]) + by * by * inv_mass(h.sv[1])) + bz * bz * inv_mass(h.sv[2])) + inv_mass(h.dv[0]);
		}
		const float a0 = h.bary[0], a1 = 1.0f - h.bary[0], b0 = h.bary[1], b1 = 1.0f - h.bary[1];
		return ((a0 * a0 * inv_mass(h.sv[0]) + a1 * a1 * inv_mass(h.sv[1])) + b0 * b0 * inv_mass(h.dv[0])) + b1 * b1 * inv_mass(h.dv[1]);
	}

	// get_hit_characteristic_normal (resolver2.cpp:1232-1256), at the current positions
	V3 hit_normal(const MeshIn& m, const Hit& h)
	{
		auto X = [&](uint v)
		{ return v3(m.x[3 * v], m.x[3 * v + 1], m.x[3 * v + 2]); };
		if (h.type == VF)
			return cross(X(h.dv[1]) - X(h.dv[0]), X(h.dv[2]) - X(h.dv[0]));
		if (h.type == FV)
			return cross(X(h.sv[1]) - X(h.sv[0]), X(h.sv[2]) - X(h.sv[0]));
		const V3 p0 = X(h.sv[0]), p1 = X(h.sv[1]), q0 = X(h.dv[0]), q1 = X(h.dv[1]);
		V3 c = cross(p1 - p0, q1 - q0);
		if (length(c) < 1e-8f)
			c = (q0 * h.bary[1] + q1 * (1.0f - h.bary[1])) - (p0 * h.bary[0] + p1 * (1.0f - h.bary[0]));
		return c;
	}

	struct DirStep
	{
		V3 dir = v3(0.0f);
		float predicted = 0.0f, gnorm = 0.0f;
		bool valid = false;
	};

	// prp_compute_direction_optimization_step (resolver2.cpp:1268-1368). The gradient and
	// Hessian sums run in the canonical 32-lane strided order over the hits in key order.
	DirStep direction_step(const MeshIn& m, const std::vector<Hit>& hits, V3 input_dir, float trust)
	{
		DirStep out;
		if (hits.empty() || !valid_dir(input_dir))
			return out;
		const V3 r = normalize(input_dir);
		const float off = 3e-3f; // prp_response_depth_offset (intersection_resolver2.h:98)
		const uint n = uint(hits.size());
		// per-hit terms: g[3], H[9] (row-major), contributes
		std::vector<float> T(size_t(n) * 13, 0.0f);
		uint contributing = 0;
		for (uint i = 0; i < n; i++)
		{
			const Hit& h = hits[i];
			const V3 raw = hit_normal(m, h);
			const float nl = length(raw);
			if (!finitef(nl) || nl < 1e-8f)
				continue;
			const V3 nn = raw / nl;
			const float ndr = dot(nn, r);
			if (!finitef(ndr) || std::fabs(ndr) < 1e-6f)
				continue;
			const float e = eff_inv_mass(m, h);
			if (!finitef(e) || e <= 1e-8f)
				continue;
			const float w = 1.0f / e;
			const float d = h.dist;
			const V3 dd = (nn * (-d)) / ndr;
			const V3 g = dd * ((2.0f * w) * (d + off));
			const float hs = ((2.0f * w) / (ndr * ndr)) * ((3.0f * d) * d + (2.0f * d) * off);
			float* t = &T[size_t(i) * 13];
			t[0] = g.x;
			t[1] = g.y;
			t[2] = g.z;
			const float nv[3] = { nn.x, nn.y, nn.z };
			for (int a = 0; a < 3; a++)
				for (int b2 = 0; b2 < 3; b2++)
					t[3 + 3 * a + b2] = hs * (nv[a] * nv[b2]);
			t[12] = 1.0f;
			contributing++;
		}
		if (contributing == 0)
			return out;
		float G[3], H[9];
		for (int q = 0; q < 3; q++)
			G[q] = lane_sum(n, [&](uint i)
				{ return T[size_t(i) * 13 + q]; });
		for (int q = 0; q < 9; q++)
			H[q] = lane_sum(n, [&](uint i)
				{ return T[size_t(i) * 13 + 3 + q]; });
		const V3 grad = v3(G[0], G[1], G[2]);
		auto Hmul = [&](V3 v)
		{
			return v3((H[0] * v.x + H[1] * v.y) + H[2] * v.z, (H[3] * v.x + H[4] * v.y) + H[5] * v.z,
				(H[6] * v.x + H[7] * v.y) + H[8] * v.z);
		};
		const V3 tg = grad - r * dot(r, grad);
		const V3 axis = std::fabs(r.y) < 0.9f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
		const V3 e1 = normalize(cross(axis, r));
		const V3 e2 = normalize(cross(r, e1));
		const float g0 = dot(e1, tg), g1 = dot(e2, tg);
		const float gnorm = std::sqrt(g0 * g0 + g1 * g1);
		if (!finitef(gnorm) || gnorm < 1e-6f)
			return out;
		const float h00 = dot(e1, Hmul(e1)), h01 = dot(e1, Hmul(e2)), h10 = dot(e2, Hmul(e1)), h11 = dot(e2, Hmul(e2));
		const float det = h00 * h11 - h01 * h10;
		float d0, d1;
		if (finitef(det) && det > 1e-10f && h00 > 0.0f)
		{
			d0 = -(h11 * g0 - h01 * g1) / det;
			d1 = -(h00 * g1 - h10 * g0) / det;
		}
		else
		{
			const float gg = g0 * g0 + g1 * g1;
			const float ghg = g0 * (h00 * g0 + h01 * g1) + g1 * (h10 * g0 + h11 * g1);
			const float alpha = ghg > 1e-10f ? gg / ghg : trust / (gnorm + 1e-20f);
			d0 = -alpha * g0;
			d1 = -alpha * g1;
		}
		const float sn = std::sqrt(d0 * d0 + d1 * d1);
		if (!finitef(sn) || sn < 1e-7f)
			return out;
		if (sn > trust)
		{
			const float sc = trust / sn;
			d0 = d0 * sc;
			d1 = d1 * sc;
		}
		const V3 trial = (r + e1 * d0) + e2 * d1;
		if (!valid_dir(trial))
			return out;
		out.dir = normalize(trial);
		out.predicted = std::fmax(0.0f, -(g0 * d0 + g1 * d1));
		out.gnorm = gnorm;
		out.valid = true;
		return out;
	}

	int select_best(const Runtime& r)
	{
		int sel = -1;
		for (size_t ci = 0; ci < r.results.size(); ci++)
		{
			if (!has_valid(r.results[ci]))
				continue;
			if (sel < 0 || response_is_better(r.results[ci], r.results[sel]))
				sel = int(ci);
		}
		return sel;
	}

	// trust-region loop over the batch's contours; each trial re-runs the k-ring
	// evaluation of the one refined direction from the initial level
	void optimize_directions(Scene& S, const std::vector<uint>& batch, uint iterations)
	{
		if (iterations == 0 || batch.empty())
			return;
		struct St
		{
			int combo = -1;
			uint attempted = 0, accepted = 0;
			float trust = 0.3f;
			bool done = false;
		};
		std::vector<St> st(batch.size());
		for (size_t i = 0; i < batch.size(); i++)
		{
			const Runtime& r = S.rt[batch[i]];
			const int sel = select_best(r);
			if (sel < 0 || r.results[sel].hits.empty())
				st[i].done = true;
			else
				st[i].combo = sel;
		}
		for (uint it = 0; it < iterations; it++)
		{
			std::vector<ComboInfo> acc(batch.size());
			std::vector<V3> acc_dir(batch.size(), v3(0.0f));
			std::vector<float> pred(batch.size(), 0.0f), gn(batch.size(), 0.0f);
			std::vector<uint> trials;
			std::vector<size_t> trial_slot;
			for (size_t i = 0; i < batch.size(); i++)
			{
				St& s = st[i];
				Runtime& r = S.rt[batch[i]];
				if (s.done)
					continue;
				const ComboInfo& a = r.results[s.combo];
				const DirStep step = direction_step(S.m, a.hits, a.dir, s.trust);
				if (!step.valid)
				{
					s.done = true;
					continue;
				}
				s.attempted++;
				acc[i] = a;
				acc_dir[i] = r.dirs[s.combo];
				pred[i] = step.predicted;
				gn[i] = step.gnorm;
				r.dirs[s.combo] = step.dir;
				std::fill(r.active.begin(), r.active.end(), 0);
				r.active[s.combo] = 1;
				trials.push_back(batch[i]);
				trial_slot.push_back(i);
			}
			if (trials.empty())
				break;
			evaluate_directions(S, trials);
			for (size_t j = 0; j < trials.size(); j++)
			{
				const size_t i = trial_slot[j];
				St& s = st[i];
				Runtime& r = S.rt[trials[j]];
				std::fill(r.active.begin(), r.active.end(), 1);
				ComboInfo& trial = r.results[s.combo];
				// prp_select_response over {accepted, trial}: the trial wins only if strictly better
				const bool take = has_valid(trial) && (!has_valid(acc[i]) || response_is_better(trial, acc[i]));
				if (take)
				{
					s.accepted++;
					trial.opt_attempted = s.attempted;
					trial.opt_accepted = s.accepted;
					r.dirs[s.combo] = trial.dir;
					const float actual = response_objective(acc[i]) - response_objective(trial);
					if (pred[i] > 1e-20f && actual / pred[i] > 0.75f)
						s.trust = std::fmin(1.0f, s.trust * 2.0f);
				}
				else
				{
					r.results[s.combo] = acc[i];
					r.results[s.combo].opt_attempted = s.attempted;
					r.results[s.combo].opt_accepted = s.accepted;
					r.dirs[s.combo] = acc_dir[i];
					s.trust = std::fmax(0.01f, s.trust * 0.5f);
					if (s.trust <= 0.01f || gn[i] < 1e-6f)
						s.done = true;
				}
			}
		}
	}

	// get_adj_contours (intersection_resolver2.cpp:413-451) for one hit
	void adj_contours(const Scene& S, const Hit& h, uint c, std::set<uint>& out)
	{
		std::vector<uint> sv, dv;
		for (int k = 0; k < 3; k++)
			if (h.sv[k] != kInf)
				sv.push_back(h.sv[k]);
		for (int k = 0; k < 3; k++)
			if (h.dv[k] != kInf)
				dv.push_back(h.dv[k]);
		auto inter = [&](const std::vector<uint>& vs)
		{
			std::vector<uint> acc = S.vflags[vs.front()];
			for (uint v : vs)
			{
				std::vector<uint> t;
				std::set_intersection(S.vflags[v].begin(), S.vflags[v].end(), acc.begin(), acc.end(), std::back_inserter(t));
				acc.swap(t);
			}
			std::vector<uint> t;
			const uint rm[2] = { 2 * c, 2 * c + 1 };
			std::set_difference(acc.begin(), acc.end(), rm, rm + 2, std::back_inserter(t));
			return t;
		};
		const auto sf = inter(sv), df = inter(dv);
		for (uint a : sf)
			for (uint b : df)
				if (a == (b ^ 1u))
					out.insert(a / 2);
	}

	// prp_select_pre_finalize_contours_to_suppress (intersection_resolver2.cpp:453-592):
	// contours with merge partners, by pre-finalize area (descending, then index), each
	// unsuppressed owner suppresses the active contours its support reaches
	void suppress_contours(const std::vector<std::vector<uint>>& merge_adj, const std::vector<float>& pre_area,
		const std::vector<uint>& active, std::vector<uint8_t>& suppressed)
	{
		std::vector<uint> conflicting;
		for (uint c : active)
			if (!merge_adj[c].empty())
				conflicting.push_back(c);
		std::sort(conflicting.begin(), conflicting.end(), [&](uint a, uint b)
			{
				if (pre_area[a] != pre_area[b]) return pre_area[a] > pre_area[b];
				return a < b; });
		std::vector<uint8_t> is_active(merge_adj.size(), 0);
		for (uint c : active)
			is_active[c] = 1;
		for (uint owner : conflicting)
		{
			if (suppressed[owner])
				continue;
			for (uint a : merge_adj[owner])
				if (a != owner && is_active[a])
					suppressed[a] = 1;
		}
	}

	void run(Scene& S)
	{
		const MeshIn& m = S.m;
		preprocess(S);
		contours(S);
		normals(S);
		const uint nc = uint(S.contours.size());
		S.rt.resize(nc);
		S.selected.assign(nc, ComboInfo{});
		S.processed.assign(nc, 0);
		S.suppressed.assign(nc, 0);
		S.pre_area.assign(nc, 0.0f);
		S.merge_adj.assign(nc, {});
		if (!S.p.brute_force_raycast)
		{
			S.face_bvh.resize(m.num_objects);
			S.edge_bvh.resize(m.num_objects);
			parallel_for(m.num_objects * 2, [&](uint i)
				{
					const uint obj = i / 2;
					std::vector<uint> ids;
					if (i % 2 == 0)
					{
						for (uint f = m.prefix_faces[obj]; f < m.prefix_faces[obj + 1]; f++) ids.push_back(f);
						S.face_bvh[obj] = std::make_unique<CachedBVH>();
						S.face_bvh[obj]->build(ids, m, true);
					}
					else
					{
						for (uint e = m.prefix_edges[obj]; e < m.prefix_edges[obj + 1]; e++) ids.push_back(e);
						S.edge_bvh[obj] = std::make_unique<CachedBVH>();
						S.edge_bvh[obj]->build(ids, m, false);
					} }, 1);
		}
		std::vector<uint> active;
		const uint stride = std::max(1u, S.p.contour_stride);
		for (uint c = 0; c < nc && c < S.p.max_contours; c++)
			if (c % stride == S.p.contour_offset % stride)
				active.push_back(c);
		const uint bs = std::max(1u, S.p.batch_size);
		for (size_t b0 = 0; b0 < active.size(); b0 += bs)
		{
			std::vector<uint> batch(active.begin() + b0, active.begin() + std::min(active.size(), b0 + bs));
			parallel_for(uint(batch.size()), [&](uint i)
				{ init_runtime(S, S.rt[batch[i]], batch[i]); }, 1);
			evaluate_directions(S, batch);
			optimize_directions(S, batch, S.p.opt_iterations);
			// select_runtime_best_results + pre-finalize merge capture + finalize
			for (uint c : batch)
			{
				Runtime& r = S.rt[c];
				S.processed[c] = 1;
				int sel = -1;
				for (size_t ci = 0; ci < r.results.size(); ci++)
				{
					if (!has_valid(r.results[ci]))
						continue;
					if (sel < 0 || response_is_better(r.results[ci], r.results[sel]))
						sel = int(ci);
				}
				ComboInfo best;
				if (sel >= 0)
					best = r.results[sel];
				S.selected[c] = best;
				S.pre_area[c] = best.area;
				std::set<uint> adjc;
				for (const Hit& h : best.hits)
				{
					std::set<uint> t;
					adj_contours(S, h, c, t);
					for (uint o : t)
					{
						// same unordered object pair; a contour whose runtime was never built
						// (a later batch, or past max_contours) has no object ids yet and
						// never matches (contour_object_ids sentinel, resolver2.cpp:472-481)
						if (o == c || o >= nc || !S.rt[o].inited)
							continue;
						const Runtime& ro = S.rt[o];
						if (std::min(ro.object_ids[0], ro.object_ids[1]) == std::min(r.object_ids[0], r.object_ids[1])
							&& std::max(ro.object_ids[0], ro.object_ids[1]) == std::max(r.object_ids[0], r.object_ids[1]))
							adjc.insert(o);
					}
				}
				S.merge_adj[c].assign(adjc.begin(), adjc.end());
				// finalize: re-evaluate the selected support (identical arithmetic here)
				if (sel >= 0)
					fill_metrics(S, r, S.selected[c]);
			}
			for (uint c : batch)
			{
				Runtime& r = S.rt[c];
				r.hop[0].clear();
				r.hop[1].clear();
				r.geo[0].clear();
				r.geo[1].clear();
				r.cur_dist[0].clear();
				r.cur_dist[1].clear();
			}
		}
		suppress_contours(S.merge_adj, S.pre_area, active, S.suppressed);
		for (uint c = 0; c < nc; c++)
			if (S.suppressed[c])
				S.selected[c] = ComboInfo{};
	}

	// ---- response assembly (make_response_from_min_hitinfo, intersection_resolver2.cpp:2105-2221)
	// and region labels (host_apply_untangling_constraint, intersection_resolver2.cpp:2296-2427)
	struct PairTemplate // CollisionPair::CollisionPairTemplate, collision_data.h:48-140
	{
		uint idx[4];
		float vec1[4], vec2[4], vec3[4];
	};
	struct Response
	{
		std::vector<PairTemplate> pairs;
		std::vector<uint> info; // [pairs][4]: src id, dst id, packed region, type (0 VF, 1 FV, 2 EE)
		std::vector<uint> vert_csr, edge_csr, face_csr; // upload_2d_csr_from layout, buffer_allocator.h:26-59
	};

	// prp_classify_hit_solution (intersection_resolver2.cpp:37-107): 3 x sign code of the
	// source normal's projection on r + the target's; |q| <= 0.1 (or not finite) is 0
	uint solution_key(V3 n_src, V3 n_dst, V3 r)
	{
		const float rl = length(r), sl = length(n_src), dl = length(n_dst);
		const float sq = rl > 1e-12f && sl > 1e-12f ? dot(n_src / sl, r / rl) : 0.0f;
		const float dq = rl > 1e-12f && dl > 1e-12f ? dot(n_dst / dl, r / rl) : 0.0f;
		auto code = [](float q)
		{
			if (!std::isfinite(q) || std::fabs(q) <= 0.1f)
				return 1u;
			return q > 0.0f ? 2u : 0u;
		};
		return 3u * code(sq) + code(dq);
	}

	// region label of a response pair: 2 (256 contour + solution key) + source mesh role
	// (prp_pack_response_region_label, intersection_resolver2.cpp:112-121). The ray casts
	// create every hit with source role 0 (cached_bvh.cpp:271-277, 513).
	inline uint pack_region(uint contour, uint key, uint mesh) { return 2u * (256u * contour + (key & 255u)) + (mesh & 1u); }
	inline uint semantic_region(uint packed) { return 2u * ((packed >> 1) / 256u) + (packed & 1u); }

	std::vector<uint> csr_of(const std::vector<std::vector<uint>>& rows)
	{
		const uint n = uint(rows.size());
		std::vector<uint> out(n + 1);
		uint at = n + 1;
		for (uint i = 0; i < n; i++)
		{
			out[i] = at;
			at += uint(rows[i].size());
		}
		out[n] = at;
		for (const auto& r : rows)
			out.insert(out.end(), r.begin(), r.end());
		return out;
	}

	Response make_response(const Scene& S, float depth_threshold, float stiffness)
	{
		const MeshIn& m = S.m;
		Response R;
		for (uint c = 0; c < uint(S.selected.size()); c++)
		{
			const ComboInfo& ci = S.selected[c];
			const float C = std::max(-ci.depth - 3e-3f, -depth_threshold);
			for (const Hit& h : ci.hits)
			{
				PairTemplate t{};
				V3 n_src, n_dst, normal = ci.dir;
				float a_src, a_dst;
				uint type;
				if (h.type == VF)
				{
					n_src = S.vn[h.src_id];
					n_dst = S.fn[h.dst_id];
					a_src = m.rest_vert_area[h.src_id];
					a_dst = m.rest_face_area[h.dst_id];
					type = 0;
				}
				else if (h.type == FV)
				{
					n_src = S.fn[h.src_id];
					n_dst = S.vn[h.dst_id];
					a_src = m.rest_face_area[h.src_id];
					a_dst = m.rest_vert_area[h.dst_id];
					type = 1;
				}
				else
				{
					n_src = S.en[h.src_id];
					n_dst = S.en[h.dst_id];
					a_src = m.rest_edge_area[h.src_id];
					a_dst = m.rest_edge_area[h.dst_id];
					type = 2;
				}
				const uint region = pack_region(c, solution_key(n_src, n_dst, ci.dir), 0u);
				const float area = std::max(0.5f * (a_src + a_dst), 3e-6f);
				const float stiff = area * stiffness;
				float k1 = stiff * C, k2 = stiff;
				if (type == 0 && (!std::isfinite(k1) || !std::isfinite(k2)))
					k1 = k2 = 0.0f;
				if (type == 0)
				{
					t.idx[0] = h.sv[0];
					t.idx[1] = h.dv[0];
					t.idx[2] = h.dv[1] | 0x80000000u;
					t.idx[3] = h.dv[2];
				}
				else if (type == 1)
				{
					// the FV pair enters as a VF pair of the target vertex, normal reversed
					t.idx[0] = h.dv[0];
					t.idx[1] = h.sv[0];
					t.idx[2] = h.sv[1] | 0x80000000u;
					t.idx[3] = h.sv[2];
					normal = -1.0f * normal;
				}
				else
				{
					t.idx[0] = h.sv[0];
					t.idx[1] = h.sv[1];
					t.idx[2] = h.dv[0];
					t.idx[3] = h.dv[1] | 0x80000000u;
				}
				t.vec1[0] = normal.x;
				t.vec1[1] = normal.y;
				t.vec1[2] = normal.z;
				t.vec1[3] = area;
				t.vec2[0] = k1;
				t.vec2[1] = k2;
				t.vec2[2] = h.bary[0];
				t.vec2[3] = h.bary[1];
				R.pairs.push_back(t);
				const uint info[4] = { type == 2 ? h.src_id : h.vid(), type == 2 ? h.dst_id : h.fid(), region, type };
				R.info.insert(R.info.end(), info, info + 4);
			}
		}
		// vertex regions: each pair's 4 vertices (source side: its semantic region, target
		// side: the other mesh role) and each EF pair's edge / face vertices
		std::vector<std::vector<uint>> vr(m.num_verts), er(m.num_edges), fr(m.num_faces);
		for (size_t i = 0; i < R.pairs.size(); i++)
		{
			const uint r = semantic_region(R.info[4 * i + 2]), type = R.info[4 * i + 3];
			const uint lab[3][4] = { { r, r ^ 1u, r ^ 1u, r ^ 1u }, { r ^ 1u, r, r, r }, { r, r, r ^ 1u, r ^ 1u } };
			for (int k = 0; k < 4; k++)
				vr[R.pairs[i].idx[k] & 0x7fffffffu].push_back(lab[type][k]);
		}
		for (size_t p = 0; p < S.ef.size(); p++)
		{
			const uint er_ = 2u * S.contour_index[p] + S.mesh_index[p], fr_ = er_ ^ 1u;
			const uint e = S.ef_e[p], f = S.ef_f[p];
			vr[edge_of(m, e, 0)].push_back(er_);
			vr[edge_of(m, e, 1)].push_back(er_);
			for (int k = 0; k < 3; k++)
				vr[face_of(m, f, k)].push_back(fr_);
		}
		for (auto& r : vr)
		{
			std::sort(r.begin(), r.end());
			r.erase(std::unique(r.begin(), r.end()), r.end());
		}
		for (uint f = 0; f < m.num_faces; f++)
		{
			std::set<uint> u;
			for (int k = 0; k < 3; k++)
				u.insert(vr[face_of(m, f, k)].begin(), vr[face_of(m, f, k)].end());
			fr[f].assign(u.begin(), u.end());
		}
		for (uint e = 0; e < m.num_edges; e++)
		{
			std::set<uint> u;
			for (int k = 0; k < 2; k++)
				u.insert(vr[edge_of(m, e, k)].begin(), vr[edge_of(m, e, k)].end());
			er[e].assign(u.begin(), u.end());
		}
		R.vert_csr = csr_of(vr);
		R.edge_csr = csr_of(er);
		R.face_csr = csr_of(fr);
		return R;
	}
} // namespace

// ---- C ABI of the oracle (ctypes) --------------------------------------------------
struct OraclePrpResult
{
	uint contour_idx, contour_type, num_pairs, combo_idx;
	uint num_dirs, hit_count, unculled_hit_count, covered_anchor_count;
	uint boundary_anchor_count, eval_k_src, eval_k_dst, max_frontier_hop_src;
	uint max_frontier_hop_dst, expansion_level_count, flags, object_id0;
	uint object_id1, init_k_src, init_k_dst, diam_src;
	uint diam_dst, num_boundary_src, num_boundary_dst, opt_attempted;
	float dir[3];
	float depth, volume, objective, area, displacement_cost, coverage, normalized_objective, pre_finalize_area;
	uint opt_accepted;
};
static_assert(sizeof(OraclePrpResult) == 24 * 4 + 12 * 4, "result record");

struct OracleHitRec
{
	uint type, src_id, dst_id, sv[3], dv[3];
	float bary[2], dist;
};
static_assert(sizeof(OracleHitRec) == 48, "hit record");

extern "C"
{
	void* oracle_prp_run(const MeshIn* mesh, const void* ef_pairs, const uint* ef_indices, uint num_pairs, const Params* params)
	{
		Scene* S = new Scene();
		S->m = *mesh;
		S->p = *params;
		const EfPair* e = static_cast<const EfPair*>(ef_pairs);
		S->ef.assign(e, e + num_pairs);
		for (uint i = 0; i < num_pairs; i++)
		{
			S->ef_e.push_back(ef_indices[2 * i]);
			S->ef_f.push_back(ef_indices[2 * i + 1]);
		}
		run(*S);
		return S;
	}
	void oracle_prp_free(void* h) { delete static_cast<Scene*>(h); }
	uint oracle_prp_num_pairs(void* h) { return uint(static_cast<Scene*>(h)->ef.size()); }
	uint oracle_prp_num_orig_pairs(void* h) { return static_cast<Scene*>(h)->num_orig_pairs; }
	void oracle_prp_pairs(void* h, void* out_pairs, uint* out_idx, uint* out_mesh_index, uint* out_contour_index, float* out_len)
	{
		Scene* S = static_cast<Scene*>(h);
		for (size_t i = 0; i < S->ef.size(); i++)
		{
			static_cast<EfPair*>(out_pairs)[i] = S->ef[i];
			out_idx[2 * i] = S->ef_e[i];
			out_idx[2 * i + 1] = S->ef_f[i];
			out_mesh_index[i] = S->mesh_index[i];
			out_contour_index[i] = S->contour_index[i];
			out_len[i] = S->length[i];
		}
	}
	uint oracle_prp_num_contours(void* h) { return uint(static_cast<Scene*>(h)->contours.size()); }
	uint oracle_prp_contour(void* h, uint c, uint* out)
	{
		Scene* S = static_cast<Scene*>(h);
		const auto& v = S->contours[c];
		if (out)
			std::copy(v.begin(), v.end(), out);
		return uint(v.size());
	}
	void oracle_prp_result(void* h, uint c, OraclePrpResult* out)
	{
		Scene* S = static_cast<Scene*>(h);
		OraclePrpResult r{};
		const ComboInfo& s = S->selected[c];
		r.contour_idx = c;
		r.contour_type = S->contour_type[c];
		r.num_pairs = uint(S->contours[c].size());
		r.combo_idx = s.present && !s.hits.empty() ? s.combo_idx : 0xFFFFFFFFu;
		r.hit_count = uint(s.hits.size());
		r.unculled_hit_count = s.unculled;
		r.covered_anchor_count = s.covered;
		r.boundary_anchor_count = s.anchors;
		r.eval_k_src = s.eval_k_src;
		r.eval_k_dst = s.eval_k_dst;
		r.max_frontier_hop_src = s.max_front_src;
		r.max_frontier_hop_dst = s.max_front_dst;
		r.expansion_level_count = s.levels;
		const bool processed = c < S->processed.size() && S->processed[c];
		const Runtime& rt = S->rt[c];
		r.flags = (s.eligible ? 1u : 0u) | (processed && rt.no_response ? 2u : 0u) | (S->suppressed[c] ? 4u : 0u) | (s.full_mesh ? 8u : 0u) | (processed ? 16u : 0u);
		if (processed)
		{
			r.num_dirs = uint(rt.dirs.size());
			r.object_id0 = rt.object_ids[0];
			r.object_id1 = rt.object_ids[1];
			r.init_k_src = rt.init_k[0];
			r.init_k_dst = rt.init_k[1];
			r.diam_src = rt.diam[0];
			r.diam_dst = rt.diam[1];
			r.num_boundary_src = uint(rt.boundary[0].size());
			r.num_boundary_dst = uint(rt.boundary[1].size());
		}
		r.dir[0] = s.dir.x;
		r.dir[1] = s.dir.y;
		r.dir[2] = s.dir.z;
		r.depth = s.depth;
		r.volume = s.volume;
		r.objective = s.objective;
		r.area = s.area;
		r.displacement_cost = s.cost;
		r.coverage = s.coverage;
		r.normalized_objective = response_objective(s);
		r.pre_finalize_area = S->pre_area[c];
		r.opt_attempted = s.opt_attempted;
		r.opt_accepted = s.opt_accepted;
		*out = r;
	}
	uint oracle_prp_hits(void* h, uint c, OracleHitRec* out)
	{
		Scene* S = static_cast<Scene*>(h);
		const auto& hits = S->selected[c].hits;
		if (out)
			for (size_t i = 0; i < hits.size(); i++)
			{
				OracleHitRec& o = out[i];
				o.type = hits[i].type;
				o.src_id = hits[i].src_id;
				o.dst_id = hits[i].dst_id;
				for (int k = 0; k < 3; k++)
				{
					o.sv[k] = hits[i].sv[k];
					o.dv[k] = hits[i].dv[k];
				}
				o.bary[0] = hits[i].bary[0];
				o.bary[1] = hits[i].bary[1];
				o.dist = hits[i].dist;
			}
		return uint(hits.size());
	}
	uint oracle_prp_directions(void* h, uint c, float* out)
	{
		Scene* S = static_cast<Scene*>(h);
		const auto& d = S->rt[c].dirs;
		if (out)
			for (size_t i = 0; i < d.size(); i++)
			{
				out[3 * i] = d[i].x;
				out[3 * i + 1] = d[i].y;
				out[3 * i + 2] = d[i].z;
			}
		return uint(d.size());
	}
	void oracle_prp_stats(void* h, uint64_t* out2)
	{
		Scene* S = static_cast<Scene*>(h);
		out2[0] = S->tested;
		out2[1] = S->requests;
		out2[2] = S->pairs;
	}
	// FP64 recheck counts of the ray casts (fp64_recheck set): rechecked, flipped
	void oracle_prp_recheck(void* h, uint64_t* out2)
	{
		Scene* S = static_cast<Scene*>(h);
		out2[0] = S->rechecks;
		out2[1] = S->flips;
	}
	// The selected supports in FP64 (the double instantiation of prp_eval_penetration_v2's
	// depth, D_C and J, intersection_resolver2.cpp:1883-1954): per contour with a response,
	// out[c] = {J_64, D_C_64, max relative depth error, tie, flip} (tie: the two largest FP32
	// depths lie within 4 g D_C of each other; flip: the FP64 argmax is another hit), and
	// zeros elsewhere. Hits in canonical order; sums and maxima sequential in double.
	void oracle_prp_fp64(void* h, double* out5)
	{
		Scene* S = static_cast<Scene*>(h);
		const MeshIn& m = S->m;
		for (uint c = 0; c < uint(S->selected.size()); c++)
		{
			double* o = out5 + 5 * size_t(c);
			o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
			const ComboInfo& ci = S->selected[c];
			if (!ci.present || ci.hits.empty())
				continue;
			std::vector<Hit> hs = ci.hits;
			std::sort(hs.begin(), hs.end(), [](const Hit& a, const Hit& b)
				{ return a.type != b.type ? a.type < b.type : (a.src_id != b.src_id ? a.src_id < b.src_id : a.dst_id < b.dst_id); });
			// source areas summed as the kernel's warp does: 32 strided partial sums (hit i into
			// lane i % 32, in hit order), then the xor butterfly (lane l adds lane l ^ 16, ^ 8, ..., ^ 1)
			double lane_area[32] = { 0.0 };
			double dc64 = -1.0, derr = 0.0;
			float m32 = -1.0f, s32 = -1.0f;
			size_t arg32 = 0, arg64 = 0;
			for (size_t i = 0; i < hs.size(); i++)
			{
				const Hit& hh = hs[i];
				double d64;
				if (hh.type == EE)
				{
					const D3 p0 = d3(load3(m.x, m.edges[2 * hh.src_id])), p1 = d3(load3(m.x, m.edges[2 * hh.src_id + 1]));
					const D3 q0 = d3(load3(m.x, m.edges[2 * hh.dst_id])), q1 = d3(load3(m.x, m.edges[2 * hh.dst_id + 1]));
					const D3 n = crossd(p1 - p0, q1 - q0);
					const double det = -dotd(d3(ci.dir), n);
					d64 = det != 0.0 ? -dotd(q0 - p0, n) / det : double(hh.dist);
				}
				else
				{
					const bool fv = hh.type == FV;
					const uint v = fv ? hh.dst_id : hh.src_id, f = fv ? hh.src_id : hh.dst_id;
					const V3 orig = load3(m.x, v);
					const V3 end = orig + (fv ? -ci.dir : ci.dir) * 1.0f;
					D3 b64;
					double t64;
					d64 = seg_tri_f64(d3(orig), d3(end), d3(load3(m.x, m.faces[3 * f])), d3(load3(m.x, m.faces[3 * f + 1])),
							  d3(load3(m.x, m.faces[3 * f + 2])), b64, t64)
						? t64 * 1.0
						: double(hh.dist);
				}
				lane_area[i % 32] += double(hh.type == VF ? m.rest_vert_area[hh.src_id] : hh.type == EE ? m.rest_edge_area[hh.src_id] : m.rest_face_area[hh.src_id]);
				if (d64 > dc64)
				{
					dc64 = d64;
					arg64 = i;
				}
				if (hh.dist > m32)
				{
					s32 = m32;
					m32 = hh.dist;
					arg32 = i;
				}
				else if (hh.dist > s32)
					s32 = hh.dist;
				if (d64 > 0.0)
					derr = std::fmax(derr, std::fabs(double(hh.dist) - d64) / d64);
			}
			for (int off = 16; off > 0; off >>= 1)
			{
				double nv[32];
				for (int l = 0; l < 32; l++)
					nv[l] = lane_area[l] + lane_area[l ^ off];
				std::copy(nv, nv + 32, lane_area);
			}
			const double area = lane_area[0];
			const bool tie = hs.size() > 1 && m32 - s32 <= 4.0f * kGamma * m32;
			o[0] = area * dc64 * dc64;
			o[1] = dc64;
			o[2] = derr;
			o[3] = tie ? 1.0 : 0.0;
			o[4] = (tie && arg64 != arg32) ? 1.0 : 0.0;
		}
	}
	// Summation-order sensitivity of the selected supports' FP32 metrics: per contour with a
	// response, out[c] = the largest relative difference of area, volume, displacement cost and
	// J between the canonical order (the kernels' and this oracle's) and the reference's block
	// reduce over the hits in key order and in `nperm` seeded shuffles (the reference's hit order
	// at that point follows its ray-casting output); 0 elsewhere.
	void oracle_prp_order_spread(void* h, uint nperm, uint seed, double* out)
	{
		Scene* S = static_cast<Scene*>(h);
		auto rel = [](float a, float b)
		{ return a == b ? 0.0 : std::fabs(double(a) - double(b)) / std::fmax(std::fabs(double(a)), 1e-30); };
		for (uint c = 0; c < uint(S->selected.size()); c++)
		{
			out[c] = 0.0;
			const ComboInfo& ci = S->selected[c];
			if (!ci.present || ci.hits.empty())
				continue;
			std::vector<Hit> hs = ci.hits;
			std::sort(hs.begin(), hs.end(), [](const Hit& a, const Hit& b)
				{ return a.key() < b.key(); });
			const PenMetrics base = penetration_metrics(S->m, S->vn.data(), S->en.data(), S->fn.data(), ci.dir, hs);
			std::mt19937 rng(seed + c);
			double worst = 0.0;
			for (uint k = 0; k <= nperm; k++)
			{
				if (k > 0)
					std::shuffle(hs.begin(), hs.end(), rng);
				const PenMetrics r = penetration_metrics(S->m, S->vn.data(), S->en.data(), S->fn.data(), ci.dir, hs, true);
				worst = std::fmax(worst, std::fmax(std::fmax(rel(base.area, r.area), rel(base.volume, r.volume)),
											 std::fmax(rel(base.cost, r.cost), rel(base.objective, r.objective))));
			}
			out[c] = worst;
		}
	}
	// response pairs and region CSRs of a finished run; returns the pair count. Any output
	// may be null (sizes: pairs 64 B each, info 4 words each, CSRs *_len words).
	uint oracle_prp_response(void* h, float depth_threshold, float stiffness, void* pairs, uint* info, uint* vert_csr, uint* edge_csr,
		uint* face_csr, uint* lens3)
	{
		Scene* S = static_cast<Scene*>(h);
		const Response R = make_response(*S, depth_threshold, stiffness);
		if (pairs)
			std::memcpy(pairs, R.pairs.data(), R.pairs.size() * sizeof(PairTemplate));
		if (info)
			std::copy(R.info.begin(), R.info.end(), info);
		if (vert_csr)
			std::copy(R.vert_csr.begin(), R.vert_csr.end(), vert_csr);
		if (edge_csr)
			std::copy(R.edge_csr.begin(), R.edge_csr.end(), edge_csr);
		if (face_csr)
			std::copy(R.face_csr.begin(), R.face_csr.end(), face_csr);
		if (lens3)
		{
			lens3[0] = uint(R.vert_csr.size());
			lens3[1] = uint(R.edge_csr.size());
			lens3[2] = uint(R.face_csr.size());
		}
		return uint(R.pairs.size());
	}
	uint oracle_region_pack(uint contour, uint key, uint mesh) { return pack_region(contour, key, mesh); }
	uint oracle_region_semantic(uint packed) { return semantic_region(packed); }
	uint oracle_solution_key(const float* n_src, const float* n_dst, const float* r)
	{
		return solution_key(v3(n_src[0], n_src[1], n_src[2]), v3(n_dst[0], n_dst[1], n_dst[2]), v3(r[0], r[1], r[2]));
	}
	void oracle_eigen3(const float* S9, float* out9)
	{
		Mat3 S;
		for (int c = 0; c < 3; c++)
			S.c[c] = v3(S9[3 * c], S9[3 * c + 1], S9[3 * c + 2]);
		V3 ev[3];
		all_eigenvectors(S, ev);
		for (int k = 0; k < 3; k++)
		{
			out9[3 * k] = ev[k].x;
			out9[3 * k + 1] = ev[k].y;
			out9[3 * k + 2] = ev[k].z;
		}
	}

	// ---- unit entry points of the PRP decision rules (known-answer tests) ----

	int oracle_ccr_owns(float own, float opp, float tau) { return owns_1(own, opp, tau) ? 1 : 0; }
	int oracle_ccr_owns_dual(float ro, float rp, float co, float cp, float tau, int use_rest, int use_cur)
	{
		return owns_dual(ro, rp, co, cp, tau, use_rest != 0, use_cur != 0) ? 1 : 0;
	}
	int oracle_ccr_owns_blended(float ro, float rp, float co, float cp, float tau, float w) { return owns_blended(ro, rp, co, cp, tau, w) ? 1 : 0; }
	float oracle_ccr_blended_phi(float ro, float rp, float co, float cp, float w) { return blended_phi(ro, rp, co, cp, w); }
	int oracle_ccr_roles_share(uint o0, uint o1, uint c0, uint c1)
	{
		const uint o[2] = { o0, o1 }, c[2] = { c0, c1 };
		return roles_share_topology(o, c) ? 1 : 0;
	}
	int oracle_ccr_applies(int enabled, uint o0, uint o1, uint c0, uint c1, int use_deformed)
	{
		const uint o[2] = { o0, o1 }, c[2] = { c0, c1 };
		return ccr_applies(enabled != 0, o, c, use_deformed != 0) ? 1 : 0;
	}

	struct OracleResp
	{
		float objective, coverage, depth, cost;
		uint hit_count, covered, eligible, pad;
	};
	static ComboInfo combo_from(const OracleResp& q, uint idx)
	{
		ComboInfo c;
		c.present = true;
		c.combo_idx = idx;
		c.objective = q.objective;
		c.coverage = q.coverage;
		c.depth = q.depth;
		c.cost = q.cost;
		c.hit_count = q.hit_count;
		c.hits.resize(q.hit_count);
		c.covered = q.covered;
		c.anchors = q.covered;
		c.eligible = q.eligible != 0;
		return c;
	}
	// prp_select_response: index of the best valid response, -1 when none
	int oracle_select_response(uint n, const OracleResp* q)
	{
		std::vector<ComboInfo> v;
		for (uint i = 0; i < n; i++)
			v.push_back(combo_from(q[i], i));
		int sel = -1;
		for (uint i = 0; i < n; i++)
		{
			if (!has_valid(v[i]))
				continue;
			if (sel < 0 || response_is_better(v[i], v[sel]))
				sel = int(i);
		}
		return sel;
	}
	float oracle_response_objective(float objective, float coverage) { return objective_div_cov2(objective, coverage); }

	// flood_components over a CSR graph (row_ptr[n + 1], col[m], flip[m]): root[i] = the seed
	// (smallest node) of i's component, parity[i]; returns 1 when some component is inconsistent
	uint oracle_flood_components(uint n, const uint* row_ptr, const uint* col, const uint* flip, uint* root, uint* parity)
	{
		std::vector<std::vector<uint>> adj(n), w(n);
		for (uint u = 0; u < n; u++)
			for (uint e = row_ptr[u]; e < row_ptr[u + 1]; e++)
			{
				adj[u].push_back(col[e]);
				w[u].push_back(flip[e] & 1u);
			}
		std::vector<uint> par;
		std::vector<std::vector<uint>> comps;
		const bool bad = flood_components(n, adj, w, par, comps);
		for (const auto& c : comps)
			for (uint p : c)
				root[p] = c.front();
		for (uint i = 0; i < n; i++)
			parity[i] = par[i];
		return bad ? 1u : 0u;
	}
	uint oracle_classify_contour(uint n, const uint8_t* is_loop, const uint8_t* is_bnd, const uint* deg, const uint* mesh_index)
	{
		return classify_contour(n, is_loop, is_bnd, deg, mesh_index);
	}

	void oracle_suppress(uint nc, const uint* adj_off, const uint* adj, const float* pre_area, uint nactive, const uint* active, uint8_t* out)
	{
		std::vector<std::vector<uint>> m(nc);
		for (uint c = 0; c < nc; c++)
			m[c].assign(adj + adj_off[c], adj + adj_off[c + 1]);
		std::vector<float> area(pre_area, pre_area + nc);
		std::vector<uint> act(active, active + nactive);
		std::vector<uint8_t> sup(nc, 0);
		suppress_contours(m, area, act, sup);
		std::memcpy(out, sup.data(), nc);
	}

	static std::vector<Hit> hits_from(uint n, const OracleHitRec* h)
	{
		std::vector<Hit> v(n);
		for (uint i = 0; i < n; i++)
		{
			v[i].type = h[i].type;
			v[i].src_id = h[i].src_id;
			v[i].dst_id = h[i].dst_id;
			for (int k = 0; k < 3; k++)
			{
				v[i].sv[k] = h[i].sv[k];
				v[i].dv[k] = h[i].dv[k];
			}
			v[i].bary[0] = h[i].bary[0];
			v[i].bary[1] = h[i].bary[1];
			v[i].dist = h[i].dist;
		}
		return v;
	}

	// prp_eval_penetration_v2 on a hit list: out = depth, volume, area, objective, cost
	void oracle_penetration(uint n, const OracleHitRec* hits, const float* dir, uint nv, uint ne, uint nf, const float* vert_area,
		const float* edge_area, const float* face_area, const float* vert_mass, const float* vn, const float* en, const float* fn, float* out5)
	{
		MeshIn m{};
		m.num_verts = nv;
		m.num_edges = ne;
		m.num_faces = nf;
		m.rest_vert_area = vert_area;
		m.rest_edge_area = edge_area;
		m.rest_face_area = face_area;
		m.vert_mass = vert_mass;
		auto v3s = [](const float* p, uint k)
		{
			std::vector<V3> r(k);
			for (uint i = 0; i < k; i++)
				r[i] = v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
			return r;
		};
		const std::vector<V3> VN = v3s(vn, nv), EN = v3s(en, ne), FN = v3s(fn, nf);
		std::vector<Hit> H = hits_from(n, hits);
		std::sort(H.begin(), H.end(), [](const Hit& a, const Hit& b)
			{ return a.key() < b.key(); });
		const PenMetrics pm = penetration_metrics(m, VN.data(), EN.data(), FN.data(), v3(dir[0], dir[1], dir[2]), H);
		out5[0] = pm.depth;
		out5[1] = pm.volume;
		out5[2] = pm.area;
		out5[3] = pm.objective;
		out5[4] = pm.cost;
	}

	// get_raycasting_direction on explicit inputs; returns the direction count (<= 26)
	uint oracle_seed_directions(uint mode, uint npts, const float* pts, const float* w, uint nb0, const uint* b0, uint nb1, const uint* b1,
		uint nv, const float* x, const float* vert_area, float* out)
	{
		std::vector<V3> P(npts);
		std::vector<float> W(w, w + npts);
		for (uint i = 0; i < npts; i++)
			P[i] = v3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
		std::vector<uint> B[2] = { std::vector<uint>(b0, b0 + nb0), std::vector<uint>(b1, b1 + nb1) };
		const std::vector<V3> d = seed_directions(mode, P, W, B, x, vert_area, nv);
		for (size_t i = 0; i < d.size() && i < 26; i++)
		{
			out[3 * i] = d[i].x;
			out[3 * i + 1] = d[i].y;
			out[3 * i + 2] = d[i].z;
		}
		return uint(std::min<size_t>(d.size(), 26));
	}

	struct OracleKInfo
	{
		uint hit_count, covered, anchors, mfs, mfd, eligible;
		float objective, coverage;
	};
	typedef int (*OracleKEval)(uint level, uint k_src, uint k_dst, uint combo, OracleKInfo* out);

	// The adaptive k-ring control of one runtime with a scripted evaluator (cb). cached holds
	// the stored results of inactive directions (or null). trace receives (k_src, k_dst) of
	// every level; state = finished, no_response, evaluations, levels; eligible per direction.
	void oracle_kring_trace(const uint* init_k, const uint* diam, uint ndirs, const uint8_t* active, const OracleKInfo* cached, OracleKEval cb,
		uint* trace, uint max_levels, uint* state, uint8_t* eligible)
	{
		Runtime r;
		r.dirs.assign(ndirs, v3(0.0f, 1.0f, 0.0f));
		r.results.assign(ndirs, ComboInfo{});
		r.converged.assign(ndirs, 0);
		r.pruned.assign(ndirs, 0);
		r.present.assign(ndirs, 0);
		r.active.assign(active, active + ndirs);
		r.init_k[0] = init_k[0];
		r.init_k[1] = init_k[1];
		r.diam[0] = diam[0];
		r.diam[1] = diam[1];
		auto to_info = [](const OracleKInfo& q, uint combo)
		{
			ComboInfo c;
			c.present = true;
			c.combo_idx = combo;
			c.hit_count = q.hit_count;
			c.hits.resize(q.hit_count);
			c.covered = q.covered;
			c.anchors = q.anchors;
			c.max_front_src = q.mfs;
			c.max_front_dst = q.mfd;
			c.objective = q.objective;
			c.coverage = q.coverage;
			c.eligible = q.eligible != 0;
			return c;
		};
		if (cached)
			for (uint d = 0; d < ndirs; d++)
				if (!r.active[d])
				{
					r.results[d] = to_info(cached[d], d);
					r.present[d] = 1;
				}
		uint levels = 0, evals = 0;
		std::vector<Runtime*> rts{ &r };
		kring_levels(
			rts, [&](const std::vector<Runtime*>&)
			{
				if (levels < max_levels)
				{
					trace[2 * levels] = r.k[0];
					trace[2 * levels + 1] = r.k[1];
				}
				levels++; },
			[&](Runtime& rr, uint combo)
			{
				OracleKInfo q{};
				cb(levels - 1, rr.k[0], rr.k[1], combo, &q);
				evals++;
				return to_info(q, combo);
			},
			false);
		state[0] = r.finished ? 1 : 0;
		state[1] = r.no_response ? 1 : 0;
		state[2] = evals;
		state[3] = levels;
		for (uint d = 0; d < ndirs; d++)
			eligible[d] = r.results[d].eligible ? 1 : 0;
	}

	// prp_compute_direction_optimization_step: out = dir[3], predicted reduction, gradient norm, valid
	void oracle_direction_step(uint n, const OracleHitRec* hits, uint nv, const float* x, const float* vert_mass, const float* dir, float trust,
		float* out6)
	{
		MeshIn m{};
		m.num_verts = nv;
		m.x = x;
		m.vert_mass = vert_mass;
		std::vector<Hit> H = hits_from(n, hits);
		std::sort(H.begin(), H.end(), [](const Hit& a, const Hit& b)
			{ return a.key() < b.key(); });
		const DirStep st = direction_step(m, H, v3(dir[0], dir[1], dir[2]), trust);
		out6[0] = st.dir.x;
		out6[1] = st.dir.y;
		out6[2] = st.dir.z;
		out6[3] = st.predicted;
		out6[4] = st.gnorm;
		out6[5] = st.valid ? 1.0f : 0.0f;
	}
}
