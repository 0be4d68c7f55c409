// Test infrastructure (oracle): CPU restatement of the reference LBVH.
//   Solver/CollisionDetector/lbvh.cpp  (global AABB 372-452, 454-496, 988-1021;
//   Morton 84-135, 512-528; sort 1023-1047; Karras 206-293, 546-601; leaf AABB
//   621-688; refit 694-758; query 295-363, 780-894) and aabb.h:94-98.
// Loaded only by tests/ and bench.py's cpu_baseline leg.
#include "oracle_common.h"

namespace u26o
{
	int oracle_threads()
	{
		const char* env = std::getenv("U26_ORACLE_THREADS");
		if (env != nullptr)
			return std::max(1, std::atoi(env));
		unsigned hc = std::thread::hardware_concurrency();
		return hc == 0 ? 1 : int(hc);
	}

	void parallel_for(uint n, const std::function<void(uint)>& fn, uint block)
	{
		const int nthreads = oracle_threads();
		if (n == 0)
			return;
		if (nthreads <= 1 || n <= block)
		{
			for (uint i = 0; i < n; i++)
				fn(i);
			return;
		}
		std::atomic<uint> next{ 0 };
		auto worker = [&]()
		{
			for (;;)
			{
				const uint begin = next.fetch_add(block);
				if (begin >= n)
					break;
				const uint end = std::min(n, begin + block);
				for (uint i = begin; i < end; i++)
					fn(i);
			}
		};
		std::vector<std::thread> pool;
		for (int t = 1; t < nthreads; t++)
			pool.emplace_back(worker);
		worker();
		for (auto& t : pool)
			t.join();
	}
} // namespace u26o

using namespace u26o;

namespace
{
	enum TreeType
	{
		kVert = 0,
		kFace = 1,
		kEdge = 2
	};

	inline uint prim_arity(int tree_type) { return tree_type == kFace ? 3u : (tree_type == kEdge ? 2u : 1u); }

	inline uint prim_vert(int tree_type, const uint* prims, uint pid, uint k)
	{
		return tree_type == kVert ? pid : prims[prim_arity(tree_type) * pid + k];
	}

	// lbvh.cpp:88-95
	inline uint expand_bits(uint v)
	{
		v = (v | (v << 16)) & 0x030000FFu;
		v = (v | (v << 8)) & 0x0300F00Fu;
		v = (v | (v << 4)) & 0x030C30C3u;
		return (v | (v << 2)) & 0x09249249u;
	}

	inline float clampf(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }

	// lbvh.cpp:115-126: 10 bits per axis, x*1024 clamped to [0, 1023] then truncated.
	inline uint morton32(V3 p)
	{
		const float x = clampf(p.x * 1024.0f, 0.0f, 1023.0f);
		const float y = clampf(p.y * 1024.0f, 0.0f, 1023.0f);
		const float z = clampf(p.z * 1024.0f, 0.0f, 1023.0f);
		return (expand_bits(uint(x)) << 2) | (expand_bits(uint(y)) << 1) | expand_bits(uint(z));
	}

	inline uint64_t morton64(V3 p, uint index) { return (uint64_t(morton32(p)) << 32) | uint64_t(index); }

	// Leaf centre and primitive AABB as the reduce kernels form them (lbvh.cpp:454-496).
	inline void leaf_center_aabb(int tree_type, const float* x, const uint* prims, uint lid, V3& c, V3& mn, V3& mx)
	{
		if (tree_type == kFace)
		{
			const V3 a = load3(x, prims[3 * lid + 0]), b = load3(x, prims[3 * lid + 1]), d = load3(x, prims[3 * lid + 2]);
			c = 0.333333f * ((a + b) + d);
			mn = vmin(a, vmin(b, d));
			mx = vmax(a, vmax(b, d));
		}
		else if (tree_type == kEdge)
		{
			const V3 a = load3(x, prims[2 * lid + 0]), b = load3(x, prims[2 * lid + 1]);
			c = 0.5f * (a + b);
			mn = vmin(a, b);
			mx = vmax(a, b);
		}
		else
		{
			c = load3(x, lid);
			mn = c;
			mx = c;
		}
	}

	inline int clz64(uint64_t v) { return v == 0 ? 64 : __builtin_clzll(v); }

	// lbvh.cpp:183-193: common prefix of key i with key j, -1 outside [0, n).
	inline int cp_ij(const uint64_t* keys, uint64_t mi, int j, int n)
	{
		if (j < 0 || j >= n)
			return -1;
		return clz64(mi ^ keys[j]);
	}

	// lbvh.cpp:206-246
	inline void determine_range(const uint64_t* keys, int n, int i, int& out_i, int& out_j)
	{
		const uint64_t mi = keys[i];
		const int cp_left = cp_ij(keys, mi, i - 1, n);
		const int cp_right = cp_ij(keys, mi, i + 1, n);
		const int d = cp_left < cp_right ? 1 : -1;
		const int cp_min = std::min(cp_left, cp_right);
		int lmax = 2;
		while (cp_ij(keys, mi, i + lmax * d, n) > cp_min)
			lmax <<= 1;
		int l = 0;
		for (int t = lmax >> 1; t >= 1; t >>= 1)
			if (cp_ij(keys, mi, i + (l + t) * d, n) > cp_min)
				l += t;
		out_i = i;
		out_j = i + l * d;
	}

	// lbvh.cpp:248-293
	inline int find_split(const uint64_t* keys, int ri, int rj)
	{
		int i = ri, j = rj;
		if (!(ri < rj))
			std::swap(i, j);
		const uint64_t mi = keys[i], mj = keys[j];
		const int cp_node = clz64(mi ^ mj);
		if (mi == mj)
			return (i + j) >> 1;
		int t = j - i;
		int split = i;
		for (;;)
		{
			t = (t + 1) >> 1;
			const int ns = split + t;
			if (ns < j && clz64(mi ^ keys[ns]) > cp_node)
				split = ns;
			if (!(t > 1))
				break;
		}
		return split;
	}

	// aabb.h:94-98: strict overlap on all three axes.
	inline bool overlap(const float* node_aabb, V3 qmn, V3 qmx)
	{
		return node_aabb[0] < qmx.x && node_aabb[1] < qmx.y && node_aabb[2] < qmx.z && node_aabb[4] > qmn.x && node_aabb[5] > qmn.y && node_aabb[6] > qmn.z;
	}
} // namespace

extern "C"
{
	// Global AABB with the reference's second-pass quirk: only the first
	// ceil(num_verts/256) blocks of 256 leaves are reduced (lbvh.cpp:999-1021; the vert
	// tree reduces every block). Blocks past the leaf count are clamped away.
	void oracle_lbvh_global_aabb(int tree_type, const float* x, uint num_verts, const uint* prims, uint n, float* out6)
	{
		const uint nblocks_leaf = (n + 255u) / 256u;
		const uint nblocks_ref = (num_verts + 255u) / 256u;
		const uint nblocks = tree_type == kVert ? nblocks_leaf : std::min(nblocks_leaf, nblocks_ref);
		const uint last = std::min(n, nblocks * 256u);
		V3 gmn = v3(0.0f), gmx = v3(0.0f);
		for (uint lid = 0; lid < last; lid++)
		{
			V3 c, mn, mx;
			leaf_center_aabb(tree_type, x, prims, lid, c, mn, mx);
			if (lid == 0)
			{
				gmn = mn;
				gmx = mx;
			}
			else
			{
				gmn = vmin(gmn, mn);
				gmx = vmax(gmx, mx);
			}
		}
		out6[0] = gmn.x;
		out6[1] = gmn.y;
		out6[2] = gmn.z;
		out6[3] = gmx.x;
		out6[4] = gmx.y;
		out6[5] = gmx.z;
	}

	// Morton keys (lbvh.cpp:512-528) from the global AABB.
	void oracle_lbvh_mortons(int tree_type, const float* x, const uint* prims, uint n, const float* gaabb, uint64_t* keys)
	{
		const V3 mn = v3(gaabb[0], gaabb[1], gaabb[2]);
		const V3 mx = v3(gaabb[3], gaabb[4], gaabb[5]);
		const V3 ext = vmax(mx - mn, v3(1e-6f));
		const V3 inv = v3(1.0f / ext.x, 1.0f / ext.y, 1.0f / ext.z);
		parallel_for(n, [&](uint lid)
			{
				V3 c, a, b;
				leaf_center_aabb(tree_type, x, prims, lid, c, a, b);
				const V3 np = (c - mn) * inv;
				keys[lid] = morton64(np, lid); });
	}

	// Karras inner nodes over sorted keys (lbvh.cpp:546-601). Node layout: inner
	// [0, n-2], leaves [n-1, 2n-2]; parent[0] = ~0.
	void oracle_lbvh_karras(const uint64_t* keys_sorted, uint n, uint* parent, uint* children)
	{
		const int num_inner = int(n) - 1;
		if (n == 0)
			return;
		parent[0] = ~0u;
		for (int nid = 0; nid < num_inner; nid++)
		{
			int i = 0, j = num_inner;
			if (nid != 0)
				determine_range(keys_sorted, int(n), nid, i, j);
			const int split = find_split(keys_sorted, i, j);
			int cl = (std::min(i, j) == split) ? num_inner + split : split;
			int cr = (std::max(i, j) == split + 1) ? num_inner + split + 1 : split + 1;
			if (cr >= num_inner)
				std::swap(cl, cr);
			parent[cl] = uint(nid);
			parent[cr] = uint(nid);
			children[2 * nid + 0] = uint(cl);
			children[2 * nid + 1] = uint(cr);
		}
	}

	// Whole construct_tree (lbvh.cpp:1023-1047): global AABB, Morton keys, sort by key,
	// leaves, Karras. Outputs per node arrays of size 2n-1 and per leaf arrays of size n.
	int oracle_lbvh_build(int tree_type, const float* x, uint num_verts, const uint* prims, uint n,
		float* gaabb6, uint64_t* keys_sorted, uint* sorted_get_original, uint* parent, uint* children, uint* object_idx)
	{
		if (n == 0)
			return 0;
		oracle_lbvh_global_aabb(tree_type, x, num_verts, prims, n, gaabb6);
		std::vector<uint64_t> keys(n);
		oracle_lbvh_mortons(tree_type, x, prims, n, gaabb6, keys.data());
		std::vector<uint> order(n);
		for (uint i = 0; i < n; i++)
			order[i] = i;
		std::sort(order.begin(), order.end(), [&](uint a, uint b)
			{ return keys[a] < keys[b]; });
		const uint num_inner = n - 1;
		const uint num_nodes = 2 * n - 1;
		for (uint i = 0; i < num_nodes; i++)
			object_idx[i] = ~0u;
		for (uint lid = 0; lid < n; lid++)
		{
			sorted_get_original[lid] = order[lid];
			keys_sorted[lid] = keys[order[lid]];
			children[2 * (num_inner + lid) + 0] = order[lid];
			children[2 * (num_inner + lid) + 1] = order[lid];
			object_idx[num_inner + lid] = order[lid];
		}
		oracle_lbvh_karras(keys_sorted, n, parent, children);
		// fn_check_construction (lbvh.cpp:603-616)
		for (uint nid = 0; nid < num_inner; nid++)
			if (parent[children[2 * nid]] != nid || parent[children[2 * nid + 1]] != nid)
				return 1;
		return 0;
	}

	// Leaf AABBs (lbvh.cpp:621-688) and the bottom-up union (lbvh.cpp:694-758). node_aabb
	// is float[8] per node: (min.xyz, 0, max.xyz, 0); the refit flags of the .w lanes are
	// not restated. Union by min/max is exact, so the result is order independent.
	void oracle_lbvh_refit(int tree_type, uint n, const float* x0, const float* x1, const float* thickness,
		const uint* prims, const uint* sorted_get_original, const uint* children, float* node_aabb)
	{
		if (n == 0)
			return;
		const uint num_inner = n - 1;
		const uint k = prim_arity(tree_type);
		parallel_for(n, [&](uint lid)
			{
				const uint pid = sorted_get_original[lid];
				V3 mn = v3(0.0f), mx = v3(0.0f);
				if (tree_type == kFace)
				{
					const uint a = prims[3 * pid], b = prims[3 * pid + 1], c = prims[3 * pid + 2];
					const V3 s0 = load3(x0, a), s1 = load3(x0, b), s2 = load3(x0, c);
					const V3 e0 = load3(x1, a), e1 = load3(x1, b), e2 = load3(x1, c);
					const V3 smn = vmin(s0, vmin(s1, s2)), smx = vmax(s0, vmax(s1, s2));
					const V3 emn = vmin(e0, vmin(e1, e2)), emx = vmax(e0, vmax(e1, e2));
					mn = vmin(smn, emn);
					mx = vmax(smx, emx);
				}
				else if (tree_type == kEdge)
				{
					const uint a = prims[2 * pid], b = prims[2 * pid + 1];
					const V3 s0 = load3(x0, a), s1 = load3(x0, b), e0 = load3(x1, a), e1 = load3(x1, b);
					mn = vmin(vmin(s0, s1), vmin(e0, e1));
					mx = vmax(vmax(s0, s1), vmax(e0, e1));
				}
				else
				{
					const V3 s0 = load3(x0, pid), e0 = load3(x1, pid);
					mn = vmin(s0, e0);
					mx = vmax(s0, e0);
				}
				const float t = thickness[prim_vert(tree_type, prims, pid, 0)];
				mn = mn - v3(t);
				mx = mx + v3(t);
				float* o = node_aabb + 8 * (num_inner + lid);
				o[0] = mn.x; o[1] = mn.y; o[2] = mn.z; o[3] = 0.0f;
				o[4] = mx.x; o[5] = mx.y; o[6] = mx.z; o[7] = 0.0f; });
		(void)k;
		// Post-order union from the root.
		if (num_inner == 0)
			return;
		std::vector<uint> stack;
		std::vector<uint8_t> state(num_inner, 0);
		stack.push_back(0);
		while (!stack.empty())
		{
			const uint nid = stack.back();
			if (state[nid] == 0)
			{
				state[nid] = 1;
				for (int c = 1; c >= 0; c--)
				{
					const uint ch = children[2 * nid + c];
					if (ch < num_inner)
						stack.push_back(ch);
				}
				continue;
			}
			stack.pop_back();
			const float* l = node_aabb + 8 * children[2 * nid];
			const float* r = node_aabb + 8 * children[2 * nid + 1];
			float* o = node_aabb + 8 * nid;
			for (int a = 0; a < 3; a++)
			{
				o[a] = std::fmin(l[a], r[a]);
				o[4 + a] = std::fmax(l[4 + a], r[4 + a]);
			}
			o[3] = 0.0f;
			o[7] = 0.0f;
		}
	}

	// Stack-32 traversal (lbvh.cpp:295-363). Query AABB per mode:
	//   mode 0 verts:   AABB(x0[v], x1[v]) +- (thickness[v] + d_hat[v]), all leaves
	//   mode 1 edges:   AABB of both edge ends at x0, x1 +- (thickness[e0] + d_hat[e0]), keep eid < adj
	//   mode 2 edges unculled: as mode 1, keep every leaf
	// Pairs are (query id, leaf object id), grouped by query id in traversal order.
	// Returns the total number found (can exceed max_pairs; extra pairs are dropped).
	// overflow_out (optional) receives the number of queries whose stack overflowed.
	uint64_t oracle_lbvh_query(int mode, uint num_queries, const float* x0, const float* x1, const uint* edges,
		const float* d_hat, const float* thickness, uint n, const uint* children, const uint* object_idx,
		const float* node_aabb, uint* pairs, uint64_t max_pairs, uint* overflow_out)
	{
		std::vector<std::vector<uint>> per(num_queries);
		std::atomic<uint> overflow{ 0 };
		parallel_for(num_queries, [&](uint q)
			{
				V3 mn, mx;
				float pad;
				if (mode == 0)
				{
					const V3 a = load3(x0, q), b = load3(x1, q);
					mn = vmin(a, b);
					mx = vmax(a, b);
					pad = thickness[q] + d_hat[q];
				}
				else
				{
					const uint e0 = edges[2 * q], e1 = edges[2 * q + 1];
					const V3 p1 = load3(x0, e0), p2 = load3(x0, e1), p3 = load3(x1, e0), p4 = load3(x1, e1);
					mn = vmin(vmin(p1, p2), vmin(p3, p4));
					mx = vmax(vmax(p1, p2), vmax(p3, p4));
					pad = thickness[e0] + d_hat[e0];
				}
				mn = mn - v3(pad);
				mx = mx + v3(pad);
				auto& out = per[q];
				uint stack[32];
				int sp = 0;
				stack[sp++] = 0u;
				uint loop = 0;
				bool stop = false;
				while (sp > 0 && !stop)
				{
					const uint node = stack[--sp];
					for (int ii = 0; ii < 2 && !stop; ii++)
					{
						const uint cs = children[2 * node + ii];
						if (overlap(node_aabb + 8 * cs, mn, mx))
						{
							const uint adj = object_idx[cs];
							if (adj != ~0u)
							{
								const bool valid = mode == 1 ? (q < adj) : true;
								if (valid)
								{
									out.push_back(q);
									out.push_back(adj);
								}
							}
							else if (sp < 32)
								stack[sp++] = cs;
							else
							{
								stop = true;
								overflow.fetch_add(1);
							}
						}
					}
					loop += 1;
					if (loop > 100000)
						stop = true;
				}
			});
		uint64_t total = 0;
		for (uint q = 0; q < num_queries; q++)
		{
			for (size_t i = 0; i + 1 < per[q].size(); i += 2)
			{
				if (total < max_pairs)
				{
					pairs[2 * total] = per[q][i];
					pairs[2 * total + 1] = per[q][i + 1];
				}
				total++;
			}
		}
		if (overflow_out)
			*overflow_out = overflow.load();
		(void)n;
		return total;
	}

	// Standalone Morton helpers for the reference's unit test (lbvh.cpp:920-984).
	uint oracle_morton32(float px, float py, float pz) { return morton32(v3(px, py, pz)); }
	uint64_t oracle_morton64(float px, float py, float pz, uint index) { return morton64(v3(px, py, pz), index); }
	void oracle_determine_range(const uint64_t* keys, uint n, uint i, int* out_ij)
	{
		determine_range(keys, int(n), int(i), out_ij[0], out_ij[1]);
	}
	int oracle_find_split(const uint64_t* keys, int i, int j) { return find_split(keys, i, j); }
	int oracle_threads_used() { return oracle_threads(); }
}
