// LBVH build / refit / broad-phase query on sm_100a.
//
// Reference: Solver/CollisionDetector/lbvh.cpp. Construction: global AABB
// (372-452, 454-496, 988-1021), Morton keys (84-135, 512-528), sort (1037-1040, here a
// device radix sort), Karras emission (206-293, 546-601), check (603-616). Refit:
// leaf AABBs (621-688) and the bottom-up union (694-758), here with a per-node arrival
// counter instead of the reference's float-CAS flags and spin-waits: the second thread
// to reach a node owns it, so no thread ever waits on another. Query: stack-32
// traversal with strict overlap (295-363, 780-894), in the reference's visit order so
// that the stack-overflow cut-off drops the same pairs.
#include <algorithm>

#include <cuda/atomic>

#include "lbvh_internal.h"

namespace u26
{
	namespace
	{
		template <int TYPE>
		__device__ __forceinline__ void prim_center_aabb(const float* __restrict__ x, const uint32_t* __restrict__ prims, uint32_t lid,
			f3& c, f3& mn, f3& mx)
		{
			if constexpr (TYPE == U26_TREE_FACE)
			{
				const uint32_t a = __ldg(prims + 3 * lid), b = __ldg(prims + 3 * lid + 1), d = __ldg(prims + 3 * lid + 2);
				const f3 pa = ld3(x, a), pb = ld3(x, b), pd = ld3(x, d);
				c = 0.333333f * ((pa + pb) + pd);
				mn = vmin(pa, vmin(pb, pd));
				mx = vmax(pa, vmax(pb, pd));
			}
			else if constexpr (TYPE == U26_TREE_EDGE)
			{
				const uint32_t a = __ldg(prims + 2 * lid), b = __ldg(prims + 2 * lid + 1);
				const f3 pa = ld3(x, a), pb = ld3(x, b);
				c = 0.5f * (pa + pb);
				mn = vmin(pa, pb);
				mx = vmax(pa, pb);
			}
			else
			{
				c = ld3(x, lid);
				mn = c;
				mx = c;
			}
		}

		__device__ __forceinline__ float warp_min(float v)
		{
#pragma unroll
			for (int o = 16; o > 0; o >>= 1)
				v = fminf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
			return v;
		}
		__device__ __forceinline__ float warp_max(float v)
		{
#pragma unroll
			for (int o = 16; o > 0; o >>= 1)
				v = fmaxf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
			return v;
		}

		// Per-256 block AABB of the primitives (fn_reduce_*_tree_global_aabb). Lanes past n
		// contribute +-inf, which leaves the block AABB of the valid leaves unchanged.
		template <int TYPE>
		__global__ void __launch_bounds__(256) reduce_blocks_kernel(const float* __restrict__ x, const uint32_t* __restrict__ prims,
			uint32_t n, float* __restrict__ block_aabb)
		{
			__shared__ float s[6][8];
			const uint32_t lid = blockIdx.x * 256u + threadIdx.x;
			f3 mn = mk3(INFINITY), mx = mk3(-INFINITY);
			if (lid < n)
			{
				f3 c;
				prim_center_aabb<TYPE>(x, prims, lid, c, mn, mx);
			}
			float v[6] = { warp_min(mn.x), warp_min(mn.y), warp_min(mn.z), warp_max(mx.x), warp_max(mx.y), warp_max(mx.z) };
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			if (lane == 0)
				for (int k = 0; k < 6; k++)
					s[k][warp] = v[k];
			__syncthreads();
			if (warp == 0)
			{
				float r[6];
				for (int k = 0; k < 6; k++)
				{
					float t = lane < 8 ? s[k][lane] : (k < 3 ? INFINITY : -INFINITY);
					r[k] = k < 3 ? warp_min(t) : warp_max(t);
				}
				if (lane == 0)
					for (int k = 0; k < 6; k++)
						block_aabb[6 * blockIdx.x + k] = r[k];
			}
		}

		// Second pass (fn_reduce_aabb_2_pass[_atomic]) over the first `nb` block AABBs.
		__global__ void __launch_bounds__(256) reduce_final_kernel(const float* __restrict__ block_aabb, uint32_t nb, float* __restrict__ out)
		{
			__shared__ float s[6][8];
			float v[6] = { INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY };
			for (uint32_t b = threadIdx.x; b < nb; b += 256)
			{
				for (int k = 0; k < 3; k++)
					v[k] = fminf(v[k], block_aabb[6 * b + k]);
				for (int k = 3; k < 6; k++)
					v[k] = fmaxf(v[k], block_aabb[6 * b + k]);
			}
			for (int k = 0; k < 6; k++)
				v[k] = k < 3 ? warp_min(v[k]) : warp_max(v[k]);
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			if (lane == 0)
				for (int k = 0; k < 6; k++)
					s[k][warp] = v[k];
			__syncthreads();
			if (warp == 0)
			{
				for (int k = 0; k < 6; k++)
				{
					float t = lane < 8 ? s[k][lane] : (k < 3 ? INFINITY : -INFINITY);
					t = k < 3 ? warp_min(t) : warp_max(t);
					if (lane == 0)
						out[k] = t;
				}
			}
		}

		__device__ __forceinline__ uint32_t expand_bits(uint32_t v)
		{
			v = (v | (v << 16)) & 0x030000FFu;
			v = (v | (v << 8)) & 0x0300F00Fu;
			v = (v | (v << 4)) & 0x030C30C3u;
			return (v | (v << 2)) & 0x09249249u;
		}

		__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

		__device__ __forceinline__ uint32_t morton32(f3 p)
		{
			const float x = clampf(p.x * 1024.0f, 0.0f, 1023.0f);
			const float y = clampf(p.y * 1024.0f, 0.0f, 1023.0f);
			const float z = clampf(p.z * 1024.0f, 0.0f, 1023.0f);
			return (expand_bits(uint32_t(x)) << 2) | (expand_bits(uint32_t(y)) << 1) | expand_bits(uint32_t(z));
		}

		// fn_compute_mortons: key = morton32(normalised centre) << 32 | leaf id; value = leaf id.
		template <int TYPE>
		__global__ void __launch_bounds__(256) morton_kernel(const float* __restrict__ x, const uint32_t* __restrict__ prims, uint32_t n,
			const float* __restrict__ gaabb, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals)
		{
			const uint32_t lid = blockIdx.x * blockDim.x + threadIdx.x;
			if (lid >= n)
				return;
			const f3 mn = mk3(gaabb[0], gaabb[1], gaabb[2]);
			const f3 mx = mk3(gaabb[3], gaabb[4], gaabb[5]);
			const f3 ext = vmax(mx - mn, mk3(1e-6f));
			const f3 inv = mk3(1.0f / ext.x, 1.0f / ext.y, 1.0f / ext.z);
			f3 c, a, b;
			prim_center_aabb<TYPE>(x, prims, lid, c, a, b);
			const f3 np = (c - mn) * inv;
			keys[lid] = (uint64_t(morton32(np)) << 32) | uint64_t(lid);
			vals[lid] = lid;
		}

		// fn_reset_tree + fn_apply_sorted.
		__global__ void __launch_bounds__(256) apply_sorted_kernel(const uint32_t* __restrict__ sorted_vals, uint32_t n,
			uint2* __restrict__ children, uint32_t* __restrict__ object_idx, uint32_t* __restrict__ parent,
			uint32_t* __restrict__ health)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			const uint32_t ni = n - 1;
			if (i == 0)
			{
				parent[0] = kInvalid;
				*health = 1u;
			}
			if (i < ni)
				object_idx[i] = kInvalid;
			if (i < n)
			{
				const uint32_t orig = sorted_vals[i];
				children[ni + i] = make_uint2(orig, orig);
				object_idx[ni + i] = orig;
			}
		}

		__device__ __forceinline__ int cp_ij(const uint64_t* __restrict__ keys, uint64_t mi, int j, int n)
		{
			if (j < 0 || j >= n)
				return -1;
			return __clzll(mi ^ __ldg(keys + j));
		}

		// fn_build_inner_nodes: determineRange + findSplit (Karras 2012) over unique keys.
		__global__ void __launch_bounds__(256) karras_kernel(const uint64_t* __restrict__ keys, uint32_t n, uint2* __restrict__ children,
			uint32_t* __restrict__ parent, uint32_t* __restrict__ node_range)
		{
			const int nid = blockIdx.x * blockDim.x + threadIdx.x;
			const int num_inner = int(n) - 1;
			if (nid >= num_inner)
				return;
			int i = 0, j = num_inner;
			if (nid != 0)
			{
				const uint64_t mi = keys[nid];
				const int cl = cp_ij(keys, mi, nid - 1, int(n));
				const int cr = cp_ij(keys, mi, nid + 1, int(n));
				const int d = cl < cr ? 1 : -1;
				const int cp_min = min(cl, cr);
				int lmax = 2;
				while (cp_ij(keys, mi, nid + lmax * d, int(n)) > cp_min)
					lmax <<= 1;
				int l = 0;
				for (int t = lmax >> 1; t >= 1; t >>= 1)
					if (cp_ij(keys, mi, nid + (l + t) * d, int(n)) > cp_min)
						l += t;
				i = nid;
				j = nid + l * d;
			}
			int lo = i, hi = j;
			if (!(i < j))
			{
				lo = j;
				hi = i;
			}
			const uint64_t mlo = keys[lo], mhi = keys[hi];
			int split;
			if (mlo == mhi)
				split = (lo + hi) >> 1;
			else
			{
				const int cp_node = __clzll(mlo ^ mhi);
				int t = hi - lo;
				split = lo;
				for (;;)
				{
					t = (t + 1) >> 1;
					const int ns = split + t;
					if (ns < hi && __clzll(mlo ^ __ldg(keys + ns)) > cp_node)
						split = ns;
					if (!(t > 1))
						break;
				}
			}
			int c_left = (min(i, j) == split) ? num_inner + split : split;
			int c_right = (max(i, j) == split + 1) ? num_inner + split + 1 : split + 1;
			if (c_right >= num_inner)
			{
				const int tmp = c_left;
				c_left = c_right;
				c_right = tmp;
			}
			parent[c_left] = uint32_t(nid);
			parent[c_right] = uint32_t(nid);
			children[nid] = make_uint2(uint32_t(c_left), uint32_t(c_right));
			node_range[nid] = uint32_t(j);
		}

		// fn_check_construction.
		__global__ void __launch_bounds__(256) check_kernel(const uint2* __restrict__ children, const uint32_t* __restrict__ parent, uint32_t ni,
			uint32_t* __restrict__ health)
		{
			const uint32_t nid = blockIdx.x * blockDim.x + threadIdx.x;
			if (nid >= ni)
				return;
			const uint2 c = children[nid];
			if (parent[c.x] != nid || parent[c.y] != nid)
				*health = 0u;
		}

		template <int TYPE>
		__device__ __forceinline__ void leaf_box(const float* __restrict__ x0, const float* __restrict__ x1, const float* __restrict__ thickness,
			const uint32_t* __restrict__ prims, uint32_t pid, f3& mn, f3& mx)
		{
			uint32_t first;
			// x_start == x_end (a refit at one state): min(v, v) = v, so one set of loads gives the
			// same box bit for bit
			const bool same = x0 == x1;
			if constexpr (TYPE == U26_TREE_FACE)
			{
				const uint32_t a = __ldg(prims + 3 * pid), b = __ldg(prims + 3 * pid + 1), c = __ldg(prims + 3 * pid + 2);
				const f3 s0 = ld3(x0, a), s1 = ld3(x0, b), s2 = ld3(x0, c);
				if (same)
				{
					mn = vmin(s0, vmin(s1, s2));
					mx = vmax(s0, vmax(s1, s2));
				}
				else
				{
					const f3 e0 = ld3(x1, a), e1 = ld3(x1, b), e2 = ld3(x1, c);
					mn = vmin(vmin(s0, vmin(s1, s2)), vmin(e0, vmin(e1, e2)));
					mx = vmax(vmax(s0, vmax(s1, s2)), vmax(e0, vmax(e1, e2)));
				}
				first = a;
			}
			else if constexpr (TYPE == U26_TREE_EDGE)
			{
				const uint32_t a = __ldg(prims + 2 * pid), b = __ldg(prims + 2 * pid + 1);
				const f3 s0 = ld3(x0, a), s1 = ld3(x0, b);
				if (same)
				{
					mn = vmin(s0, s1);
					mx = vmax(s0, s1);
				}
				else
				{
					const f3 e0 = ld3(x1, a), e1 = ld3(x1, b);
					mn = vmin(vmin(s0, s1), vmin(e0, e1));
					mx = vmax(vmax(s0, s1), vmax(e0, e1));
				}
				first = a;
			}
			else
			{
				const f3 s0 = ld3(x0, pid);
				if (same)
				{
					mn = s0;
					mx = s0;
				}
				else
				{
					const f3 e0 = ld3(x1, pid);
					mn = vmin(s0, e0);
					mx = vmax(s0, e0);
				}
				first = pid;
			}
			const float t = __ldg(thickness + first);
			mn = mn - mk3(t);
			mx = mx + mk3(t);
		}

		// fn_update_*_tree_leave_aabb_v2: flags (0, 1) as in the reference.
		template <int TYPE>
		__global__ void __launch_bounds__(256) leaf_update_kernel(const uint32_t* __restrict__ sorted_get_original, NodeBox* __restrict__ boxes,
			const float* __restrict__ x0, const float* __restrict__ x1, const float* __restrict__ thickness,
			const uint32_t* __restrict__ prims, uint32_t n)
		{
			const uint32_t lid = blockIdx.x * blockDim.x + threadIdx.x;
			if (lid >= n)
				return;
			f3 mn, mx;
			leaf_box<TYPE>(x0, x1, thickness, prims, __ldg(sorted_get_original + lid), mn, mx);
			NodeBox b;
			b.mn = make_float4(mn.x, mn.y, mn.z, 0.0f);
			b.mx = make_float4(mx.x, mx.y, mx.z, 1.0f);
			boxes[n - 1 + lid] = b;
		}

		// Bottom-up union (fn_refit_tree_aabb, lbvh.cpp:694-758) without atomics or waits, level
		// by level. construct_tree prepares, once per topology:
		//  * the height of every inner node (1 + the larger child height, leaves 0); a Karras
		//    tree over unique 64-bit keys is at most 64 deep, so a height fits a byte;
		//  * treelets: the maximal subtrees of at most kTreelet leaves (each a contiguous leaf
		//    range, Karras 2012), packed in leaf order into chunks of at most kTreelet leaves;
		//  * the top nodes (more than kTreelet leaves) sorted by height, their children as
		//    compact ids (top node j, or 0x80000000 | treelet b).
		// refit_chunk_kernel: one block per chunk. Leaf boxes, the chunk's inner nodes (child
		// links and heights) and their boxes live in shared memory; the nodes of height h are
		// united in step h, after a barrier, so every union reads finished children without
		// atomics or fences. Boxes go out coalesced.
		// refit_top_kernel: one block for the top tree. The treelet roots' boxes are read once,
		// then the top nodes height by height, in shared memory when the tree fits, else
		// through L2.
		// Unions keep the (first child, second child) operand order of the reference.
		constexpr uint32_t kTreelet = 1024;
		constexpr uint32_t kTopRoot = 0x80000000u;
		constexpr uint32_t kMaxHeight = 64;
		constexpr size_t kTopSharedBytes = 226u * 1024u; // the top tree in shared memory up to this size (227 KB per block, less static)
		constexpr size_t kChunkSmem = 2 * 24 * kTreelet + sizeof(uint32_t) * kTreelet;
		struct Box6
		{
			float v[6];
		};
		__device__ __forceinline__ Box6 unite(const Box6& a, const Box6& b)
		{
			return Box6{ { fminf(a.v[0], b.v[0]), fminf(a.v[1], b.v[1]), fminf(a.v[2], b.v[2]), fmaxf(a.v[3], b.v[3]), fmaxf(a.v[4], b.v[4]),
				fmaxf(a.v[5], b.v[5]) } };
		}
		__device__ __forceinline__ void store_box6(NodeBox* p, const Box6& b, float w_mx)
		{
			__stcg(&p->mn, make_float4(b.v[0], b.v[1], b.v[2], 0.0f));
			__stcg(&p->mx, make_float4(b.v[3], b.v[4], b.v[5], w_mx));
		}
		__device__ __forceinline__ Box6 load_box6(const NodeBox* p)
		{
			const float4 a = __ldcg(&p->mn), b = __ldcg(&p->mx);
			return Box6{ { a.x, a.y, a.z, b.x, b.y, b.z } };
		}
		// leaf order -> primitive table, permuted once per construction
		template <int K>
		__global__ void __launch_bounds__(256) permute_prims_kernel(const uint32_t* __restrict__ sorted_get_original,
			const uint32_t* __restrict__ prims, uint32_t n, uint32_t* __restrict__ out)
		{
			const uint32_t lid = blockIdx.x * blockDim.x + threadIdx.x;
			if (lid >= n)
				return;
			const uint32_t p = sorted_get_original[lid];
#pragma unroll
			for (int k = 0; k < K; k++)
				out[size_t(K) * lid + k] = prims[size_t(K) * p + k];
		}

		// ---- construction: heights, treelets, top nodes
		// heights: a thread per leaf climbs; at each inner node the first arrival stops and the
		// second (acquiring the first's height) stores 1 + the larger child height. counters are
		// zero on entry. Bounded by the tree depth (<= 64 levels, capped at kMaxClimb).
		__global__ void __launch_bounds__(256) height_kernel(const uint32_t* __restrict__ parent, const uint2* __restrict__ children, uint32_t n,
			uint32_t* __restrict__ counters, uint8_t* __restrict__ height, uint32_t* __restrict__ health)
		{
			const uint32_t lid = blockIdx.x * blockDim.x + threadIdx.x;
			if (lid >= n)
				return;
			const uint32_t ni = n - 1;
			uint32_t node = parent[ni + lid];
			uint32_t steps = 0;
			while (node != kInvalid)
			{
				if (++steps > 100000u || node >= ni)
				{
					atomicExch(health, 0u);
					return;
				}
				if (cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(counters[node]).fetch_add(1u, cuda::memory_order_acq_rel) == 0u)
					return;
				const uint2 c = children[node];
				// the sibling's height, ordered after its store by the arrival's acquire
				const uint32_t ha = c.x >= ni ? 0u : height[c.x];
				const uint32_t hb = c.y >= ni ? 0u : height[c.y];
				const uint32_t h = 1u + max(ha, hb);
				if (h > kMaxHeight)
				{
					atomicExch(health, 0u);
					return;
				}
				height[node] = uint8_t(h);
				node = parent[node];
			}
		}
		__device__ __forceinline__ uint32_t node_size(uint32_t x, uint32_t ni, const uint32_t* __restrict__ range)
		{
			if (x >= ni)
				return 1u;
			const uint32_t r = range[x];
			return (x > r ? x - r : r - x) + 1u;
		}
		// treelet roots (key: first leaf) and top nodes (key: height, node) appended to two lists
		__global__ void __launch_bounds__(256) treelet_mark_kernel(const uint32_t* __restrict__ parent, const uint32_t* __restrict__ range,
			const uint8_t* __restrict__ height, uint32_t n, uint32_t* __restrict__ counts, uint64_t* __restrict__ top_keys,
			uint32_t* __restrict__ top_vals, uint64_t* __restrict__ root_keys, uint32_t* __restrict__ root_vals)
		{
			const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
			const uint32_t ni = n - 1;
			if (x >= 2 * n - 1)
				return;
			const uint32_t sz = node_size(x, ni, range);
			if (sz > kTreelet)
			{
				const uint32_t j = atomicAdd(counts + 0, 1u);
				top_keys[j] = (uint64_t(height[x]) << 32) | x;
				top_vals[j] = x;
				return;
			}
			const uint32_t p = parent[x];
			if (p == kInvalid || node_size(p, ni, range) > kTreelet)
			{
				const uint32_t lo = x >= ni ? x - ni : min(x, range[x]);
				const uint32_t b = atomicAdd(counts + 1, 1u);
				root_keys[b] = lo;
				root_vals[b] = x;
			}
		}
		// compact ids of the sorted lists, then each top node's children as compact ids, the end
		// of each height's run, and the treelets' leaf ranges
		__global__ void __launch_bounds__(256) treelet_map_kernel(const uint32_t* __restrict__ top_nodes, uint32_t m,
			const uint32_t* __restrict__ roots, uint32_t nt, uint32_t* __restrict__ cmap)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i < m)
				cmap[top_nodes[i]] = i;
			else if (i < m + nt)
				cmap[roots[i - m]] = kTopRoot | (i - m);
		}
		__global__ void __launch_bounds__(256) treelet_links_kernel(const uint32_t* __restrict__ top_nodes, uint32_t m,
			const uint2* __restrict__ children, const uint32_t* __restrict__ cmap, const uint8_t* __restrict__ height,
			uint2* __restrict__ top_links, uint32_t* __restrict__ height_end, const uint32_t* __restrict__ roots, uint32_t nt,
			const uint32_t* __restrict__ range, uint32_t n, uint32_t* __restrict__ root_size, uint8_t* __restrict__ top_height)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i < m)
			{
				const uint32_t x = top_nodes[i];
				const uint2 c = children[x];
				top_links[i] = make_uint2(cmap[c.x], cmap[c.y]);
				const uint32_t h = height[x];
				top_height[i] = uint8_t(h);
				if (i + 1 == m || height[top_nodes[i + 1]] != h)
					height_end[h] = i + 1;
			}
			if (i < nt)
				root_size[i] = node_size(roots[i], n - 1, range);
		}
		// treelets (in leaf order) packed greedily into chunks of at most kTreelet leaves; one
		// thread (a few thousand treelets)
		// (chunk_tb: each chunk's first treelet, then nt)
		__global__ void treelet_chunks_kernel(const uint32_t* __restrict__ root_size, uint32_t nt, uint32_t* __restrict__ chunk_lo,
			uint32_t* __restrict__ chunk_tb, uint32_t* __restrict__ nchunks)
		{
			if (threadIdx.x != 0 || blockIdx.x != 0)
				return;
			uint32_t k = 0, lo = 0, fill = 0, tb = 0;
			for (uint32_t b = 0; b < nt; b++)
			{
				const uint32_t sz = root_size[b];
				if (fill > 0 && fill + sz > kTreelet)
				{
					chunk_tb[k] = tb;
					chunk_lo[k++] = lo;
					lo += fill;
					fill = 0;
					tb = b;
				}
				fill += sz;
			}
			chunk_tb[k] = tb;
			chunk_lo[k++] = lo;
			chunk_lo[k] = lo + fill;
			chunk_tb[k] = nt;
			*nchunks = k;
		}

		// ---- refit
		// a box in shared memory: six floats on an 8-byte boundary (three 8-byte accesses)
		struct __align__(8) SBox
		{
			float2 v[3]; // (mn.x, mn.y), (mn.z, mx.x), (mx.y, mx.z)
		};
		__device__ __forceinline__ SBox sbox(f3 mn, f3 mx)
		{
			return SBox{ { make_float2(mn.x, mn.y), make_float2(mn.z, mx.x), make_float2(mx.y, mx.z) } };
		}
		__device__ __forceinline__ SBox unite_s(const SBox& a, const SBox& b)
		{
			return SBox{ { make_float2(fminf(a.v[0].x, b.v[0].x), fminf(a.v[0].y, b.v[0].y)),
				make_float2(fminf(a.v[1].x, b.v[1].x), fmaxf(a.v[1].y, b.v[1].y)),
				make_float2(fmaxf(a.v[2].x, b.v[2].x), fmaxf(a.v[2].y, b.v[2].y)) } };
		}
		__device__ __forceinline__ void store_sbox(NodeBox* p, const SBox& b)
		{
			__stcg(&p->mn, make_float4(b.v[0].x, b.v[0].y, b.v[1].x, 0.0f));
			__stcg(&p->mx, make_float4(b.v[1].y, b.v[2].x, b.v[2].y, 1.0f));
		}
		// One 512-thread block per chunk of at most 1024 leaves, two leaves and two inner-node
		// slots per thread, so that four chunks share an SM and one chunk's loads overlap another's
		// height steps.
		constexpr uint32_t kChunkThreads = 512;
		template <int TYPE, bool FUSED>
		__global__ void __launch_bounds__(kChunkThreads, 4) refit_chunk_kernel(const uint32_t* __restrict__ sorted_get_original,
			NodeBox* __restrict__ boxes, const float* __restrict__ x0, const float* __restrict__ x1, const float* __restrict__ thickness,
			const uint32_t* __restrict__ prims, bool prims_in_leaf_order, const uint2* __restrict__ children,
			const uint32_t* __restrict__ node_range, const uint8_t* __restrict__ height, const uint32_t* __restrict__ chunk_lo, uint32_t n,
			const uint32_t* __restrict__ chunk_tb, const uint32_t* __restrict__ roots, SBox* __restrict__ root_box, uint32_t* __restrict__ health)
		{
			// dynamic shared memory (kChunkSmem bytes, four blocks per SM): leaf boxes, inner boxes,
			// child links as two 16-bit chunk-local slots (bit 15: leaf)
			extern __shared__ __align__(16) unsigned char s_raw[];
			SBox* s_leaf = reinterpret_cast<SBox*>(s_raw);
			SBox* s_inner = s_leaf + kTreelet;
			uint32_t* s_child = reinterpret_cast<uint32_t*>(s_inner + kTreelet);
			__shared__ uint32_t s_hmax;
			const uint32_t base = chunk_lo[blockIdx.x];
			const uint32_t cnt = chunk_lo[blockIdx.x + 1] - base;
			const uint32_t ni = n - 1;
			const uint32_t t = threadIdx.x;
			if (cnt > kTreelet || base + cnt > n)
			{
				// a plan that does not match the tree: nothing is read or written
				if (t == 0)
					atomicExch(health, 0u);
				return;
			}
			if (t == 0)
				s_hmax = 0u;
			// inner nodes base + t and base + t + 512: links and heights when their leaf ranges lie
			// inside the chunk
			uint32_t h[2] = { 0u, 0u };
#pragma unroll
			for (int q = 0; q < 2; q++)
			{
				const uint32_t tq = t + q * kChunkThreads, x = base + tq;
				if (tq < cnt && x < ni)
				{
					const uint32_t r = __ldg(node_range + x);
					if (min(x, r) >= base && max(x, r) < base + cnt)
					{
						// children of a node inside the chunk are inside it too (checked, not assumed)
						const uint2 c = __ldg(children + x);
						const uint32_t ia = c.x >= ni ? c.x - ni - base : c.x - base, ib = c.y >= ni ? c.y - ni - base : c.y - base;
						if (ia < cnt && ib < cnt)
						{
							s_child[tq] = (ia | (c.x >= ni ? 0x8000u : 0u)) | ((ib | (c.y >= ni ? 0x8000u : 0u)) << 16);
							h[q] = __ldg(height + x);
						}
						else
							atomicExch(health, 0u);
					}
				}
			}
#pragma unroll
			for (int q = 0; q < 2; q++)
			{
				const uint32_t tq = t + q * kChunkThreads, lid = base + tq;
				if (tq < cnt)
				{
					f3 mn, mx;
					if constexpr (FUSED)
					{
						if (prims_in_leaf_order)
							leaf_box<TYPE>(x0, x1, thickness, prims, lid, mn, mx);
						else
							leaf_box<TYPE>(x0, x1, thickness, prims, __ldg(sorted_get_original + lid), mn, mx);
					}
					else
					{
						const float4 a = __ldcg(&boxes[ni + lid].mn), b = __ldcg(&boxes[ni + lid].mx);
						mn = mk3(a.x, a.y, a.z);
						mx = mk3(b.x, b.y, b.z);
					}
					s_leaf[tq] = sbox(mn, mx);
				}
			}
			const uint32_t wmax = __reduce_max_sync(0xFFFFFFFFu, max(h[0], h[1]));
			if ((t & 31) == 0 && wmax)
				atomicMax(&s_hmax, wmax);
			__syncthreads();
			const uint32_t hmax = s_hmax;
			for (uint32_t lv = 1; lv <= hmax; lv++)
			{
#pragma unroll
				for (int q = 0; q < 2; q++)
				{
					if (h[q] != lv)
						continue;
					const uint32_t tq = t + q * kChunkThreads;
					const uint32_t c = s_child[tq], ca = c & 0xFFFFu, cb = c >> 16;
					s_inner[tq] = unite_s((ca & 0x8000u) ? s_leaf[ca & 0x3FFu] : s_inner[ca & 0x3FFu],
						(cb & 0x8000u) ? s_leaf[cb & 0x3FFu] : s_inner[cb & 0x3FFu]);
				}
				__syncthreads();
			}
#pragma unroll
			for (int q = 0; q < 2; q++)
			{
				const uint32_t tq = t + q * kChunkThreads;
				if (tq < cnt)
				{
					store_sbox(boxes + ni + base + tq, s_leaf[tq]);
					if (h[q])
						store_sbox(boxes + base + tq, s_inner[tq]);
				}
			}
			// the chunk's treelet roots' boxes, also in a compact array for the top-tree launch
			if (root_box)
			{
				const uint32_t tb0 = chunk_tb[blockIdx.x], tb1 = chunk_tb[blockIdx.x + 1];
				for (uint32_t b = tb0 + t; b < tb1; b += kChunkThreads)
				{
					const uint32_t x = roots[b];
					const uint32_t k = x >= ni ? x - ni - base : x - base;
					if (k < cnt)
						root_box[b] = x >= ni ? s_leaf[k] : s_inner[k];
					else
						atomicExch(health, 0u);
				}
			}
		}

		// The top tree in one block: the treelet roots' boxes are read once, then the top nodes are
		// united height by height. SHARED (every box fits in shared memory, at most kTopSlots x 1024
		// top nodes): each thread holds its nodes' links, ids and heights in registers, so a height
		// step touches shared memory only (its box stores go out behind it). Otherwise the
		// children are read back through L2 (the block's barrier orders its own stores before the
		// next height's loads).
		constexpr uint32_t kTopSlots = 8;
		template <bool SHARED>
		__global__ void __launch_bounds__(1024) refit_top_kernel(NodeBox* __restrict__ boxes, const uint32_t* __restrict__ top_nodes,
			const uint2* __restrict__ top_links, const uint32_t* __restrict__ height_end, uint32_t m, const uint32_t* __restrict__ roots,
			uint32_t nt, const uint8_t* __restrict__ top_height, const SBox* __restrict__ root_box, uint32_t* __restrict__ health)
		{
			extern __shared__ SBox s_box[]; // [nt] treelet roots, then [m] top nodes
			const uint32_t t = threadIdx.x;
			auto valid = [&](uint32_t id, uint32_t j) { return (id & kTopRoot) ? (id & ~kTopRoot) < nt : id < j; };
			if constexpr (SHARED)
			{
				uint2 l[kTopSlots];
				uint32_t node[kTopSlots], hh[kTopSlots];
				uint32_t hmax = 0, hmin = kMaxHeight + 1;
#pragma unroll
				for (uint32_t k = 0; k < kTopSlots; k++)
				{
					const uint32_t j = t + k * blockDim.x;
					hh[k] = 0;
					if (j < m)
					{
						l[k] = top_links[j];
						node[k] = top_nodes[j];
						hh[k] = top_height[j];
						hmax = max(hmax, hh[k]);
						hmin = min(hmin, hh[k]);
					}
				}
				// the treelet roots' boxes: one coalesced read of the compact copy
				for (uint32_t b = t; b < nt; b += blockDim.x)
					s_box[b] = root_box[b];
				// the heights present: the loop runs from the lowest top node's height to the root's
				hmax = __reduce_max_sync(0xFFFFFFFFu, hmax);
				hmin = __reduce_min_sync(0xFFFFFFFFu, hmin);
				__shared__ uint32_t s_hmax, s_hmin;
				if (t == 0)
				{
					s_hmax = 0;
					s_hmin = kMaxHeight + 1;
				}
				__syncthreads();
				if ((t & 31) == 0)
				{
					atomicMax(&s_hmax, hmax);
					atomicMin(&s_hmin, hmin);
				}
				__syncthreads();
				hmax = s_hmax;
				for (uint32_t lv = s_hmin; lv <= hmax; lv++)
				{
#pragma unroll
					for (uint32_t k = 0; k < kTopSlots; k++)
					{
						if (hh[k] != lv)
							continue;
						const uint32_t j = t + k * blockDim.x;
						if (!valid(l[k].x, j) || !valid(l[k].y, j))
						{
							atomicExch(health, 0u);
							continue;
						}
						const SBox a = (l[k].x & kTopRoot) ? s_box[l[k].x & ~kTopRoot] : s_box[nt + l[k].x];
						const SBox c = (l[k].y & kTopRoot) ? s_box[l[k].y & ~kTopRoot] : s_box[nt + l[k].y];
						const SBox u = unite_s(a, c);
						s_box[nt + j] = u;
						store_sbox(boxes + node[k], u);
					}
					__syncthreads();
				}
			}
			else
			{
				uint32_t begin = 0;
				for (uint32_t h = 1; h <= kMaxHeight && begin < m; h++)
				{
					const uint32_t end = max(begin, height_end[h]);
					for (uint32_t j = begin + t; j < end && j < m; j += blockDim.x)
					{
						const uint2 l = top_links[j];
						if (!valid(l.x, j) || !valid(l.y, j))
						{
							atomicExch(health, 0u);
							continue;
						}
						auto child = [&](uint32_t id) { return load_box6(boxes + ((id & kTopRoot) ? roots[id & ~kTopRoot] : top_nodes[id])); };
						store_box6(boxes + top_nodes[j], unite(child(l.x), child(l.y)), 1.0f);
					}
					begin = end;
					__syncthreads();
				}
			}
		}

		// query_template2 with the reference's visit order: pop, test child 0 then child 1,
		// push inner children, stop the whole traversal when the 32-entry stack is full.
		template <int MODE>
		__global__ void __launch_bounds__(128) query_kernel(TreeView tv, const float* __restrict__ xb, const float* __restrict__ xe,
			const uint32_t* __restrict__ edges, uint32_t nq, const float* __restrict__ d_hat,
			const float* __restrict__ thickness, uint32_t* __restrict__ count, uint32_t* __restrict__ pairs,
			uint32_t max_pairs, uint32_t* __restrict__ dev_err)
		{
			const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
			if (q >= nq)
				return;
			if (*tv.health == 0u)
				return;
			f3 mn, mx;
			float pad;
			if constexpr (MODE == U26_QUERY_VERTS)
			{
				const f3 a = ld3(xb, q), b = ld3(xe, q);
				mn = vmin(a, b);
				mx = vmax(a, b);
				pad = __ldg(thickness + q) + __ldg(d_hat + q);
			}
			else
			{
				const uint32_t e0 = __ldg(edges + 2 * q), e1 = __ldg(edges + 2 * q + 1);
				const f3 p1 = ld3(xb, e0), p2 = ld3(xb, e1), p3 = ld3(xe, e0), p4 = ld3(xe, e1);
				mn = vmin(vmin(p1, p2), vmin(p3, p4));
				mx = vmax(vmax(p1, p2), vmax(p3, p4));
				pad = __ldg(thickness + e0) + __ldg(d_hat + e0);
			}
			mn = mn - mk3(pad);
			mx = mx + mk3(pad);
			uint32_t stack[32];
			int sp = 0;
			stack[sp++] = 0u;
			uint32_t loop = 0;
			while (sp > 0)
			{
				const uint32_t node = stack[--sp];
				const uint2 ch = __ldg(tv.children + node);
				bool stop = false;
#pragma unroll
				for (int ii = 0; ii < 2; ii++)
				{
					if (stop)
						break;
					const uint32_t cs = ii == 0 ? ch.x : ch.y;
					NodeBox b;
					b.mn = __ldg(&tv.boxes[cs].mn);
					b.mx = __ldg(&tv.boxes[cs].mx);
					if (overlap_strict(b, mn, mx))
					{
						const uint32_t adj = __ldg(tv.object_idx + cs);
						if (adj != kInvalid)
						{
							bool valid = true;
							if constexpr (MODE == U26_QUERY_EDGES)
								valid = q < adj;
							if (valid)
							{
								const uint32_t idx = atomicAdd(count, 1u);
								if (idx < max_pairs)
								{
									pairs[2 * idx] = q;
									pairs[2 * idx + 1] = adj;
								}
							}
						}
						else if (sp < 32)
							stack[sp++] = cs;
						else
						{
							atomicOr(dev_err, U26_DEVERR_STACK_OVERFLOW);
							stop = true;
						}
					}
				}
				if (stop)
					break;
				if (++loop > 100000u)
				{
					atomicOr(dev_err, U26_DEVERR_ITERATION_CAP);
					break;
				}
			}
		}

	} // namespace

	// ---- host side ------------------------------------------------------------------

	static u26_status lbvh_alloc(u26_lbvh* t)
	{
		u26_ctx* ctx = t->ctx;
		const uint32_t n = t->n;
		const uint32_t nn = 2 * n - 1;
		U26_CUDA(ctx, t->morton_sorted.reserve(sizeof(uint64_t) * n));
		U26_CUDA(ctx, t->sorted_get_original.reserve(sizeof(uint32_t) * n));
		U26_CUDA(ctx, t->parent.reserve(sizeof(uint32_t) * nn));
		U26_CUDA(ctx, t->children.reserve(sizeof(uint2) * nn));
		U26_CUDA(ctx, t->object_idx.reserve(sizeof(uint32_t) * nn));
		U26_CUDA(ctx, t->node_aabb.reserve(sizeof(NodeBox) * nn));
		U26_CUDA(ctx, t->block_aabb.reserve(sizeof(float) * 6 * div_up(n, 256)));
		U26_CUDA(ctx, t->global_aabb.reserve(sizeof(float) * 6));
		U26_CUDA(ctx, t->refit_flags.reserve(sizeof(uint32_t) * std::max<uint32_t>(n - 1, 1)));
		U26_CUDA(ctx, t->node_range.reserve(sizeof(uint32_t) * std::max<uint32_t>(n - 1, 1)));
		U26_CUDA(ctx, t->height.reserve(std::max<uint32_t>(n - 1, 1)));
		U26_CUDA(ctx, t->height_end.reserve(sizeof(uint32_t) * (kMaxHeight + 1)));
		if (t->type != U26_TREE_VERT)
			U26_CUDA(ctx, t->leaf_prims.reserve(sizeof(uint32_t) * (t->type == U26_TREE_FACE ? 3u : 2u) * size_t(n)));
		U26_CUDA(ctx, t->health.reserve(sizeof(uint32_t)));
		U26_CUDA(ctx, cudaMemsetAsync(t->health.ptr, 0, sizeof(uint32_t), ctx->stream));
		U26_CUDA(ctx, cudaMemsetAsync(t->node_aabb.ptr, 0, sizeof(NodeBox) * nn, ctx->stream));
		return U26_OK;
	}
} // namespace u26

using namespace u26;

#define U26_DISPATCH_TYPE(type, KERNEL, GRID, BLOCK, STREAM, ...)                        \
	do                                                                                   \
	{                                                                                    \
		if ((type) == U26_TREE_FACE)                                                     \
			KERNEL<U26_TREE_FACE><<<(GRID), (BLOCK), 0, (STREAM)>>>(__VA_ARGS__);        \
		else if ((type) == U26_TREE_EDGE)                                                \
			KERNEL<U26_TREE_EDGE><<<(GRID), (BLOCK), 0, (STREAM)>>>(__VA_ARGS__);        \
		else                                                                             \
			KERNEL<U26_TREE_VERT><<<(GRID), (BLOCK), 0, (STREAM)>>>(__VA_ARGS__);        \
	}                                                                                    \
	while (0)

U26_API u26_status u26_lbvh_create(u26_ctx* ctx, int tree_type, uint32_t num_leaves, u26_lbvh** out)
{
	if (!ctx || !out)
		return U26_ERR_INVALID_INPUT;
	*out = nullptr;
	if (tree_type < U26_TREE_VERT || tree_type > U26_TREE_EDGE)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_create: bad tree type %d", tree_type);
	if (num_leaves == 0 || num_leaves > 0x7FFFFFFFu)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_create: num_leaves %u out of range", num_leaves);
	U26_CUDA(ctx, cudaSetDevice(ctx->device));
	u26_lbvh* t = new u26_lbvh();
	t->ctx = ctx;
	t->type = tree_type;
	t->n = num_leaves;
	const u26_status st = lbvh_alloc(t);
	if (st != U26_OK)
	{
		u26_lbvh_destroy(t);
		return st;
	}
	*out = t;
	return U26_OK;
}

U26_API void u26_lbvh_destroy(u26_lbvh* t)
{
	if (!t)
		return;
	t->morton_sorted.release();
	t->sorted_get_original.release();
	t->parent.release();
	t->children.release();
	t->object_idx.release();
	t->node_aabb.release();
	t->block_aabb.release();
	t->global_aabb.release();
	t->refit_flags.release();
	t->node_range.release();
	t->height.release();
	t->chunk_lo.release();
	t->top_nodes.release();
	t->top_links.release();
	t->height_end.release();
	t->roots.release();
	t->chunk_tb.release();
	t->top_height.release();
	t->root_box.release();
	t->plan_scratch.release();
	t->leaf_prims.release();
	t->health.release();
	t->sorter.release();
	delete t;
}

U26_API u26_status u26_lbvh_reduce_aabb(u26_lbvh* t, const float* x, uint32_t num_verts, const uint32_t* prims)
{
	if (!t || !x || (t->type != U26_TREE_VERT && !prims))
		return t ? set_error(t->ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_reduce_aabb: null input") : U26_ERR_INVALID_INPUT;
	u26_ctx* ctx = t->ctx;
	const uint32_t nb_leaf = div_up(t->n, 256);
	// lbvh.cpp:999-1021: the edge/face trees reduce ceil(num_verts/256) blocks in the second pass.
	uint32_t nb = (t->type == U26_TREE_VERT || t->full_global_aabb) ? nb_leaf : std::min(nb_leaf, div_up(num_verts, 256));
	if (nb == 0)
		nb = 1;
	U26_DISPATCH_TYPE(t->type, reduce_blocks_kernel, nb_leaf, 256, ctx->stream, x, prims, t->n, t->block_aabb.as<float>());
	U26_TRY(after_launch(ctx, "reduce_blocks_kernel"));
	reduce_final_kernel<<<1, 256, 0, ctx->stream>>>(t->block_aabb.as<float>(), nb, t->global_aabb.as<float>());
	U26_TRY(after_launch(ctx, "reduce_final_kernel"));
	t->last_x = x;
	t->last_prims = prims;
	t->last_num_verts = num_verts;
	return U26_OK;
}

// The refit plan of a constructed tree (heights, treelets, chunks, top nodes by height).
static u26_status refit_plan(u26_lbvh* t)
{
	u26_ctx* ctx = t->ctx;
	cudaStream_t st = ctx->stream;
	const uint32_t n = t->n, ni = n - 1, nn = 2 * n - 1;
	uint32_t* health = t->health.as<uint32_t>();
	// heights
	U26_CUDA(ctx, cudaMemsetAsync(t->refit_flags.ptr, 0, sizeof(uint32_t) * ni, st));
	U26_CUDA(ctx, cudaMemsetAsync(t->height.ptr, 0, ni, st));
	height_kernel<<<div_up(n, 256), 256, 0, st>>>(t->parent.as<uint32_t>(), t->children.as<uint2>(), n, t->refit_flags.as<uint32_t>(),
		t->height.as<uint8_t>(), health);
	U26_TRY(after_launch(ctx, "height_kernel"));
	// scratch: counts[2], top keys / vals [ni], root keys / vals [n], compact map [nn], root sizes [n]
	// every region starts on a 256-byte boundary
	auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
	const size_t off_tk = 256, off_tv = up(off_tk + 8 * size_t(ni)), off_rk = up(off_tv + 4 * size_t(ni)), off_rv = up(off_rk + 8 * size_t(n)),
				 off_map = up(off_rv + 4 * size_t(n)), off_sz = up(off_map + 4 * size_t(nn)), total = up(off_sz + 4 * size_t(n));
	U26_CUDA(ctx, t->plan_scratch.reserve(total));
	unsigned char* sc = static_cast<unsigned char*>(t->plan_scratch.ptr);
	uint32_t* counts = reinterpret_cast<uint32_t*>(sc);
	uint64_t* top_keys = reinterpret_cast<uint64_t*>(sc + off_tk);
	uint32_t* top_vals = reinterpret_cast<uint32_t*>(sc + off_tv);
	uint64_t* root_keys = reinterpret_cast<uint64_t*>(sc + off_rk);
	uint32_t* root_vals = reinterpret_cast<uint32_t*>(sc + off_rv);
	uint32_t* cmap = reinterpret_cast<uint32_t*>(sc + off_map);
	uint32_t* root_size = reinterpret_cast<uint32_t*>(sc + off_sz);
	U26_CUDA(ctx, cudaMemsetAsync(counts, 0, 2 * sizeof(uint32_t), st));
	treelet_mark_kernel<<<div_up(nn, 256), 256, 0, st>>>(t->parent.as<uint32_t>(), t->node_range.as<uint32_t>(), t->height.as<uint8_t>(), n,
		counts, top_keys, top_vals, root_keys, root_vals);
	U26_TRY(after_launch(ctx, "treelet_mark_kernel"));
	uint32_t mt[2] = { 0, 0 };
	U26_CUDA(ctx, cudaMemcpyAsync(mt, counts, sizeof(mt), cudaMemcpyDeviceToHost, st));
	U26_CUDA(ctx, cudaStreamSynchronize(st));
	const uint32_t m = mt[0], nt = mt[1];
	if (nt == 0 || nt > n || m > ni)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "refit plan: %u treelets, %u top nodes for %u leaves", nt, m, n);
	if (m > 1)
		U26_TRY(t->sorter.sort(ctx, top_keys, top_vals, m, 0, 40));
	if (nt > 1)
		U26_TRY(t->sorter.sort(ctx, root_keys, root_vals, nt, 0, 32));
	U26_CUDA(ctx, t->top_nodes.reserve(sizeof(uint32_t) * std::max(m, 1u)));
	U26_CUDA(ctx, t->top_links.reserve(sizeof(uint2) * std::max(m, 1u)));
	U26_CUDA(ctx, t->roots.reserve(sizeof(uint32_t) * nt));
	U26_CUDA(ctx, t->chunk_lo.reserve(sizeof(uint32_t) * (nt + 2)));
	U26_CUDA(ctx, t->chunk_tb.reserve(sizeof(uint32_t) * (nt + 2)));
	U26_CUDA(ctx, t->top_height.reserve(std::max(m, 1u)));
	U26_CUDA(ctx, t->root_box.reserve(sizeof(SBox) * nt));
	if (m)
		U26_CUDA(ctx, cudaMemcpyAsync(t->top_nodes.ptr, top_vals, sizeof(uint32_t) * m, cudaMemcpyDeviceToDevice, st));
	U26_CUDA(ctx, cudaMemcpyAsync(t->roots.ptr, root_vals, sizeof(uint32_t) * nt, cudaMemcpyDeviceToDevice, st));
	treelet_map_kernel<<<div_up(m + nt, 256), 256, 0, st>>>(t->top_nodes.as<uint32_t>(), m, t->roots.as<uint32_t>(), nt, cmap);
	U26_TRY(after_launch(ctx, "treelet_map_kernel"));
	U26_CUDA(ctx, cudaMemsetAsync(t->height_end.ptr, 0, sizeof(uint32_t) * (kMaxHeight + 1), st));
	treelet_links_kernel<<<div_up(std::max(m, nt), 256), 256, 0, st>>>(t->top_nodes.as<uint32_t>(), m, t->children.as<uint2>(), cmap,
		t->height.as<uint8_t>(), t->top_links.as<uint2>(), t->height_end.as<uint32_t>(), t->roots.as<uint32_t>(), nt,
		t->node_range.as<uint32_t>(), n, root_size, t->top_height.as<uint8_t>());
	U26_TRY(after_launch(ctx, "treelet_links_kernel"));
	treelet_chunks_kernel<<<1, 32, 0, st>>>(root_size, nt, t->chunk_lo.as<uint32_t>(), t->chunk_tb.as<uint32_t>(), counts);
	U26_TRY(after_launch(ctx, "treelet_chunks_kernel"));
	U26_CUDA(ctx, cudaMemcpyAsync(mt, counts, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
	U26_CUDA(ctx, cudaStreamSynchronize(st));
	t->nchunks = mt[0];
	t->ntop = m;
	t->ntreelets = nt;
	const size_t top_bytes = sizeof(SBox) * (size_t(m) + nt);
	t->top_in_shared = top_bytes <= kTopSharedBytes && m <= kTopSlots * 1024u;
	if (t->top_in_shared && m)
		U26_CUDA(ctx, cudaFuncSetAttribute(refit_top_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTopSharedBytes)));
	// the chunk kernels' dynamic shared memory (above the 48 KB default)
	const void* chunk_kernels[] = { (const void*)refit_chunk_kernel<U26_TREE_VERT, false>, (const void*)refit_chunk_kernel<U26_TREE_VERT, true>,
		(const void*)refit_chunk_kernel<U26_TREE_EDGE, false>, (const void*)refit_chunk_kernel<U26_TREE_EDGE, true>,
		(const void*)refit_chunk_kernel<U26_TREE_FACE, false>, (const void*)refit_chunk_kernel<U26_TREE_FACE, true> };
	for (const void* k : chunk_kernels)
		U26_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kChunkSmem)));
	// the lists and the compact map (about 40 B per leaf) are needed at construction only; the
	// stream is idle here (synchronised above)
	t->plan_scratch.release();
	return U26_OK;
}

U26_API u26_status u26_lbvh_construct_tree(u26_lbvh* t)
{
	if (!t)
		return U26_ERR_INVALID_INPUT;
	u26_ctx* ctx = t->ctx;
	if (!t->last_x)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_construct_tree: call u26_lbvh_reduce_aabb first");
	const uint32_t n = t->n;
	uint64_t* keys = t->morton_sorted.as<uint64_t>();
	uint32_t* vals = t->sorted_get_original.as<uint32_t>();
	U26_DISPATCH_TYPE(t->type, morton_kernel, div_up(n, 256), 256, ctx->stream, t->last_x, t->last_prims, n,
		t->global_aabb.as<float>(), keys, vals);
	U26_TRY(after_launch(ctx, "morton_kernel"));
	// Keys are unique and values start as the identity: a stable sort of the Morton bits
	// [32, 62) reproduces the 64-bit key order.
	U26_TRY(t->sorter.sort(ctx, keys, vals, n, 32, 62));
	apply_sorted_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(vals, n, t->children.as<uint2>(), t->object_idx.as<uint32_t>(),
		t->parent.as<uint32_t>(), t->health.as<uint32_t>());
	U26_TRY(after_launch(ctx, "apply_sorted_kernel"));
	if (n > 1)
	{
		karras_kernel<<<div_up(n - 1, 256), 256, 0, ctx->stream>>>(keys, n, t->children.as<uint2>(), t->parent.as<uint32_t>(),
			t->node_range.as<uint32_t>());
		U26_TRY(after_launch(ctx, "karras_kernel"));
		check_kernel<<<div_up(n - 1, 256), 256, 0, ctx->stream>>>(t->children.as<uint2>(), t->parent.as<uint32_t>(), n - 1,
			t->health.as<uint32_t>());
		U26_TRY(after_launch(ctx, "check_kernel"));
	}
	// the primitive table in leaf order, for the refits' coalesced leaf reads (the mesh
	// topology is fixed between constructions; a refit given another table gathers)
	t->leaf_prims_src = nullptr;
	if (t->type == U26_TREE_FACE)
	{
		permute_prims_kernel<3><<<div_up(n, 256), 256, 0, ctx->stream>>>(vals, t->last_prims, n, t->leaf_prims.as<uint32_t>());
		U26_TRY(after_launch(ctx, "permute_prims_kernel"));
		t->leaf_prims_src = t->last_prims;
	}
	else if (t->type == U26_TREE_EDGE)
	{
		permute_prims_kernel<2><<<div_up(n, 256), 256, 0, ctx->stream>>>(vals, t->last_prims, n, t->leaf_prims.as<uint32_t>());
		U26_TRY(after_launch(ctx, "permute_prims_kernel"));
		t->leaf_prims_src = t->last_prims;
	}
	if (n > 1)
		U26_TRY(refit_plan(t));
	t->built = true;
	return U26_OK;
}

U26_API u26_status u26_lbvh_update_leaves(u26_lbvh* t, const float* thickness, const float* x_start, const float* x_end,
	const uint32_t* prims)
{
	if (!t || !thickness || !x_start || !x_end || (t->type != U26_TREE_VERT && !prims))
		return t ? set_error(t->ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_update_leaves: null input") : U26_ERR_INVALID_INPUT;
	u26_ctx* ctx = t->ctx;
	U26_DISPATCH_TYPE(t->type, leaf_update_kernel, div_up(t->n, 256), 256, ctx->stream, t->sorted_get_original.as<uint32_t>(),
		t->node_aabb.as<NodeBox>(), x_start, x_end, thickness, prims, t->n);
	return after_launch(ctx, "leaf_update_kernel");
}

static u26_status refit_impl(u26_lbvh* t, bool fused, const float* thickness, const float* x0, const float* x1,
	const uint32_t* prims)
{
	u26_ctx* ctx = t->ctx;
	if (t->n <= 1)
	{
		if (fused)
			return u26_lbvh_update_leaves(t, thickness, x0, x1, prims);
		return U26_OK;
	}
	if (!t->built)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "refit: call u26_lbvh_construct_tree first");
	const bool sorted = fused && prims && prims == t->leaf_prims_src;
	SBox* root_box = (t->ntop && t->top_in_shared) ? t->root_box.as<SBox>() : nullptr;
	const uint32_t* lp = sorted ? t->leaf_prims.as<uint32_t>() : prims;
#define U26_REFIT(T, F)                                                                                                          \
	refit_chunk_kernel<T, F><<<t->nchunks, kChunkThreads, kChunkSmem, ctx->stream>>>(t->sorted_get_original.as<uint32_t>(), t->node_aabb.as<NodeBox>(), \
		x0, x1, thickness, lp, sorted, t->children.as<uint2>(), t->node_range.as<uint32_t>(), t->height.as<uint8_t>(),                  \
		t->chunk_lo.as<uint32_t>(), t->n, t->chunk_tb.as<uint32_t>(), t->roots.as<uint32_t>(), root_box, t->health.as<uint32_t>())
	if (t->type == U26_TREE_FACE)
	{
		if (fused)
			U26_REFIT(U26_TREE_FACE, true);
		else
			U26_REFIT(U26_TREE_FACE, false);
	}
	else if (t->type == U26_TREE_EDGE)
	{
		if (fused)
			U26_REFIT(U26_TREE_EDGE, true);
		else
			U26_REFIT(U26_TREE_EDGE, false);
	}
	else if (fused)
		U26_REFIT(U26_TREE_VERT, true);
	else
		U26_REFIT(U26_TREE_VERT, false);
#undef U26_REFIT
	U26_TRY(after_launch(ctx, "refit_chunk_kernel"));
	if (t->ntop == 0)
		return U26_OK;
	if (t->top_in_shared)
		refit_top_kernel<true><<<1, 1024, sizeof(SBox) * (size_t(t->ntop) + t->ntreelets), ctx->stream>>>(t->node_aabb.as<NodeBox>(),
			t->top_nodes.as<uint32_t>(), t->top_links.as<uint2>(), t->height_end.as<uint32_t>(), t->ntop, t->roots.as<uint32_t>(), t->ntreelets,
			t->top_height.as<uint8_t>(), t->root_box.as<SBox>(), t->health.as<uint32_t>());
	else
		refit_top_kernel<false><<<1, 1024, 0, ctx->stream>>>(t->node_aabb.as<NodeBox>(), t->top_nodes.as<uint32_t>(), t->top_links.as<uint2>(),
			t->height_end.as<uint32_t>(), t->ntop, t->roots.as<uint32_t>(), t->ntreelets, t->top_height.as<uint8_t>(), nullptr,
			t->health.as<uint32_t>());
	return after_launch(ctx, "refit_top_kernel");
}

U26_API u26_status u26_lbvh_refit(u26_lbvh* t)
{
	if (!t)
		return U26_ERR_INVALID_INPUT;
	return refit_impl(t, false, nullptr, nullptr, nullptr, nullptr);
}

U26_API u26_status u26_lbvh_update_and_refit(u26_lbvh* t, const float* thickness, const float* x_start, const float* x_end,
	const uint32_t* prims)
{
	if (!t || !thickness || !x_start || !x_end || (t->type != U26_TREE_VERT && !prims))
		return t ? set_error(t->ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_update_and_refit: null input") : U26_ERR_INVALID_INPUT;
	return refit_impl(t, true, thickness, x_start, x_end, prims);
}

U26_API u26_status u26_lbvh_query(u26_lbvh* t, int mode, const float* x_begin, const float* x_end, const uint32_t* edges,
	uint32_t num_queries, const float* d_hat, const float* thickness, uint32_t* count, uint32_t* pairs, uint32_t max_pairs)
{
	if (!t || !x_begin || !x_end || !d_hat || !thickness || !count || (!pairs && max_pairs))
		return t ? set_error(t->ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_query: null input") : U26_ERR_INVALID_INPUT;
	if (mode != U26_QUERY_VERTS && !edges)
		return set_error(t->ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_query: edges required for edge queries");
	if (num_queries == 0)
		return U26_OK;
	u26_ctx* ctx = t->ctx;
	const TreeView tv = tree_view(t);
	const uint32_t grid = div_up(num_queries, 128);
	if (mode == U26_QUERY_VERTS)
		query_kernel<U26_QUERY_VERTS><<<grid, 128, 0, ctx->stream>>>(tv, x_begin, x_end, edges, num_queries, d_hat, thickness, count,
			pairs, max_pairs, ctx->dev_err);
	else if (mode == U26_QUERY_EDGES)
		query_kernel<U26_QUERY_EDGES><<<grid, 128, 0, ctx->stream>>>(tv, x_begin, x_end, edges, num_queries, d_hat, thickness, count,
			pairs, max_pairs, ctx->dev_err);
	else if (mode == U26_QUERY_EDGES_UNCULLED)
		query_kernel<U26_QUERY_EDGES_UNCULLED><<<grid, 128, 0, ctx->stream>>>(tv, x_begin, x_end, edges, num_queries, d_hat, thickness,
			count, pairs, max_pairs, ctx->dev_err);
	else
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_query: bad mode %d", mode);
	return after_launch(ctx, "query_kernel");
}

U26_API u26_status u26_lbvh_check_health(u26_lbvh* t, int* healthy)
{
	if (!t || !healthy)
		return U26_ERR_INVALID_INPUT;
	u26_ctx* ctx = t->ctx;
	U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, t->health.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
	U26_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	*healthy = *ctx->host_word != 0u ? 1 : 0;
	return U26_OK;
}

U26_API u26_status u26_lbvh_arrays_get(const u26_lbvh* t, u26_lbvh_arrays* out)
{
	if (!t || !out)
		return U26_ERR_INVALID_INPUT;
	out->num_leaves = t->n;
	out->num_nodes = t->num_nodes();
	out->morton_sorted = t->morton_sorted.as<uint64_t>();
	out->sorted_get_original = t->sorted_get_original.as<uint32_t>();
	out->parent = t->parent.as<uint32_t>();
	out->children = t->children.as<uint32_t>();
	out->object_idx = t->object_idx.as<uint32_t>();
	out->node_aabb = t->node_aabb.as<float>();
	out->global_aabb = t->global_aabb.as<float>();
	return U26_OK;
}

U26_API u26_status u26_lbvh_set_option(u26_lbvh* t, int option, int value)
{
	if (!t)
		return U26_ERR_INVALID_INPUT;
	if (option == U26_LBVH_OPT_FULL_GLOBAL_AABB)
	{
		t->full_global_aabb = value != 0;
		return U26_OK;
	}
	return set_error(t->ctx, U26_ERR_INVALID_INPUT, "u26_lbvh_set_option: unknown option %d", option);
}
