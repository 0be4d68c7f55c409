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
			if constexpr (TYPE == U26_TREE_FACE)
			{
				const uint32_t a = __ldg(prims + 3 * pid), b = __ldg(prims + 3 * pid + 1), c = __ldg(prims + 3 * pid + 2);
				const f3 s0 = ld3(x0, a), s1 = ld3(x0, b), s2 = ld3(x0, c);
				const f3 e0 = ld3(x1, a), e1 = ld3(x1, b), e2 = ld3(x1, c);
				mn = vmin(vmin(s0, vmin(s1, s2)), vmin(e0, vmin(e1, e2)));
				mx = vmax(vmax(s0, vmax(s1, s2)), vmax(e0, vmax(e1, e2)));
				first = a;
			}
			else if constexpr (TYPE == U26_TREE_EDGE)
			{
				const uint32_t a = __ldg(prims + 2 * pid), b = __ldg(prims + 2 * pid + 1);
				const f3 s0 = ld3(x0, a), s1 = ld3(x0, b), e0 = ld3(x1, a), e1 = ld3(x1, b);
				mn = vmin(vmin(s0, s1), vmin(e0, e1));
				mx = vmax(vmax(s0, s1), vmax(e0, e1));
				first = a;
			}
			else
			{
				const f3 s0 = ld3(x0, pid), e0 = ld3(x1, pid);
				mn = vmin(s0, e0);
				mx = vmax(s0, e0);
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

		// Bottom-up union (fn_refit_tree_aabb, lbvh.cpp:694-758) without spin-waits. One thread
		// per leaf climbs; at each inner node the first arrival stops and the second owns the
		// union. The climb stays inside its block while it can: block b owns the leaves
		// [b * kRefitBlock, (b + 1) * kRefitBlock), and an inner node's leaves form a contiguous
		// range with the node's own index at one end (Karras 2012), so a node whose range lies
		// inside the block is reached by the block's threads only. Its arrival counter and its
		// box live in shared memory (the box is written out as well). A node whose range
		// crosses a block boundary, and every ancestor of it, joins through a device counter
		// that gains 2 per refit: an even value before the increment marks the first arrival,
		// so the counters need no reset between refits. The leaf update runs in the same
		// thread when FUSED. Every climb is bounded by kMaxClimb steps.
		constexpr uint32_t kRefitBlock = 512;
		struct Box6
		{
			float v[6];
		};
		__device__ __forceinline__ void load_box6_cg(const NodeBox* p, f3& mn, f3& mx)
		{
			const float4 a = __ldcg(&p->mn), b = __ldcg(&p->mx);
			mn = mk3(a.x, a.y, a.z);
			mx = mk3(b.x, b.y, b.z);
		}
		template <int TYPE, bool FUSED>
		__global__ void __launch_bounds__(kRefitBlock) refit_block_kernel(const uint32_t* __restrict__ sorted_get_original,
			NodeBox* __restrict__ boxes, const float* __restrict__ x0, const float* __restrict__ x1, const float* __restrict__ thickness,
			const uint32_t* __restrict__ prims, const uint32_t* __restrict__ parent, const uint2* __restrict__ children,
			const uint32_t* __restrict__ node_range, uint32_t* __restrict__ flags, uint32_t n, uint32_t* __restrict__ health)
		{
			__shared__ uint32_t s_cnt[kRefitBlock];
			__shared__ Box6 s_leaf[kRefitBlock];
			__shared__ Box6 s_inner[kRefitBlock];
			// topology of the inner nodes [base, base + cnt), read once with coalesced loads, so
			// that the climb's dependent lookups inside the block hit shared memory
			__shared__ uint2 s_child[kRefitBlock];
			__shared__ uint32_t s_parent[kRefitBlock], s_range[kRefitBlock];
			const uint32_t base = blockIdx.x * kRefitBlock;
			const uint32_t cnt = min(kRefitBlock, n - base);
			const uint32_t ni = n - 1;
			const uint32_t t = threadIdx.x;
			s_cnt[t] = 0u;
			bool inner_local = false; // inner node base + t lies inside the block (its box is written below)
			if (base + t < ni)
			{
				s_child[t] = __ldg(children + base + t);
				s_parent[t] = __ldg(parent + base + t);
				const uint32_t r = __ldg(node_range + base + t);
				s_range[t] = r;
				inner_local = min(base + t, r) >= base && max(base + t, r) < base + cnt;
			}
			// phase 1: leaf boxes (into shared memory; written out in phase 3)
			const uint32_t lid = base + t;
			if (t < cnt)
			{
				f3 mn, mx;
				if constexpr (FUSED)
					leaf_box<TYPE>(x0, x1, thickness, prims, __ldg(sorted_get_original + lid), mn, mx);
				else
					load_box6_cg(boxes + ni + lid, mn, mx);
				s_leaf[t] = Box6{ { mn.x, mn.y, mn.z, mx.x, mx.y, mx.z } };
			}
			__syncthreads();
			// phase 2: the climb through the nodes inside the block, in shared memory only (no device
			// stores in flight, so the block-scope fences stay cheap). A thread that reaches a node
			// crossing the block boundary keeps it as `pending` for phase 4.
			constexpr uint32_t kMaxClimb = 100000u;
			uint32_t pending = kInvalid;
			if (t < cnt)
			{
				uint32_t node = __ldg(parent + ni + lid);
				uint32_t steps = 0;
				while (node != kInvalid)
				{
					if (++steps > kMaxClimb || node >= ni)
					{
						atomicExch(health, 0u);
						node = kInvalid;
						break;
					}
					const uint32_t k = node - base;
					if (!(k < cnt && min(node, s_range[k]) >= base && max(node, s_range[k]) < base + cnt))
					{
						pending = node; // crosses the block boundary
						break;
					}
					__threadfence_block(); // this thread's shared boxes before its arrival
					if (atomicAdd(&s_cnt[k], 1u) == 0u)
						break;
					__threadfence_block();
					const uint2 c = s_child[k];
					// children of a node inside the block are inside it too (checked, not assumed)
					const uint32_t ia = c.x >= ni ? c.x - ni - base : c.x - base, ib = c.y >= ni ? c.y - ni - base : c.y - base;
					if (ia >= cnt || ib >= cnt)
					{
						atomicExch(health, 0u);
						break;
					}
					const Box6 ba = c.x >= ni ? s_leaf[ia] : s_inner[ia];
					const Box6 bb = c.y >= ni ? s_leaf[ib] : s_inner[ib];
					s_inner[k] = Box6{ { fminf(ba.v[0], bb.v[0]), fminf(ba.v[1], bb.v[1]), fminf(ba.v[2], bb.v[2]), fmaxf(ba.v[3], bb.v[3]),
						fmaxf(ba.v[4], bb.v[4]), fmaxf(ba.v[5], bb.v[5]) } };
					node = s_parent[k];
				}
			}
			__syncthreads();
			// phase 3: the block's leaf boxes and local inner boxes, written out coalesced
			if (t < cnt)
			{
				const Box6 l = s_leaf[t];
				__stcg(&boxes[ni + lid].mn, make_float4(l.v[0], l.v[1], l.v[2], 0.0f));
				__stcg(&boxes[ni + lid].mx, make_float4(l.v[3], l.v[4], l.v[5], 1.0f));
			}
			if (inner_local)
			{
				const Box6 b = s_inner[t];
				__stcg(&boxes[base + t].mn, make_float4(b.v[0], b.v[1], b.v[2], 0.0f));
				__stcg(&boxes[base + t].mx, make_float4(b.v[3], b.v[4], b.v[5], 1.0f));
			}
			__syncthreads();
			if (pending == kInvalid)
				return;
			// phase 4: nodes crossing block boundaries, through device counters that gain 2 per refit
			// (an even value before the increment marks the first arrival). The acq_rel arrival
			// releases the block's boxes written above (ordered before it by the barrier) and the
			// second arrival acquires the sibling's.
			__threadfence(); // the block's phase 3 stores, ordered by the barrier, before the release below
			uint32_t node = pending;
			uint32_t steps = 0;
			while (node != kInvalid)
			{
				if (++steps > kMaxClimb || node >= ni)
				{
					atomicExch(health, 0u);
					return;
				}
				const uint32_t arrived = cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(flags[node]).fetch_add(1u,
					cuda::memory_order_acq_rel);
				if ((arrived & 1u) == 0u)
					return;
				const uint2 c = __ldg(children + node);
				f3 amn, amx, bmn, bmx;
				load_box6_cg(boxes + c.x, amn, amx);
				load_box6_cg(boxes + c.y, bmn, bmx);
				const f3 mn = vmin(amn, bmn), mx = vmax(amx, bmx);
				__stcg(&boxes[node].mn, make_float4(mn.x, mn.y, mn.z, 0.0f));
				__stcg(&boxes[node].mx, make_float4(mx.x, mx.y, mx.z, 1.0f));
				node = __ldg(parent + node);
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
		U26_CUDA(ctx, cudaMemsetAsync(t->refit_flags.ptr, 0, sizeof(uint32_t) * std::max<uint32_t>(n - 1, 1), ctx->stream));
		U26_CUDA(ctx, t->node_range.reserve(sizeof(uint32_t) * std::max<uint32_t>(n - 1, 1)));
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
	const uint32_t grid = div_up(t->n, kRefitBlock);
#define U26_REFIT(T, F)                                                                                                          \
	refit_block_kernel<T, F><<<grid, kRefitBlock, 0, ctx->stream>>>(t->sorted_get_original.as<uint32_t>(), t->node_aabb.as<NodeBox>(), \
		x0, x1, thickness, prims, t->parent.as<uint32_t>(), t->children.as<uint2>(), t->node_range.as<uint32_t>(),                   \
		t->refit_flags.as<uint32_t>(), t->n, t->health.as<uint32_t>())
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
	return after_launch(ctx, "refit_block_kernel");
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
