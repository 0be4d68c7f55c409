// PRP contour evaluation on sm_100a: the reference's host_resolve_intersections_PRP /
// device_resolve_intersections_PRP (intersection_resolver2.cpp:2750-4072,
// intersection_resolver_gpu.cpp:2792-4460) with every (contour, direction) task of an
// adaptive k-ring level evaluated in one batch of launches.
//
// Host (C++ below, like the reference's own GPU evaluator): EF adjacency and loop-vertex
// pairs (intersection_resolver.cpp:431-558, 683-1096), contour flood fill and types
// (intersection_resolver2.cpp:254-375), vertex boundary flags (2646-2680), side identity
// and boundary anchors (2428-2585), candidate directions (1488-1569) with a 3x3 Jacobi
// eigen solver, the k-ring growth decisions (1058-1230), selection (h:852-912),
// pre-finalize merge data and suppression (453-592).
//
// Device (kernels below):
//   normals_kernel            face / edge / vertex normals (2605-2644)
//   distances_kernel          one CTA per (contour, side): BFS hop distance and rest-geodesic
//                             distance to the contour boundary over the side's object
//                             (618-722); the geodesic is a worklist Bellman-Ford whose least
//                             fixpoint equals Dijkstra's result in float (monotone relax)
//   candidates_kernel         one CTA per (contour, side): the k-ring vertices are a prefix
//                             of the BFS order; contour-side ownership (CCR, 1571-1804,
//                             h:405-506); candidate edge / face lists and membership bitmaps
//   raycast_kernel            one thread per VF / EE / FV request of all tasks, traversal of
//                             the scene face / edge LBVH with conservative (epsilon-grown)
//                             node tests and the exact reference primitive tests
//                             (cached_bvh.cpp:131-555, helper.cpp:319-514)
//   radix sort                hits by (task, type, source, target)
//   init/union/compress       product-complex adjacency (helper.cpp:771-902) as exact key
//                             lookups in the task's sorted hits, lock-free union-find
//   task_kernel               one CTA per task: boundary-attached components, EF-anchor
//                             coverage, best component (3506-3685), J / volume / area /
//                             displacement cost (1806-1954) with a canonical reduction order
//   gather_kernel             selected supports S(r) compacted for the host
#include <algorithm>
#include <functional>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <set>
#include <atomic>
#include <thread>
#include <unistd.h>
#include <vector>

#include <cooperative_groups.h>

#include "lbvh_internal.h"
#include "predicates.cuh"

namespace cg = cooperative_groups;

namespace u26
{
	struct EfPairH
	{
		uint32_t idx[5];
		float bary[3];
		float grad[3];
		float stiff;
		bool is_loop() const { return idx[0] == idx[1]; }
	};
	static_assert(sizeof(EfPairH) == 48, "EfPair");

	// ---------------------------------------------------------------- device helpers
	__device__ __forceinline__ bool ray_tri(f3 start, f3 dir, float ray_len, f3 A, f3 B, f3 C, float& out_t, f3& out_bary)
	{
		const f3 AB = B - A;
		const f3 AC = C - A;
		const f3 N = cross(AB, AC);
		const f3 neg = -dir;
		const float den = dot(neg, N);
		const f3 to_a = start - A;
		const float tnum = dot(to_a, N);
		// misses decided before the square root and the division, only where the exact test
		// below must also reject: t = tnum / den surely negative (opposite signs, magnitudes far
		// from underflow), or surely beyond ray_len (1e-5 relative margin)
		const float aden = fabsf(den), anum = fabsf(tnum);
		const bool den_ok = aden >= 1e-30f && aden <= 1e20f; // 1 / den neither overflows nor underflows
		if (den_ok && anum >= 1e-20f && ((tnum > 0.0f) != (den > 0.0f)))
			return false;
		if (aden >= 1e-30f && anum > aden * ray_len * (1.0f + 1e-5f) && ((tnum > 0.0f) == (den > 0.0f)))
			return false;
		// the barycentric numerators (uu = nu / den, vv = nv / den): a numerator of the other sign
		// than den makes its coordinate negative, and nu + nv beyond den (1e-5 relative margin,
		// both of den's sign by then) puts uu + vv above 1 - 1e-6; both rejections the exact test
		// below makes too, here without its square root and division
		const f3 cx = cross(neg, to_a);
		const float nu = dot(AC, cx), nv = -dot(AB, cx);
		if (den_ok)
		{
			if ((nu > 0.0f && den < 0.0f) || (nu < 0.0f && den > 0.0f) || (nv > 0.0f && den < 0.0f) || (nv < 0.0f && den > 0.0f))
				return false;
			if (fabsf(nu + nv) > aden * (1.0f + 1e-5f))
				return false;
		}
		const float nlen = length(N);
		if (fabsf(den) < nlen * 1e-6f)
			return false;
		const float inv_den = 1.0f / den;
		const float t = tnum * inv_den;
		if (t < 0.0f || t > ray_len)
			return false;
		const float uu = nu * inv_den;
		if (uu < 1e-6f || uu > (1.0f - 1e-6f))
			return false;
		const float vv = nv * inv_den;
		if (vv < 1e-6f || (vv + uu) > (1.0f - 1e-6f))
			return false;
		out_t = t;
		out_bary = mk3(1.0f - uu - vv, uu, vv);
		return true;
	}

	__device__ __forceinline__ bool seg_tri(f3 p0, f3 p1, f3 A, f3 B, f3 C, f3& out_bary, float& out_time)
	{
		const f3 d = p1 - p0;
		const float len_sq = length_sq(d);
		if (len_sq < 1e-6f * 1e-6f)
			return false;
		const float len = sqrtf(len_sq);
		const float inv_len = 1.0f / len;
		const f3 ray = d * inv_len;
		if (ray_tri(p0, ray, len, A, B, C, out_time, out_bary))
		{
			out_time = out_time * inv_len;
			return true;
		}
		return false;
	}

	__device__ __forceinline__ uint32_t float_bits(float f) { return __float_as_uint(f); }

	namespace
	{
		constexpr uint32_t kInf = 0xFFFFFFFFu;
		constexpr float kGeoInf = 3.402823466e+38f;

		// ------------------------------------------------------------ normals
		__global__ void normals_face_kernel(const float* __restrict__ x, const uint32_t* __restrict__ faces, const uint32_t* __restrict__ vobj,
			const uint32_t* __restrict__ orient, uint32_t nf, float* __restrict__ fn)
		{
			const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
			if (f >= nf)
				return;
			const uint32_t a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
			const f3 pa = ld3(x, a), pb = ld3(x, b), pc = ld3(x, c);
			f3 n = cross(pb - pa, pc - pa);
			const float l2 = dot(n, n);
			n = l2 > 1e-20f ? n / sqrtf(l2) : mk3(0.0f);
			const float s = orient[vobj[a]] == 0u ? 1.0f : -1.0f;
			n = s * n;
			fn[3 * f] = n.x;
			fn[3 * f + 1] = n.y;
			fn[3 * f + 2] = n.z;
		}

		// area-weighted sum of incident face normals, sequential in CSR order
		__global__ void normals_accum_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj,
			const float* __restrict__ face_area, const float* __restrict__ fn, uint32_t n, float* __restrict__ out)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			f3 s = mk3(0.0f);
			for (uint32_t k = off[i]; k < off[i + 1]; k++)
			{
				const uint32_t f = adj[k];
				s = s + face_area[f] * mk3(fn[3 * f], fn[3 * f + 1], fn[3 * f + 2]);
			}
			const float l2 = dot(s, s);
			s = l2 > 1e-20f ? s / sqrtf(l2) : mk3(0.0f);
			out[3 * i] = s.x;
			out[3 * i + 1] = s.y;
			out[3 * i + 2] = s.z;
		}

		struct Slot
		{
			uint32_t v_lo, v_cnt, e_lo, e_cnt, f_lo, f_cnt;
			uint32_t bnd_off, bnd_cnt;
			uint32_t k;
			uint32_t diam;
			uint32_t pad[2]; // [0] contour-side restriction applies, [1] object of the side
		};

		// ------------------------------------------------------------ distances
		// One CTA per slot. hop/geo/order/mark are slot-strided (stride = largest object).
		__global__ void __launch_bounds__(256) distances_kernel(Slot* __restrict__ slots, const uint32_t* __restrict__ slot_ids,
			const uint32_t* __restrict__ bnd, const uint32_t* __restrict__ vav_off, const uint32_t* __restrict__ vav,
			const float* __restrict__ rest_x, uint32_t stride, uint32_t* __restrict__ hop, float* __restrict__ geo,
			uint32_t* __restrict__ order, uint32_t* __restrict__ level_end, uint32_t* __restrict__ work, uint32_t* __restrict__ mark,
			uint32_t* __restrict__ dev_err)
		{
			const uint32_t s = slot_ids[blockIdx.x];
			Slot sl = slots[s];
			const uint32_t lo = sl.v_lo, cnt = sl.v_cnt;
			uint32_t* hs = hop + size_t(s) * stride;
			float* gs = geo + size_t(s) * stride;
			uint32_t* os = order + size_t(s) * stride;
			uint32_t* ms = mark + size_t(s) * stride;
			uint32_t* le = level_end + size_t(s) * (stride + 1);
			uint32_t* wa = work + size_t(s) * 2 * stride;
			uint32_t* wb = wa + stride;
			__shared__ uint32_t s_tail, s_n;
			for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
			{
				hs[i] = kInf;
				gs[i] = kGeoInf;
				ms[i] = 0u;
			}
			__syncthreads();
			for (uint32_t j = threadIdx.x; j < sl.bnd_cnt; j += blockDim.x)
			{
				// the host only forms slots whose anchors lie in the side's object
				const uint32_t v = min(bnd[sl.bnd_off + j] - lo, cnt - 1u);
				hs[v] = 0u;
				gs[v] = 0.0f;
				os[j] = v;
				wa[j] = v;
			}
			if (threadIdx.x == 0)
			{
				s_tail = sl.bnd_cnt;
				le[0] = sl.bnd_cnt;
			}
			__syncthreads();
			// BFS: the order array is the queue; level_end[h] = #vertices with hop <= h
			uint32_t head = 0, tail = sl.bnd_cnt, level = 0;
			while (head < tail)
			{
				for (uint32_t i = head + threadIdx.x; i < tail; i += blockDim.x)
				{
					const uint32_t v = os[i];
					const uint32_t gv = lo + v;
					for (uint32_t k = vav_off[gv]; k < vav_off[gv + 1]; k++)
					{
						const uint32_t a = vav[k];
						if (a < lo || a >= lo + cnt)
							continue;
						if (atomicCAS(hs + (a - lo), kInf, level + 1u) == kInf)
							os[atomicAdd(&s_tail, 1u)] = a - lo;
					}
				}
				__syncthreads();
				head = tail;
				tail = s_tail;
				level++;
				if (threadIdx.x == 0)
					le[level] = tail;
				__syncthreads();
			}
			if (threadIdx.x == 0)
			{
				slots[s].diam = level > 0 ? level - 1u : 0u;
				if (sl.bnd_cnt == 0)
					slots[s].diam = 0u;
			}
			// rest-geodesic distance: worklist relaxation to the least fixpoint
			uint32_t ncur = sl.bnd_cnt;
			uint32_t* cur = wa;
			uint32_t* nxt = wb;
			uint32_t rounds = 0;
			const uint32_t max_rounds = 8u * cnt + 64u;
			while (ncur > 0)
			{
				if (threadIdx.x == 0)
					s_n = 0u;
				__syncthreads();
				for (uint32_t i = threadIdx.x; i < ncur; i += blockDim.x)
				{
					const uint32_t v = cur[i];
					const uint32_t gv = lo + v;
					const float d = __uint_as_float(atomicAdd(reinterpret_cast<uint32_t*>(gs + v), 0u));
					const f3 pv = ld3(rest_x, gv);
					for (uint32_t k = vav_off[gv]; k < vav_off[gv + 1]; k++)
					{
						const uint32_t a = vav[k];
						if (a < lo || a >= lo + cnt)
							continue;
						const float nd = d + length(pv - ld3(rest_x, a));
						const uint32_t nb = __float_as_uint(nd);
						const uint32_t old = atomicMin(reinterpret_cast<uint32_t*>(gs + (a - lo)), nb);
						if (nb < old && atomicExch(ms + (a - lo), 1u) == 0u)
							nxt[atomicAdd(&s_n, 1u)] = a - lo;
					}
				}
				__syncthreads();
				const uint32_t nn = s_n;
				for (uint32_t i = threadIdx.x; i < nn; i += blockDim.x)
					ms[nxt[i]] = 0u;
				__syncthreads();
				uint32_t* t = cur;
				cur = nxt;
				nxt = t;
				ncur = nn;
				if (++rounds > max_rounds)
				{
					if (threadIdx.x == 0)
						atomicOr(dev_err, U26_DEVERR_ITERATION_CAP);
					break;
				}
			}
		}

		// per-slot bitmap of the contour-boundary vertices (object-local index)
		__global__ void bnd_bits_kernel(const Slot* __restrict__ slots, const uint32_t* __restrict__ bnd, uint32_t v_stride,
			uint32_t* __restrict__ bits)
		{
			const uint32_t s = blockIdx.x;
			const Slot sl = slots[s];
			uint32_t* b = bits + size_t(s) * (v_stride / 32 + 1);
			for (uint32_t j = threadIdx.x; j < sl.bnd_cnt; j += blockDim.x)
			{
				const uint32_t v = bnd[sl.bnd_off + j] - sl.v_lo;
				if (v < sl.v_cnt)
					atomicOr(b + (v >> 5), 1u << (v & 31));
			}
		}

		// ------------------------------------------------------------ candidates
		// contour-side ownership (intersection_resolver2.h:431-506)
		__device__ __forceinline__ bool reachable(float d) { return isfinite(d) && d < 3.402823466e+38f * 0.5f; }
		__device__ __forceinline__ float normalized_phi(float own, float opp)
		{
			const bool g0 = reachable(own), g1 = reachable(opp);
			if (!g0 && !g1)
				return 0.0f;
			if (!g0)
				return 1.0f;
			if (!g1)
				return -1.0f;
			return (own - opp) / (own + opp + 1e-6f);
		}
		__device__ __forceinline__ bool owns1(float own, float opp, float tau)
		{
			if (!reachable(own))
				return false;
			if (!reachable(opp))
				return true;
			return normalized_phi(own, opp) <= tau;
		}
		__device__ __forceinline__ bool owns_blended(float ro, float rp, float co, float cp, float tau, float w)
		{
			float phi;
			if (!isfinite(w) || (!reachable(ro) && !reachable(co)))
				phi = INFINITY;
			else if (!(reachable(ro) && reachable(rp)))
				phi = normalized_phi(co, cp);
			else if (!(reachable(co) && reachable(cp)))
				phi = normalized_phi(ro, rp);
			else
			{
				const float wc = fminf(fmaxf(w, 0.0f), 1.0f);
				phi = wc * normalized_phi(ro, rp) + (1.0f - wc) * normalized_phi(co, cp);
			}
			return phi <= tau;
		}

		// Current-space distance of each k-ring vertex to the nearest boundary anchor of its own
		// side and of the opposite side (deformed_boundary_distance, intersection_resolver2.cpp:
		// 1706-1738), cached across the levels of a pass (NaN = not yet computed). One warp per
		// vertex, lanes over the anchors; min over squared distances, then one sqrt (sqrt is
		// monotone and correctly rounded, so this equals the min of the lengths). Only the
		// vertices whose ownership test reads the current distances are computed.
		__global__ void __launch_bounds__(256) ccr_current_kernel(const Slot* __restrict__ slots, const uint32_t* __restrict__ slot_ids,
			const uint32_t* __restrict__ bnd, const float* __restrict__ x, uint32_t v_stride, const float* __restrict__ geo,
			const uint32_t* __restrict__ order, const uint32_t* __restrict__ level_end, uint32_t ccr_rest, uint32_t ccr_blend, float tau,
			uint32_t blocks_per_slot, float* __restrict__ cur_own, float* __restrict__ cur_opp)
		{
			const uint32_t s = slot_ids[blockIdx.x / blocks_per_slot];
			const uint32_t o = s ^ 1u;
			const Slot sl = slots[s];
			if (sl.pad[0] == 0u)
				return;
			const Slot so = slots[o];
			const uint32_t nk = level_end[size_t(s) * (v_stride + 1) + min(sl.k, sl.diam)];
			const float* gs = geo + size_t(s) * v_stride;
			const float* go = geo + size_t(o) * v_stride;
			const uint32_t* os = order + size_t(s) * v_stride;
			float* co_out = cur_own + size_t(s) * v_stride;
			float* cp_out = cur_opp + size_t(s) * v_stride;
			const int lane = threadIdx.x & 31;
			const uint32_t wid = (blockIdx.x % blocks_per_slot) * (blockDim.x >> 5) + (threadIdx.x >> 5);
			const uint32_t nw = blocks_per_slot * (blockDim.x >> 5);
			const bool blend = ccr_blend && ccr_rest;
			for (uint32_t i = wid; i < nk; i += nw)
			{
				const uint32_t v = os[i];
				if (!isnan(co_out[v]))
					continue;
				const uint32_t gv = sl.v_lo + v;
				if (!blend && ccr_rest)
				{
					float rp = kGeoInf;
					if (gv >= so.v_lo && gv < so.v_lo + so.v_cnt)
						rp = go[gv - so.v_lo];
					if (!owns1(gs[v], rp, tau))
						continue;
				}
				const f3 xv = ld3(x, gv);
				float m_own = INFINITY, m_opp = INFINITY;
				for (uint32_t j = lane; j < sl.bnd_cnt; j += 32)
				{
					const f3 d = xv - ld3(x, bnd[sl.bnd_off + j]);
					m_own = fminf(m_own, dot(d, d));
				}
				for (uint32_t j = lane; j < so.bnd_cnt; j += 32)
				{
					const f3 d = xv - ld3(x, bnd[so.bnd_off + j]);
					m_opp = fminf(m_opp, dot(d, d));
				}
#pragma unroll
				for (int off = 16; off >= 1; off >>= 1)
				{
					m_own = fminf(m_own, __shfl_xor_sync(0xFFFFFFFFu, m_own, off));
					m_opp = fminf(m_opp, __shfl_xor_sync(0xFFFFFFFFu, m_opp, off));
				}
				if (lane == 0)
				{
					co_out[v] = fminf(3.402823466e+38f, sqrtf(m_own));
					cp_out[v] = fminf(3.402823466e+38f, sqrtf(m_opp));
				}
			}
		}

		__global__ void __launch_bounds__(256) candidates_kernel(const Slot* __restrict__ slots, const uint32_t* __restrict__ slot_ids,
			const uint32_t* __restrict__ bnd, const float* __restrict__ x, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, const uint32_t* __restrict__ vae_off, const uint32_t* __restrict__ vae,
			const uint32_t* __restrict__ vaf_off, const uint32_t* __restrict__ vaf, uint32_t v_stride, uint32_t e_stride,
			uint32_t f_stride, const uint32_t* __restrict__ hop, const float* __restrict__ geo, const uint32_t* __restrict__ order,
			const uint32_t* __restrict__ level_end, uint32_t ccr_rest, uint32_t ccr_current, uint32_t ccr_blend, float tau,
			float blend_w, uint8_t* __restrict__ owns, uint32_t* __restrict__ cand_v, uint32_t* __restrict__ cand_e, uint32_t* __restrict__ cand_f,
			uint32_t* __restrict__ counts, uint32_t* __restrict__ bits_e, uint32_t* __restrict__ bits_f, float* __restrict__ slot_box,
			const float* __restrict__ cur_own, const float* __restrict__ cur_opp)
		{
			const uint32_t s = slot_ids[blockIdx.x];
			const uint32_t o = s ^ 1u; // the other side of the same contour
			// AABB of the candidate faces / edges (targets of the rays cast at this slot)
			f3 fmn = mk3(INFINITY), fmx = mk3(-INFINITY), emn = mk3(INFINITY), emx = mk3(-INFINITY);
			const Slot sl = slots[s];
			const Slot so = slots[o];
			const uint32_t lo = sl.v_lo;
			const uint32_t* hs = hop + size_t(s) * v_stride;
			const float* gs = geo + size_t(s) * v_stride;
			const float* go = geo + size_t(o) * v_stride;
			const uint32_t* os = order + size_t(s) * v_stride;
			const uint32_t* le = level_end + size_t(s) * (v_stride + 1);
			uint8_t* ow = owns + size_t(s) * v_stride;
			uint32_t* be = bits_e + size_t(s) * (e_stride / 32 + 1);
			uint32_t* bf = bits_f + size_t(s) * (f_stride / 32 + 1);
			__shared__ uint32_t nvc, nec, nfc;
			if (threadIdx.x == 0)
			{
				nvc = 0;
				nec = 0;
				nfc = 0;
			}
			for (uint32_t i = threadIdx.x; i < sl.e_cnt / 32 + 1; i += blockDim.x)
				be[i] = 0u;
			for (uint32_t i = threadIdx.x; i < sl.f_cnt / 32 + 1; i += blockDim.x)
				bf[i] = 0u;
			const uint32_t k = sl.k;
			const uint32_t nk = le[min(k, sl.diam)];
			__syncthreads();
			const bool applies = sl.pad[0] != 0u; // prp_intrinsic_contour_side_restriction_applies, per contour
			const bool blend = ccr_blend && ccr_rest && ccr_current;
			for (uint32_t i = threadIdx.x; i < nk; i += blockDim.x)
			{
				const uint32_t v = os[i];
				const uint32_t gv = lo + v;
				bool own = true;
				if (applies)
				{
					const float ro = gs[v];
					float rp = kGeoInf;
					if (gv >= so.v_lo && gv < so.v_lo + so.v_cnt)
						rp = go[gv - so.v_lo];
					if (!blend && ccr_rest && !owns1(ro, rp, tau))
						own = false;
					else if (ccr_current)
					{
						const float co = cur_own[size_t(s) * v_stride + v], cp = cur_opp[size_t(s) * v_stride + v];
						own = blend ? owns_blended(ro, rp, co, cp, tau, blend_w) : ((!ccr_rest || owns1(ro, rp, tau)) && owns1(co, cp, tau));
					}
				}
				ow[v] = own ? 1 : 0;
				if (own)
					cand_v[size_t(s) * v_stride + atomicAdd(&nvc, 1u)] = gv;
			}
			__syncthreads();
			for (uint32_t i = threadIdx.x; i < nk; i += blockDim.x)
			{
				const uint32_t v = os[i];
				const uint32_t gv = lo + v;
				const bool ov = ow[v] != 0;
				for (uint32_t kk = vae_off[gv]; kk < vae_off[gv + 1]; kk++)
				{
					const uint32_t e = vae[kk];
					const uint2 ev = edges[e];
					if (ev.x != gv)
						continue;
					const uint32_t b = ev.y - lo;
					if (hs[b] > k)
						continue;
					if (applies && !ov && !ow[b])
						continue;
					cand_e[size_t(s) * e_stride + atomicAdd(&nec, 1u)] = e;
					atomicOr(be + ((e - sl.e_lo) >> 5), 1u << ((e - sl.e_lo) & 31));
					const f3 pa = ld3(x, ev.x), pb = ld3(x, ev.y);
					emn = vmin(emn, vmin(pa, pb));
					emx = vmax(emx, vmax(pa, pb));
				}
				for (uint32_t kk = vaf_off[gv]; kk < vaf_off[gv + 1]; kk++)
				{
					const uint32_t f = vaf[kk];
					const uint32_t a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
					if (min(a, min(b, c)) != gv)
						continue;
					if (hs[a - lo] > k || hs[b - lo] > k || hs[c - lo] > k)
						continue;
					if (applies && !ow[a - lo] && !ow[b - lo] && !ow[c - lo])
						continue;
					cand_f[size_t(s) * f_stride + atomicAdd(&nfc, 1u)] = f;
					atomicOr(bf + ((f - sl.f_lo) >> 5), 1u << ((f - sl.f_lo) & 31));
					const f3 pa = ld3(x, a), pb = ld3(x, b), pc = ld3(x, c);
					fmn = vmin(fmn, vmin(pa, vmin(pb, pc)));
					fmx = vmax(fmx, vmax(pa, vmax(pb, pc)));
				}
			}
			// block min / max of the candidate boxes
			__shared__ float red[12][8];
			float v12[12] = { fmn.x, fmn.y, fmn.z, fmx.x, fmx.y, fmx.z, emn.x, emn.y, emn.z, emx.x, emx.y, emx.z };
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
			for (int q = 0; q < 12; q++)
			{
				float v = v12[q];
				const bool is_min = (q % 6) < 3;
				for (int off = 16; off > 0; off >>= 1)
				{
					const float w = __shfl_xor_sync(0xFFFFFFFFu, v, off);
					v = is_min ? fminf(v, w) : fmaxf(v, w);
				}
				if (lane == 0)
					red[q][warp] = v;
			}
			__syncthreads();
			if (threadIdx.x < 12)
			{
				const int q = threadIdx.x;
				const bool is_min = (q % 6) < 3;
				float v = red[q][0];
				for (int w = 1; w < 8; w++)
					v = is_min ? fminf(v, red[q][w]) : fmaxf(v, red[q][w]);
				slot_box[12 * size_t(s) + q] = v;
			}
			if (threadIdx.x == 0)
			{
				counts[3 * s] = nvc;
				counts[3 * s + 1] = nec;
				counts[3 * s + 2] = nfc;
			}
		}

		// ------------------------------------------------------------ request order
		// Candidate vertices / edges of each slot ordered by the Morton code of their rest
		// position (edge midpoint), so that the 32 requests of a warp packet start from a
		// compact patch. Only the request order changes: hits are keyed by primitive ids.
		// Dense request-order ranks, made once per scene: the position of each vertex (edge) in
		// the order of (Morton code, id). Candidates keyed by (slot, rank) sort into the
		// (slot, code, id) order over the slot and id bits alone.
		__global__ void rank_keys_kernel(const uint32_t* __restrict__ code, uint32_t n, int id_bits, uint64_t* __restrict__ keys,
			uint32_t* __restrict__ vals)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			keys[i] = (uint64_t(code[i]) << id_bits) | i;
			vals[i] = i;
		}
		__global__ void rank_scatter_kernel(const uint32_t* __restrict__ sorted_ids, uint32_t n, uint32_t* __restrict__ rank)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			rank[sorted_ids[i]] = i;
		}
		__global__ void cand_keys_kernel(const uint32_t* __restrict__ slot_ids, const uint32_t* __restrict__ off, uint32_t nsid,
			const uint32_t* __restrict__ cand, uint32_t stride, const uint32_t* __restrict__ rank, int id_bits, uint64_t* __restrict__ keys,
			uint32_t* __restrict__ vals)
		{
			const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
			if (g >= off[nsid])
				return;
			uint32_t lo = 0, hi = nsid;
			while (hi - lo > 1)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (off[mid] <= g)
					lo = mid;
				else
					hi = mid;
			}
			const uint32_t id = cand[size_t(slot_ids[lo]) * stride + (g - off[lo])];
			// (slot, dense rank of (Morton code, id)): unique keys, so the request order (and the
			// packets) do not depend on the order the candidates were found in
			keys[g] = (uint64_t(lo) << id_bits) | rank[id];
			vals[g] = id;
		}
		__global__ void cand_scatter_kernel(const uint32_t* __restrict__ slot_ids, const uint32_t* __restrict__ off, uint32_t nsid,
			const uint32_t* __restrict__ vals, uint32_t* __restrict__ cand, uint32_t stride)
		{
			const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
			if (g >= off[nsid])
				return;
			uint32_t lo = 0, hi = nsid;
			while (hi - lo > 1)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (off[mid] <= g)
					lo = mid;
				else
					hi = mid;
			}
			cand[size_t(slot_ids[lo]) * stride + (g - off[lo])] = vals[g];
		}

		// ------------------------------------------------------------ ray casting
		struct Task
		{
			uint32_t slot0, slot1, contour_local, combo;
			float dir[3];
			float ee_pmin, ee_pmax;
			uint32_t req_begin, n_vf, n_ee, n_fv;
			uint32_t contour_global;
			uint32_t pad;
		};

		// EE projection bounds of the target edges of each task (prp_compute_edge_projection_bounds)
		__global__ void proj_bounds_kernel(Task* __restrict__ tasks, uint32_t ntasks, const uint32_t* __restrict__ counts,
			const uint32_t* __restrict__ cand_e, uint32_t e_stride, const uint2* __restrict__ edges, const float* __restrict__ x)
		{
			const uint32_t t = blockIdx.x;
			if (t >= ntasks)
				return;
			const Task tk = tasks[t];
			const f3 d = mk3(tk.dir[0], tk.dir[1], tk.dir[2]);
			const uint32_t n = counts[3 * tk.slot1 + 1];
			float mn = 3.402823466e+38f, mx = -3.402823466e+38f;
			for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
			{
				const uint2 e = edges[cand_e[size_t(tk.slot1) * e_stride + i]];
				const float a = dot(ld3(x, e.x), d), b = dot(ld3(x, e.y), d);
				mn = fminf(mn, fminf(a, b));
				mx = fmaxf(mx, fmaxf(a, b));
			}
			__shared__ float smn[256], smx[256];
			smn[threadIdx.x] = mn;
			smx[threadIdx.x] = mx;
			__syncthreads();
			for (uint32_t w = blockDim.x / 2; w > 0; w >>= 1)
			{
				if (threadIdx.x < w)
				{
					smn[threadIdx.x] = fminf(smn[threadIdx.x], smn[threadIdx.x + w]);
					smx[threadIdx.x] = fmaxf(smx[threadIdx.x], smx[threadIdx.x + w]);
				}
				__syncthreads();
			}
			if (threadIdx.x == 0)
			{
				tasks[t].ee_pmin = smn[0];
				tasks[t].ee_pmax = smx[0];
			}
		}

		__device__ __forceinline__ bool bit_test(const uint32_t* bits, uint32_t lo, uint32_t cnt, uint32_t id)
		{
			if (id < lo || id >= lo + cnt)
				return false;
			const uint32_t l = id - lo;
			return (__ldg(bits + (l >> 5)) >> (l & 31)) & 1u;
		}

		// conservative ray / box test against a box grown by eps, over [t_lo, t_hi]
		__device__ __forceinline__ bool ray_box_range(f3 o, f3 d, float t_lo, float t_hi, const float* lo, const float* hi, float& out_lo,
			float& out_hi)
		{
			float tmin = t_lo, tmax = t_hi;
			const float oo[3] = { o.x, o.y, o.z }, dd[3] = { d.x, d.y, d.z };
#pragma unroll
			for (int a = 0; a < 3; a++)
			{
				const float eps = 1e-5f * (1.0f + fmaxf(fabsf(lo[a]), fabsf(hi[a])));
				const float l = lo[a] - eps, h = hi[a] + eps;
				if (fabsf(dd[a]) < 1e-30f)
				{
					if (oo[a] < l || oo[a] > h)
						return false;
					continue;
				}
				const float inv = 1.0f / dd[a];
				float t0 = (l - oo[a]) * inv, t1 = (h - oo[a]) * inv;
				if (t0 > t1)
				{
					const float t = t0;
					t0 = t1;
					t1 = t;
				}
				tmin = fmaxf(tmin, t0);
				tmax = fminf(tmax, t1);
			}
			out_lo = tmin;
			out_hi = tmax;
			return tmin <= tmax;
		}

		// Conservative node margins, applied to every node once per pass so that the traversals
		// read grown boxes: eps = 1e-5 (1 + max |bound|) per axis for the ray slab tests, one eps
		// from all six bounds for the swept-edge box tests (the epsilon-grown node tests that
		// keep the traversal a superset of the exact primitive tests).
		// The w lanes carry the node's links, so one 32-byte load serves a visit: inner node
		// (mn.w, mx.w) = (left, right child); leaf (mn.w, mx.w) = (primitive, ~0).
		// node_off / prim_off place one object's tree in the forest of all objects' trees
		__global__ void grow_boxes_kernel(const NodeBox* __restrict__ boxes, const uint2* __restrict__ children,
			const uint32_t* __restrict__ object_idx, uint32_t n, int isotropic, uint32_t node_off, uint32_t prim_off, NodeBox* __restrict__ out)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const NodeBox b = boxes[i];
			NodeBox g;
			if (isotropic)
			{
				const float e = 1e-5f * (1.0f + fmaxf(fmaxf(fabsf(b.mn.x), fabsf(b.mx.x)), fmaxf(fmaxf(fabsf(b.mn.y), fabsf(b.mx.y)), fmaxf(fabsf(b.mn.z), fabsf(b.mx.z)))));
				g.mn = make_float4(b.mn.x - e, b.mn.y - e, b.mn.z - e, 0.0f);
				g.mx = make_float4(b.mx.x + e, b.mx.y + e, b.mx.z + e, 0.0f);
			}
			else
			{
				const float ex = 1e-5f * (1.0f + fmaxf(fabsf(b.mn.x), fabsf(b.mx.x)));
				const float ey = 1e-5f * (1.0f + fmaxf(fabsf(b.mn.y), fabsf(b.mx.y)));
				const float ez = 1e-5f * (1.0f + fmaxf(fabsf(b.mn.z), fabsf(b.mx.z)));
				g.mn = make_float4(b.mn.x - ex, b.mn.y - ey, b.mn.z - ez, 0.0f);
				g.mx = make_float4(b.mx.x + ex, b.mx.y + ey, b.mx.z + ez, 0.0f);
			}
			const uint32_t obj = object_idx[i];
			if (obj != kInvalid)
			{
				g.mn.w = __uint_as_float(obj + prim_off);
				g.mx.w = __uint_as_float(kInvalid);
			}
			else
			{
				const uint2 ch = children[i];
				g.mn.w = __uint_as_float(ch.x + node_off);
				g.mx.w = __uint_as_float(ch.y + node_off);
			}
			out[node_off + i] = g;
		}

		// The subtree roots that split one traversal across `split` parts (4, 8 or 16): the nodes
		// at depth log2(split) below the root, or shallower leaves; unused entries ~0. One object's
		// frontiers for the three splits sit at [0, 4), [4, 12) and [12, 28) of its kFrontStride
		// words.
		constexpr uint32_t kMaxSplit = 16, kFrontStride = 28;
		__host__ __device__ constexpr uint32_t front_offset(uint32_t split) { return split == 4u ? 0u : split == 8u ? 4u : 12u; }
		__global__ void frontier_kernel(const uint2* __restrict__ children, const uint32_t* __restrict__ object_idx, uint32_t n_nodes,
			uint32_t node_off, uint32_t* __restrict__ out)
		{
			if (threadIdx.x != 0 || blockIdx.x != 0)
				return;
			uint32_t cur[kMaxSplit], nxt[kMaxSplit];
			uint32_t nc = 0;
			if (n_nodes > 0)
				cur[nc++] = 0u;
			for (uint32_t d = 1; d < kMaxSplit; d <<= 1)
			{
				uint32_t nn = 0;
				for (uint32_t i = 0; i < nc; i++)
				{
					const uint32_t v = cur[i];
					if (object_idx[v] != kInvalid)
						nxt[nn++] = v;
					else
					{
						nxt[nn++] = children[v].x;
						nxt[nn++] = children[v].y;
					}
				}
				for (uint32_t i = 0; i < nn; i++)
					cur[i] = nxt[i];
				nc = nn;
				if (2u * d >= 4u)
					for (uint32_t i = 0; i < 2u * d; i++)
						out[front_offset(2u * d) + i] = i < nc ? cur[i] + node_off : kInvalid;
			}
		}

		// slab test of a grown box with the ray's reciprocals hoisted (same values as ray_box:
		// t0 <= t1 follows from the reciprocal's sign)
		// Slab test against the grown node boxes: t = box * inv - o * inv, one explicit fma per
		// plane. The boxes carry the conservative margin 1e-5 (1 + |c|), far above the rounding of
		// this form (a few ulp of o * inv), so no box the ray meets is rejected; a slab the ray
		// runs parallel to (|d| < 1e-30) gets inv = +-1e30, which turns the same arithmetic into
		// the inside-the-slab test. Node tests only prune: the leaf tests decide the hits.
		struct RaySlab
		{
			float inv[3], oinv[3];
		};
		__device__ __forceinline__ RaySlab make_slab(f3 o, f3 d)
		{
			RaySlab r;
			const float oo[3] = { o.x, o.y, o.z }, dd[3] = { d.x, d.y, d.z };
#pragma unroll
			for (int a = 0; a < 3; a++)
			{
				r.inv[a] = fabsf(dd[a]) < 1e-30f ? copysignf(1e30f, dd[a]) : 1.0f / dd[a];
				r.oinv[a] = oo[a] * r.inv[a];
			}
			return r;
		}
		__device__ __forceinline__ bool ray_grown_box(const RaySlab& r, float t_lo, float t_hi, const NodeBox& g)
		{
			const float ax = __fmaf_rn(g.mn.x, r.inv[0], -r.oinv[0]), bx = __fmaf_rn(g.mx.x, r.inv[0], -r.oinv[0]);
			const float ay = __fmaf_rn(g.mn.y, r.inv[1], -r.oinv[1]), by = __fmaf_rn(g.mx.y, r.inv[1], -r.oinv[1]);
			const float az = __fmaf_rn(g.mn.z, r.inv[2], -r.oinv[2]), bz = __fmaf_rn(g.mx.z, r.inv[2], -r.oinv[2]);
			const float tmin = fmaxf(fmaxf(t_lo, fminf(ax, bx)), fmaxf(fminf(ay, by), fminf(az, bz)));
			const float tmax = fminf(fminf(t_hi, fmaxf(ax, bx)), fminf(fmaxf(ay, by), fmaxf(az, bz)));
			return tmin <= tmax;
		}

		struct HitSink
		{
			uint64_t* keys;
			uint32_t* vals;
			float* payload;
			uint32_t* count;
			uint32_t cap;
			int b;
		};

		// one counter atomic per group of lanes emitting together (slot order does not matter:
		// hit keys are unique and sorted afterwards)
		__device__ __forceinline__ void emit(const HitSink& hs, uint32_t task, uint32_t type, uint32_t src, uint32_t dst, float b0, float b1,
			float dist)
		{
			cg::coalesced_group g = cg::coalesced_threads();
			uint32_t base = 0;
			if (g.thread_rank() == 0)
				base = atomicAdd(hs.count, g.size());
			const uint32_t slot = g.shfl(base, 0) + g.thread_rank();
			if (slot >= hs.cap)
				return;
			const uint64_t key = (uint64_t(task) << (2 + 2 * hs.b)) | (uint64_t(type) << (2 * hs.b)) | (uint64_t(src) << hs.b) | uint64_t(dst);
			hs.keys[slot] = key;
			hs.vals[slot] = slot;
			hs.payload[3 * slot] = b0;
			hs.payload[3 * slot + 1] = b1;
			hs.payload[3 * slot + 2] = dist;
		}

		// FP64 rechecks (predicates.cuh) of one VF / FV ray - triangle test and one swept edge -
		// edge test whose FP32 decision lies inside its error band: bit 0 set, bit 1 when the FP64
		// decision differs from hit32 (the FP32 decision, which the hit sets keep). Out of line:
		// they run for a small fraction of the leaf tests, and keep their registers off the
		// traversal loop (the band test itself is inline).
		__device__ __noinline__ uint32_t recheck_vf(f3 orig, f3 cast, f3 A, f3 B, f3 C, bool hit32)
		{
			const f3 end = orig + cast * 1.0f;
			d3 b64;
			double t64;
			const bool h64 = line_intersection_f64(dd(orig), dd(end), dd(A), dd(B), dd(C), b64, t64) && t64 >= 0.0 && t64 <= 1.0;
			return 1u | (h64 != hit32 ? 2u : 0u);
		}
		__device__ __noinline__ uint32_t recheck_ee(f3 p0, f3 e1, f3 dir, float ray_max, f3 q0, f3 q1, bool hit32)
		{
			const bool h64 = edge_edge_f64(dd(p0), dd(p0 + e1), dd(dir), double(ray_max), dd(q0), dd(q1));
			return 1u | (h64 != hit32 ? 2u : 0u);
		}

		// Packet traversal: a warp takes 32 consecutive requests (one task's candidate vertices
		// or edges in BFS order: one direction, nearby origins) and walks the union of their
		// paths with one shared stack, every lane testing its own ray against each popped node
		// (one broadcast load per node) and its own leaf primitives. Face-tree requests (VF,
		// FV) and edge-tree requests (EE) of a warp take one packet walk each. The grid is
		// `split` parts x the requests rounded up to warps; part p starts at the p-th node of the
		// target tree's frontier for that split, so every (ray, leaf) pair is decided once.
		// MINB: resident 128-thread blocks per SM the registers are sized for.
		constexpr int kStack = 64;
		template <bool RECHECK, int MINB, bool QUEUE>
		__global__ void __launch_bounds__(128, MINB) raycast_kernel(const Task* __restrict__ tasks, uint32_t ntasks, uint32_t total,
			const Slot* __restrict__ slots, const uint32_t* __restrict__ cand_v, const uint32_t* __restrict__ cand_e, uint32_t v_stride,
			uint32_t e_stride, uint32_t f_stride, const uint32_t* __restrict__ bits_e, const uint32_t* __restrict__ bits_f,
			const NodeBox* __restrict__ fgrow, const NodeBox* __restrict__ egrow, const uint32_t* __restrict__ ffront,
			const uint32_t* __restrict__ efront, const float* __restrict__ x, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, const float* __restrict__ slot_box, HitSink sink, unsigned long long* __restrict__ stats,
			uint32_t split, uint32_t* __restrict__ queue, uint32_t* __restrict__ dev_err)
		{
			const int lane = threadIdx.x & 31;
			// the packet's traversal stack lives in registers across the warp: entry k in lane k & 31
			// of s_lo (k < 32) or s_hi (k >= 32); every lane holds the same stack pointer
			uint32_t s_lo = 0u, s_hi = 0u;
			const uint32_t warps_per_part = (total + 31u) >> 5;
			const uint32_t items = split * warps_per_part; // (part, packet) work items
			uint32_t tested = 0, visited = 0, etested = 0, ctested = 0, rechecks = 0, flips = 0, reqs = 0;
			uint32_t fetch_nodes = 0, fetch_tris = 0, fetch_edges = 0; // warp-uniform: data each packet brings in
			uint32_t ray_visits = 0; // the node tests this ray alone would make: its start + 2 per inner node it enters
			// QUEUE (persistent form): every warp takes work items from a device counter until none is
			// left, so no warp idles while the other warps of its block finish; otherwise the grid
			// has one warp per item
			// warp index from the block index (a level's grid can exceed 2^32 threads: requests x parts)
			uint32_t wi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
			for (;;)
			{
			if constexpr (QUEUE)
			{
				uint32_t it = 0;
				if (lane == 0)
					it = atomicAdd(queue, 1u);
				wi = __shfl_sync(0xFFFFFFFFu, it, 0);
			}
			if (wi >= items)
				break; // whole warps only
			const uint32_t part = wi / warps_per_part; // warp-uniform
			const uint32_t r = (wi - part * warps_per_part) * 32u + uint32_t(lane);
			reqs += (part == 0 && r < total) ? 1u : 0u;

			// ---- per-lane request
			int kind = 0; // 1: VF / FV ray on the face tree, 2: EE swept edge on the edge tree
			uint32_t t = 0, vid = 0, eid = 0, tobj = 0;
			bool fv = false;
			const uint32_t* bits = nullptr;
			uint32_t tgt_lo = 0, tgt_cnt = 0;
			f3 dir = mk3(0.0f), orig = mk3(0.0f), sray = mk3(0.0f);
			float slen = 0.0f, inv_len = 0.0f, t_lo = 0.0f, t_hi = 1.0f;
			bool seg_ok = false;
			RaySlab slab{};
			bool ee_req = false; // an EE request: its swept-edge state is set up after the face walk
			uint32_t ee_slot = 0;
			float ee_pmax = 0.0f, ee_pmin = 0.0f;
			if (r < total)
			{
				// task of this request: last task with req_begin <= r
				uint32_t lo = 0, hi = ntasks;
				while (hi - lo > 1)
				{
					const uint32_t mid = (lo + hi) >> 1;
					if (tasks[mid].req_begin <= r)
						lo = mid;
					else
						hi = mid;
				}
				t = lo;
				const Task tk = tasks[t];
				const uint32_t local = r - tk.req_begin;
				dir = mk3(tk.dir[0], tk.dir[1], tk.dir[2]);
				if (local < tk.n_vf + tk.n_ee + tk.n_fv && (local < tk.n_vf || local >= tk.n_vf + tk.n_ee))
				{
					// VF: vertex of side 0 along +dir onto faces of side 1;
					// FV: vertex of side 1 along -dir onto faces of side 0
					fv = local >= tk.n_vf;
					vid = fv ? cand_v[size_t(tk.slot1) * v_stride + (local - tk.n_vf - tk.n_ee)] : cand_v[size_t(tk.slot0) * v_stride + local];
					const Slot tgt = slots[fv ? tk.slot0 : tk.slot1];
					tgt_lo = tgt.f_lo;
					tgt_cnt = tgt.f_cnt;
					tobj = tgt.pad[1];
					bits = bits_f + size_t(fv ? tk.slot0 : tk.slot1) * (f_stride / 32 + 1);
					const f3 cast = fv ? -dir : dir;
					orig = ld3(x, vid);
					const f3 end = orig + cast * 1.0f;
					// segment constants of seg_tri, once per ray
					const f3 sd = end - orig;
					const float len_sq = length_sq(sd);
					seg_ok = !(len_sq < 1e-6f * 1e-6f);
					slen = sqrtf(len_sq);
					inv_len = 1.0f / slen;
					sray = sd * inv_len;
					slab = make_slab(orig, cast);
					// clip the ray to the grown AABB of the candidate target faces
					const float* tb = slot_box + 12 * size_t(fv ? tk.slot0 : tk.slot1);
					if (ray_box_range(orig, cast, 0.0f, 1.0f, tb, tb + 3, t_lo, t_hi))
						kind = 1;
				}
				else if (local < tk.n_vf + tk.n_ee)
				{
					// EE: swept edge of side 0 along dir onto edges of side 1
					eid = cand_e[size_t(tk.slot0) * e_stride + (local - tk.n_vf)];
					bits = bits_e + size_t(tk.slot1) * (e_stride / 32 + 1);
					const Slot s1 = slots[tk.slot1];
					tgt_lo = s1.e_lo;
					tgt_cnt = s1.e_cnt;
					tobj = s1.pad[1];
					ee_req = true;
					ee_slot = tk.slot1;
					ee_pmax = tk.ee_pmax;
					ee_pmin = tk.ee_pmin;
				}
			}

			// ---- face tree: VF / FV rays of the warp
			// each lane starts at its target object's subtree root of this part; lanes with the
			// same start walk together
			const uint32_t foff = front_offset(split);
			const uint32_t fstart_l = kind == 1 ? ffront[size_t(tobj) * kFrontStride + foff + part] : kInvalid;
			uint32_t fpending = __ballot_sync(0xFFFFFFFFu, fstart_l != kInvalid);
			while (fpending != 0u)
			{
				const uint32_t fstart = __shfl_sync(0xFFFFFFFFu, fstart_l, __ffs(fpending) - 1);
				const bool on = fstart_l == fstart;
				fpending &= ~__ballot_sync(0xFFFFFFFFu, on);
				ray_visits += on ? 1u : 0u;
				// depth first: a hit inner node continues with its first child and stacks the second
				uint32_t node = fstart;
				int sp = 0;
				uint32_t loop = 0;
				for (;;)
				{
					NodeBox b;
					b.mn = __ldg(&fgrow[node].mn);
					b.mx = __ldg(&fgrow[node].mx);
					visited += on ? 1u : 0u;
					fetch_nodes++;
					const bool hit = on && ray_grown_box(slab, t_lo, t_hi, b);
					const uint32_t link_a = __float_as_uint(b.mn.w), link_b = __float_as_uint(b.mx.w);
					bool descend = false;
					if (__ballot_sync(0xFFFFFFFFu, hit) == 0u)
					{
					}
					else if (link_b == kInvalid)
					{
						const uint32_t fid = link_a;
						fetch_tris++;
						if (hit)
						{
							tested++;
							if (bit_test(bits, tgt_lo, tgt_cnt, fid))
							{
								ctested++;
								const uint32_t f0 = faces[3 * fid], f1 = faces[3 * fid + 1], f2 = faces[3 * fid + 2];
								if (vid != f0 && vid != f1 && vid != f2 && seg_ok)
								{
									f3 bary;
									float tt;
									const f3 A = ld3(x, f0), B = ld3(x, f1), C = ld3(x, f2);
									bool hit32 = false;
									if (ray_tri(orig, sray, slen, A, B, C, tt, bary))
									{
										tt = tt * inv_len;
										hit32 = tt >= 0.0f && tt <= 1.0f;
										if (hit32)
											emit(sink, t, fv ? 2u : 0u, fv ? fid : vid, fv ? vid : fid, bary.x, bary.y, tt * 1.0f);
									}
									if (RECHECK && tri_needs_recheck(orig, sray, slen, A, B, C))
									{
										const uint32_t rc = recheck_vf(orig, fv ? -dir : dir, A, B, C, hit32);
										rechecks += rc & 1u;
										flips += rc >> 1;
									}
								}
							}
						}
						__syncwarp();
					}
					else
					{
						ray_visits += hit ? 2u : 0u;
						if (sp + 1 > kStack)
						{
							if (lane == 0)
								atomicOr(dev_err, U26_DEVERR_STACK_OVERFLOW);
							break;
						}
						if (lane == (sp & 31))
						{
							if (sp < 32)
								s_lo = link_b;
							else
								s_hi = link_b;
						}
						sp++;
						node = link_a;
						descend = true;
					}
					if (++loop > 4000000u)
					{
						if (lane == 0)
							atomicOr(dev_err, U26_DEVERR_ITERATION_CAP);
						break;
					}
					if (descend)
						continue;
					if (sp == 0)
						break;
					sp--;
					node = __shfl_sync(0xFFFFFFFFu, sp < 32 ? s_lo : s_hi, sp & 31);
				}
				__syncwarp();
			}

			// ---- edge tree: EE swept edges of the warp (their state set up here, after the face
			// rays' state is dead)
			uint2 ev = make_uint2(0u, 0u);
			f3 p0 = mk3(0.0f), e1 = mk3(0.0f), pn = mk3(0.0f), smn = mk3(0.0f), smx = mk3(0.0f);
			float pd = 0.0f, ray_max = 0.0f, proj_lo = 0.0f, proj_hi = 0.0f;
			bool plane = false;
			if (ee_req)
			{
				ev = edges[eid];
				p0 = ld3(x, ev.x);
				const f3 p1 = ld3(x, ev.y);
				const float dl2 = dot(dir, dir);
				ray_max = 1.0f;
				if (!(dl2 <= 1e-12f))
				{
					const float smin = fminf(dot(p0, dir), dot(p1, dir));
					ray_max = fminf(fmaxf((ee_pmax - smin) / dl2 + 1e-5f, 0.0f), 1.0f);
				}
				if (ray_max > 0.0f)
				{
					// the swept edge's extent along dir (prp_compute_edge_projection_bounds with the
					// target edges' lower bound, cached_bvh.cpp:377-473), widened by 1e-6
					const float ep0 = dot(p0, dir), ep1 = dot(p1, dir);
					proj_lo = fmaxf(fminf(ep0, ep1), ee_pmin - 1e-5f) - 1e-6f;
					proj_hi = (fmaxf(ep0, ep1) + ray_max * dl2) + 1e-6f;
					e1 = p1 - p0;
					pn = cross(e1, dir);
					const float nl = length(pn);
					plane = nl >= 1e-10f;
					if (plane)
					{
						pn = pn / nl;
						pd = dot(pn, p0);
					}
					const f3 a_end = p0 + dir * ray_max, b_end = p1 + dir * ray_max;
					smn = vmin(vmin(p0, p1), vmin(a_end, b_end));
					smx = vmax(vmax(p0, p1), vmax(a_end, b_end));
					// intersect the swept box with the grown AABB of the candidate target edges
					const float* tb = slot_box + 12 * size_t(ee_slot) + 6;
					const float g0 = 1e-5f * (1.0f + fmaxf(fabsf(tb[0]), fabsf(tb[3])));
					const float g1 = 1e-5f * (1.0f + fmaxf(fabsf(tb[1]), fabsf(tb[4])));
					const float g2 = 1e-5f * (1.0f + fmaxf(fabsf(tb[2]), fabsf(tb[5])));
					smn = vmax(smn, mk3(tb[0] - g0, tb[1] - g1, tb[2] - g2));
					smx = vmin(smx, mk3(tb[3] + g0, tb[4] + g1, tb[5] + g2));
					if (smn.x <= smx.x && smn.y <= smx.y && smn.z <= smx.z)
						kind = 2;
				}
			}
			const uint32_t estart_l = kind == 2 ? efront[size_t(tobj) * kFrontStride + foff + part] : kInvalid;
			uint32_t epending = __ballot_sync(0xFFFFFFFFu, estart_l != kInvalid);
			while (epending != 0u)
			{
				const uint32_t estart = __shfl_sync(0xFFFFFFFFu, estart_l, __ffs(epending) - 1);
				const bool on = estart_l == estart;
				epending &= ~__ballot_sync(0xFFFFFFFFu, on);
				ray_visits += on ? 1u : 0u;
				uint32_t node = estart;
				int sp = 0;
				uint32_t loop = 0;
				for (;;)
				{
					NodeBox g;
					g.mn = __ldg(&egrow[node].mn);
					g.mx = __ldg(&egrow[node].mx);
					visited += on ? 1u : 0u;
					fetch_nodes++;
					bool hit = on && (smn.x <= g.mx.x) & (smx.x >= g.mn.x) & (smn.y <= g.mx.y) & (smx.y >= g.mn.y) & (smn.z <= g.mx.z) &
						(smx.z >= g.mn.z);
					// the swept edge lies in the plane (pn, pd): a box that keeps clear of the slab
					// |dot(pn, q) - pd| <= 1e-6 holds only edges the leaf's separating-plane test
					// rejects (cached_bvh.cpp:433-473 prunes its nodes the same way). The boxes carry
					// the 1e-5 (1 + |c|) margin, far above the rounding of this test, so no edge the
					// leaf test keeps is pruned.
					// and a box whose extent along dir misses the swept edge's holds no edge it reaches
					if (hit)
					{
						const f3 c = mk3(0.5f * (g.mn.x + g.mx.x), 0.5f * (g.mn.y + g.mx.y), 0.5f * (g.mn.z + g.mx.z));
						const f3 h = mk3(0.5f * (g.mx.x - g.mn.x), 0.5f * (g.mx.y - g.mn.y), 0.5f * (g.mx.z - g.mn.z));
						const float cp = dot(c, dir);
						const float pr = (h.x * fabsf(dir.x) + h.y * fabsf(dir.y)) + h.z * fabsf(dir.z);
						hit = !(cp + pr < proj_lo || cp - pr > proj_hi);
						if (hit && plane)
						{
							const float rad = (h.x * fabsf(pn.x) + h.y * fabsf(pn.y)) + h.z * fabsf(pn.z);
							hit = fabsf(dot(pn, c) - pd) <= rad + 1e-6f;
						}
					}
					const uint32_t link_a = __float_as_uint(g.mn.w), link_b = __float_as_uint(g.mx.w);
					bool descend = false;
					if (__ballot_sync(0xFFFFFFFFu, hit) == 0u)
					{
					}
					else if (link_b == kInvalid)
					{
						const uint32_t e2 = link_a;
						fetch_edges++;
						if (hit)
						{
							tested++;
							etested++;
							if (bit_test(bits, tgt_lo, tgt_cnt, e2))
							{
								ctested++;
								const uint2 qv = edges[e2];
								if (!(ev.x == qv.x || ev.x == qv.y || ev.y == qv.x || ev.y == qv.y))
								{
									const f3 q0 = ld3(x, qv.x), q1 = ld3(x, qv.y);
									bool sep = false, ee_hit = false;
									if (plane)
									{
										const float d0 = dot(pn, q0) - pd;
										const float d1 = dot(pn, q1) - pd;
										sep = (d0 > 1e-6f && d1 > 1e-6f) || (d0 < -1e-6f && d1 < -1e-6f);
									}
									if (!sep)
									{
										const f3 e2v = q1 - q0;
										const f3 rr = q0 - p0;
										const f3 n = cross(e1, e2v);
										const float det = -dot(dir, n);
										if (!(fabsf(det) < 1e-10f))
										{
											// x = n_x / det. Misses decided before the division, only where the test
											// below rejects too: a numerator (|n| >= 1e-20, so n / det stays nonzero) of
											// the other sign than det, or t1, t2 beyond 1 / sv beyond ray_max by a 1e-5
											// relative margin; each numerator is computed once the earlier ones pass
											const float n_sv = -dot(rr, cross(e1, e2v));
											const float adet = fabsf(det);
											const bool screen = adet <= 1e20f;
											auto neg = [&](float v)
											{ return fabsf(v) >= 1e-20f && ((v > 0.0f) != (det > 0.0f)); };
											const float lim = adet * (1.0f + 1e-5f);
											bool maybe = !(screen && (neg(n_sv) || (ray_max >= 1e-20f && fabsf(n_sv) > lim * ray_max)));
											float n_t1 = 0.0f, n_t2 = 0.0f;
											if (maybe)
											{
												n_t1 = -dot(dir, cross(rr, e2v));
												maybe = !(screen && (neg(n_t1) || fabsf(n_t1) > lim));
											}
											if (maybe)
											{
												n_t2 = dot(dir, cross(e1, rr));
												maybe = !(screen && (neg(n_t2) || fabsf(n_t2) > lim));
											}
											if (maybe)
											{
												const float inv = 1.0f / det;
												const float sv = n_sv * inv;
												const float t1 = n_t1 * inv;
												const float t2 = n_t2 * inv;
												if (sv >= 0.0f && sv <= ray_max && t1 >= 0.0f && t1 <= 1.0f && t2 >= 0.0f && t2 <= 1.0f)
												{
													ee_hit = true;
													emit(sink, t, 1u, eid, e2, 1.0f - t1, 1.0f - t2, sv);
												}
											}
										}
									}
									Band bd;
									if (RECHECK)
										edge_edge_band(p0, e1, dir, ray_max, plane, pn, pd, q0, q1, bd);
									if (RECHECK && bd.recheck())
									{
										const uint32_t rc = recheck_ee(p0, e1, dir, ray_max, q0, q1, ee_hit);
										rechecks += rc & 1u;
										flips += rc >> 1;
									}
								}
							}
						}
						__syncwarp();
					}
					else
					{
						ray_visits += hit ? 2u : 0u;
						if (sp + 1 > kStack)
						{
							if (lane == 0)
								atomicOr(dev_err, U26_DEVERR_STACK_OVERFLOW);
							break;
						}
						if (lane == (sp & 31))
						{
							if (sp < 32)
								s_lo = link_b;
							else
								s_hi = link_b;
						}
						sp++;
						node = link_a;
						descend = true;
					}
					if (++loop > 4000000u)
					{
						if (lane == 0)
							atomicOr(dev_err, U26_DEVERR_ITERATION_CAP);
						break;
					}
					if (descend)
						continue;
					if (sp == 0)
						break;
					sp--;
					node = __shfl_sync(0xFFFFFFFFu, sp < 32 ? s_lo : s_hi, sp & 31);
				}
				__syncwarp();
			}
			if constexpr (!QUEUE)
				break;
			}
			if (stats)
			{
				const uint32_t tsum = __reduce_add_sync(0xFFFFFFFFu, tested);
				const uint32_t rsum = __reduce_add_sync(0xFFFFFFFFu, reqs);
				const uint32_t vsum = __reduce_add_sync(0xFFFFFFFFu, visited);
				const uint32_t esum = __reduce_add_sync(0xFFFFFFFFu, etested);
				const uint32_t rvsum = __reduce_add_sync(0xFFFFFFFFu, ray_visits);
				const uint32_t csum = __reduce_add_sync(0xFFFFFFFFu, ctested);
				const uint32_t rcsum = __reduce_add_sync(0xFFFFFFFFu, rechecks);
				const uint32_t flsum = __reduce_add_sync(0xFFFFFFFFu, flips);
				if (lane == 0)
				{
					// [0] leaf primitive tests, [1] requests, [2] ray-node tests, [3] edge leaf tests,
					// [4] node fetches, [5] triangle fetches, [6] edge fetches (per packet),
					// [7] single-ray node visits, [8] leaf tests of candidate targets
					atomicAdd(stats + 7, (unsigned long long)rvsum);
					atomicAdd(stats + 8, (unsigned long long)csum);
					// [9] FP64 rechecks of leaf tests inside their error band, [10] FP32 / FP64 flips
					if (rcsum)
						atomicAdd(stats + 9, (unsigned long long)rcsum);
					if (flsum)
						atomicAdd(stats + 10, (unsigned long long)flsum);
					atomicAdd(stats + 0, (unsigned long long)tsum);
					atomicAdd(stats + 1, (unsigned long long)rsum);
					atomicAdd(stats + 2, (unsigned long long)vsum);
					atomicAdd(stats + 3, (unsigned long long)esum);
					atomicAdd(stats + 4, (unsigned long long)fetch_nodes);
					atomicAdd(stats + 5, (unsigned long long)fetch_tris);
					atomicAdd(stats + 6, (unsigned long long)fetch_edges);
				}
			}
		}

		// The traversal configurations the autotuner chooses from: subtree parts per request
		// (4, 8, 16) x resident blocks of 128 threads per SM the registers are sized for (6, 7, 8:
		// at most 80, 72 or 64 registers per thread) x the grid form (one warp per work item, or a
		// persistent grid of warps taking items from a queue). The packet is the warp (32 requests).
		struct RaycastConfig
		{
			uint32_t split;
			int min_blocks;
			bool queue;
		};
		constexpr RaycastConfig kRaycastConfigs[] = { { 4, 6, false }, { 4, 7, false }, { 4, 8, false }, { 8, 6, false }, { 8, 7, false },
			{ 8, 8, false }, { 16, 6, false }, { 16, 7, false }, { 16, 8, false }, { 4, 6, true }, { 4, 7, true }, { 4, 8, true }, { 8, 6, true },
			{ 8, 7, true }, { 8, 8, true }, { 16, 6, true }, { 16, 7, true }, { 16, 8, true } };
		constexpr int kNumRaycastConfigs = 18, kDefaultRaycastConfig = 4; // 8 parts, 7 blocks per SM, a warp per item
		using RaycastFn = decltype(&raycast_kernel<false, 7, false>);
		template <bool R, bool Q>
		inline RaycastFn raycast_variant_q(int min_blocks)
		{
			return min_blocks == 6 ? &raycast_kernel<R, 6, Q> : min_blocks == 8 ? &raycast_kernel<R, 8, Q> : &raycast_kernel<R, 7, Q>;
		}
		inline RaycastFn raycast_variant(bool recheck, int min_blocks, bool queue)
		{
			if (recheck)
				return queue ? raycast_variant_q<true, true>(min_blocks) : raycast_variant_q<true, false>(min_blocks);
			return queue ? raycast_variant_q<false, true>(min_blocks) : raycast_variant_q<false, false>(min_blocks);
		}

		// ---- the plain form (the comparison baseline of the batched, filtered form above):
		// one thread per request with a private stack from the root, the epsilon-grown node
		// tests evaluated per visit, no clipping to the candidate boxes, one launch per contour.
		// It decides the same (request, primitive) pairs with the same exact tests.
		__device__ __forceinline__ bool ray_box_plain(f3 o, f3 d, const NodeBox& b)
		{
			float tmin = 0.0f, tmax = 1.0f;
			const float lo[3] = { b.mn.x, b.mn.y, b.mn.z }, hi[3] = { b.mx.x, b.mx.y, b.mx.z };
			const float oo[3] = { o.x, o.y, o.z }, dd[3] = { d.x, d.y, d.z };
#pragma unroll
			for (int a = 0; a < 3; a++)
			{
				const float eps = 1e-5f * (1.0f + fmaxf(fabsf(lo[a]), fabsf(hi[a])));
				const float l = lo[a] - eps, h = hi[a] + eps;
				if (fabsf(dd[a]) < 1e-30f)
				{
					if (oo[a] < l || oo[a] > h)
						return false;
					continue;
				}
				const float inv = 1.0f / dd[a];
				float t0 = (l - oo[a]) * inv, t1 = (h - oo[a]) * inv;
				if (t0 > t1)
				{
					const float tt = t0;
					t0 = t1;
					t1 = tt;
				}
				tmin = fmaxf(tmin, t0);
				tmax = fminf(tmax, t1);
			}
			return tmin <= tmax;
		}

		__global__ void __launch_bounds__(128) raycast_plain_kernel(const Task* __restrict__ tasks, uint32_t t_first, uint32_t ntasks,
			uint32_t r_first, uint32_t count, const Slot* __restrict__ slots, const uint32_t* __restrict__ cand_v,
			const uint32_t* __restrict__ cand_e, uint32_t v_stride, uint32_t e_stride, uint32_t f_stride, const uint32_t* __restrict__ bits_e,
			const uint32_t* __restrict__ bits_f, TreeView ftree, TreeView etree, const float* __restrict__ x, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, HitSink sink, unsigned long long* __restrict__ stats, uint32_t* __restrict__ dev_err)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			uint32_t tested = 0, visited = 0, etested = 0;
			if (i < count)
			{
				const uint32_t r = r_first + i;
				uint32_t lo = t_first, hi = t_first + ntasks;
				while (hi - lo > 1)
				{
					const uint32_t mid = (lo + hi) >> 1;
					if (tasks[mid].req_begin <= r)
						lo = mid;
					else
						hi = mid;
				}
				const uint32_t t = lo;
				const Task tk = tasks[t];
				const uint32_t local = r - tk.req_begin;
				const f3 dir = mk3(tk.dir[0], tk.dir[1], tk.dir[2]);
				uint32_t stack[64];
				int sp = 0;
				if (local < tk.n_vf || local >= tk.n_vf + tk.n_ee)
				{
					const bool fv = local >= tk.n_vf;
					const uint32_t vid = fv ? cand_v[size_t(tk.slot1) * v_stride + (local - tk.n_vf - tk.n_ee)] : cand_v[size_t(tk.slot0) * v_stride + local];
					const Slot tgt = slots[fv ? tk.slot0 : tk.slot1];
					const uint32_t* bits = bits_f + size_t(fv ? tk.slot0 : tk.slot1) * (f_stride / 32 + 1);
					const f3 cast = fv ? -dir : dir;
					const f3 orig = ld3(x, vid);
					const f3 end = orig + cast * 1.0f;
					if (ftree.n)
						stack[sp++] = 0u;
					for (uint32_t loop = 0; sp > 0; loop++)
					{
						const uint32_t node = stack[--sp];
						visited++;
						NodeBox b;
						b.mn = __ldg(&ftree.boxes[node].mn);
						b.mx = __ldg(&ftree.boxes[node].mx);
						if (!ray_box_plain(orig, cast, b))
							continue;
						const uint32_t fid = __ldg(ftree.object_idx + node);
						if (fid != kInvalid)
						{
							tested++;
							if (!bit_test(bits, tgt.f_lo, tgt.f_cnt, fid))
								continue;
							const uint32_t f0 = faces[3 * fid], f1 = faces[3 * fid + 1], f2 = faces[3 * fid + 2];
							if (vid == f0 || vid == f1 || vid == f2)
								continue;
							f3 bary;
							float tt;
							if (seg_tri(orig, end, ld3(x, f0), ld3(x, f1), ld3(x, f2), bary, tt) && tt >= 0.0f && tt <= 1.0f)
								emit(sink, t, fv ? 2u : 0u, fv ? fid : vid, fv ? vid : fid, bary.x, bary.y, tt * 1.0f);
							continue;
						}
						if (sp + 2 > 64 || loop > 4000000u)
						{
							atomicOr(dev_err, sp + 2 > 64 ? U26_DEVERR_STACK_OVERFLOW : U26_DEVERR_ITERATION_CAP);
							break;
						}
						const uint2 ch = __ldg(ftree.children + node);
						stack[sp++] = ch.y;
						stack[sp++] = ch.x;
					}
				}
				else
				{
					const uint32_t eid = cand_e[size_t(tk.slot0) * e_stride + (local - tk.n_vf)];
					const uint32_t* bits = bits_e + size_t(tk.slot1) * (e_stride / 32 + 1);
					const Slot s1 = slots[tk.slot1];
					const uint2 ev = edges[eid];
					const f3 p0 = ld3(x, ev.x), p1 = ld3(x, ev.y);
					const float dl2 = dot(dir, dir);
					float ray_max = 1.0f;
					if (!(dl2 <= 1e-12f))
					{
						const float smin = fminf(dot(p0, dir), dot(p1, dir));
						ray_max = fminf(fmaxf((tk.ee_pmax - smin) / dl2 + 1e-5f, 0.0f), 1.0f);
					}
					const f3 e1 = p1 - p0;
					f3 pn = cross(e1, dir);
					const float nl = length(pn);
					const bool plane = nl >= 1e-10f;
					float pd = 0.0f;
					if (plane)
					{
						pn = pn / nl;
						pd = dot(pn, p0);
					}
					const f3 a_end = p0 + dir * ray_max, b_end = p1 + dir * ray_max;
					const f3 smn = vmin(vmin(p0, p1), vmin(a_end, b_end));
					const f3 smx = vmax(vmax(p0, p1), vmax(a_end, b_end));
					if (ray_max > 0.0f && etree.n)
						stack[sp++] = 0u;
					for (uint32_t loop = 0; sp > 0; loop++)
					{
						const uint32_t node = stack[--sp];
						visited++;
						NodeBox b;
						b.mn = __ldg(&etree.boxes[node].mn);
						b.mx = __ldg(&etree.boxes[node].mx);
						const float e = 1e-5f * (1.0f + fmaxf(fmaxf(fmaxf(fabsf(b.mn.x), fabsf(b.mx.x)), fmaxf(fabsf(b.mn.y), fabsf(b.mx.y))),
															   fmaxf(fabsf(b.mn.z), fabsf(b.mx.z))));
						if (!((smn.x <= b.mx.x + e) & (smx.x >= b.mn.x - e) & (smn.y <= b.mx.y + e) & (smx.y >= b.mn.y - e) & (smn.z <= b.mx.z + e) &
								(smx.z >= b.mn.z - e)))
							continue;
						const uint32_t e2 = __ldg(etree.object_idx + node);
						if (e2 != kInvalid)
						{
							tested++;
							etested++;
							if (!bit_test(bits, s1.e_lo, s1.e_cnt, e2))
								continue;
							const uint2 qv = edges[e2];
							if (ev.x == qv.x || ev.x == qv.y || ev.y == qv.x || ev.y == qv.y)
								continue;
							const f3 q0 = ld3(x, qv.x), q1 = ld3(x, qv.y);
							if (plane)
							{
								const float d0 = dot(pn, q0) - pd;
								const float d1 = dot(pn, q1) - pd;
								if ((d0 > 1e-6f && d1 > 1e-6f) || (d0 < -1e-6f && d1 < -1e-6f))
									continue;
							}
							const f3 e2v = q1 - q0;
							const f3 rr = q0 - p0;
							const f3 n = cross(e1, e2v);
							const float det = -dot(dir, n);
							if (fabsf(det) < 1e-10f)
								continue;
							const float inv = 1.0f / det;
							const float d_r_e1_e2 = dot(rr, cross(e1, e2v));
							const float d_dir_r_e2 = dot(dir, cross(rr, e2v));
							const float d_dir_e1_r = dot(dir, cross(e1, rr));
							const float sv = -d_r_e1_e2 * inv;
							const float t1 = -d_dir_r_e2 * inv;
							const float t2 = d_dir_e1_r * inv;
							if (sv >= 0.0f && sv <= ray_max && t1 >= 0.0f && t1 <= 1.0f && t2 >= 0.0f && t2 <= 1.0f)
								emit(sink, t, 1u, eid, e2, 1.0f - t1, 1.0f - t2, sv);
							continue;
						}
						if (sp + 2 > 64 || loop > 4000000u)
						{
							atomicOr(dev_err, sp + 2 > 64 ? U26_DEVERR_STACK_OVERFLOW : U26_DEVERR_ITERATION_CAP);
							break;
						}
						const uint2 ch = __ldg(etree.children + node);
						stack[sp++] = ch.y;
						stack[sp++] = ch.x;
					}
				}
			}
			if (stats)
			{
				const uint32_t mask = __activemask();
				const uint32_t tsum = __reduce_add_sync(mask, tested);
				const uint32_t rsum = __reduce_add_sync(mask, i < count ? 1u : 0u);
				const uint32_t vsum = __reduce_add_sync(mask, visited);
				const uint32_t esum = __reduce_add_sync(mask, etested);
				if ((threadIdx.x & 31) == uint32_t(__ffs(mask) - 1))
				{
					atomicAdd(stats + 0, (unsigned long long)tsum);
					atomicAdd(stats + 1, (unsigned long long)rsum);
					atomicAdd(stats + 2, (unsigned long long)vsum);
					atomicAdd(stats + 3, (unsigned long long)esum);
					atomicAdd(stats + 4, (unsigned long long)vsum);
					atomicAdd(stats + 5, (unsigned long long)(tsum - esum));
					atomicAdd(stats + 6, (unsigned long long)esum);
					atomicAdd(stats + 7, (unsigned long long)vsum);
				}
			}
		}

		// ------------------------------------------------------------ post-processing
		struct HitKeyCodec
		{
			int b;
			__device__ __forceinline__ uint32_t task(uint64_t k) const { return uint32_t(k >> (2 + 2 * b)); }
			__device__ __forceinline__ uint32_t type(uint64_t k) const { return uint32_t(k >> (2 * b)) & 3u; }
			__device__ __forceinline__ uint32_t src(uint64_t k) const { return uint32_t(k >> b) & ((1u << b) - 1u); }
			__device__ __forceinline__ uint32_t dst(uint64_t k) const { return uint32_t(k) & ((1u << b) - 1u); }
			__device__ __forceinline__ uint64_t make(uint32_t t, uint32_t ty, uint32_t s, uint32_t d) const
			{
				return (uint64_t(t) << (2 + 2 * b)) | (uint64_t(ty) << (2 * b)) | (uint64_t(s) << b) | uint64_t(d);
			}
		};

		__global__ void segments_kernel(const uint64_t* __restrict__ keys, uint32_t n, HitKeyCodec cd, uint32_t ntasks, uint32_t* __restrict__ seg)
		{
			const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
			if (t > ntasks)
				return;
			const uint64_t key = uint64_t(t) << (2 + 2 * cd.b);
			uint32_t lo = 0, hi = n;
			while (lo < hi)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (keys[mid] < key)
					lo = mid + 1;
				else
					hi = mid;
			}
			seg[t] = lo;
		}

		__device__ __forceinline__ void hit_verts(uint32_t type, uint32_t src, uint32_t dst, const uint2* edges, const uint32_t* faces,
			uint32_t sv[3], uint32_t dv[3])
		{
			sv[0] = sv[1] = sv[2] = kInf;
			dv[0] = dv[1] = dv[2] = kInf;
			if (type == 0u)
			{
				sv[0] = src;
				dv[0] = faces[3 * dst];
				dv[1] = faces[3 * dst + 1];
				dv[2] = faces[3 * dst + 2];
			}
			else if (type == 1u)
			{
				const uint2 a = edges[src], b = edges[dst];
				sv[0] = a.x;
				sv[1] = a.y;
				dv[0] = b.x;
				dv[1] = b.y;
			}
			else
			{
				sv[0] = faces[3 * src];
				sv[1] = faces[3 * src + 1];
				sv[2] = faces[3 * src + 2];
				dv[0] = dst;
			}
		}

		__device__ __forceinline__ bool has_flag(const uint32_t* off, const uint32_t* fl, uint32_t v, uint32_t flag)
		{
			uint32_t lo = off[v], hi = off[v + 1];
			while (lo < hi)
			{
				const uint32_t mid = (lo + hi) >> 1;
				const uint32_t x = fl[mid];
				if (x == flag)
					return true;
				if (x < flag)
					lo = mid + 1;
				else
					hi = mid;
			}
			return false;
		}

		__global__ void init_hits_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ perm, const float* __restrict__ pay_in,
			float* __restrict__ pay, uint32_t n, HitKeyCodec cd, const Task* __restrict__ tasks, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, const uint32_t* __restrict__ vf_off, const uint32_t* __restrict__ vf,
			uint32_t* __restrict__ parent, uint8_t* __restrict__ attached, uint32_t* __restrict__ comp_size, uint32_t* __restrict__ comp_att)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint32_t j = perm[i];
			pay[3 * i] = pay_in[3 * j];
			pay[3 * i + 1] = pay_in[3 * j + 1];
			pay[3 * i + 2] = pay_in[3 * j + 2];
			parent[i] = i;
			comp_size[i] = 0u;
			comp_att[i] = 0u;
			const uint64_t k = keys[i];
			const uint32_t c = tasks[cd.task(k)].contour_global;
			uint32_t sv[3], dv[3];
			hit_verts(cd.type(k), cd.src(k), cd.dst(k), edges, faces, sv, dv);
			bool ok = true;
			for (int q = 0; q < 3; q++)
				if (sv[q] != kInf)
					ok = ok && has_flag(vf_off, vf, sv[q], 2u * c);
			for (int q = 0; q < 3; q++)
				if (dv[q] != kInf)
					ok = ok && has_flag(vf_off, vf, dv[q], 2u * c + 1u);
			attached[i] = ok ? 1 : 0;
		}

		__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x)
		{
			uint32_t p = parent[x];
			while (p != x)
			{
				const uint32_t gp = parent[p];
				if (gp != p)
					parent[x] = gp; // path halving (benign race)
				x = p;
				p = gp;
			}
			return x;
		}

		__device__ __forceinline__ void uf_union(uint32_t* parent, uint32_t a, uint32_t b, uint32_t* dev_err)
		{
			for (int it = 0; it < 1 << 20; it++)
			{
				a = uf_find(parent, a);
				b = uf_find(parent, b);
				if (a == b)
					return;
				if (a > b)
				{
					const uint32_t t = a;
					a = b;
					b = t;
				}
				// hook the larger root under the smaller
				const uint32_t old = atomicCAS(parent + b, b, a);
				if (old == b)
					return;
				b = old;
			}
			atomicOr(dev_err, U26_DEVERR_ITERATION_CAP);
		}

		__device__ __forceinline__ uint32_t find_key(const uint64_t* keys, uint32_t lo, uint32_t hi, uint64_t key)
		{
			while (lo < hi)
			{
				const uint32_t mid = (lo + hi) >> 1;
				const uint64_t k = keys[mid];
				if (k == key)
					return mid;
				if (k < key)
					lo = mid + 1;
				else
					hi = mid;
			}
			return kInf;
		}

		// ---- run directory: every (task, type, source) run of the sorted hits, in an
		// open-addressing hash table keyed by that prefix (value: run id; run r spans
		// [heads[r], heads[r + 1]))
		struct RunDir
		{
			const uint64_t* hkeys; // prefix + 1 (0: empty slot)
			const uint32_t* hvals;
			const uint32_t* heads;
			uint32_t mask;
		};
		__device__ __forceinline__ uint32_t run_hash(uint64_t p)
		{
			p ^= p >> 33;
			p *= 0xff51afd7ed558ccdull;
			p ^= p >> 33;
			p *= 0xc4ceb9fe1a85ec53ull;
			p ^= p >> 33;
			return uint32_t(p);
		}
		__global__ void run_flags_kernel(const uint64_t* __restrict__ keys, uint32_t n, int b, uint32_t* __restrict__ flag)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i > n)
				return;
			flag[i] = (i < n && (i == 0 || (keys[i] >> b) != (keys[i - 1] >> b))) ? 1u : 0u;
		}
		// flag[] scanned in place: flag[i] = run id of a head i; flag[n] = number of runs
		__global__ void run_insert_kernel(const uint64_t* __restrict__ keys, uint32_t n, int b, const uint32_t* __restrict__ scanned,
			uint32_t* __restrict__ heads, uint64_t* __restrict__ hkeys, uint32_t* __restrict__ hvals, uint32_t mask, uint32_t* __restrict__ dev_err)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i > n)
				return;
			if (i == n)
			{
				heads[scanned[n]] = n;
				return;
			}
			if (!(i == 0 || (keys[i] >> b) != (keys[i - 1] >> b)))
				return;
			const uint32_t r = scanned[i];
			heads[r] = i;
			const uint64_t k = (keys[i] >> b) + 1u;
			uint32_t h = run_hash(k) & mask;
			for (uint32_t it = 0; it <= mask; it++)
			{
				const unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(hkeys + h), 0ull, (unsigned long long)k);
				if (old == 0ull)
				{
					hvals[h] = r;
					return;
				}
				h = (h + 1u) & mask;
			}
			atomicOr(dev_err, U26_DEVERR_ITERATION_CAP);
		}
		// [rb, re) of the run with this prefix (empty when absent)
		__device__ __forceinline__ void run_lookup(const RunDir& d, uint64_t prefix, uint32_t& rb, uint32_t& re)
		{
			const uint64_t k = prefix + 1u;
			uint32_t h = run_hash(k) & d.mask;
			rb = re = 0;
			for (uint32_t it = 0; it <= d.mask; it++)
			{
				const uint64_t v = d.hkeys[h];
				if (v == k)
				{
					const uint32_t r = d.hvals[h];
					rb = d.heads[r];
					re = d.heads[r + 1];
					return;
				}
				if (v == 0ull)
					return;
				h = (h + 1u) & d.mask;
			}
		}

		// find_adjacent_hits rules as exact key lookups inside the task segment. Lookups that
		// share a (type, source) first find that source's run of hits once, then search the
		// targets inside the (short) run. Every rule is symmetric (its mirror rule from the
		// other hit's type gives the same pair, since the adjacency lists are the mesh's
		// incidence relations), so each unordered pair is looked up from one side only:
		// same-type pairs from the smaller adjacent id, VF-FV pairs from the FV hit, VF-EE and
		// FV-EE pairs from the EE hit (the sides with the fewest lookups). The components are
		// those of the two-sided rules.
		__global__ void union_kernel(const uint64_t* __restrict__ keys, uint32_t n, HitKeyCodec cd, const uint32_t* __restrict__ seg,
			const uint2* __restrict__ edges, const uint32_t* __restrict__ faces, const uint32_t* __restrict__ fae,
			const uint32_t* __restrict__ vav_off, const uint32_t* __restrict__ vav, const uint32_t* __restrict__ vae_off,
			const uint32_t* __restrict__ vae, const uint32_t* __restrict__ vaf_off, const uint32_t* __restrict__ vaf,
			const uint32_t* __restrict__ eaf_off, const uint32_t* __restrict__ eaf, const uint32_t* __restrict__ eae_off,
			const uint32_t* __restrict__ eae, RunDir dir, uint32_t* __restrict__ parent, uint32_t* __restrict__ dev_err)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint64_t k = keys[i];
			const uint32_t t = cd.task(k), ty = cd.type(k), s = cd.src(k), d = cd.dst(k);
			// [rb, re): the hits of (t, ty2, src2), from the run directory
			auto run = [&](uint32_t ty2, uint32_t src2, uint32_t& rb, uint32_t& re)
			{ run_lookup(dir, cd.make(t, ty2, src2, 0u) >> cd.b, rb, re); };
			auto link_in = [&](uint32_t rb, uint32_t re, uint32_t nty, uint32_t ns, uint32_t nd)
			{
				if (rb >= re)
					return;
				const uint32_t j = find_key(keys, rb, re, cd.make(t, nty, ns, nd));
				if (j != kInf && j != i)
					uf_union(parent, i, j, dev_err);
			};
			auto link = [&](uint32_t nty, uint32_t ns, uint32_t nd)
			{
				uint32_t rb2, re2;
				run(nty, ns, rb2, re2);
				link_in(rb2, re2, nty, ns, nd);
			};
			uint32_t rb, re;
			if (ty == 0u)
			{
				// VF(v, f) - VF(v', f), v' adjacent to v (VF-FV and VF-EE pairs come from the other side)
				for (uint32_t q = vav_off[s]; q < vav_off[s + 1]; q++)
					if (vav[q] > s)
						link(0u, vav[q], d);
			}
			else if (ty == 2u)
			{
				// FV(f, w)
				for (int c = 0; c < 3; c++)
				{
					run(0u, faces[3 * s + c], rb, re);
					for (uint32_t q = vaf_off[d]; q < vaf_off[d + 1]; q++)
						link_in(rb, re, 0u, faces[3 * s + c], vaf[q]);
				}
				run(2u, s, rb, re);
				for (uint32_t q = vav_off[d]; q < vav_off[d + 1]; q++)
					if (vav[q] > d)
						link_in(rb, re, 2u, s, vav[q]);
			}
			else
			{
				// EE(e1, e2)
				const uint2 a = edges[s], b = edges[d];
				uint32_t rb2, re2;
				run(0u, a.x, rb, re);
				run(0u, a.y, rb2, re2);
				for (uint32_t q = eaf_off[d]; q < eaf_off[d + 1]; q++)
				{
					link_in(rb, re, 0u, a.x, eaf[q]);
					link_in(rb2, re2, 0u, a.y, eaf[q]);
				}
				for (uint32_t q = eaf_off[s]; q < eaf_off[s + 1]; q++)
				{
					run(2u, eaf[q], rb, re);
					link_in(rb, re, 2u, eaf[q], b.x);
					link_in(rb, re, 2u, eaf[q], b.y);
				}
				run(1u, s, rb, re);
				for (uint32_t q = eae_off[d]; q < eae_off[d + 1]; q++)
					if (eae[q] > d)
						link_in(rb, re, 1u, s, eae[q]);
				for (uint32_t q = eae_off[s]; q < eae_off[s + 1]; q++)
					if (eae[q] > s)
						link(1u, eae[q], d);
			}
		}

		// ---- solid-interior links (intersection_resolver2.cpp:3298-3464): hits sharing a
		// source vertex (VF), target vertex (FV) or source edge (EE), ordered by (distance,
		// key), link each hit to its successor when both targets lie on one solid mesh, the
		// distance grows by more than eps_d and the ray enters the first target and leaves
		// through the second. Each thread finds its hit's successor in its group.
		struct SolidParams
		{
			const float* fn;
			const float* en;
			const uint32_t* vobj;
			const uint8_t* vsolid;
			uint32_t all;
			float eps_n, eps_d;
		};
		__device__ __forceinline__ bool solid_link_ok(const SolidParams& sp, uint32_t ty, uint32_t ta, uint32_t tb, float da_, float db_, f3 r,
			const uint2* __restrict__ edges, const uint32_t* __restrict__ faces)
		{
			// ta / tb: the targets (faces for VF / FV, second edges for EE) of the hit and its successor
			const uint32_t va = ty == 1u ? edges[ta].x : faces[3 * ta], vb = ty == 1u ? edges[tb].x : faces[3 * tb];
			if (sp.vobj[va] != sp.vobj[vb] || !(sp.all || sp.vsolid[va]) || !(db_ - da_ > sp.eps_d))
				return false;
			const float* nrm = ty == 1u ? sp.en : sp.fn;
			const float a = dot(mk3(nrm[3 * ta], nrm[3 * ta + 1], nrm[3 * ta + 2]), r);
			const float b = dot(mk3(nrm[3 * tb], nrm[3 * tb + 1], nrm[3 * tb + 2]), r);
			if (ty == 2u)
				return a > sp.eps_n && b < -sp.eps_n;
			return a < -sp.eps_n && b > sp.eps_n;
		}

		// VF and EE groups are runs of the sorted hits (same task, type, source)
		__global__ void solid_runs_kernel(const uint64_t* __restrict__ keys, uint32_t n, HitKeyCodec cd, const uint32_t* __restrict__ seg,
			const float* __restrict__ pay, const Task* __restrict__ tasks, const uint2* __restrict__ edges, const uint32_t* __restrict__ faces,
			SolidParams sp, uint32_t* __restrict__ parent, uint32_t* __restrict__ dev_err)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint64_t k = keys[i];
			const uint32_t ty = cd.type(k);
			if (ty == 2u)
				return;
			const uint32_t t = cd.task(k), s = cd.src(k);
			const uint32_t lo = seg[t], hi = seg[t + 1];
			const uint64_t k0 = cd.make(t, ty, s, 0u), k1 = k0 + (uint64_t(1) << cd.b);
			// the run around i
			uint32_t rb = i, re = i + 1;
			for (int it = 0; it < (1 << 22) && rb > lo && keys[rb - 1] >= k0; it++)
				rb--;
			for (int it = 0; it < (1 << 22) && re < hi && keys[re] < k1; it++)
				re++;
			const float di = pay[3 * i + 2];
			uint32_t nxt = kInf;
			float dn = 0.0f;
			for (uint32_t j = rb; j < re; j++)
			{
				if (j == i)
					continue;
				const float dj = pay[3 * j + 2];
				const bool after = dj > di || (dj == di && j > i);
				if (after && (nxt == kInf || dj < dn || (dj == dn && j < nxt)))
				{
					nxt = j;
					dn = dj;
				}
			}
			if (nxt == kInf)
				return;
			const Task tk = tasks[t];
			if (solid_link_ok(sp, ty, cd.dst(k), cd.dst(keys[nxt]), di, dn, mk3(tk.dir[0], tk.dir[1], tk.dir[2]), edges, faces))
				uf_union(parent, i, nxt, dev_err);
		}

		// FV groups share a target vertex: the FV hits re-keyed by (task, target vertex)
		__global__ void solid_fv_keys_kernel(const uint64_t* __restrict__ keys, uint32_t n, HitKeyCodec cd, uint64_t* __restrict__ k2,
			uint32_t* __restrict__ v2, uint32_t* __restrict__ count)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint64_t k = keys[i];
			if (cd.type(k) != 2u)
				return;
			cg::coalesced_group g = cg::coalesced_threads();
			uint32_t base = 0;
			if (g.thread_rank() == 0)
				base = atomicAdd(count, g.size());
			const uint32_t slot = g.shfl(base, 0) + g.thread_rank();
			k2[slot] = (uint64_t(cd.task(k)) << cd.b) | cd.dst(k);
			v2[slot] = i;
		}
		__global__ void solid_fv_kernel(const uint64_t* __restrict__ k2, const uint32_t* __restrict__ v2, uint32_t m, const uint64_t* __restrict__ keys,
			HitKeyCodec cd, const float* __restrict__ pay, const Task* __restrict__ tasks, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, SolidParams sp, uint32_t* __restrict__ parent, uint32_t* __restrict__ dev_err)
		{
			const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
			if (q >= m)
				return;
			const uint64_t g = k2[q];
			uint32_t rb = q, re = q + 1;
			for (int it = 0; it < (1 << 22) && rb > 0 && k2[rb - 1] == g; it++)
				rb--;
			for (int it = 0; it < (1 << 22) && re < m && k2[re] == g; it++)
				re++;
			const uint32_t i = v2[q];
			const float di = pay[3 * i + 2];
			uint32_t nxt = kInf;
			float dn = 0.0f;
			for (uint32_t p = rb; p < re; p++)
			{
				const uint32_t j = v2[p];
				if (j == i)
					continue;
				const float dj = pay[3 * j + 2];
				const bool after = dj > di || (dj == di && j > i);
				if (after && (nxt == kInf || dj < dn || (dj == dn && j < nxt)))
				{
					nxt = j;
					dn = dj;
				}
			}
			if (nxt == kInf)
				return;
			const Task tk = tasks[cd.task(keys[i])];
			if (solid_link_ok(sp, 2u, cd.src(keys[i]), cd.src(keys[nxt]), di, dn, mk3(tk.dir[0], tk.dir[1], tk.dir[2]), edges, faces))
				uf_union(parent, i, nxt, dev_err);
		}

		__global__ void compress_kernel(uint32_t* __restrict__ parent, uint32_t n, const uint8_t* __restrict__ attached,
			uint32_t* __restrict__ comp_size, uint32_t* __restrict__ comp_att, uint32_t* __restrict__ root)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			const bool valid = i < n;
			uint32_t r = kInf;
			bool att = false;
			if (valid)
			{
				r = i;
				for (int it = 0; it < 1 << 22; it++)
				{
					const uint32_t p = parent[r];
					if (p == r)
						break;
					r = p;
				}
				// path compression: every pointer on the walked path now names the root
				// (concurrent readers see an old ancestor or the root, both valid)
				uint32_t v = i;
				for (int it = 0; it < 1 << 22 && v != r; it++)
				{
					const uint32_t p = parent[v];
					parent[v] = r;
					v = p;
				}
				root[i] = r;
				att = attached[i] != 0;
			}
			// one atomic per (warp, component): hits of a task's large components are adjacent
			const uint32_t peers = __match_any_sync(0xFFFFFFFFu, r);
			const uint32_t att_peers = __ballot_sync(0xFFFFFFFFu, att) & peers;
			if (valid && (threadIdx.x & 31) == uint32_t(__ffs(peers) - 1))
			{
				atomicAdd(comp_size + r, uint32_t(__popc(peers)));
				if (att_peers)
					atomicOr(comp_att + r, 1u);
			}
		}

		// support entries (side, vertex, component) of hits in boundary-attached components
		// Only contour-boundary vertices are entered: the coverage test queries (side, v)
		// for v in the contour's side-`side` anchors, which are that side's boundary verts.
		__global__ void entries_kernel(const uint64_t* __restrict__ keys, uint32_t n, HitKeyCodec cd, const uint32_t* __restrict__ seg,
			const uint32_t* __restrict__ root, const uint32_t* __restrict__ comp_att, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, int vb, int rb, uint64_t* __restrict__ ekeys, uint32_t* __restrict__ evals,
			uint32_t* __restrict__ ecount, uint32_t cap, const Task* __restrict__ tasks, const Slot* __restrict__ slots,
			const uint32_t* __restrict__ bnd_bits, uint32_t v_stride)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint32_t r = root[i];
			if (!comp_att[r])
				return;
			const uint64_t k = keys[i];
			const uint32_t t = cd.task(k);
			const uint32_t rl = r - seg[t];
			uint32_t sv[3], dv[3];
			hit_verts(cd.type(k), cd.src(k), cd.dst(k), edges, faces, sv, dv);
			const Task tk = tasks[t];
			for (int side = 0; side < 2; side++)
				for (int q = 0; q < 3; q++)
				{
					const uint32_t v = side == 0 ? sv[q] : dv[q];
					if (v == kInf)
						continue;
					const uint32_t sl_id = side == 0 ? tk.slot0 : tk.slot1;
					const uint32_t lv = v - slots[sl_id].v_lo;
					if (!((bnd_bits[size_t(sl_id) * (v_stride / 32 + 1) + (lv >> 5)] >> (lv & 31)) & 1u))
						continue;
					// one counter atomic per group of lanes (entries are sorted afterwards)
					cg::coalesced_group g = cg::coalesced_threads();
					uint32_t base = 0;
					if (g.thread_rank() == 0)
						base = atomicAdd(ecount, g.size());
					const uint32_t slot = g.shfl(base, 0) + g.thread_rank();
					if (slot < cap)
					{
						ekeys[slot] = (uint64_t(t) << (1 + vb + rb)) | (uint64_t(side) << (vb + rb)) | (uint64_t(v) << rb) | uint64_t(rl);
						evals[slot] = slot;
					}
				}
		}

		// boundary-attached component roots of each task (order does not matter: the
		// selection rule is a strict total order)
		__global__ void cand_roots_kernel(const uint64_t* __restrict__ keys, uint32_t n, HitKeyCodec cd, const uint32_t* __restrict__ seg,
			const uint32_t* __restrict__ root, const uint32_t* __restrict__ comp_att, uint32_t* __restrict__ ncand,
			uint32_t* __restrict__ cand_roots)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n || root[i] != i || !comp_att[i])
				return;
			const uint32_t t = cd.task(keys[i]);
			cand_roots[seg[t] + atomicAdd(ncand + t, 1u)] = i;
		}

		__device__ __forceinline__ uint32_t lower_bound64(const uint64_t* __restrict__ a, uint32_t n, uint64_t key)
		{
			uint32_t lo = 0, hi = n;
			while (lo < hi)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (a[mid] < key)
					lo = mid + 1;
				else
					hi = mid;
			}
			return lo;
		}

		// The component ids (root - segment start) entered for one (task, side, vertex): a
		// sorted run of the support entries (with repeats).
		struct EntryRun
		{
			uint32_t b, e;
		};
		// the run of keys with the given (task, side, vertex) prefix inside [lo, hi): two binary searches
		__device__ __forceinline__ EntryRun entry_run(const uint64_t* __restrict__ ek, uint32_t lo, uint32_t hi, uint64_t prefix, int rb)
		{
			const uint32_t b = lo + lower_bound64(ek + lo, hi - lo, prefix);
			const uint32_t e = b + lower_bound64(ek + b, hi - b, prefix + (uint64_t(1) << rb));
			return EntryRun{ b, e };
		}
		// each task's range of the sorted support entries (tasks without entries keep [0, 0))
		__global__ void entry_ranges_kernel(const uint64_t* __restrict__ ek, uint32_t n, int shift, uint32_t* __restrict__ tbeg,
			uint32_t* __restrict__ tend)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint64_t t = ek[i] >> shift;
			if (i == 0 || (ek[i - 1] >> shift) != t)
				tbeg[t] = i;
			if (i + 1 == n || (ek[i + 1] >> shift) != t)
				tend[t] = i + 1;
		}
		__device__ __forceinline__ bool run_has(const uint64_t* __restrict__ ek, EntryRun r, uint64_t key)
		{
			uint32_t lo = r.b, hi = r.e;
			while (lo < hi)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (ek[mid] < key)
					lo = mid + 1;
				else
					hi = mid;
			}
			return lo < r.e && ek[lo] == key;
		}

		// EF-anchor coverage counted per anchor (prp_fill_combo_eval_info, intersection_
		// resolver2.cpp:1806-1881): one thread per (task, anchor); every boundary-attached
		// component that holds a vertex of the anchor's edge on side m and a vertex of its face
		// on side m^1 gains one covered anchor (cov[] is indexed by the component's root).
		__global__ void coverage_count_kernel(const Task* __restrict__ tasks, uint32_t ntasks, const uint32_t* __restrict__ task_anchor_begin,
			const uint32_t* __restrict__ anchor_off, const uint32_t* __restrict__ anchors, const uint64_t* __restrict__ ekeys, uint32_t nentries,
			const uint32_t* __restrict__ tbeg, const uint32_t* __restrict__ tend, int vb, int rb, const uint32_t* __restrict__ seg,
			uint32_t* __restrict__ cov)
		{
			const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
			if (g >= task_anchor_begin[ntasks])
				return;
			uint32_t lo = 0, hi = ntasks;
			while (hi - lo > 1)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (task_anchor_begin[mid] <= g)
					lo = mid;
				else
					hi = mid;
			}
			const uint32_t t = lo;
			const uint32_t c = tasks[t].contour_local;
			const uint32_t* A = anchors + 6 * size_t(anchor_off[c] + (g - task_anchor_begin[t]));
			const uint32_t m = A[0];
			const uint64_t tb = uint64_t(t) << (1 + vb + rb);
			auto prefix = [&](uint32_t side, uint32_t v)
			{ return tb | (uint64_t(side) << (vb + rb)) | (uint64_t(v) << rb); };
			const uint32_t lo_t = min(tbeg[t], nentries), hi_t = min(max(tend[t], lo_t), nentries);
			const EntryRun E0 = entry_run(ekeys, lo_t, hi_t, prefix(m, A[1]), rb);
			const EntryRun E1 = entry_run(ekeys, lo_t, hi_t, prefix(m, A[2]), rb);
			if (E0.b == E0.e && E1.b == E1.e)
				return;
			const EntryRun F[3] = { entry_run(ekeys, lo_t, hi_t, prefix(m ^ 1u, A[3]), rb), entry_run(ekeys, lo_t, hi_t, prefix(m ^ 1u, A[4]), rb),
				entry_run(ekeys, lo_t, hi_t, prefix(m ^ 1u, A[5]), rb) };
			if (F[0].b == F[0].e && F[1].b == F[1].e && F[2].b == F[2].e)
				return;
			const uint64_t rmask = (uint64_t(1) << rb) - 1u;
			const uint32_t s0 = seg[t];
			// distinct components of E0 u E1 in increasing order (two-pointer merge)
			uint32_t i0 = E0.b, i1 = E1.b;
			uint32_t last = kInf;
			for (int it = 0; it < (1 << 22) && (i0 < E0.e || i1 < E1.e); it++)
			{
				uint32_t rl;
				if (i1 >= E1.e || (i0 < E0.e && (ekeys[i0] & rmask) <= (ekeys[i1] & rmask)))
					rl = uint32_t(ekeys[i0++] & rmask);
				else
					rl = uint32_t(ekeys[i1++] & rmask);
				if (rl == last)
					continue;
				last = rl;
				bool in_f = false;
				for (int q = 0; q < 3 && !in_f; q++)
					in_f = run_has(ekeys, F[q], prefix(m ^ 1u, A[3 + q]) | rl);
				if (in_f)
					atomicAdd(cov + s0 + rl, 1u);
			}
		}

		// One warp per task: the best candidate component, maximal coverage, then more hits,
		// then the smaller canonical key (= smaller root index).
		__global__ void best_component_kernel(uint32_t ntasks, const uint32_t* __restrict__ seg, const uint32_t* __restrict__ ncand_arr,
			const uint32_t* __restrict__ cand_roots, const uint32_t* __restrict__ comp_size, const uint32_t* __restrict__ cov,
			uint32_t* __restrict__ best_out, uint32_t* __restrict__ bestcov_out)
		{
			const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
			const int lane = threadIdx.x & 31;
			if (t >= ntasks)
				return;
			const uint32_t lo = seg[t], ncand = ncand_arr[t];
			uint32_t best = kInf, bc = 0, bn = 0;
			for (uint32_t j = lane; j < ncand; j += 32)
			{
				const uint32_t r = cand_roots[lo + j];
				const uint32_t cv = cov[r], nh = comp_size[r];
				if (best == kInf || cv > bc || (cv == bc && (nh > bn || (nh == bn && r < best))))
				{
					best = r;
					bc = cv;
					bn = nh;
				}
			}
#pragma unroll
			for (int off = 16; off >= 1; off >>= 1)
			{
				const uint32_t ob = __shfl_xor_sync(0xFFFFFFFFu, best, off);
				const uint32_t oc = __shfl_xor_sync(0xFFFFFFFFu, bc, off);
				const uint32_t on = __shfl_xor_sync(0xFFFFFFFFu, bn, off);
				if (ob != kInf && (best == kInf || oc > bc || (oc == bc && (on > bn || (on == bn && ob < best)))))
				{
					best = ob;
					bc = oc;
					bn = on;
				}
			}
			if (lane == 0)
			{
				best_out[t] = best;
				bestcov_out[t] = best == kInf ? 0u : bc;
			}
		}

		__device__ __forceinline__ uint32_t selected_flag(const uint64_t* keys, const uint32_t* root, const uint32_t* best, HitKeyCodec cd,
			uint32_t i, uint32_t n)
		{
			if (i >= n)
				return 0u;
			return root[i] == best[cd.task(keys[i])] ? 1u : 0u;
		}

		// exclusive scan of the "selected" flags (hits of each task's best component), in
		// three phases over blocks of 1024 hits
		__global__ void __launch_bounds__(256) sel_block_sums_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ root,
			const uint32_t* __restrict__ best, HitKeyCodec cd, uint32_t n, uint32_t* __restrict__ bsum)
		{
			const uint32_t base = blockIdx.x * 1024u;
			uint32_t c = 0;
			for (uint32_t k = threadIdx.x; k < 1024u; k += 256u)
				c += selected_flag(keys, root, best, cd, base + k, n);
			c = __reduce_add_sync(0xFFFFFFFFu, c);
			__shared__ uint32_t w[8];
			if ((threadIdx.x & 31) == 0)
				w[threadIdx.x >> 5] = c;
			__syncthreads();
			if (threadIdx.x == 0)
			{
				uint32_t t = 0;
				for (int q = 0; q < 8; q++)
					t += w[q];
				bsum[blockIdx.x] = t;
			}
		}

		__global__ void __launch_bounds__(1024) scan_one_block_kernel(uint32_t* __restrict__ v, uint32_t n, uint32_t* __restrict__ total)
		{
			__shared__ uint32_t ws[32];
			const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
			const uint32_t b = threadIdx.x * per, e = min(n, b + per);
			uint32_t local = 0;
			for (uint32_t i = b; i < e; i++)
				local += v[i];
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			uint32_t x = local;
			for (int o = 1; o < 32; o <<= 1)
			{
				const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
				if (lane >= o)
					x += y;
			}
			if (lane == 31)
				ws[warp] = x;
			__syncthreads();
			if (warp == 0)
			{
				uint32_t y = ws[lane];
				for (int o = 1; o < 32; o <<= 1)
				{
					const uint32_t z = __shfl_up_sync(0xFFFFFFFFu, y, o);
					if (lane >= o)
						y += z;
				}
				ws[lane] = y;
			}
			__syncthreads();
			uint32_t run = x - local + (warp > 0 ? ws[warp - 1] : 0u);
			for (uint32_t i = b; i < e; i++)
			{
				const uint32_t c = v[i];
				v[i] = run;
				run += c;
			}
			if (threadIdx.x == blockDim.x - 1)
				*total = run;
		}

		// position of every selected hit in the compact canonical order, and its metric terms
		__global__ void __launch_bounds__(256) sel_terms_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ root,
			const uint32_t* __restrict__ best, HitKeyCodec cd, uint32_t n, const uint32_t* __restrict__ bsum, const Task* __restrict__ tasks,
			const float* __restrict__ pay, const uint2* __restrict__ edges, const uint32_t* __restrict__ faces, const float* __restrict__ vert_area,
			const float* __restrict__ edge_area, const float* __restrict__ face_area, const float* __restrict__ vert_mass,
			const float* __restrict__ vn, const float* __restrict__ en, const float* __restrict__ fnn, const Slot* __restrict__ slots,
			const uint32_t* __restrict__ hop, uint32_t v_stride, uint32_t* __restrict__ pos, float* __restrict__ terms,
			uint32_t* __restrict__ task_max, u26_prp_hit* __restrict__ out_hits)
		{
			__shared__ uint32_t wsum[8];
			const uint32_t base = blockIdx.x * 1024u;
			uint32_t f[4];
			uint32_t loc = 0;
#pragma unroll
			for (int q = 0; q < 4; q++)
			{
				f[q] = selected_flag(keys, root, best, cd, base + 4 * threadIdx.x + q, n);
				loc += f[q];
			}
			// exclusive scan of per-thread counts across the block
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			uint32_t x = loc;
			for (int o = 1; o < 32; o <<= 1)
			{
				const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
				if (lane >= o)
					x += y;
			}
			if (lane == 31)
				wsum[warp] = x;
			__syncthreads();
			uint32_t wbase = 0;
			for (int q = 0; q < warp; q++)
				wbase += wsum[q];
			uint32_t p = bsum[blockIdx.x] + wbase + x - loc;
			// running maxima of depth (float bits) and frontier hops of the thread's current
			// task; flushed when the task changes, then reduced across the warp by task segment
			uint32_t cur_t = kInf, m_dist = 0u, m_fs = 0u, m_fd = 0u;
#pragma unroll
			for (int q = 0; q < 4; q++)
			{
				const uint32_t i = base + 4 * threadIdx.x + q;
				if (!f[q])
					continue;
				pos[i] = p;
				const uint64_t k = keys[i];
				const uint32_t t = cd.task(k), ty = cd.type(k), sid = cd.src(k), did = cd.dst(k);
				const Task tk = tasks[t];
				const f3 dir = mk3(tk.dir[0], tk.dir[1], tk.dir[2]);
				const float b0 = pay[3 * i], b1 = pay[3 * i + 1], dist = pay[3 * i + 2];
				float area, alpha;
				if (ty == 0u)
				{
					area = vert_area[sid];
					alpha = fabsf(dot(mk3(vn[3 * sid], vn[3 * sid + 1], vn[3 * sid + 2]), dir));
				}
				else if (ty == 1u)
				{
					area = edge_area[sid];
					alpha = fabsf(dot(mk3(en[3 * sid], en[3 * sid + 1], en[3 * sid + 2]), dir));
				}
				else
				{
					area = face_area[sid];
					alpha = fabsf(dot(mk3(fnn[3 * sid], fnn[3 * sid + 1], fnn[3 * sid + 2]), dir));
				}
				uint32_t sv3[3], dv3[3];
				hit_verts(ty, sid, did, edges, faces, sv3, dv3);
				auto im = [&](uint32_t v)
				{ return 1.0f / fmaxf(vert_mass[v], 1e-8f); };
				float e;
				if (ty == 0u)
				{
					const float bx = b0, by = b1, bz = 1.0f - b0 - b1;
					e = ((im(sv3[0]) + bx * bx * im(dv3[0])) + by * by * im(dv3[1])) + bz * bz * im(dv3[2]);
				}
				else if (ty == 2u)
				{
					const float bx = b0, by = b1, bz = 1.0f - b0 - b1;
					e = ((bx * bx * im(sv3[0]) + by * by * im(sv3[1])) + bz * bz * im(sv3[2])) + im(dv3[0]);
				}
				else
				{
					const float a0 = b0, a1 = 1.0f - b0, c0 = b1, c1 = 1.0f - b1;
					e = ((a0 * a0 * im(sv3[0]) + a1 * a1 * im(sv3[1])) + c0 * c0 * im(dv3[0])) + c1 * c1 * im(dv3[1]);
				}
				const float sd = dist + 3e-3f;
				terms[3 * size_t(p)] = area;
				terms[3 * size_t(p) + 1] = (area * alpha) * dist;
				terms[3 * size_t(p) + 2] = e > 1e-8f ? (sd * sd) / e : 0.0f;
				// depth (non-negative float bits order like uints) and frontier hops
				if (t != cur_t)
				{
					if (cur_t != kInf)
					{
						atomicMax(task_max + 3 * cur_t, m_dist);
						atomicMax(task_max + 3 * cur_t + 1, m_fs);
						atomicMax(task_max + 3 * cur_t + 2, m_fd);
					}
					cur_t = t;
					m_dist = m_fs = m_fd = 0u;
				}
				m_dist = max(m_dist, __float_as_uint(dist));
				const Slot s0 = slots[tk.slot0], s1 = slots[tk.slot1];
				const uint32_t* h0 = hop + size_t(tk.slot0) * v_stride;
				const uint32_t* h1 = hop + size_t(tk.slot1) * v_stride;
				uint32_t mfs = 0, mfd = 0;
				for (int q2 = 0; q2 < 3; q2++)
				{
					if (sv3[q2] != kInf)
					{
						const uint32_t hv = h0[sv3[q2] - s0.v_lo];
						if (hv != kInf)
							mfs = max(mfs, hv);
					}
					if (dv3[q2] != kInf)
					{
						const uint32_t hv = h1[dv3[q2] - s1.v_lo];
						if (hv != kInf)
							mfd = max(mfd, hv);
					}
				}
				m_fs = max(m_fs, mfs);
				m_fd = max(m_fd, mfd);
				if (out_hits)
				{
					u26_prp_hit h;
					h.type = ty;
					h.src_id = sid;
					h.dst_id = did;
					for (int q2 = 0; q2 < 3; q2++)
					{
						h.src_verts[q2] = sv3[q2];
						h.dst_verts[q2] = dv3[q2];
					}
					h.bary[0] = b0;
					h.bary[1] = b1;
					h.dist = dist;
					out_hits[p] = h;
				}
				p++;
			}
			// segmented max across the warp: each lane's last task is non-decreasing along the
			// lanes (lanes without selected hits carry kInf), a run's first lane holds the run's
			// maxima after the shuffle steps and flushes them (max is idempotent, so a run that
			// also reaches past an empty lane is harmless)
#pragma unroll
			for (int off = 1; off < 32; off <<= 1)
			{
				const uint32_t ot = __shfl_down_sync(0xFFFFFFFFu, cur_t, off);
				const uint32_t od = __shfl_down_sync(0xFFFFFFFFu, m_dist, off);
				const uint32_t of = __shfl_down_sync(0xFFFFFFFFu, m_fs, off);
				const uint32_t og = __shfl_down_sync(0xFFFFFFFFu, m_fd, off);
				if (lane + off < 32 && ot == cur_t)
				{
					m_dist = max(m_dist, od);
					m_fs = max(m_fs, of);
					m_fd = max(m_fd, og);
				}
			}
			const uint32_t prev_t = __shfl_up_sync(0xFFFFFFFFu, cur_t, 1);
			if (cur_t != kInf && (lane == 0 || prev_t != cur_t))
			{
				atomicMax(task_max + 3 * cur_t, m_dist);
				atomicMax(task_max + 3 * cur_t + 1, m_fs);
				atomicMax(task_max + 3 * cur_t + 2, m_fd);
			}
		}

		struct TaskOut
		{
			uint32_t hit_begin, hit_end, best_root, hit_count;
			uint32_t unculled, covered, anchors, max_front_src;
			uint32_t max_front_dst, sel_offset, ncand, pad;
			float depth, volume, area, kappa;
		};

		// one warp per task: canonical 32-lane strided sums over its contiguous selected terms
		// The metrics' canonical sum of n interleaved triples (area, volume, kappa terms): each
		// lane adds its strided terms in order (the loads of 8 steps issued ahead), then an xor
		// butterfly. Lists longer than kSumChunk are summed per chunk of kSumChunk from their
		// start (chunk_sum_kernel, in parallel) and the chunk sums summed the same way.
		constexpr uint32_t kSumChunk = 8192;
		__device__ __forceinline__ void lane_sum3(const float* __restrict__ terms, uint32_t cnt, int lane, float& sa, float& sv, float& sk)
		{
			sa = sv = sk = 0.0f;
			uint32_t i = lane;
			for (; i + 7u * 32u < cnt; i += 8u * 32u)
			{
				float ta[8], tv[8], tk8[8];
#pragma unroll
				for (int u = 0; u < 8; u++)
				{
					const float* tt = terms + 3 * size_t(i + 32u * u);
					ta[u] = tt[0];
					tv[u] = tt[1];
					tk8[u] = tt[2];
				}
#pragma unroll
				for (int u = 0; u < 8; u++)
				{
					sa = sa + ta[u];
					sv = sv + tv[u];
					sk = sk + tk8[u];
				}
			}
			for (; i < cnt; i += 32)
			{
				const float* tt = terms + 3 * size_t(i);
				sa = sa + tt[0];
				sv = sv + tt[1];
				sk = sk + tt[2];
			}
			for (int off = 16; off >= 1; off >>= 1)
			{
				sa = sa + __shfl_xor_sync(0xFFFFFFFFu, sa, off);
				sv = sv + __shfl_xor_sync(0xFFFFFFFFu, sv, off);
				sk = sk + __shfl_xor_sync(0xFFFFFFFFu, sk, off);
			}
		}

		// chunks of the supports longer than kSumChunk: nchunk[t], then (after an exclusive
		// scan) one warp per chunk
		__global__ void chunk_count_kernel(uint32_t ntasks, const uint32_t* __restrict__ best, const uint32_t* __restrict__ comp_size,
			uint32_t* __restrict__ nchunk)
		{
			const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
			if (t > ntasks)
				return;
			uint32_t c = 0;
			if (t < ntasks)
			{
				const uint32_t b = best[t];
				const uint32_t cnt = b != kInf ? comp_size[b] : 0u;
				c = cnt > kSumChunk ? (cnt + kSumChunk - 1) / kSumChunk : 0u;
			}
			nchunk[t] = c;
		}
		__global__ void chunk_sum_kernel(uint32_t ntasks, uint32_t nchunks, const uint32_t* __restrict__ chunk_off, const uint32_t* __restrict__ best,
			const uint32_t* __restrict__ comp_size, const uint32_t* __restrict__ sel_begin, const float* __restrict__ terms,
			float* __restrict__ csum)
		{
			const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
			const int lane = threadIdx.x & 31;
			if (g >= nchunks)
				return;
			uint32_t lo = 0, hi = ntasks;
			while (hi - lo > 1)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (chunk_off[mid] <= g)
					lo = mid;
				else
					hi = mid;
			}
			// lo: the last task whose chunks begin at or before g (tasks without chunks share offsets)
			const uint32_t t = lo;
			const uint32_t cnt = comp_size[best[t]];
			const uint32_t j = g - chunk_off[t];
			const uint32_t b0 = j * kSumChunk;
			float sa, sv, sk;
			lane_sum3(terms + 3 * size_t(sel_begin[t] + b0), min(kSumChunk, cnt - b0), lane, sa, sv, sk);
			if (lane == 0)
			{
				csum[3 * size_t(g)] = sa;
				csum[3 * size_t(g) + 1] = sv;
				csum[3 * size_t(g) + 2] = sk;
			}
		}

		// one warp per task: the canonical sums of its selected terms and the task's outputs
		__global__ void task_sum_kernel(uint32_t ntasks, const Task* __restrict__ tasks, const uint32_t* __restrict__ seg,
			const uint32_t* __restrict__ best, const uint32_t* __restrict__ bestcov, const uint32_t* __restrict__ comp_size,
			const uint32_t* __restrict__ ncand, const uint32_t* __restrict__ sel_begin, const float* __restrict__ terms,
			const uint32_t* __restrict__ task_max, const uint32_t* __restrict__ anchor_off, const uint32_t* __restrict__ chunk_off,
			const float* __restrict__ csum, TaskOut* __restrict__ out)
		{
			const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
			const int lane = threadIdx.x & 31;
			if (t >= ntasks)
				return;
			const uint32_t b = best[t];
			const uint32_t cnt = b != kInf ? comp_size[b] : 0u;
			const uint32_t p0 = sel_begin[t];
			float sa, sv, sk;
			if (cnt <= kSumChunk)
				lane_sum3(terms + 3 * size_t(p0), cnt, lane, sa, sv, sk);
			else
				lane_sum3(csum + 3 * size_t(chunk_off[t]), chunk_off[t + 1] - chunk_off[t], lane, sa, sv, sk);
			if (lane == 0)
			{
				const Task tk = tasks[t];
				TaskOut o;
				o.hit_begin = seg[t];
				o.hit_end = seg[t + 1];
				o.best_root = b;
				o.hit_count = cnt;
				o.unculled = seg[t + 1] - seg[t];
				o.covered = b != kInf ? bestcov[t] : 0u;
				o.anchors = anchor_off[tk.contour_local + 1] - anchor_off[tk.contour_local];
				o.max_front_src = task_max[3 * t + 1];
				o.max_front_dst = task_max[3 * t + 2];
				o.sel_offset = p0;
				o.ncand = ncand[t];
				o.pad = 0u;
				o.depth = __uint_as_float(task_max[3 * t]);
				o.volume = sv;
				o.area = sa;
				o.kappa = sk;
				out[t] = o;
			}
		}

		// ------------------------------------------------------------ S^2 direction step
		struct StepIn
		{
			float dir[3];
			float trust;
			uint32_t hit_begin, hit_count;
		};
		struct StepOut
		{
			float dir[3];
			float predicted, gnorm;
			uint32_t valid, contributing, pad;
		};

		__device__ __forceinline__ bool valid_dir(f3 v)
		{
			return isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && length_sq(v) > 1e-12f;
		}

		// compute_effective_inverse_mass_weight (intersection_resolver_helper.cpp:611-645)
		__device__ __forceinline__ float hit_eff_inv_mass(const u26_prp_hit& h, const float* __restrict__ vert_mass)
		{
			auto im = [&](uint32_t v)
			{ return 1.0f / fmaxf(vert_mass[v], 1e-8f); };
			const float b0 = h.bary[0], b1 = h.bary[1];
			if (h.type == 0u)
			{
				const float bz = 1.0f - b0 - b1;
				return ((im(h.src_verts[0]) + b0 * b0 * im(h.dst_verts[0])) + b1 * b1 * im(h.dst_verts[1])) + bz * bz * im(h.dst_verts[2]);
			}
			if (h.type == 2u)
			{
				const float bz = 1.0f - b0 - b1;
				return ((b0 * b0 * im(h.src_verts[0]) + b1 * b1 * im(h.src_verts[1])) + bz * bz * im(h.src_verts[2])) + im(h.dst_verts[0]);
			}
			const float a1 = 1.0f - b0, c1 = 1.0f - b1;
			return ((b0 * b0 * im(h.src_verts[0]) + a1 * a1 * im(h.src_verts[1])) + b1 * b1 * im(h.dst_verts[0])) + c1 * c1 * im(h.dst_verts[1]);
		}

		// get_hit_characteristic_normal (intersection_resolver2.cpp:1232-1256) at x
		__device__ __forceinline__ f3 hit_normal(const u26_prp_hit& h, const float* __restrict__ x)
		{
			if (h.type == 0u)
			{
				const f3 A = ld3(x, h.dst_verts[0]), B = ld3(x, h.dst_verts[1]), C = ld3(x, h.dst_verts[2]);
				return cross(B - A, C - A);
			}
			if (h.type == 2u)
			{
				const f3 A = ld3(x, h.src_verts[0]), B = ld3(x, h.src_verts[1]), C = ld3(x, h.src_verts[2]);
				return cross(B - A, C - A);
			}
			const f3 p0 = ld3(x, h.src_verts[0]), p1 = ld3(x, h.src_verts[1]), q0 = ld3(x, h.dst_verts[0]), q1 = ld3(x, h.dst_verts[1]);
			f3 c = cross(p1 - p0, q1 - q0);
			if (length(c) < 1e-8f)
				c = (q0 * h.bary[1] + q1 * (1.0f - h.bary[1])) - (p0 * h.bary[0] + p1 * (1.0f - h.bary[0]));
			return c;
		}

		// One warp per contour under refinement: the gradient and Gauss-Newton Hessian of
		// sum_h w_h (delta_h + delta_0)^2 with respect to the direction r over the accepted
		// support (delta_h' = -delta_h n_h / (n_h . r)), projected to the tangent plane of S^2,
		// then a Newton step when the 2x2 tangent Hessian is positive definite, else a Cauchy
		// step, clipped to the trust radius (prp_compute_direction_optimization_step,
		// intersection_resolver2.cpp:1268-1368). Sums: canonical 32-lane strided order over
		// the hits in key order; a skipped hit adds zeros.
		__global__ void dir_step_kernel(uint32_t n, const StepIn* __restrict__ in, const u26_prp_hit* __restrict__ hits,
			const float* __restrict__ x, const float* __restrict__ vert_mass, StepOut* __restrict__ out)
		{
			const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
			const int lane = threadIdx.x & 31;
			if (t >= n)
				return;
			const StepIn si = in[t];
			const f3 r0 = mk3(si.dir[0], si.dir[1], si.dir[2]);
			StepOut o{};
			if (si.hit_count == 0u || !valid_dir(r0))
			{
				if (lane == 0)
					out[t] = o;
				return;
			}
			const f3 r = normalize(r0);
			const float off = 3e-3f; // prp_response_depth_offset (intersection_resolver2.h:98)
			float acc[12];
#pragma unroll
			for (int q = 0; q < 12; q++)
				acc[q] = 0.0f;
			uint32_t contributing = 0;
			for (uint32_t i = lane; i < si.hit_count; i += 32)
			{
				const u26_prp_hit h = hits[si.hit_begin + i];
				float term[12];
#pragma unroll
				for (int q = 0; q < 12; q++)
					term[q] = 0.0f;
				const f3 raw = hit_normal(h, x);
				const float nl = length(raw);
				bool use = isfinite(nl) && !(nl < 1e-8f);
				f3 nn = mk3(0.0f);
				float ndr = 0.0f, e = 0.0f;
				if (use)
				{
					nn = raw / nl;
					ndr = dot(nn, r);
					use = isfinite(ndr) && !(fabsf(ndr) < 1e-6f);
				}
				if (use)
				{
					e = hit_eff_inv_mass(h, vert_mass);
					use = isfinite(e) && !(e <= 1e-8f);
				}
				if (use)
				{
					const float w = 1.0f / e;
					const float d = h.dist;
					const f3 dd = (nn * (-d)) / ndr;
					const f3 g = dd * ((2.0f * w) * (d + off));
					const float hs = ((2.0f * w) / (ndr * ndr)) * ((3.0f * d) * d + (2.0f * d) * off);
					const float nv[3] = { nn.x, nn.y, nn.z };
					term[0] = g.x;
					term[1] = g.y;
					term[2] = g.z;
#pragma unroll
					for (int a = 0; a < 3; a++)
#pragma unroll
						for (int b2 = 0; b2 < 3; b2++)
							term[3 + 3 * a + b2] = hs * (nv[a] * nv[b2]);
					contributing++;
				}
#pragma unroll
				for (int q = 0; q < 12; q++)
					acc[q] = acc[q] + term[q];
			}
#pragma unroll
			for (int q = 0; q < 12; q++)
				for (int sh = 16; sh >= 1; sh >>= 1)
					acc[q] = acc[q] + __shfl_xor_sync(0xFFFFFFFFu, acc[q], sh);
			contributing = __reduce_add_sync(0xFFFFFFFFu, contributing);
			if (lane != 0)
				return;
			o.contributing = contributing;
			if (contributing == 0u)
			{
				out[t] = o;
				return;
			}
			const float* H = acc + 3;
			auto hmul = [&](f3 v)
			{
				return mk3((H[0] * v.x + H[1] * v.y) + H[2] * v.z, (H[3] * v.x + H[4] * v.y) + H[5] * v.z,
					(H[6] * v.x + H[7] * v.y) + H[8] * v.z);
			};
			const f3 grad = mk3(acc[0], acc[1], acc[2]);
			const f3 tg = grad - r * dot(r, grad);
			const f3 axis = fabsf(r.y) < 0.9f ? mk3(0.0f, 1.0f, 0.0f) : mk3(1.0f, 0.0f, 0.0f);
			const f3 e1 = normalize(cross(axis, r));
			const f3 e2 = normalize(cross(r, e1));
			const float g0 = dot(e1, tg), g1 = dot(e2, tg);
			const float gnorm = sqrtf(g0 * g0 + g1 * g1);
			if (!isfinite(gnorm) || gnorm < 1e-6f)
			{
				out[t] = o;
				return;
			}
			const float h00 = dot(e1, hmul(e1)), h01 = dot(e1, hmul(e2)), h10 = dot(e2, hmul(e1)), h11 = dot(e2, hmul(e2));
			const float det = h00 * h11 - h01 * h10;
			float d0, d1;
			if (isfinite(det) && det > 1e-10f && h00 > 0.0f)
			{
				d0 = -(h11 * g0 - h01 * g1) / det;
				d1 = -(h00 * g1 - h10 * g0) / det;
			}
			else
			{
				const float gg = g0 * g0 + g1 * g1;
				const float ghg = g0 * (h00 * g0 + h01 * g1) + g1 * (h10 * g0 + h11 * g1);
				const float alpha = ghg > 1e-10f ? gg / ghg : si.trust / (gnorm + 1e-20f);
				d0 = -alpha * g0;
				d1 = -alpha * g1;
			}
			const float sn = sqrtf(d0 * d0 + d1 * d1);
			if (!isfinite(sn) || sn < 1e-7f)
			{
				out[t] = o;
				return;
			}
			if (sn > si.trust)
			{
				const float sc = si.trust / sn;
				d0 = d0 * sc;
				d1 = d1 * sc;
			}
			const f3 trial = (r + e1 * d0) + e2 * d1;
			if (!valid_dir(trial))
			{
				out[t] = o;
				return;
			}
			const f3 nd = normalize(trial);
			o.dir[0] = nd.x;
			o.dir[1] = nd.y;
			o.dir[2] = nd.z;
			o.predicted = fmaxf(0.0f, -(g0 * d0 + g1 * d1));
			o.gnorm = gnorm;
			o.valid = 1u;
			out[t] = o;
		}

		// The selected support of each listed task in canonical (key) order: one CTA per task
		// compacts the hits of its best component out of the task's sorted segment.
		__global__ void __launch_bounds__(256) capture_kernel(const uint32_t* __restrict__ list, const uint32_t* __restrict__ out_off,
			const uint64_t* __restrict__ keys, const uint32_t* __restrict__ root, const uint32_t* __restrict__ best,
			const uint32_t* __restrict__ seg, const float* __restrict__ pay, HitKeyCodec cd, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, u26_prp_hit* __restrict__ out)
		{
			__shared__ uint32_t wsum[8];
			__shared__ uint32_t base;
			const uint32_t t = list[blockIdx.x];
			const uint32_t b = best[t];
			const uint32_t lo = seg[t], hi = seg[t + 1];
			if (threadIdx.x == 0)
				base = out_off[blockIdx.x];
			__syncthreads();
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			for (uint32_t i0 = lo; i0 < hi; i0 += blockDim.x)
			{
				const uint32_t i = i0 + threadIdx.x;
				const bool sel = i < hi && root[i] == b;
				const uint32_t m = __ballot_sync(0xFFFFFFFFu, sel);
				if (lane == 0)
					wsum[warp] = __popc(m);
				__syncthreads();
				uint32_t off = base;
				for (int w = 0; w < warp; w++)
					off += wsum[w];
				off += __popc(m & ((1u << lane) - 1u));
				if (sel)
				{
					const uint64_t k = keys[i];
					u26_prp_hit h;
					h.type = cd.type(k);
					h.src_id = cd.src(k);
					h.dst_id = cd.dst(k);
					uint32_t sv3[3], dv3[3];
					hit_verts(h.type, h.src_id, h.dst_id, edges, faces, sv3, dv3);
					for (int q = 0; q < 3; q++)
					{
						h.src_verts[q] = sv3[q];
						h.dst_verts[q] = dv3[q];
					}
					h.bary[0] = pay[3 * i];
					h.bary[1] = pay[3 * i + 1];
					h.dist = pay[3 * i + 2];
					out[off] = h;
				}
				__syncthreads();
				if (threadIdx.x == 0)
				{
					uint32_t tot = 0;
					for (int w = 0; w < 8; w++)
						tot += wsum[w];
					base += tot;
				}
				__syncthreads();
			}
		}

		// selected-hit offset of each task: the scanned position of its first hit
		__global__ void sel_begin_kernel(uint32_t ntasks, const uint32_t* __restrict__ seg, const uint32_t* __restrict__ bsum_scanned,
			const uint64_t* __restrict__ keys, const uint32_t* __restrict__ root, const uint32_t* __restrict__ best, HitKeyCodec cd,
			uint32_t n, uint32_t* __restrict__ sel_begin)
		{
			const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
			if (t >= ntasks)
				return;
			// count selected flags in [block start, seg[t]) on top of the block prefix
			const uint32_t i0 = seg[t];
			const uint32_t blk = i0 / 1024u;
			uint32_t p = bsum_scanned[blk];
			for (uint32_t i = blk * 1024u; i < i0; i++)
				p += selected_flag(keys, root, best, cd, i, n);
			sel_begin[t] = p;
		}

		// ---- FP64 evaluation of the selected supports (prp_eval_penetration_v2's terms,
		// intersection_resolver2.cpp:1883-1954): every hit's depth delta recomputed in FP64 from
		// the float positions (the ray / swept-edge test of its kind along the contour's
		// direction), D_C = max delta, J = (sum of the source rest areas) D_C^2, all in double
		// and in the hits' canonical order; and the D_C tie check: when the largest and second
		// largest FP32 depths lie within the depth's error band, the argmax is re-decided in FP64.
		// copies of captured supports out of the pass's support store: block q copies
		// [off[q], off[q] + cnt[q]) to [pos[q], ...)
		__global__ void __launch_bounds__(256) support_gather_kernel(const u26_prp_hit* __restrict__ store, const uint64_t* __restrict__ off,
			const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ pos, u26_prp_hit* __restrict__ out)
		{
			const uint32_t q = blockIdx.x;
			const u26_prp_hit* src = store + off[q];
			u26_prp_hit* dst = out + pos[q];
			for (uint32_t i = threadIdx.x; i < cnt[q]; i += blockDim.x)
				dst[i] = src[i];
		}

		struct Fp64In
		{
			uint32_t hit_begin, hit_end;
			float dir[3];
			float j32, dc32;
		};
		struct Fp64Out
		{
			double j64, dc64, delta_err;
			uint32_t tie, flip;
		};
		__device__ __forceinline__ double hit_delta_f64(const u26_prp_hit& h, f3 dir, const float* __restrict__ x, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces)
		{
			if (h.type == 1u)
			{
				const uint2 a = edges[h.src_id], b = edges[h.dst_id];
				const d3 p0 = dd(ld3(x, a.x)), p1 = dd(ld3(x, a.y)), q0 = dd(ld3(x, b.x)), q1 = dd(ld3(x, b.y));
				const d3 n = cross(p1 - p0, q1 - q0);
				const double det = -dot(dd(dir), n);
				return det != 0.0 ? -dot(q0 - p0, n) / det : double(h.dist);
			}
			const bool fv = h.type == 2u;
			const uint32_t v = fv ? h.dst_id : h.src_id, f = fv ? h.src_id : h.dst_id;
			const f3 orig = ld3(x, v);
			const f3 end = orig + (fv ? -dir : dir) * 1.0f;
			d3 b64;
			double t64;
			if (!line_intersection_f64(dd(orig), dd(end), dd(ld3(x, faces[3 * f])), dd(ld3(x, faces[3 * f + 1])), dd(ld3(x, faces[3 * f + 2])),
					b64, t64))
				return double(h.dist); // FP64 misses the hit (an FP32 / FP64 flip): keep its FP32 depth
			return t64 * 1.0;
		}
		// The FP64 depth of every selected support hit, a thread per hit (the contours' supports are
		// consecutive ranges of the hit list).
		__global__ void fp64_depths_kernel(uint32_t nc, const Fp64In* __restrict__ in, uint32_t nh, const u26_prp_hit* __restrict__ hits,
			const float* __restrict__ x, const uint2* __restrict__ edges, const uint32_t* __restrict__ faces, double* __restrict__ d64)
		{
			const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
			if (h >= nh)
				return;
			uint32_t lo = 0, hi = nc;
			while (hi - lo > 1)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (in[mid].hit_begin <= h)
					lo = mid;
				else
					hi = mid;
			}
			const Fp64In ci = in[lo];
			if (h < ci.hit_begin || h >= ci.hit_end)
				return;
			d64[h] = hit_delta_f64(hits[h], mk3(ci.dir[0], ci.dir[1], ci.dir[2]), x, edges, faces);
		}
		// Warp per contour. Each lane takes the hits h = begin + lane, begin + lane + 32, ...: their
		// FP64 depths, its partial source-area sum (in that order), the maxima; the partial sums
		// then combine by the xor butterfly (lane l adds lane l ^ 16, ^ 8, ^ 4, ^ 2, ^ 1), a fixed
		// order the oracle restates. Ties of a maximum keep the smallest hit index.
		__global__ void fp64_metrics_kernel(uint32_t nc, const Fp64In* __restrict__ in, const u26_prp_hit* __restrict__ hits,
			const double* __restrict__ d64s, const float* __restrict__ varea, const float* __restrict__ earea, const float* __restrict__ farea,
			Fp64Out* __restrict__ out)
		{
			const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
			const uint32_t lane = threadIdx.x & 31u;
			if (c >= nc)
				return;
			const Fp64In ci = in[c];
			double area = 0.0, dc64 = -1.0, derr = 0.0;
			float m32 = -1.0f, s32 = -1.0f;
			uint32_t arg32 = kInvalid, arg64 = kInvalid;
			for (uint32_t h = ci.hit_begin + lane; h < ci.hit_end; h += 32u)
			{
				const u26_prp_hit hh = hits[h];
				const double d64 = d64s[h];
				area += double(hh.type == 0u ? varea[hh.src_id] : hh.type == 1u ? earea[hh.src_id] : farea[hh.src_id]);
				if (d64 > dc64)
				{
					dc64 = d64;
					arg64 = h;
				}
				if (hh.dist > m32)
				{
					s32 = m32;
					m32 = hh.dist;
					arg32 = h;
				}
				else if (hh.dist > s32)
					s32 = hh.dist;
				if (d64 > 0.0)
					derr = fmax(derr, fabs(double(hh.dist) - d64) / d64);
			}
			for (int off = 16; off > 0; off >>= 1)
			{
				area += __shfl_xor_sync(0xFFFFFFFFu, area, off);
				derr = fmax(derr, __shfl_xor_sync(0xFFFFFFFFu, derr, off));
				const double od = __shfl_xor_sync(0xFFFFFFFFu, dc64, off);
				const uint32_t oa = __shfl_xor_sync(0xFFFFFFFFu, arg64, off);
				if (od > dc64 || (od == dc64 && oa < arg64))
				{
					dc64 = od;
					arg64 = oa;
				}
				// the two largest FP32 depths of both lanes (a multiset: equal values both count)
				const float om = __shfl_xor_sync(0xFFFFFFFFu, m32, off), os = __shfl_xor_sync(0xFFFFFFFFu, s32, off);
				const uint32_t oa32 = __shfl_xor_sync(0xFFFFFFFFu, arg32, off);
				if (om > m32 || (om == m32 && oa32 < arg32))
				{
					s32 = fmaxf(m32, os);
					m32 = om;
					arg32 = oa32;
				}
				else
					s32 = fmaxf(s32, om);
			}
			if (lane != 0u)
				return;
			Fp64Out o;
			o.j64 = area * dc64 * dc64;
			o.dc64 = dc64;
			o.delta_err = derr;
			o.tie = (ci.hit_end - ci.hit_begin > 1u && m32 - s32 <= 4.0f * kBandGamma * m32) ? 1u : 0u;
			o.flip = (o.tie && arg64 != arg32) ? 1u : 0u;
			out[c] = o;
		}
	} // namespace
} // namespace u26

using namespace u26;

// ==================================================================== host side
namespace
{
	constexpr uint32_t kInfH = 0xFFFFFFFFu;

	struct V3h
	{
		float x, y, z;
	};
	inline V3h mkv(float x, float y, float z) { return V3h{ x, y, z }; }
	inline V3h operator+(V3h a, V3h b) { return mkv(a.x + b.x, a.y + b.y, a.z + b.z); }
	inline V3h operator-(V3h a, V3h b) { return mkv(a.x - b.x, a.y - b.y, a.z - b.z); }
	inline V3h operator-(V3h a) { return mkv(-a.x, -a.y, -a.z); }
	inline V3h operator*(V3h a, float s) { return mkv(a.x * s, a.y * s, a.z * s); }
	inline V3h operator/(V3h a, float s) { return mkv(a.x / s, a.y / s, a.z / s); }
	inline float hdot(V3h a, V3h b)
	{
		float s = a.x * b.x;
		s = s + a.y * b.y;
		s = s + a.z * b.z;
		return s;
	}
	inline float hlen(V3h a) { return std::sqrt(hdot(a, a)); }
	inline V3h hnorm(V3h a) { return a * (1.0f / hlen(a)); }
	inline bool hvalid(V3h v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z) && hdot(v, v) > 1e-12f; }

	// cyclic Jacobi on a symmetric 3x3 (double): eigenvalues ascending, each
	// eigenvector signed so that its largest-magnitude component is positive
	void sym_eigen3(const double A0[3][3], double V_out[3][3])
	{
		double A[3][3], V[3][3] = { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
		std::memcpy(A, A0, sizeof(A));
		static const int P[3] = { 0, 0, 1 }, Q[3] = { 1, 2, 2 };
		for (int sweep = 0; sweep < 64; sweep++)
		{
			const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
			const double dg = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
			if (off <= 1e-30 * dg || off == 0.0)
				break;
			for (int k = 0; k < 3; k++)
			{
				const int p = P[k], q = Q[k];
				if (A[p][q] == 0.0)
					continue;
				const double th = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
				const double tt = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
				const double c = 1.0 / std::sqrt(tt * tt + 1.0), s = tt * c;
				for (int r = 0; r < 3; r++)
				{
					const double x = A[r][p], y = A[r][q];
					A[r][p] = c * x - s * y;
					A[r][q] = s * x + c * y;
				}
				for (int r = 0; r < 3; r++)
				{
					const double x = A[p][r], y = A[q][r];
					A[p][r] = c * x - s * y;
					A[q][r] = s * x + c * y;
				}
				for (int r = 0; r < 3; r++)
				{
					const double x = V[r][p], y = V[r][q];
					V[r][p] = c * x - s * y;
					V[r][q] = s * x + c * y;
				}
			}
		}
		int ord[3] = { 0, 1, 2 };
		std::stable_sort(ord, ord + 3, [&](int a, int b)
			{ return A[a][a] < A[b][b]; });
		for (int k = 0; k < 3; k++)
		{
			const int c = ord[k];
			int big = 0;
			for (int r = 1; r < 3; r++)
				if (std::fabs(V[r][c]) > std::fabs(V[big][c]))
					big = r;
			const double sg = V[big][c] < 0 ? -1.0 : 1.0;
			for (int r = 0; r < 3; r++)
				V_out[r][k] = sg * V[r][c];
		}
	}

	struct ComboState
	{
		bool present = false, eligible = false, full_mesh = false;
		uint32_t levels = 0, eval_k_src = kInfH, eval_k_dst = kInfH;
		uint32_t hit_count = 0, unculled = 0, covered = 0, anchors = 0, mfs = 0, mfd = 0;
		float depth = 0, volume = 0, area = 0, cost = 0, objective = 0, coverage = 0;
		uint32_t opt_attempted = 0, opt_accepted = 0; // direction_optimization_{iteration,accepted}_count
		std::vector<u26_prp_hit> hits;
		// the support, when captured on the device: [store_off, store_off + hit_count) of the
		// pass's support store (hits stays empty until the support is fetched)
		uint64_t store_off = ~0ull;
		bool in_store() const { return store_off != ~0ull; }
	};

	inline bool usable(const ComboState& c)
	{
		return c.hit_count > 0 && c.covered > 0 && std::isfinite(c.objective) && std::isfinite(c.coverage) && c.coverage > 0.0f;
	}
	inline bool valid_resp(const ComboState& c) { return c.eligible && usable(c); }
	inline float resp_obj(const ComboState& c)
	{
		if (!std::isfinite(c.objective) || !std::isfinite(c.coverage) || c.coverage <= 0.0f)
			return std::numeric_limits<float>::infinity();
		const double o = double(c.objective) / (double(c.coverage) * double(c.coverage));
		return (std::isfinite(o) && o <= double(std::numeric_limits<float>::max())) ? float(o) : std::numeric_limits<float>::infinity();
	}
	inline int fcmp(float l, float r)
	{
		const bool lf = std::isfinite(l), rf = std::isfinite(r);
		if (lf != rf)
			return lf ? -1 : 1;
		if (!lf)
			return 0;
		const float tol = 1e-7f + 1e-5f * std::fmax(std::fabs(l), std::fabs(r));
		if (l + tol < r)
			return -1;
		if (r + tol < l)
			return 1;
		return 0;
	}
	inline bool better_resp(const ComboState& a, uint32_t ai, const ComboState& b, uint32_t bi)
	{
		int c = fcmp(resp_obj(a), resp_obj(b));
		if (c)
			return c < 0;
		c = fcmp(a.depth, b.depth);
		if (c)
			return c < 0;
		c = fcmp(a.cost, b.cost);
		if (c)
			return c < 0;
		if (a.hit_count != b.hit_count)
			return a.hit_count < b.hit_count;
		return ai < bi;
	}

	struct ContourRT
	{
		uint32_t contour = 0;
		uint32_t obj[2] = { 0, 0 };
		std::vector<uint32_t> bnd[2];
		std::vector<V3h> dirs;
		std::vector<ComboState> res;
		std::vector<uint8_t> conv, pruned, present;
		std::vector<uint8_t> active; // active_combos as a mask: all directions, or the one under refinement
		uint32_t diam[2] = { 0, 0 }, k0[2] = { 0, 0 }, k[2] = { 0, 0 };
		bool finished = false, no_resp = false;
		uint32_t levels = 0;
	};
} // namespace

struct u26_scene
{
	u26_ctx* ctx = nullptr;
	uint32_t nv = 0, ne = 0, nf = 0, nobj = 0;
	std::vector<float> rest_x;
	std::vector<uint32_t> edges, faces, fae, vav_off, vav, vae_off, vae, vaf_off, vaf, eaf_off, eaf, eae_off, eae;
	std::vector<uint32_t> pv, pe, pf, vobj, vcomp, orient, oscene;
	std::vector<float> varea, earea, farea, vmass;
	DevBuf d_rest_x, d_edges, d_faces, d_fae, d_vav_off, d_vav, d_vae_off, d_vae, d_vaf_off, d_vaf, d_eaf_off, d_eaf, d_eae_off, d_eae;
	DevBuf d_vobj, d_varea, d_earea, d_farea, d_vmass, d_orient;
	DevBuf d_fn, d_en, d_vn;
	// per pass
	DevBuf d_slots, d_slot_ids, d_bnd, d_hop, d_geo, d_order, d_level_end, d_work, d_mark, d_owns;
	DevBuf d_cand_v, d_cand_e, d_cand_f, d_counts, d_bits_e, d_bits_f;
	DevBuf d_tasks, d_keys, d_vals, d_pay_in, d_pay, d_hitcount, d_stats, d_seg, d_parent, d_root, d_att, d_csize, d_catt;
	DevBuf d_ekeys, d_evals, d_ecount, d_cand_roots, d_vf_off, d_vf, d_anchor_off, d_anchors, d_out, d_sel;
	DevBuf d_bnd_bits, d_slot_box, d_ncand, d_best, d_bsum, d_task_max, d_selbegin, d_pos, d_terms;
	DevBuf d_step_in, d_step_hits, d_step_out;
	DevBuf d_f64in, d_f64hits, d_f64delta, d_f64out; // FP64 evaluation of the selected supports
	DevBuf d_queue;									  // work-item counter of the persistent ray casts
	DevBuf d_fgrow, d_egrow, d_front, d_cur_own, d_cur_opp, d_tab, d_cov;
	DevBuf d_trange; // per task: first and past-the-end index of its support entries
	DevBuf d_store;	 // the pass's captured supports (u26_prp_hit), grown with its contents kept
	uint64_t store_used = 0;
	DevBuf d_fetch_off, d_fetch_cnt, d_fetch_pos;
	DevBuf d_vrank, d_erank, d_cand_off, d_ckeys, d_cvals, d_cap_list, d_cap_off, d_capture, d_chunk_off, d_csum, scan_tmp, d_vsolid, d_fvk, d_fvv, d_rflag, d_heads, d_hkeys, d_hvals, d_zero_th;
	RadixSorter sorter, esorter, csorter, fvsorter;
	std::vector<uint8_t> vsolid; // per vertex: its object is rigid / tetrahedral
	bool any_solid = false;
	std::vector<u26_lbvh*> otree_f, otree_e; // per-object ray-casting trees (built at the first pass)
	// the per-pass refit + grow of those trees as one CUDA graph, captured at the second pass
	// for the positions pointer forest_x and replayed while it stays the same
	cudaStream_t forest_stream = nullptr;
	cudaGraphExec_t forest_exec = nullptr;
	const float* forest_x = nullptr;
	uint64_t forest_launches = 0;
	bool forest_graph_failed = false;
	bool otrees_built = false, fronts_built = false;
	uint32_t vmax_obj = 0, emax_obj = 0, fmax_obj = 0;
	uint32_t hit_cap = 0, e_cap = 0; // capacities that survive between passes
	int tuned_cfg = -1;				  // autotuned ray-casting configuration (-1: not tuned yet)
	uint32_t num_sms = 148;			  // the device's SM count (the persistent grid's size)
	uint64_t passes = 0;			  // completed u26_prp_resolve calls (the normals d_fn / d_en / d_vn are the last one's)
	void* cap_host = nullptr;		  // pinned staging of the captured supports (grow-only)
	size_t cap_host_bytes = 0;
	ResponseState resp;
};

struct u26_prp_output
{
	std::vector<EfPairH> pairs;
	std::vector<uint32_t> pair_idx, mesh_index, contour_index, contour_offsets, contour_pairs, hit_offsets;
	std::vector<float> pair_length, directions;
	std::vector<u26_prp_result> results;
	std::vector<u26_prp_hit> hits;
	uint32_t num_orig_pairs = 0, levels = 0, dev_err = 0;
	uint64_t ray_tests = 0, ray_requests = 0, ray_pairs = 0;
	double stage_ms[8] = { 0 };
	double gpu_ms[6] = { 0 };
	uint64_t ray_nodes = 0, ray_edge_tests = 0, ray_node_fetches = 0, ray_tri_fetches = 0, ray_edge_fetches = 0, ray_visits = 0, ray_candidate_tests = 0;
	uint64_t fp64_rechecks = 0, fp64_flips = 0, dc_tie_rechecks = 0, dc_tie_flips = 0;
	double tune_ms[18] = { 0 }; // autotuner: ray-casting time of each configuration over the tuning pass
	int raycast_cfg = -1;	   // configuration the scene's launches use from now on (index of the table)
	uint32_t tuned = 0;		   // this pass ran the autotuner
	double fp64_delta_rel_err = 0.0, fp64_dc_rel_err = 0.0, fp64_j_rel_err = 0.0;
	const u26_scene* scene = nullptr; // the pass this output came from
	uint64_t pass = 0;
};

template <typename T>
static u26_status upload(u26_ctx* ctx, DevBuf& b, const std::vector<T>& v)
{
	U26_CUDA(ctx, b.reserve(std::max<size_t>(sizeof(T) * v.size(), 16)));
	if (!v.empty())
		U26_CUDA(ctx, cudaMemcpyAsync(b.ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, ctx->stream));
	return U26_OK;
}

template <typename T>
static u26_status download(u26_ctx* ctx, std::vector<T>& v, const void* p, size_t n)
{
	v.resize(n);
	if (n)
		U26_CUDA(ctx, cudaMemcpyAsync(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
	return U26_OK;
}

U26_API u26_status u26_scene_create(u26_ctx* ctx, const u26_mesh_desc* m, u26_scene** out)
{
	if (!ctx || !m || !out)
		return U26_ERR_INVALID_INPUT;
	*out = nullptr;
	if (!m->rest_x || !m->edges || !m->faces || !m->face_adj_edges || !m->vert_adj_verts_offsets || !m->prefix_num_verts)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_scene_create: missing mesh table");
	std::unique_ptr<u26_scene> s(new u26_scene());
	s->ctx = ctx;
	int sms = 0;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) == cudaSuccess && sms > 0)
		s->num_sms = uint32_t(sms);
	U26_CUDA(ctx, s->d_queue.reserve(sizeof(uint32_t)));
	s->nv = m->num_verts;
	s->ne = m->num_edges;
	s->nf = m->num_faces;
	s->nobj = m->num_objects;
	auto cp = [](std::vector<uint32_t>& d, const uint32_t* p, size_t n)
	{ d.assign(p, p + n); };
	auto cpf = [](std::vector<float>& d, const float* p, size_t n)
	{ d.assign(p, p + n); };
	cpf(s->rest_x, m->rest_x, 3 * size_t(s->nv));
	cp(s->edges, m->edges, 2 * size_t(s->ne));
	cp(s->faces, m->faces, 3 * size_t(s->nf));
	cp(s->fae, m->face_adj_edges, 3 * size_t(s->nf));
	cp(s->vav_off, m->vert_adj_verts_offsets, s->nv + 1);
	cp(s->vav, m->vert_adj_verts, s->vav_off.back());
	cp(s->vae_off, m->vert_adj_edges_offsets, s->nv + 1);
	cp(s->vae, m->vert_adj_edges, s->vae_off.back());
	cp(s->vaf_off, m->vert_adj_faces_offsets, s->nv + 1);
	cp(s->vaf, m->vert_adj_faces, s->vaf_off.back());
	cp(s->eaf_off, m->edge_adj_faces_offsets, s->ne + 1);
	cp(s->eaf, m->edge_adj_faces, s->eaf_off.back());
	cp(s->eae_off, m->edge_adj_edges_offsets, s->ne + 1);
	cp(s->eae, m->edge_adj_edges, s->eae_off.back());
	cp(s->pv, m->prefix_num_verts, s->nobj + 1);
	cp(s->pe, m->prefix_num_edges, s->nobj + 1);
	cp(s->pf, m->prefix_num_faces, s->nobj + 1);
	cp(s->vobj, m->vert_object, s->nv);
	if (m->vert_component)
		cp(s->vcomp, m->vert_component, s->nv);
	else
		s->vcomp.assign(s->nv, 0u);
	if (m->mesh_orientation)
		cp(s->orient, m->mesh_orientation, s->nobj);
	else
		s->orient.assign(std::max(1u, s->nobj), 0u);
	if (m->object_scene)
		cp(s->oscene, m->object_scene, s->nobj);
	else
		s->oscene.assign(std::max(1u, s->nobj), 0u);
	cpf(s->varea, m->rest_vert_area, s->nv);
	cpf(s->earea, m->rest_edge_area, s->ne);
	cpf(s->farea, m->rest_face_area, s->nf);
	cpf(s->vmass, m->vert_mass, s->nv);
	s->vsolid.assign(std::max(1u, s->nv), 0u);
	if (m->object_solid)
		for (uint32_t v = 0; v < s->nv; v++)
		{
			s->vsolid[v] = m->object_solid[s->vobj[v]] ? 1u : 0u;
			s->any_solid = s->any_solid || s->vsolid[v];
		}
	for (uint32_t o = 0; o < s->nobj; o++)
	{
		s->vmax_obj = std::max(s->vmax_obj, s->pv[o + 1] - s->pv[o]);
		s->emax_obj = std::max(s->emax_obj, s->pe[o + 1] - s->pe[o]);
		s->fmax_obj = std::max(s->fmax_obj, s->pf[o + 1] - s->pf[o]);
	}
	U26_TRY(upload(ctx, s->d_rest_x, s->rest_x));
	U26_TRY(upload(ctx, s->d_edges, s->edges));
	U26_TRY(upload(ctx, s->d_faces, s->faces));
	U26_TRY(upload(ctx, s->d_fae, s->fae));
	U26_TRY(upload(ctx, s->d_vav_off, s->vav_off));
	U26_TRY(upload(ctx, s->d_vav, s->vav));
	U26_TRY(upload(ctx, s->d_vae_off, s->vae_off));
	U26_TRY(upload(ctx, s->d_vae, s->vae));
	U26_TRY(upload(ctx, s->d_vaf_off, s->vaf_off));
	U26_TRY(upload(ctx, s->d_vaf, s->vaf));
	U26_TRY(upload(ctx, s->d_eaf_off, s->eaf_off));
	U26_TRY(upload(ctx, s->d_eaf, s->eaf));
	U26_TRY(upload(ctx, s->d_eae_off, s->eae_off));
	U26_TRY(upload(ctx, s->d_eae, s->eae));
	U26_TRY(upload(ctx, s->d_vobj, s->vobj));
	U26_TRY(upload(ctx, s->d_varea, s->varea));
	U26_TRY(upload(ctx, s->d_earea, s->earea));
	U26_TRY(upload(ctx, s->d_farea, s->farea));
	U26_TRY(upload(ctx, s->d_vmass, s->vmass));
	U26_TRY(upload(ctx, s->d_orient, s->orient));
	U26_TRY(upload(ctx, s->d_vsolid, s->vsolid));
	{
		// 30-bit Morton codes of the rest positions (vertices) and rest edge midpoints over
		// the rest AABB: the request order of the ray casts
		float lo[3] = { INFINITY, INFINITY, INFINITY }, hi[3] = { -INFINITY, -INFINITY, -INFINITY };
		for (uint32_t v = 0; v < s->nv; v++)
			for (int a = 0; a < 3; a++)
			{
				lo[a] = std::fmin(lo[a], s->rest_x[3 * v + a]);
				hi[a] = std::fmax(hi[a], s->rest_x[3 * v + a]);
			}
		auto spread = [](uint32_t q)
		{
			q = (q * 0x00010001u) & 0xFF0000FFu;
			q = (q * 0x00000101u) & 0x0F00F00Fu;
			q = (q * 0x00000011u) & 0xC30C30C3u;
			q = (q * 0x00000005u) & 0x49249249u;
			return q;
		};
		auto code = [&](const float* p)
		{
			uint32_t c = 0;
			for (int a = 0; a < 3; a++)
			{
				const float ext = hi[a] - lo[a];
				const float u = ext > 0.0f ? (p[a] - lo[a]) / ext : 0.0f;
				const uint32_t q = uint32_t(std::fmin(std::fmax(u * 1024.0f, 0.0f), 1023.0f));
				c |= spread(q) << (2 - a);
			}
			return c;
		};
		std::vector<uint32_t> vr(std::max(1u, s->nv)), er(std::max(1u, s->ne));
		for (uint32_t v = 0; v < s->nv; v++)
			vr[v] = code(&s->rest_x[3 * v]);
		for (uint32_t e = 0; e < s->ne; e++)
		{
			const uint32_t a = s->edges[2 * e], b = s->edges[2 * e + 1];
			const float mid[3] = { 0.5f * (s->rest_x[3 * a] + s->rest_x[3 * b]), 0.5f * (s->rest_x[3 * a + 1] + s->rest_x[3 * b + 1]),
				0.5f * (s->rest_x[3 * a + 2] + s->rest_x[3 * b + 2]) };
			er[e] = code(mid);
		}
		U26_TRY(upload(ctx, s->d_vrank, vr));
		U26_TRY(upload(ctx, s->d_erank, er));
		// the codes become dense ranks of (code, id), in place
		auto dense = [&](DevBuf& rank, uint32_t n) -> u26_status
		{
			if (n < 2)
			{
				U26_CUDA(ctx, cudaMemsetAsync(rank.ptr, 0, sizeof(uint32_t), ctx->stream));
				return U26_OK;
			}
			int id_bits = 1;
			while (id_bits < 32 && (uint64_t(1) << id_bits) < n)
				id_bits++;
			U26_CUDA(ctx, s->d_ckeys.reserve(sizeof(uint64_t) * n));
			U26_CUDA(ctx, s->d_cvals.reserve(sizeof(uint32_t) * n));
			rank_keys_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(rank.as<uint32_t>(), n, id_bits, s->d_ckeys.as<uint64_t>(),
				s->d_cvals.as<uint32_t>());
			U26_TRY(after_launch(ctx, "rank_keys_kernel"));
			U26_TRY(s->csorter.sort(ctx, s->d_ckeys.as<uint64_t>(), s->d_cvals.as<uint32_t>(), n, 0, 30 + id_bits));
			rank_scatter_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(s->d_cvals.as<uint32_t>(), n, rank.as<uint32_t>());
			return after_launch(ctx, "rank_scatter_kernel");
		};
		U26_TRY(dense(s->d_vrank, s->nv));
		U26_TRY(dense(s->d_erank, s->ne));
	}
	U26_CUDA(ctx, s->d_fn.reserve(sizeof(float) * 3 * std::max(1u, s->nf)));
	U26_CUDA(ctx, s->d_en.reserve(sizeof(float) * 3 * std::max(1u, s->ne)));
	U26_CUDA(ctx, s->d_vn.reserve(sizeof(float) * 3 * std::max(1u, s->nv)));
	U26_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	*out = s.release();
	return U26_OK;
}

U26_API void u26_scene_destroy(u26_scene* s)
{
	if (!s)
		return;
	DevBuf* bufs[] = { &s->d_rest_x, &s->d_edges, &s->d_faces, &s->d_fae, &s->d_vav_off, &s->d_vav, &s->d_vae_off, &s->d_vae,
		&s->d_vaf_off, &s->d_vaf, &s->d_eaf_off, &s->d_eaf, &s->d_eae_off, &s->d_eae, &s->d_vobj, &s->d_varea, &s->d_earea,
		&s->d_farea, &s->d_vmass, &s->d_orient, &s->d_fn, &s->d_en, &s->d_vn, &s->d_slots, &s->d_slot_ids, &s->d_bnd, &s->d_hop,
		&s->d_geo, &s->d_order, &s->d_level_end, &s->d_work, &s->d_mark, &s->d_owns, &s->d_cand_v, &s->d_cand_e, &s->d_cand_f,
		&s->d_counts, &s->d_bits_e, &s->d_bits_f, &s->d_tasks, &s->d_keys, &s->d_vals, &s->d_pay_in, &s->d_pay, &s->d_hitcount,
		&s->d_stats, &s->d_seg, &s->d_parent, &s->d_root, &s->d_att, &s->d_csize, &s->d_catt, &s->d_ekeys, &s->d_evals,
		&s->d_ecount, &s->d_cand_roots, &s->d_vf_off, &s->d_vf, &s->d_anchor_off, &s->d_anchors, &s->d_out, &s->d_sel, &s->d_bnd_bits,
		&s->d_slot_box, &s->d_ncand, &s->d_best, &s->d_bsum, &s->d_task_max, &s->d_selbegin, &s->d_pos, &s->d_terms, &s->d_step_in,
		&s->d_step_hits, &s->d_step_out, &s->d_f64in, &s->d_f64hits, &s->d_f64delta, &s->d_f64out, &s->d_queue, &s->d_fgrow, &s->d_egrow, &s->d_front, &s->d_cur_own,
		&s->d_cur_opp, &s->d_tab, &s->d_cov, &s->d_vrank, &s->d_erank, &s->d_cand_off, &s->d_ckeys, &s->d_cvals,
		&s->d_cap_list, &s->d_cap_off, &s->d_capture, &s->d_chunk_off, &s->d_csum, &s->scan_tmp, &s->d_vsolid,
		&s->d_fvk, &s->d_fvv, &s->d_rflag, &s->d_heads, &s->d_hkeys, &s->d_hvals,
		&s->d_zero_th, &s->d_trange, &s->d_store, &s->d_fetch_off, &s->d_fetch_cnt, &s->d_fetch_pos };
	for (DevBuf* b : bufs)
		b->release();
	s->sorter.release();
	s->esorter.release();
	s->csorter.release();
	s->fvsorter.release();
	s->resp.release();
	if (s->forest_exec)
		cudaGraphExecDestroy(s->forest_exec);
	if (s->forest_stream)
		cudaStreamDestroy(s->forest_stream);
	if (s->cap_host)
		cudaFreeHost(s->cap_host);
	for (u26_lbvh* t : s->otree_f)
		u26_lbvh_destroy(t);
	for (u26_lbvh* t : s->otree_e)
		u26_lbvh_destroy(t);
	delete s;
}

void u26_prp_release_ctx(const u26_ctx* ctx) { (void)ctx; }

namespace
{
	// host-side EF preprocessing, contours and classification (the canonical list is sorted by
	// (eid, fid), so the pairs of one edge are a contiguous run)
	struct HostGraph
	{
		std::vector<EfPairH> ef;
		std::vector<uint32_t> ee, ff;
		std::vector<std::vector<uint32_t>> adj;
		std::vector<V3h> pos3;
		std::vector<float> len;
		std::vector<std::vector<uint32_t>> contours;
		std::vector<uint32_t> mesh_index, contour_index, type;
		std::vector<uint32_t> vflag_off, vflags;
	};

	// Host worker threads, started once per process and reused by every parallel loop of a
	// pass (starting threads for each loop cost more than most loops do). One loop at a time:
	// a caller holds run_mtx while its items are handed out; the calling thread works too.
	class HostPool
	{
	public:
		// never destroyed: the workers stay parked on their condition variable until the
		// process ends (no join at exit, none in a forked child)
		static HostPool& get()
		{
			static HostPool* pool = new HostPool();
			return *pool;
		}
		uint32_t size() const { return uint32_t(workers_.size()) + 1u; }
		// job(i) for every i in [0, n), items handed out one at a time
		void run(uint32_t n, const std::function<void(uint32_t)>& job)
		{
			// a forked child has none of the workers, and a loop started inside a pool job would
			// wait for itself: both run the loop in the calling thread
			if (workers_.empty() || n <= 1 || getpid() != pid_ || in_job())
			{
				for (uint32_t i = 0; i < n; i++)
					job(i);
				return;
			}
			std::lock_guard<std::mutex> one(run_mtx_);
			InJob mark;
			{
				std::lock_guard<std::mutex> lk(mtx_);
				job_ = &job;
				n_ = n;
				next_.store(0u);
				busy_ = uint32_t(workers_.size());
				gen_++;
			}
			cv_.notify_all();
			work();
			std::unique_lock<std::mutex> lk(mtx_);
			done_cv_.wait(lk, [&] { return busy_ == 0; });
			job_ = nullptr;
		}

	private:
		HostPool() : pid_(getpid())
		{
			const uint32_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
			for (uint32_t t = 1; t < hw; t++)
				workers_.emplace_back([this] { loop(); });
		}
		void work()
		{
			for (uint32_t i = next_.fetch_add(1u); i < n_; i = next_.fetch_add(1u))
				(*job_)(i);
		}
		static bool& in_job()
		{
			thread_local bool flag = false;
			return flag;
		}
		struct InJob
		{
			InJob() { in_job() = true; }
			~InJob() { in_job() = false; }
		};
		void loop()
		{
			in_job() = true;
			uint64_t seen = 0;
			for (;;)
			{
				{
					std::unique_lock<std::mutex> lk(mtx_);
					cv_.wait(lk, [&] { return gen_ != seen; });
					seen = gen_;
				}
				work();
				{
					std::lock_guard<std::mutex> lk(mtx_);
					busy_--;
				}
				done_cv_.notify_one();
			}
		}
		pid_t pid_;
		std::vector<std::thread> workers_;
		std::mutex run_mtx_, mtx_;
		std::condition_variable cv_, done_cv_;
		const std::function<void(uint32_t)>* job_ = nullptr;
		uint32_t n_ = 0, busy_ = 0;
		uint64_t gen_ = 0;
		std::atomic<uint32_t> next_{ 0u };
	};

	// fn(i) for i in [0, n) over the host cores in contiguous chunks; fn(i) writes only what i owns
	template <typename F>
	void host_parallel_for(uint32_t n, F&& fn)
	{
		HostPool& pool = HostPool::get();
		const uint32_t nt = n < 8192 ? 1u : pool.size();
		if (nt == 1)
		{
			for (uint32_t i = 0; i < n; i++)
				fn(i);
			return;
		}
		const uint32_t chunk = (n + nt - 1) / nt;
		pool.run(nt, [&](uint32_t t)
			{
				const uint32_t e = std::min(n, (t + 1) * chunk);
				for (uint32_t i = t * chunk; i < e; i++)
					fn(i); });
	}

	// fn(i) for i in [0, n) over the host cores, items handed out one at a time (for few,
	// uneven items such as contours); fn(i) writes only what i owns
	template <typename F>
	void host_parallel_dynamic(uint32_t n, F&& fn)
	{
		HostPool::get().run(n, [&](uint32_t i) { fn(i); });
	}

	// returns the EF pair count after the degenerate filter (before loop-vertex pairs)
	uint32_t build_graph(const u26_scene& S, const std::vector<float>& x, HostGraph& G, bool ignore_near_zero,
		const std::function<void(const char*)>& mark)
	{
		uint32_t n = uint32_t(G.ef.size());
		// the canonical EF list is sorted by edge: each edge's pairs form one run, found by
		// binary search (no table over all of the mesh's edges)
		auto edge_run = [&](uint32_t e, uint32_t& b, uint32_t& t)
		{
			const auto r = std::equal_range(G.ee.begin(), G.ee.begin() + n, e);
			b = uint32_t(r.first - G.ee.begin());
			t = uint32_t(r.second - G.ee.begin());
		};
		auto build_adj = [&]()
		{
		G.adj.assign(n, {});
		host_parallel_for(n, [&](uint32_t p)
		{
			const uint32_t e = G.ee[p], f = G.ff[p];
			auto& out = G.adj[p];
			for (uint32_t k = S.eae_off[e]; k < S.eae_off[e + 1]; k++)
			{
				uint32_t b, t;
				edge_run(S.eae[k], b, t);
				for (uint32_t q = b; q < t; q++)
					if (G.ff[q] == f && q != p)
						out.push_back(q);
			}
			for (int j = 0; j < 3; j++)
			{
				uint32_t b, t;
				edge_run(S.fae[3 * f + j], b, t);
				for (uint32_t q = b; q < t; q++)
				{
					if (q == p)
						continue;
					for (uint32_t k = S.eaf_off[e]; k < S.eaf_off[e + 1]; k++)
						if (G.ff[q] == S.eaf[k] && G.ee[q] != e)
							out.push_back(q);
				}
			}
		});
		};
		build_adj();
		mark("  EF adjacency");
		// degenerate filter (intersection_resolver.cpp:841-896): with near-zero-distance pairs in
		// play, a pair with a barycentric coordinate below 1e-4 stays only when one of its
		// adjacent pairs is not degenerate; if that would remove every pair, all stay
		if (!ignore_near_zero && n > 0)
		{
			std::vector<uint8_t> deg(n);
			uint32_t ndeg = 0;
			for (uint32_t p = 0; p < n; p++)
			{
				const EfPairH& e = G.ef[p];
				const float eb0 = e.bary[0], eb1 = 1.0f - e.bary[0];
				const float f0 = e.bary[1], f1 = e.bary[2], f2 = 1.0f - e.bary[1] - e.bary[2];
				deg[p] = (std::min(eb0, eb1) < 1e-4f || std::min(std::min(f0, f1), f2) < 1e-4f) ? 1 : 0;
				ndeg += deg[p];
			}
			if (ndeg)
			{
				std::vector<uint32_t> keep;
				for (uint32_t p = 0; p < n; p++)
				{
					bool k = !deg[p];
					for (uint32_t q : G.adj[p])
						k = k || !deg[q];
					if (k)
						keep.push_back(p);
				}
				if (!keep.empty() && keep.size() < n)
				{
					std::vector<EfPairH> ef;
					std::vector<uint32_t> ee, ff;
					for (uint32_t p : keep)
					{
						ef.push_back(G.ef[p]);
						ee.push_back(G.ee[p]);
						ff.push_back(G.ff[p]);
					}
					G.ef = std::move(ef);
					G.ee = std::move(ee);
					G.ff = std::move(ff);
					n = uint32_t(keep.size());
					build_adj();
				}
			}
		}
		const uint32_t n_kept = n;
		mark("  degenerate filter");
		// loop-vertex pairs
		struct Loop
		{
			uint32_t v, p, e, f;
		};
		std::vector<std::vector<Loop>> loops_of(n);
		host_parallel_for(n, [&](uint32_t p)
		{
			const uint32_t e = G.ee[p], f = G.ff[p];
			const uint32_t ex = S.edges[2 * e], ey = S.edges[2 * e + 1];
			for (uint32_t k = S.eaf_off[e]; k < S.eaf_off[e + 1]; k++)
			{
				const uint32_t af = S.eaf[k];
				const uint32_t av = S.faces[3 * af] + S.faces[3 * af + 1] + S.faces[3 * af + 2] - ex - ey;
				if (av != S.faces[3 * f] && av != S.faces[3 * f + 1] && av != S.faces[3 * f + 2])
					continue;
				const uint32_t* fa = &S.fae[3 * af];
				auto has = [&](uint32_t ed, uint32_t v)
				{ return S.edges[2 * ed] == v || S.edges[2 * ed + 1] == v; };
				uint32_t le;
				if (e == fa[0])
					le = has(fa[1], av) ? fa[1] : fa[2];
				else if (e == fa[1])
					le = has(fa[0], av) ? fa[0] : fa[2];
				else
					le = has(fa[0], av) ? fa[0] : fa[1];
				loops_of[p].push_back({ av, p, le, f });
			}
		});
		std::vector<Loop> loops;
		for (const auto& lv : loops_of)
			loops.insert(loops.end(), lv.begin(), lv.end());
		for (const Loop& l : loops)
		{
			EfPairH lp{};
			for (int k = 0; k < 5; k++)
				lp.idx[k] = l.v;
			lp.bary[0] = 1.0f;
			lp.bary[1] = 1.0f;
			lp.bary[2] = 0.0f;
			const uint32_t np = uint32_t(G.ef.size());
			G.ef.push_back(lp);
			G.ee.push_back(l.e);
			G.ff.push_back(l.f);
			G.adj.push_back({ l.p });
			G.adj[l.p].push_back(np);
		}
		const uint32_t na = uint32_t(G.ef.size());
		auto X = [&](uint32_t v)
		{ return mkv(x[3 * v], x[3 * v + 1], x[3 * v + 2]); };
		G.pos3.resize(na);
		G.len.resize(na);
		host_parallel_for(na, [&](uint32_t p)
			{ G.pos3[p] = X(G.ef[p].idx[0]) * G.ef[p].bary[0] + X(G.ef[p].idx[1]) * (1.0f - G.ef[p].bary[0]); });
		host_parallel_for(na, [&](uint32_t p)
			{
				float s = 0.0f;
				for (uint32_t q : G.adj[p])
					s += hlen(G.pos3[q] - G.pos3[p]);
				G.len[p] = 0.5f * s; });
		mark("  loop pairs, lengths");
		// flood fill with mesh-side parity
		G.mesh_index.assign(na, kInfH);
		std::vector<uint8_t> seen(na, 0);
		for (uint32_t seed = 0; seed < na; seed++)
		{
			if (seen[seed])
				continue;
			std::vector<std::pair<uint32_t, uint32_t>> stack{ { seed, 0u } };
			std::vector<uint32_t> comp{ seed };
			G.mesh_index[seed] = 0;
			seen[seed] = 1;
			while (!stack.empty())
			{
				const auto [p, par] = stack.back();
				stack.pop_back();
				for (uint32_t q : G.adj[p])
				{
					if (seen[q])
						continue;
					seen[q] = 1;
					const bool same = G.ef[p].idx[2] == G.ef[q].idx[2] && G.ef[p].idx[3] == G.ef[q].idx[3] && G.ef[p].idx[4] == G.ef[q].idx[4];
					const uint32_t np = par + (same ? 0u : 1u);
					G.mesh_index[q] = np % 2;
					stack.push_back({ q, np });
					comp.push_back(q);
				}
			}
			G.contours.push_back(std::move(comp));
		}
		G.contour_index.assign(na, kInfH);
		for (uint32_t c = 0; c < G.contours.size(); c++)
			for (uint32_t p : G.contours[c])
				G.contour_index[p] = c;
		G.type.resize(G.contours.size());
		for (uint32_t c = 0; c < G.contours.size(); c++)
		{
			uint32_t nb = 0, nl = 0, first_b = 0, last_b = 0;
			bool closed = true;
			for (uint32_t p : G.contours[c])
			{
				const bool bnd = (S.eaf_off[G.ee[p] + 1] - S.eaf_off[G.ee[p]]) <= 1;
				if (G.ef[p].is_loop())
					nl++;
				if (bnd)
				{
					if (nb == 0)
						first_b = p;
					last_b = p;
					nb++;
					closed = false;
				}
				if (!G.ef[p].is_loop() && G.adj[p].size() == 1)
					closed = false;
			}
			uint32_t t = 0;
			if (nb == 0)
				t = (closed && nl == 0) ? 1u : (closed && nl == 1) ? 2u : (closed && nl == 2) ? 3u : 0u;
			else if (nl == 0)
				t = nb == 2 ? (G.mesh_index[first_b] == G.mesh_index[last_b] ? 7u : 6u) : 0u;
			else if (nl == 1)
				t = nb == 1 ? 4u : nb == 2 ? 5u : 0u;
			G.type[c] = t;
		}
		mark("  contours, types");
		// vertex boundary flags 2c + side (CSR, sorted unique per vertex): bucketed by vertex
		// (counting sort), then each short row sorted and deduplicated
		std::vector<uint32_t> row(S.nv + 1, 0u);
		for (uint32_t p = 0; p < na; p++)
			if (!G.ef[p].is_loop())
				for (int k = 0; k < 5; k++)
					row[G.ef[p].idx[k] + 1]++;
		for (uint32_t v = 0; v < S.nv; v++)
			row[v + 1] += row[v];
		std::vector<uint32_t> fill(row.begin(), row.end() - 1), flat(row[S.nv]);
		for (uint32_t p = 0; p < na; p++)
		{
			if (G.ef[p].is_loop())
				continue;
			const uint32_t fe = 2 * G.contour_index[p] + G.mesh_index[p];
			for (int k = 0; k < 5; k++)
				flat[fill[G.ef[p].idx[k]]++] = k < 2 ? fe : (fe ^ 1u);
		}
		G.vflag_off.assign(S.nv + 1, 0u);
		host_parallel_for(S.nv, [&](uint32_t v)
			{
				std::sort(flat.begin() + row[v], flat.begin() + row[v + 1]);
				G.vflag_off[v + 1] = uint32_t(std::unique(flat.begin() + row[v], flat.begin() + row[v + 1]) - (flat.begin() + row[v]));
			});
		for (uint32_t v = 0; v < S.nv; v++)
			G.vflag_off[v + 1] += G.vflag_off[v];
		G.vflags.resize(G.vflag_off[S.nv]);
		host_parallel_for(S.nv, [&](uint32_t v)
			{ std::copy(flat.begin() + row[v], flat.begin() + row[v] + (G.vflag_off[v + 1] - G.vflag_off[v]), G.vflags.begin() + G.vflag_off[v]); });
		return n_kept;
	}

	std::vector<V3h> directions(const u26_scene& S, const std::vector<float>& x, const HostGraph& G, const ContourRT& r, uint32_t mode,
		V3h global_centroid, bool gc_valid)
	{
		std::vector<V3h> d;
		if (mode == 1)
		{
			for (int a = -1; a <= 1; a++)
				for (int b = -1; b <= 1; b++)
					for (int c = -1; c <= 1; c++)
						if (a || b || c)
							d.push_back(hnorm(mkv(float(a), float(b), float(c))));
			return d;
		}
		auto seed = [&](V3h v)
		{
			if (hvalid(v))
				d.push_back(hnorm(v));
		};
		auto both = [&](V3h v)
		{
			seed(v);
			seed(-v);
		};
		auto X = [&](uint32_t v)
		{ return mkv(x[3 * v], x[3 * v + 1], x[3 * v + 2]); };
		const auto& cp = G.contours[r.contour];
		V3h ws = mkv(0, 0, 0), us = mkv(0, 0, 0);
		float sw = 0.0f;
		for (uint32_t p : cp)
		{
			us = us + G.pos3[p];
			ws = ws + G.pos3[p] * G.len[p];
			sw += G.len[p];
		}
		const V3h cen = sw == 0.0f ? us / float(cp.size()) : ws / sw;
		V3h mc[2] = { mkv(0, 0, 0), mkv(0, 0, 0) };
		V3h col[3] = { mkv(0, 0, 0), mkv(0, 0, 0), mkv(0, 0, 0) };
		for (int side = 0; side < 2; side++)
		{
			std::vector<float> w;
			for (uint32_t v : r.bnd[side])
			{
				const V3h p = X(v);
				const float wt = std::fmax(S.varea[v], 1e-8f);
				w.push_back(wt);
				mc[side] = mc[side] + p * wt;
				const V3h c = p - cen;
				col[0] = col[0] + (c * c.x) * wt;
				col[1] = col[1] + (c * c.y) * wt;
				col[2] = col[2] + (c * c.z) * wt;
			}
			float sum = 0.0f;
			for (float v : w)
				sum += v;
			mc[side] = sum > 1e-8f ? mc[side] / sum : cen;
		}
		V3h ev[3] = { mkv(0, 1, 0), mkv(1, 0, 0), mkv(0, 0, 1) };
		{
			bool finite = true;
			for (int c = 0; c < 3; c++)
				finite = finite && std::isfinite(col[c].x) && std::isfinite(col[c].y) && std::isfinite(col[c].z);
			const float tr = col[0].x + col[1].y + col[2].z;
			float fr = 0.0f;
			for (int c = 0; c < 3; c++)
				fr += hdot(col[c], col[c]);
			if (finite && tr >= 1e-10f && fr >= 1e-20f)
			{
				double A[3][3], V[3][3];
				for (int c = 0; c < 3; c++)
				{
					A[0][c] = col[c].x;
					A[1][c] = col[c].y;
					A[2][c] = col[c].z;
				}
				sym_eigen3(A, V);
				const V3h def[3] = { mkv(0, 1, 0), mkv(1, 0, 0), mkv(0, 0, 1) };
				for (int k = 0; k < 3; k++)
				{
					const V3h v = mkv(float(V[0][k]), float(V[1][k]), float(V[2][k]));
					ev[k] = hdot(v, v) > 1e-12f ? hnorm(v) : def[k];
				}
			}
		}
		for (int k = 0; k < 3; k++)
			both(ev[k]);
		for (int side = 0; side < 2; side++)
		{
			V3h v = cen - mc[side];
			if (!hvalid(v))
				v = ev[side + 1];
			seed(v);
		}
		if (gc_valid)
		{
			const V3h rad = cen - global_centroid;
			if (hvalid(rad))
				both(rad);
		}
		if (d.empty())
			both(mkv(0, 1, 0));
		return d;
	}

	inline int bits_for(uint64_t n)
	{
		int b = 1;
		while (b < 63 && (uint64_t(1) << b) < n)
			b++;
		return b;
	}
} // namespace

static double ms_since(std::chrono::steady_clock::time_point t0)
{
	return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// GPU-timeline markers of one level (read only when U26_PRP_TRACE is set)
struct LevelEvents
{
	cudaEvent_t e[8] = {};
	bool on = false;
	explicit LevelEvents(bool enable) : on(enable)
	{
		if (on)
			for (auto& x : e)
				cudaEventCreate(&x);
	}
	~LevelEvents()
	{
		if (on)
			for (auto& x : e)
				cudaEventDestroy(x);
	}
	void mark(int i, cudaStream_t st)
	{
		if (on)
			cudaEventRecord(e[i], st);
	}
	float ms(int a, int b) const
	{
		float t = 0.0f;
		if (on)
			cudaEventElapsedTime(&t, e[a], e[b]);
		return t;
	}
};

// The selected supports' depths, D_C and J in FP64 against their FP32 values (max relative
// errors over the pass) and the D_C tie rechecks.
static u26_status fp64_metrics(u26_scene* S, const float* d_x, u26_prp_output* out)
{
	u26_ctx* ctx = S->ctx;
	cudaStream_t st = ctx->stream;
	std::vector<Fp64In> in;
	for (size_t c = 0; c < out->results.size(); c++)
	{
		const u26_prp_result& r = out->results[c];
		if (r.combo_idx == kInf || r.hit_count == 0)
			continue;
		in.push_back(Fp64In{ out->hit_offsets[c], out->hit_offsets[c + 1], { r.dir[0], r.dir[1], r.dir[2] }, r.objective, r.depth });
	}
	if (in.empty())
		return U26_OK;
	DevBuf &d_in = S->d_f64in, &d_hits = S->d_f64hits, &d_out = S->d_f64out;
	U26_TRY(upload(ctx, d_in, in));
	U26_TRY(upload(ctx, d_hits, out->hits));
	U26_CUDA(ctx, d_out.reserve(sizeof(Fp64Out) * in.size()));
	const uint32_t nc = uint32_t(in.size());
	const uint32_t nh = uint32_t(out->hits.size());
	U26_CUDA(ctx, S->d_f64delta.reserve(sizeof(double) * nh));
	fp64_depths_kernel<<<div_up(nh, 128u), 128, 0, st>>>(nc, d_in.as<Fp64In>(), nh, d_hits.as<u26_prp_hit>(), d_x, S->d_edges.as<uint2>(),
		S->d_faces.as<uint32_t>(), S->d_f64delta.as<double>());
	U26_TRY(after_launch(ctx, "fp64_depths_kernel"));
	fp64_metrics_kernel<<<div_up(nc * 32u, 128u), 128, 0, st>>>(nc, d_in.as<Fp64In>(), d_hits.as<u26_prp_hit>(), S->d_f64delta.as<double>(),
		S->d_varea.as<float>(), S->d_earea.as<float>(), S->d_farea.as<float>(), d_out.as<Fp64Out>());
	U26_TRY(after_launch(ctx, "fp64_metrics_kernel"));
	std::vector<Fp64Out> res;
	U26_TRY(download(ctx, res, d_out.ptr, in.size()));
	U26_CUDA(ctx, cudaStreamSynchronize(st));
	for (size_t i = 0; i < res.size(); i++)
	{
		const Fp64Out& o = res[i];
		out->fp64_delta_rel_err = std::max(out->fp64_delta_rel_err, o.delta_err);
		if (o.dc64 > 0.0)
			out->fp64_dc_rel_err = std::max(out->fp64_dc_rel_err, std::fabs(double(in[i].dc32) - o.dc64) / o.dc64);
		if (o.j64 > 0.0)
			out->fp64_j_rel_err = std::max(out->fp64_j_rel_err, std::fabs(double(in[i].j32) - o.j64) / o.j64);
		out->dc_tie_rechecks += o.tie;
		out->dc_tie_flips += o.flip;
	}
	return U26_OK;
}

static u26_status prp_run(u26_scene* S, u26_lbvh* face_tree, u26_lbvh* edge_tree, const float* d_x, const void* d_pairs,
	const uint32_t* d_idx, uint32_t num_pairs, const u26_prp_params* P, u26_prp_output* out)
{
	u26_ctx* ctx = S->ctx;
	cudaStream_t st = ctx->stream;
	const auto t_total = std::chrono::steady_clock::now();
	auto t0 = t_total;
	S->store_used = 0; // the support store holds this pass's captures only
	// with U26_PRP_TRACE set: the host-side time line of the pass, printed at its end
	const bool trace_marks = std::getenv("U26_PRP_TRACE") != nullptr;
	std::vector<std::pair<const char*, double>> marks;
	auto mark = [&](const char* what)
	{
		if (trace_marks)
			marks.emplace_back(what, ms_since(t_total));
	};
	// ---- 1. host copies of positions and the canonical EF list
	std::vector<float> x;
	HostGraph G;
	U26_TRY(download(ctx, x, d_x, 3 * size_t(S->nv)));
	mark("positions downloaded");
	U26_TRY(download(ctx, G.ef, d_pairs, num_pairs));
	std::vector<uint32_t> idx;
	U26_TRY(download(ctx, idx, d_idx, 2 * size_t(num_pairs)));
	// ---- device normals at x (overlaps the host preprocessing)
	if (S->nf)
	{
		normals_face_kernel<<<div_up(S->nf, 256), 256, 0, st>>>(d_x, S->d_faces.as<uint32_t>(), S->d_vobj.as<uint32_t>(),
			S->d_orient.as<uint32_t>(), S->nf, S->d_fn.as<float>());
		U26_TRY(after_launch(ctx, "normals_face_kernel"));
		normals_accum_kernel<<<div_up(S->ne, 256), 256, 0, st>>>(S->d_eaf_off.as<uint32_t>(), S->d_eaf.as<uint32_t>(), S->d_farea.as<float>(),
			S->d_fn.as<float>(), S->ne, S->d_en.as<float>());
		U26_TRY(after_launch(ctx, "normals_accum_kernel"));
		normals_accum_kernel<<<div_up(S->nv, 256), 256, 0, st>>>(S->d_vaf_off.as<uint32_t>(), S->d_vaf.as<uint32_t>(), S->d_farea.as<float>(),
			S->d_fn.as<float>(), S->nv, S->d_vn.as<float>());
		U26_TRY(after_launch(ctx, "normals_accum_kernel"));
	}
	U26_CUDA(ctx, cudaStreamSynchronize(st));
	G.ee.resize(num_pairs);
	G.ff.resize(num_pairs);
	for (uint32_t i = 0; i < num_pairs; i++)
	{
		G.ee[i] = idx[2 * i];
		G.ff[i] = idx[2 * i + 1];
	}
	mark("EF list downloaded, normals");
	out->num_orig_pairs = build_graph(*S, x, G, P->ignore_near_zero_dist_pairs != 0, mark);
	mark("EF graph, contours");
	out->stage_ms[0] = ms_since(t0);
	const uint32_t na = uint32_t(G.ef.size());
	const uint32_t nc = uint32_t(G.contours.size());
	const uint32_t nact = std::min(nc, P->max_contours);

	// ---- 2. runtime identity, anchors, boundary verts, distances
	t0 = std::chrono::steady_clock::now();
	std::vector<ContourRT> R(nact);
	// global area-weighted centroid of each independent scene (one scene unless the mesh
	// says otherwise), summed in vertex order
	const uint32_t nscene = S->oscene.empty() ? 1u : *std::max_element(S->oscene.begin(), S->oscene.end()) + 1u;
	std::vector<V3h> gcs(nscene, mkv(0, 0, 0));
	std::vector<float> tms(nscene, 0.0f);
	{
		// each scene's sums run over its vertices in vertex order (its objects' contiguous
		// ranges, in object order); the scenes in parallel
		std::vector<std::vector<uint32_t>> objs(nscene);
		for (uint32_t o = 0; o < S->nobj; o++)
			objs[S->oscene.empty() ? 0u : S->oscene[o]].push_back(o);
		host_parallel_dynamic(nscene, [&](uint32_t sc)
		{
			V3h g = mkv(0, 0, 0);
			float tm = 0.0f;
			for (uint32_t o : objs[sc])
				for (uint32_t v = S->pv[o]; v < S->pv[o + 1]; v++)
				{
					const float w = std::fmax(S->varea[v], 1e-8f);
					g = g + mkv(x[3 * v], x[3 * v + 1], x[3 * v + 2]) * w;
					tm += w;
				}
			gcs[sc] = g;
			tms[sc] = tm;
		});
	}
	for (uint32_t sc = 0; sc < nscene; sc++)
		if (tms[sc] > 1e-8f)
			gcs[sc] = gcs[sc] / tms[sc];
	mark("  scene centroids");
	std::vector<uint32_t> anchor_off(nact + 1, 0u), anchors, bnd;
	std::vector<Slot> slots(2 * size_t(nact));
	// per contour (in parallel): objects, the restriction switch, the two sides' boundary vertices
	// (sorted unique) and the EF anchors; then the slots and the flat lists in contour order
	std::vector<uint8_t> ccr(nact, 0);
	std::vector<std::vector<uint32_t>> anch(nact);
	host_parallel_dynamic(nact, [&](uint32_t c)
	{
		ContourRT& r = R[c];
		r.contour = c;
		const uint32_t first = G.contours[c].front();
		const uint32_t es = G.mesh_index[first];
		r.obj[es] = S->vobj[G.ef[first].idx[0]];
		r.obj[es ^ 1] = S->vobj[G.ef[first].idx[2]];
		uint32_t comp[2];
		comp[es] = S->vcomp[G.ef[first].idx[0]];
		comp[es ^ 1] = S->vcomp[G.ef[first].idx[2]];
		// prp_intrinsic_contour_side_restriction_applies (intersection_resolver2.h:415-429)
		bool ccr_on = P->use_ccr && (P->ccr_use_rest || P->ccr_use_current);
		if (ccr_on && P->ccr_use_current)
			ccr_on = r.obj[0] != kInfH && r.obj[1] != kInfH;
		else if (ccr_on)
			ccr_on = r.obj[0] == r.obj[1] && comp[0] != kInfH && comp[0] == comp[1];
		ccr[c] = ccr_on ? 1 : 0;
		std::vector<uint32_t> b[2];
		std::vector<uint32_t>& an = anch[c];
		an.reserve(6 * G.contours[c].size());
		for (uint32_t p : G.contours[c])
		{
			const uint32_t mi = G.mesh_index[p];
			b[mi].push_back(G.ef[p].idx[0]);
			b[mi].push_back(G.ef[p].idx[1]);
			for (int k = 2; k < 5; k++)
				b[mi ^ 1].push_back(G.ef[p].idx[k]);
			an.insert(an.end(), { mi, G.ef[p].idx[0], G.ef[p].idx[1], G.ef[p].idx[2], G.ef[p].idx[3], G.ef[p].idx[4] });
		}
		for (int sd = 0; sd < 2; sd++)
		{
			std::sort(b[sd].begin(), b[sd].end());
			b[sd].erase(std::unique(b[sd].begin(), b[sd].end()), b[sd].end());
			r.bnd[sd] = std::move(b[sd]);
		}
	});
	for (uint32_t c = 0; c < nact; c++)
	{
		const ContourRT& r = R[c];
		anchors.insert(anchors.end(), anch[c].begin(), anch[c].end());
		anchor_off[c + 1] = uint32_t(anchors.size() / 6);
		for (int sd = 0; sd < 2; sd++)
		{
			Slot& sl = slots[2 * c + sd];
			const uint32_t o = r.obj[sd];
			sl.v_lo = S->pv[o];
			sl.v_cnt = S->pv[o + 1] - S->pv[o];
			sl.e_lo = S->pe[o];
			sl.e_cnt = S->pe[o + 1] - S->pe[o];
			sl.f_lo = S->pf[o];
			sl.f_cnt = S->pf[o + 1] - S->pf[o];
			sl.bnd_off = uint32_t(bnd.size());
			sl.bnd_cnt = uint32_t(r.bnd[sd].size());
			sl.k = 0;
			sl.diam = 0;
			sl.pad[0] = ccr[c];
			sl.pad[1] = o; // the side's object: its ray-casting trees
			bnd.insert(bnd.end(), r.bnd[sd].begin(), r.bnd[sd].end());
		}
	}
	// candidate directions of each contour (host, in parallel), while the GPU computes the
	// slots' distances below
	auto contour_directions = [&]()
	{
		host_parallel_dynamic(nact, [&](uint32_t c)
		{
			ContourRT& r = R[c];
			const uint32_t rsc = S->oscene[r.obj[0]];
			r.dirs = directions(*S, x, G, r, P->direction_mode, gcs[rsc], tms[rsc] > 1e-8f);
			const size_t nd = r.dirs.size();
			r.res.assign(nd, ComboState{});
			r.conv.assign(nd, 0);
			r.pruned.assign(nd, 0);
			r.present.assign(nd, 0);
			r.active.assign(nd, 1);
		});
	};
	mark("runtimes, anchors");
	const uint32_t nslots = 2 * nact;
	const uint32_t vs = std::max(1u, S->vmax_obj), es_ = std::max(1u, S->emax_obj), fs = std::max(1u, S->fmax_obj);
	if (nact > 0)
	{
		U26_TRY(upload(ctx, S->d_slots, slots));
		U26_TRY(upload(ctx, S->d_bnd, bnd));
		std::vector<uint32_t> ids(nslots);
		std::iota(ids.begin(), ids.end(), 0u);
		U26_TRY(upload(ctx, S->d_slot_ids, ids));
		U26_CUDA(ctx, S->d_hop.reserve(sizeof(uint32_t) * size_t(nslots) * vs));
		U26_CUDA(ctx, S->d_geo.reserve(sizeof(float) * size_t(nslots) * vs));
		U26_CUDA(ctx, S->d_order.reserve(sizeof(uint32_t) * size_t(nslots) * vs));
		U26_CUDA(ctx, S->d_level_end.reserve(sizeof(uint32_t) * size_t(nslots) * (vs + 1)));
		U26_CUDA(ctx, S->d_work.reserve(sizeof(uint32_t) * size_t(nslots) * 2 * vs));
		U26_CUDA(ctx, S->d_mark.reserve(sizeof(uint32_t) * size_t(nslots) * vs));
		U26_CUDA(ctx, S->d_owns.reserve(size_t(nslots) * vs));
		U26_CUDA(ctx, S->d_cand_v.reserve(sizeof(uint32_t) * size_t(nslots) * vs));
		U26_CUDA(ctx, S->d_cand_e.reserve(sizeof(uint32_t) * size_t(nslots) * es_));
		U26_CUDA(ctx, S->d_cand_f.reserve(sizeof(uint32_t) * size_t(nslots) * fs));
		U26_CUDA(ctx, S->d_counts.reserve(sizeof(uint32_t) * 3 * size_t(nslots)));
		U26_CUDA(ctx, S->d_bits_e.reserve(sizeof(uint32_t) * size_t(nslots) * (es_ / 32 + 1)));
		U26_CUDA(ctx, S->d_bits_f.reserve(sizeof(uint32_t) * size_t(nslots) * (fs / 32 + 1)));
		// current-space anchor distances, computed lazily per level (NaN: not yet computed)
		U26_CUDA(ctx, S->d_cur_own.reserve(sizeof(float) * size_t(nslots) * vs));
		U26_CUDA(ctx, S->d_cur_opp.reserve(sizeof(float) * size_t(nslots) * vs));
		U26_CUDA(ctx, cudaMemsetAsync(S->d_cur_own.ptr, 0xFF, sizeof(float) * size_t(nslots) * vs, st));
		U26_CUDA(ctx, cudaMemsetAsync(S->d_cur_opp.ptr, 0xFF, sizeof(float) * size_t(nslots) * vs, st));
		distances_kernel<<<nslots, 256, 0, st>>>(S->d_slots.as<Slot>(), S->d_slot_ids.as<uint32_t>(), S->d_bnd.as<uint32_t>(),
			S->d_vav_off.as<uint32_t>(), S->d_vav.as<uint32_t>(), S->d_rest_x.as<float>(), vs, S->d_hop.as<uint32_t>(),
			S->d_geo.as<float>(), S->d_order.as<uint32_t>(), S->d_level_end.as<uint32_t>(), S->d_work.as<uint32_t>(),
			S->d_mark.as<uint32_t>(), ctx->dev_err);
		U26_TRY(after_launch(ctx, "distances_kernel"));
		contour_directions();
		mark("directions (beside the distances)");
		U26_TRY(download(ctx, slots, S->d_slots.ptr, nslots));
		U26_CUDA(ctx, cudaStreamSynchronize(st));
	}
	for (uint32_t c = 0; c < nact; c++)
	{
		ContourRT& r = R[c];
		for (int sd = 0; sd < 2; sd++)
		{
			r.diam[sd] = slots[2 * c + sd].diam;
			const uint32_t bc = uint32_t(r.bnd[sd].size());
			uint32_t k0 = 3;
			if (r.diam[sd] != 0)
				k0 = std::max(3u, std::min(uint32_t(std::ceil(std::sqrt(float(bc)))), r.diam[sd]));
			r.k0[sd] = k0;
			r.k[sd] = k0;
		}
	}
	// vertex flags and anchors on the device
	U26_TRY(upload(ctx, S->d_vf_off, G.vflag_off));
	U26_TRY(upload(ctx, S->d_vf, G.vflags));
	U26_TRY(upload(ctx, S->d_anchor_off, anchor_off));
	U26_TRY(upload(ctx, S->d_anchors, anchors));
	out->stage_ms[1] = ms_since(t0);

	// ---- 3. adaptive k-ring levels, every active (contour, direction) task batched
	const int b = bits_for(std::max({ S->nv, S->ne, S->nf, 2u }));
	U26_CUDA(ctx, S->d_stats.reserve(sizeof(unsigned long long) * 16));
	U26_CUDA(ctx, cudaMemsetAsync(S->d_stats.ptr, 0, sizeof(unsigned long long) * 16, st));
	const TreeView ftv = tree_view(face_tree), etv = tree_view(edge_tree);
	// The ray casts traverse one face tree and one edge tree per object (the reference's
	// per-object CachedBVH): a ray tests only its target object's primitives. The trees are
	// built at the scene's first pass and refit on every pass; their grown node boxes (with
	// the child links in the w lanes) form one forest array, and each tree's subtree roots of
	// the split traversals sit at [object * kFrontStride, (object + 1) * kFrontStride).
	const uint32_t nobj = std::max(1u, S->nobj);
	{
		if (!S->otrees_built)
		{
			U26_CUDA(ctx, S->d_zero_th.reserve(sizeof(float) * std::max(1u, S->nv)));
			U26_CUDA(ctx, cudaMemsetAsync(S->d_zero_th.ptr, 0, sizeof(float) * std::max(1u, S->nv), st));
			S->otree_f.assign(nobj, nullptr);
			S->otree_e.assign(nobj, nullptr);
			for (uint32_t o = 0; o < S->nobj; o++)
				for (int kind = 0; kind < 2; kind++)
				{
					const uint32_t cnt = kind == 0 ? S->pf[o + 1] - S->pf[o] : S->pe[o + 1] - S->pe[o];
					if (cnt == 0)
						continue;
					const uint32_t* prims = kind == 0 ? S->d_faces.as<uint32_t>() + 3 * size_t(S->pf[o]) : S->d_edges.as<uint32_t>() + 2 * size_t(S->pe[o]);
					u26_lbvh* t = nullptr;
					U26_TRY(u26_lbvh_create(ctx, kind == 0 ? U26_TREE_FACE : U26_TREE_EDGE, cnt, &t));
					(kind == 0 ? S->otree_f : S->otree_e)[o] = t;
					U26_TRY(u26_lbvh_set_option(t, U26_LBVH_OPT_FULL_GLOBAL_AABB, 1));
					U26_TRY(u26_lbvh_reduce_aabb(t, d_x, S->nv, prims));
					U26_TRY(u26_lbvh_construct_tree(t));
				}
			S->otrees_built = true;
		}
		std::vector<uint32_t> foff(nobj + 1, 0u), eoff(nobj + 1, 0u);
		for (uint32_t o = 0; o < nobj; o++)
		{
			foff[o + 1] = foff[o] + (S->otree_f[o] ? S->otree_f[o]->num_nodes() : 0u);
			eoff[o + 1] = eoff[o] + (S->otree_e[o] ? S->otree_e[o]->num_nodes() : 0u);
		}
		U26_CUDA(ctx, S->d_fgrow.reserve(sizeof(NodeBox) * std::max(foff[nobj], 1u)));
		U26_CUDA(ctx, S->d_egrow.reserve(sizeof(NodeBox) * std::max(eoff[nobj], 1u)));
		// the split traversals' subtree roots depend on the trees' topology only: found once
		const bool fronts = !S->fronts_built;
		if (fronts)
		{
			U26_CUDA(ctx, S->d_front.reserve(sizeof(uint32_t) * 2 * size_t(nobj) * kFrontStride));
			U26_CUDA(ctx, cudaMemsetAsync(S->d_front.ptr, 0xFF, sizeof(uint32_t) * 2 * size_t(nobj) * kFrontStride, st));
		}
		// refit + grow of every object tree on stream `on` (and the frontiers when asked)
		auto forest_pass = [&](cudaStream_t on, bool with_fronts) -> u26_status
		{
			for (uint32_t o = 0; o < nobj; o++)
				for (int kind = 0; kind < 2; kind++)
				{
					u26_lbvh* t = (kind == 0 ? S->otree_f : S->otree_e)[o];
					if (!t)
						continue;
					const uint32_t* prims = kind == 0 ? S->d_faces.as<uint32_t>() + 3 * size_t(S->pf[o]) : S->d_edges.as<uint32_t>() + 2 * size_t(S->pe[o]);
					U26_TRY(u26_lbvh_update_and_refit(t, S->d_zero_th.as<float>(), d_x, d_x, prims));
					const TreeView tv = tree_view(t);
					const uint32_t nn = t->num_nodes();
					const uint32_t node_off = kind == 0 ? foff[o] : eoff[o];
					const uint32_t prim_off = kind == 0 ? S->pf[o] : S->pe[o];
					grow_boxes_kernel<<<div_up(nn, 256), 256, 0, on>>>(tv.boxes, tv.children, tv.object_idx, nn, kind, node_off, prim_off,
						(kind == 0 ? S->d_fgrow : S->d_egrow).as<NodeBox>());
					U26_TRY(after_launch(ctx, "grow_boxes_kernel"));
					if (with_fronts)
					{
						frontier_kernel<<<1, 32, 0, on>>>(tv.children, tv.object_idx, nn, node_off,
							S->d_front.as<uint32_t>() + (size_t(kind) * nobj + o) * kFrontStride);
						U26_TRY(after_launch(ctx, "frontier_kernel"));
					}
				}
			return U26_OK;
		};
		if (fronts)
			U26_TRY(forest_pass(st, true)); // first pass: trees just built, frontiers found
		else
		{
			if (S->forest_exec && S->forest_x != d_x)
			{
				cudaGraphExecDestroy(S->forest_exec);
				S->forest_exec = nullptr;
			}
			if (!S->forest_exec && !S->forest_graph_failed)
			{
				// capture the launches on a private stream (the context's may be the legacy
				// default stream, which cannot be captured); the library's launches follow the
				// context's stream, so it points at the capture stream meanwhile
				if (!S->forest_stream)
					U26_CUDA(ctx, cudaStreamCreateWithFlags(&S->forest_stream, cudaStreamNonBlocking));
				const uint64_t l0 = ctx->launches;
				cudaStream_t orig = ctx->stream;
				cudaGraph_t graph = nullptr;
				cudaError_t ce = cudaStreamBeginCapture(S->forest_stream, cudaStreamCaptureModeThreadLocal);
				u26_status fs = U26_ERR_CUDA;
				if (ce == cudaSuccess)
				{
					ctx->stream = S->forest_stream;
					fs = forest_pass(S->forest_stream, false);
					ctx->stream = orig;
					ce = cudaStreamEndCapture(S->forest_stream, &graph);
				}
				if (fs == U26_OK && ce == cudaSuccess && graph)
					ce = cudaGraphInstantiate(&S->forest_exec, graph, 0);
				if (graph)
					cudaGraphDestroy(graph);
				if (fs != U26_OK || ce != cudaSuccess || !S->forest_exec)
				{
					// not capturable here: direct launches from now on
					cudaGetLastError();
					S->forest_exec = nullptr;
					S->forest_graph_failed = true;
					ctx->last_error.clear();
				}
				else
				{
					S->forest_launches = ctx->launches - l0;
					S->forest_x = d_x;
				}
				ctx->launches = l0;
			}
			if (S->forest_exec)
			{
				U26_CUDA(ctx, cudaGraphLaunch(S->forest_exec, st));
				ctx->launches += S->forest_launches; // the graph's kernels, as launches of this pass
			}
			else
				U26_TRY(forest_pass(st, false));
		}
		S->fronts_built = true;
	}
	const uint32_t bnd_words = vs / 32 + 1;
	if (nslots)
	{
		U26_CUDA(ctx, S->d_bnd_bits.reserve(sizeof(uint32_t) * size_t(nslots) * bnd_words));
		U26_CUDA(ctx, cudaMemsetAsync(S->d_bnd_bits.ptr, 0, sizeof(uint32_t) * size_t(nslots) * bnd_words, st));
		bnd_bits_kernel<<<nslots, 256, 0, st>>>(S->d_slots.as<Slot>(), S->d_bnd.as<uint32_t>(), vs, S->d_bnd_bits.as<uint32_t>());
		U26_TRY(after_launch(ctx, "bnd_bits_kernel"));
		U26_CUDA(ctx, S->d_slot_box.reserve(sizeof(float) * 12 * size_t(nslots)));
	}
	auto grow = [](uint32_t cur, uint32_t diam) -> uint32_t
	{
		if (cur >= diam)
			return cur;
		return uint32_t(std::min<uint64_t>(diam, std::max<uint64_t>(1u, uint64_t(cur) * 2u)));
	};
	// hit capacity kept by the scene across passes; grows by 1.5x the count that overflowed
	uint32_t hit_cap = std::max<uint32_t>(S->hit_cap, 1u << 22);
	const bool trace = std::getenv("U26_PRP_TRACE") != nullptr;
	// traversal configuration: with autotune, the scene's first pass times every configuration
	// on each of its ray-casting launches and the scene keeps the fastest (summed over that
	// pass) for its later passes
	const bool forced = P->raycast_config >= 1 && P->raycast_config <= uint32_t(kNumRaycastConfigs);
	const bool tuning = !forced && P->autotune && P->form == 0 && S->tuned_cfg < 0;
	const int cfg_now = forced ? int(P->raycast_config) - 1 : S->tuned_cfg >= 0 ? S->tuned_cfg : kDefaultRaycastConfig;
	std::vector<cudaEvent_t> tune_ev;
	struct EventsGuard
	{
		std::vector<cudaEvent_t>& v;
		~EventsGuard()
		{
			for (cudaEvent_t e : v)
				cudaEventDestroy(e);
		}
	} tune_guard{ tune_ev };
	if (tuning)
		for (int i = 0; i < 2 * kNumRaycastConfigs; i++)
		{
			cudaEvent_t e;
			U26_CUDA(ctx, cudaEventCreate(&e));
			tune_ev.push_back(e);
		}
	LevelEvents ev(true);
	uint64_t alg_tests = 0;

	// candidates of the listed slots at slots[s].k
	auto build_candidates = [&](const std::vector<uint32_t>& sids, std::vector<uint32_t>& counts) -> u26_status
	{
		U26_TRY(upload(ctx, S->d_slots, slots));
		U26_TRY(upload(ctx, S->d_slot_ids, sids));
		if (P->use_ccr && P->ccr_use_current && !sids.empty())
		{
			constexpr uint32_t kBlocksPerSlot = 32;
			ccr_current_kernel<<<uint32_t(sids.size()) * kBlocksPerSlot, 256, 0, st>>>(S->d_slots.as<Slot>(), S->d_slot_ids.as<uint32_t>(),
				S->d_bnd.as<uint32_t>(), d_x, vs, S->d_geo.as<float>(), S->d_order.as<uint32_t>(), S->d_level_end.as<uint32_t>(),
				P->ccr_use_rest, P->ccr_blend, P->ccr_tau, kBlocksPerSlot, S->d_cur_own.as<float>(), S->d_cur_opp.as<float>());
			U26_TRY(after_launch(ctx, "ccr_current_kernel"));
		}
		candidates_kernel<<<uint32_t(sids.size()), 256, 0, st>>>(S->d_slots.as<Slot>(), S->d_slot_ids.as<uint32_t>(), S->d_bnd.as<uint32_t>(),
			d_x, S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(), S->d_vae_off.as<uint32_t>(), S->d_vae.as<uint32_t>(),
			S->d_vaf_off.as<uint32_t>(), S->d_vaf.as<uint32_t>(), vs, es_, fs, S->d_hop.as<uint32_t>(), S->d_geo.as<float>(),
			S->d_order.as<uint32_t>(), S->d_level_end.as<uint32_t>(), P->ccr_use_rest, P->ccr_use_current, P->ccr_blend, P->ccr_tau,
			P->ccr_blend_weight,
			S->d_owns.as<uint8_t>(), S->d_cand_v.as<uint32_t>(), S->d_cand_e.as<uint32_t>(), S->d_cand_f.as<uint32_t>(),
			S->d_counts.as<uint32_t>(), S->d_bits_e.as<uint32_t>(), S->d_bits_f.as<uint32_t>(), S->d_slot_box.as<float>(),
			S->d_cur_own.as<float>(), S->d_cur_opp.as<float>());
		U26_TRY(after_launch(ctx, "candidates_kernel"));
		U26_TRY(download(ctx, counts, S->d_counts.ptr, 3 * size_t(nslots)));
		U26_CUDA(ctx, cudaStreamSynchronize(st));
		// request order: each slot's candidate vertices and edges by rest-space Morton code
		const uint32_t nsid = uint32_t(sids.size());
		const int sid_bits = bits_for(nsid + 1);
		for (int kind = 0; kind < 2; kind++)
		{
			std::vector<uint32_t> off(nsid + 1, 0u);
			for (uint32_t j = 0; j < nsid; j++)
				off[j + 1] = off[j] + counts[3 * sids[j] + kind];
			const uint32_t total = off[nsid];
			if (total < 2)
				continue;
			U26_TRY(upload(ctx, S->d_cand_off, off));
			U26_CUDA(ctx, S->d_ckeys.reserve(sizeof(uint64_t) * total));
			U26_CUDA(ctx, S->d_cvals.reserve(sizeof(uint32_t) * total));
			uint32_t* cand = kind == 0 ? S->d_cand_v.as<uint32_t>() : S->d_cand_e.as<uint32_t>();
			const uint32_t stride = kind == 0 ? vs : es_;
			const int id_bits = bits_for(kind == 0 ? S->nv : S->ne);
			cand_keys_kernel<<<div_up(total, 256), 256, 0, st>>>(S->d_slot_ids.as<uint32_t>(), S->d_cand_off.as<uint32_t>(), nsid, cand, stride,
				kind == 0 ? S->d_vrank.as<uint32_t>() : S->d_erank.as<uint32_t>(), id_bits, S->d_ckeys.as<uint64_t>(), S->d_cvals.as<uint32_t>());
			U26_TRY(after_launch(ctx, "cand_keys_kernel"));
			U26_TRY(S->csorter.sort(ctx, S->d_ckeys.as<uint64_t>(), S->d_cvals.as<uint32_t>(), total, 0, sid_bits + id_bits));
			cand_scatter_kernel<<<div_up(total, 256), 256, 0, st>>>(S->d_slot_ids.as<uint32_t>(), S->d_cand_off.as<uint32_t>(), nsid,
				S->d_cvals.as<uint32_t>(), cand, stride);
			U26_TRY(after_launch(ctx, "cand_scatter_kernel"));
		}
		return U26_OK;
	};

	// ray casting, hit sort, product adjacency, coverage, best component and metrics of
	// the given tasks; with hits_out, also the selected supports in canonical order
	auto evaluate = [&](std::vector<Task>& tasks, const std::vector<uint32_t>& counts, std::vector<TaskOut>& tout,
						std::vector<u26_prp_hit>* hits_out) -> u26_status
	{
		auto tl = std::chrono::steady_clock::now();
		uint32_t total_req = 0;
		uint64_t total_req64 = 0;
		for (Task& t : tasks)
		{
			const uint32_t v0 = counts[3 * t.slot0], e0 = counts[3 * t.slot0 + 1], f0 = counts[3 * t.slot0 + 2];
			const uint32_t v1 = counts[3 * t.slot1], e1 = counts[3 * t.slot1 + 1], f1 = counts[3 * t.slot1 + 2];
			t.n_vf = f1 ? v0 : 0;
			t.n_ee = e1 ? e0 : 0;
			t.n_fv = f0 ? v1 : 0;
			t.req_begin = total_req;
			total_req64 += uint64_t(t.n_vf) + t.n_ee + t.n_fv;
			// request ids are 32-bit (and a launch's work items stay below 2^31)
			if (total_req64 >= (uint64_t(1) << 31))
				return set_error(ctx, U26_ERR_CAPACITY, "PRP level needs %llu ray requests (limit 2^31): lower max_contours",
					(unsigned long long)total_req64);
			total_req = uint32_t(total_req64);
			if (!hits_out)
				alg_tests += uint64_t(t.n_vf) * f1 + uint64_t(t.n_ee) * e1 + uint64_t(t.n_fv) * f0;
		}
		const uint32_t nt = uint32_t(tasks.size());
		if (trace && nt > 0)
		{
			std::vector<uint32_t> ord(nt);
			std::iota(ord.begin(), ord.end(), 0u);
			std::partial_sort(ord.begin(), ord.begin() + std::min<uint32_t>(nt, 5), ord.end(), [&](uint32_t a, uint32_t b)
				{ return tasks[a].n_vf + tasks[a].n_ee + tasks[a].n_fv > tasks[b].n_vf + tasks[b].n_ee + tasks[b].n_fv; });
			for (uint32_t q = 0; q < std::min<uint32_t>(nt, 5); q++)
			{
				const Task& t = tasks[ord[q]];
				fprintf(stderr, "[u26 prp]   task contour %u dir %u k %u/%u requests vf %u ee %u fv %u cand faces %u/%u edges %u/%u\n", t.contour_local,
					t.combo, slots[t.slot0].k, slots[t.slot1].k, t.n_vf, t.n_ee, t.n_fv, counts[3 * t.slot0 + 2], counts[3 * t.slot1 + 2],
					counts[3 * t.slot0 + 1], counts[3 * t.slot1 + 1]);
			}
		}
		const int tb = bits_for(nt + 1);
		if (2 + 2 * b + tb > 64)
			return set_error(ctx, U26_ERR_CAPACITY, "PRP hit key needs %d bits", 2 + 2 * b + tb);
		U26_TRY(upload(ctx, S->d_tasks, tasks));
		proj_bounds_kernel<<<nt, 256, 0, st>>>(S->d_tasks.as<Task>(), nt, S->d_counts.as<uint32_t>(), S->d_cand_e.as<uint32_t>(), es_,
			S->d_edges.as<uint2>(), d_x);
		U26_TRY(after_launch(ctx, "proj_bounds_kernel"));
		uint32_t nh = 0;
		for (int attempt = 0; attempt < 8; attempt++)
		{
			U26_CUDA(ctx, S->d_keys.reserve(sizeof(uint64_t) * hit_cap));
			U26_CUDA(ctx, S->d_vals.reserve(sizeof(uint32_t) * hit_cap));
			U26_CUDA(ctx, S->d_pay_in.reserve(sizeof(float) * 3 * size_t(hit_cap)));
			U26_CUDA(ctx, S->d_hitcount.reserve(sizeof(uint32_t)));
			U26_CUDA(ctx, cudaMemsetAsync(S->d_hitcount.ptr, 0, sizeof(uint32_t), st));
			HitSink sink{ S->d_keys.as<uint64_t>(), S->d_vals.as<uint32_t>(), S->d_pay_in.as<float>(), S->d_hitcount.as<uint32_t>(), hit_cap, b };
			ev.mark(0, st);
			if (total_req && P->form == 1)
			{
				// plain form: one launch per contour (its tasks are contiguous)
				for (uint32_t q = 0; q < nt;)
				{
					uint32_t e = q;
					while (e < nt && tasks[e].contour_local == tasks[q].contour_local)
						e++;
					const uint32_t r0 = tasks[q].req_begin, r1 = e < nt ? tasks[e].req_begin : total_req;
					if (r1 > r0)
					{
						raycast_plain_kernel<<<div_up(r1 - r0, 128), 128, 0, st>>>(S->d_tasks.as<Task>(), q, e - q, r0, r1 - r0, S->d_slots.as<Slot>(),
							S->d_cand_v.as<uint32_t>(), S->d_cand_e.as<uint32_t>(), vs, es_, fs, S->d_bits_e.as<uint32_t>(),
							S->d_bits_f.as<uint32_t>(), ftv, etv, d_x, S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(), sink,
							(attempt == 0 && !hits_out) ? S->d_stats.as<unsigned long long>() : nullptr, ctx->dev_err);
						U26_TRY(after_launch(ctx, "raycast_plain_kernel"));
					}
					q = e;
				}
			}
			else if (total_req)
			{
				const bool rc = attempt == 0 && !hits_out && P->fp64_recheck;
				auto launch = [&](int cfg, unsigned long long* stats) -> u26_status
				{
					const RaycastConfig c = kRaycastConfigs[cfg];
					const uint64_t nthreads = uint64_t(div_up(total_req, 32u)) * 32u * c.split;
					uint64_t blocks = div_up64(nthreads, 128);
					if (c.queue)
					{
						// persistent grid: the blocks that fit on the GPU at once, items from a counter
						blocks = std::min<uint64_t>(blocks, uint64_t(S->num_sms) * uint64_t(c.min_blocks));
						U26_CUDA(ctx, cudaMemsetAsync(S->d_queue.ptr, 0, sizeof(uint32_t), st));
					}
					const RaycastFn kern = raycast_variant(rc, c.min_blocks, c.queue);
					kern<<<uint32_t(blocks), 128, 0, st>>>(S->d_tasks.as<Task>(), nt, total_req, S->d_slots.as<Slot>(),
						S->d_cand_v.as<uint32_t>(), S->d_cand_e.as<uint32_t>(), vs, es_, fs, S->d_bits_e.as<uint32_t>(),
						S->d_bits_f.as<uint32_t>(), S->d_fgrow.as<NodeBox>(), S->d_egrow.as<NodeBox>(), S->d_front.as<uint32_t>(),
						S->d_front.as<uint32_t>() + size_t(nobj) * kFrontStride, d_x, S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(),
						S->d_slot_box.as<float>(), sink, stats, c.split, S->d_queue.as<uint32_t>(), ctx->dev_err);
					return after_launch(ctx, "raycast_kernel");
				};
				if (tuning && attempt == 0 && !hits_out)
				{
					// autotuner: every configuration on this level's launch, timed with CUDA events;
					// each trial's hits are discarded (the counter is reset) and the launch below
					// produces the level's hits and statistics
					for (int cfg = 0; cfg < kNumRaycastConfigs; cfg++)
					{
						U26_CUDA(ctx, cudaMemsetAsync(S->d_hitcount.ptr, 0, sizeof(uint32_t), st));
						U26_CUDA(ctx, cudaEventRecord(tune_ev[2 * cfg], st));
						U26_TRY(launch(cfg, nullptr));
						U26_CUDA(ctx, cudaEventRecord(tune_ev[2 * cfg + 1], st));
					}
					U26_CUDA(ctx, cudaStreamSynchronize(st));
					for (int cfg = 0; cfg < kNumRaycastConfigs; cfg++)
					{
						float ms = 0.0f;
						U26_CUDA(ctx, cudaEventElapsedTime(&ms, tune_ev[2 * cfg], tune_ev[2 * cfg + 1]));
						out->tune_ms[cfg] += ms;
					}
					U26_CUDA(ctx, cudaMemsetAsync(S->d_hitcount.ptr, 0, sizeof(uint32_t), st));
				}
				U26_TRY(launch(cfg_now, (attempt == 0 && !hits_out) ? S->d_stats.as<unsigned long long>() : nullptr));
			}
			U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, S->d_hitcount.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
			U26_CUDA(ctx, cudaStreamSynchronize(st));
			nh = *ctx->host_word;
			if (nh <= hit_cap)
				break;
			hit_cap = uint32_t(std::min<uint64_t>(0xFFFFFFF0ull, std::max<uint64_t>(uint64_t(hit_cap) * 2, uint64_t(nh) + nh / 2)));
			S->hit_cap = hit_cap;
			if (attempt == 7)
				return set_error(ctx, U26_ERR_CAPACITY, "PRP hit capacity");
		}
		out->stage_ms[3] += ms_since(tl);
		tl = std::chrono::steady_clock::now();
		ev.mark(1, st);
		U26_TRY(S->sorter.sort(ctx, S->d_keys.as<uint64_t>(), S->d_vals.as<uint32_t>(), nh, 0, 2 + 2 * b + tb));
		ev.mark(2, st);
		const HitKeyCodec cd{ b };
		U26_CUDA(ctx, S->d_seg.reserve(sizeof(uint32_t) * (nt + 1)));
		segments_kernel<<<div_up(nt + 1, 256), 256, 0, st>>>(S->d_keys.as<uint64_t>(), nh, cd, nt, S->d_seg.as<uint32_t>());
		U26_TRY(after_launch(ctx, "segments_kernel"));
		const uint32_t nh1 = std::max(nh, 1u);
		U26_CUDA(ctx, S->d_pay.reserve(sizeof(float) * 3 * size_t(nh1)));
		U26_CUDA(ctx, S->d_parent.reserve(sizeof(uint32_t) * nh1));
		U26_CUDA(ctx, S->d_root.reserve(sizeof(uint32_t) * nh1));
		U26_CUDA(ctx, S->d_att.reserve(nh1));
		U26_CUDA(ctx, S->d_csize.reserve(sizeof(uint32_t) * nh1));
		U26_CUDA(ctx, S->d_catt.reserve(sizeof(uint32_t) * nh1));
		U26_CUDA(ctx, S->d_cand_roots.reserve(sizeof(uint32_t) * nh1));
		if (nh)
		{
			init_hits_kernel<<<div_up(nh, 256), 256, 0, st>>>(S->d_keys.as<uint64_t>(), S->d_vals.as<uint32_t>(), S->d_pay_in.as<float>(),
				S->d_pay.as<float>(), nh, cd, S->d_tasks.as<Task>(), S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(),
				S->d_vf_off.as<uint32_t>(), S->d_vf.as<uint32_t>(), S->d_parent.as<uint32_t>(), S->d_att.as<uint8_t>(),
				S->d_csize.as<uint32_t>(), S->d_catt.as<uint32_t>());
			U26_TRY(after_launch(ctx, "init_hits_kernel"));
			// run directory of this level's hits
			U26_CUDA(ctx, S->d_rflag.reserve(sizeof(uint32_t) * (size_t(nh) + 1)));
			run_flags_kernel<<<div_up(nh + 1, 256), 256, 0, st>>>(S->d_keys.as<uint64_t>(), nh, b, S->d_rflag.as<uint32_t>());
			U26_TRY(after_launch(ctx, "run_flags_kernel"));
			U26_TRY(device_exclusive_scan(ctx, S->d_rflag.as<uint32_t>(), nh + 1, S->scan_tmp));
			U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, S->d_rflag.as<uint32_t>() + nh, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
			U26_CUDA(ctx, cudaStreamSynchronize(st));
			const uint32_t nruns = *ctx->host_word;
			uint32_t hsize = 1024;
			while (hsize < 2 * nruns)
				hsize <<= 1;
			U26_CUDA(ctx, S->d_heads.reserve(sizeof(uint32_t) * (size_t(nruns) + 1)));
			U26_CUDA(ctx, S->d_hkeys.reserve(sizeof(uint64_t) * hsize));
			U26_CUDA(ctx, S->d_hvals.reserve(sizeof(uint32_t) * hsize));
			U26_CUDA(ctx, cudaMemsetAsync(S->d_hkeys.ptr, 0, sizeof(uint64_t) * hsize, st));
			run_insert_kernel<<<div_up(nh + 1, 256), 256, 0, st>>>(S->d_keys.as<uint64_t>(), nh, b, S->d_rflag.as<uint32_t>(),
				S->d_heads.as<uint32_t>(), S->d_hkeys.as<uint64_t>(), S->d_hvals.as<uint32_t>(), hsize - 1, ctx->dev_err);
			U26_TRY(after_launch(ctx, "run_insert_kernel"));
			const RunDir rdir{ S->d_hkeys.as<uint64_t>(), S->d_hvals.as<uint32_t>(), S->d_heads.as<uint32_t>(), hsize - 1 };
			union_kernel<<<div_up(nh, 128), 128, 0, st>>>(S->d_keys.as<uint64_t>(), nh, cd, S->d_seg.as<uint32_t>(), S->d_edges.as<uint2>(),
				S->d_faces.as<uint32_t>(), S->d_fae.as<uint32_t>(), S->d_vav_off.as<uint32_t>(), S->d_vav.as<uint32_t>(),
				S->d_vae_off.as<uint32_t>(), S->d_vae.as<uint32_t>(), S->d_vaf_off.as<uint32_t>(), S->d_vaf.as<uint32_t>(),
				S->d_eaf_off.as<uint32_t>(), S->d_eaf.as<uint32_t>(), S->d_eae_off.as<uint32_t>(), S->d_eae.as<uint32_t>(),
				rdir, S->d_parent.as<uint32_t>(), ctx->dev_err);
			U26_TRY(after_launch(ctx, "union_kernel"));
			if (P->solid_interior && (P->solid_all || S->any_solid))
			{
				const SolidParams sp{ S->d_fn.as<float>(), S->d_en.as<float>(), S->d_vobj.as<uint32_t>(), S->d_vsolid.as<uint8_t>(), P->solid_all,
					P->solid_eps_n, P->solid_eps_d };
				solid_runs_kernel<<<div_up(nh, 128), 128, 0, st>>>(S->d_keys.as<uint64_t>(), nh, cd, S->d_seg.as<uint32_t>(), S->d_pay.as<float>(),
					S->d_tasks.as<Task>(), S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(), sp, S->d_parent.as<uint32_t>(), ctx->dev_err);
				U26_TRY(after_launch(ctx, "solid_runs_kernel"));
				U26_CUDA(ctx, S->d_fvk.reserve(sizeof(uint64_t) * nh));
				U26_CUDA(ctx, S->d_fvv.reserve(sizeof(uint32_t) * nh));
				U26_CUDA(ctx, S->d_ecount.reserve(sizeof(uint32_t)));
				U26_CUDA(ctx, cudaMemsetAsync(S->d_ecount.ptr, 0, sizeof(uint32_t), st));
				solid_fv_keys_kernel<<<div_up(nh, 256), 256, 0, st>>>(S->d_keys.as<uint64_t>(), nh, cd, S->d_fvk.as<uint64_t>(),
					S->d_fvv.as<uint32_t>(), S->d_ecount.as<uint32_t>());
				U26_TRY(after_launch(ctx, "solid_fv_keys_kernel"));
				U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, S->d_ecount.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
				U26_CUDA(ctx, cudaStreamSynchronize(st));
				const uint32_t nfv = *ctx->host_word;
				if (nfv > 1)
				{
					U26_TRY(S->fvsorter.sort(ctx, S->d_fvk.as<uint64_t>(), S->d_fvv.as<uint32_t>(), nfv, 0, b + tb));
					solid_fv_kernel<<<div_up(nfv, 128), 128, 0, st>>>(S->d_fvk.as<uint64_t>(), S->d_fvv.as<uint32_t>(), nfv, S->d_keys.as<uint64_t>(), cd,
						S->d_pay.as<float>(), S->d_tasks.as<Task>(), S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(), sp, S->d_parent.as<uint32_t>(),
						ctx->dev_err);
					U26_TRY(after_launch(ctx, "solid_fv_kernel"));
				}
			}
			compress_kernel<<<div_up(nh, 256), 256, 0, st>>>(S->d_parent.as<uint32_t>(), nh, S->d_att.as<uint8_t>(), S->d_csize.as<uint32_t>(),
				S->d_catt.as<uint32_t>(), S->d_root.as<uint32_t>());
			U26_TRY(after_launch(ctx, "compress_kernel"));
		}
		ev.mark(3, st);
		std::vector<uint32_t> seg_h;
		U26_TRY(download(ctx, seg_h, S->d_seg.ptr, nt + 1));
		U26_CUDA(ctx, cudaStreamSynchronize(st));
		uint32_t max_seg = 1;
		for (uint32_t t = 0; t < nt; t++)
			max_seg = std::max(max_seg, seg_h[t + 1] - seg_h[t]);
		const int rb = bits_for(max_seg + 1);
		const int vb = bits_for(std::max(S->nv, 2u));
		if (tb + 1 + vb + rb > 64)
			return set_error(ctx, U26_ERR_CAPACITY, "PRP support key needs %d bits", tb + 1 + vb + rb);
		U26_CUDA(ctx, S->d_ecount.reserve(sizeof(uint32_t)));
		U26_CUDA(ctx, S->d_ncand.reserve(sizeof(uint32_t) * 3 * (nt + 1)));
		U26_CUDA(ctx, cudaMemsetAsync(S->d_ncand.ptr, 0, sizeof(uint32_t) * 3 * (nt + 1), st));
		uint32_t* d_ncand = S->d_ncand.as<uint32_t>();
		uint32_t ne_entries = 0;
		if (nh)
		{
			cand_roots_kernel<<<div_up(nh, 256), 256, 0, st>>>(S->d_keys.as<uint64_t>(), nh, cd, S->d_seg.as<uint32_t>(), S->d_root.as<uint32_t>(),
				S->d_catt.as<uint32_t>(), d_ncand, S->d_cand_roots.as<uint32_t>());
			U26_TRY(after_launch(ctx, "cand_roots_kernel"));
			// support entries, with a capacity kept across levels (re-run once on overflow)
			uint32_t ecap = std::max<uint32_t>(S->e_cap, 1u << 20);
			for (int attempt = 0; attempt < 4; attempt++)
			{
				U26_CUDA(ctx, S->d_ekeys.reserve(sizeof(uint64_t) * size_t(ecap)));
				U26_CUDA(ctx, S->d_evals.reserve(sizeof(uint32_t) * size_t(ecap)));
				U26_CUDA(ctx, cudaMemsetAsync(S->d_ecount.ptr, 0, sizeof(uint32_t), st));
				entries_kernel<<<div_up(nh, 256), 256, 0, st>>>(S->d_keys.as<uint64_t>(), nh, cd, S->d_seg.as<uint32_t>(), S->d_root.as<uint32_t>(),
					S->d_catt.as<uint32_t>(), S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(), vb, rb, S->d_ekeys.as<uint64_t>(),
					S->d_evals.as<uint32_t>(), S->d_ecount.as<uint32_t>(), ecap, S->d_tasks.as<Task>(), S->d_slots.as<Slot>(),
					S->d_bnd_bits.as<uint32_t>(), vs);
				U26_TRY(after_launch(ctx, "entries_kernel"));
				U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, S->d_ecount.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
				U26_CUDA(ctx, cudaStreamSynchronize(st));
				ne_entries = *ctx->host_word;
				if (ne_entries <= ecap)
					break;
				ecap = uint32_t(std::min<uint64_t>(0xFFFFFFF0ull, uint64_t(ne_entries) + ne_entries / 2));
				S->e_cap = ecap;
				if (attempt == 3)
					return set_error(ctx, U26_ERR_CAPACITY, "PRP support entry capacity");
			}
			U26_TRY(S->esorter.sort(ctx, S->d_ekeys.as<uint64_t>(), S->d_evals.as<uint32_t>(), ne_entries, 0, tb + 1 + vb + rb));
		}
		ev.mark(4, st);
		// best component per task, selected-hit scan, metric terms, canonical sums
		U26_CUDA(ctx, S->d_best.reserve(sizeof(uint32_t) * 2 * (nt + 1)));
		uint32_t* d_best = S->d_best.as<uint32_t>();
		uint32_t* d_bestcov = d_best + (nt + 1);
		{
			// coverage per anchor, then the best component per task
			std::vector<uint32_t> tab(nt + 1, 0u);
			for (uint32_t q = 0; q < nt; q++)
				tab[q + 1] = tab[q] + (anchor_off[tasks[q].contour_local + 1] - anchor_off[tasks[q].contour_local]);
			U26_TRY(upload(ctx, S->d_tab, tab));
			U26_CUDA(ctx, S->d_cov.reserve(sizeof(uint32_t) * std::max(nh, 1u)));
			U26_CUDA(ctx, cudaMemsetAsync(S->d_cov.ptr, 0, sizeof(uint32_t) * std::max(nh, 1u), st));
			if (tab[nt] && ne_entries)
			{
				U26_CUDA(ctx, S->d_trange.reserve(sizeof(uint32_t) * 2 * size_t(nt)));
				U26_CUDA(ctx, cudaMemsetAsync(S->d_trange.ptr, 0, sizeof(uint32_t) * 2 * size_t(nt), st));
				uint32_t* tbeg = S->d_trange.as<uint32_t>();
				entry_ranges_kernel<<<div_up(ne_entries, 256), 256, 0, st>>>(S->d_ekeys.as<uint64_t>(), ne_entries, 1 + vb + rb, tbeg, tbeg + nt);
				U26_TRY(after_launch(ctx, "entry_ranges_kernel"));
				coverage_count_kernel<<<div_up(tab[nt], 256), 256, 0, st>>>(S->d_tasks.as<Task>(), nt, S->d_tab.as<uint32_t>(),
					S->d_anchor_off.as<uint32_t>(), S->d_anchors.as<uint32_t>(), S->d_ekeys.as<uint64_t>(), ne_entries, tbeg, tbeg + nt, vb, rb,
					S->d_seg.as<uint32_t>(), S->d_cov.as<uint32_t>());
				U26_TRY(after_launch(ctx, "coverage_count_kernel"));
			}
			best_component_kernel<<<div_up(32 * nt, 256), 256, 0, st>>>(nt, S->d_seg.as<uint32_t>(), d_ncand, S->d_cand_roots.as<uint32_t>(),
				S->d_csize.as<uint32_t>(), S->d_cov.as<uint32_t>(), d_best, d_bestcov);
			U26_TRY(after_launch(ctx, "best_component_kernel"));
		}
		const uint32_t nblk = div_up(nh1, 1024);
		U26_CUDA(ctx, S->d_bsum.reserve(sizeof(uint32_t) * (nblk + 2)));
		U26_CUDA(ctx, S->d_task_max.reserve(sizeof(uint32_t) * 3 * (nt + 1)));
		U26_CUDA(ctx, cudaMemsetAsync(S->d_task_max.ptr, 0, sizeof(uint32_t) * 3 * (nt + 1), st));
		U26_CUDA(ctx, S->d_selbegin.reserve(sizeof(uint32_t) * (nt + 1)));
		uint32_t nsel = 0;
		if (nh)
		{
			sel_block_sums_kernel<<<nblk, 256, 0, st>>>(S->d_keys.as<uint64_t>(), S->d_root.as<uint32_t>(), d_best, cd, nh, S->d_bsum.as<uint32_t>());
			U26_TRY(after_launch(ctx, "sel_block_sums_kernel"));
			scan_one_block_kernel<<<1, 1024, 0, st>>>(S->d_bsum.as<uint32_t>(), nblk, S->d_bsum.as<uint32_t>() + nblk + 1);
			U26_TRY(after_launch(ctx, "scan_one_block_kernel"));
			U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, S->d_bsum.as<uint32_t>() + nblk + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
			U26_CUDA(ctx, cudaStreamSynchronize(st));
			nsel = *ctx->host_word;
			U26_CUDA(ctx, S->d_pos.reserve(sizeof(uint32_t) * nh1));
			U26_CUDA(ctx, S->d_terms.reserve(sizeof(float) * 3 * size_t(std::max(nsel, 1u))));
			if (hits_out)
				U26_CUDA(ctx, S->d_sel.reserve(sizeof(u26_prp_hit) * size_t(std::max(nsel, 1u))));
			sel_terms_kernel<<<nblk, 256, 0, st>>>(S->d_keys.as<uint64_t>(), S->d_root.as<uint32_t>(), d_best, cd, nh, S->d_bsum.as<uint32_t>(),
				S->d_tasks.as<Task>(), S->d_pay.as<float>(), S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(), S->d_varea.as<float>(),
				S->d_earea.as<float>(), S->d_farea.as<float>(), S->d_vmass.as<float>(), S->d_vn.as<float>(), S->d_en.as<float>(),
				S->d_fn.as<float>(), S->d_slots.as<Slot>(), S->d_hop.as<uint32_t>(), vs, S->d_pos.as<uint32_t>(), S->d_terms.as<float>(),
				S->d_task_max.as<uint32_t>(), hits_out ? S->d_sel.as<u26_prp_hit>() : nullptr);
			U26_TRY(after_launch(ctx, "sel_terms_kernel"));
			sel_begin_kernel<<<div_up(nt, 256), 256, 0, st>>>(nt, S->d_seg.as<uint32_t>(), S->d_bsum.as<uint32_t>(), S->d_keys.as<uint64_t>(),
				S->d_root.as<uint32_t>(), d_best, cd, nh, S->d_selbegin.as<uint32_t>());
			U26_TRY(after_launch(ctx, "sel_begin_kernel"));
		}
		else
			U26_CUDA(ctx, cudaMemsetAsync(S->d_selbegin.ptr, 0, sizeof(uint32_t) * (nt + 1), st));
		U26_CUDA(ctx, S->d_out.reserve(sizeof(TaskOut) * nt));
		// chunk sums of the supports longer than kSumChunk
		U26_CUDA(ctx, S->d_chunk_off.reserve(sizeof(uint32_t) * (nt + 1)));
		chunk_count_kernel<<<div_up(nt + 1, 256), 256, 0, st>>>(nt, d_best, S->d_csize.as<uint32_t>(), S->d_chunk_off.as<uint32_t>());
		U26_TRY(after_launch(ctx, "chunk_count_kernel"));
		U26_TRY(device_exclusive_scan(ctx, S->d_chunk_off.as<uint32_t>(), nt + 1, S->scan_tmp));
		U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, S->d_chunk_off.as<uint32_t>() + nt, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
		U26_CUDA(ctx, cudaStreamSynchronize(st));
		const uint32_t nchunks = *ctx->host_word;
		U26_CUDA(ctx, S->d_csum.reserve(sizeof(float) * 3 * size_t(std::max(nchunks, 1u))));
		if (nchunks)
		{
			chunk_sum_kernel<<<div_up(32 * nchunks, 256), 256, 0, st>>>(nt, nchunks, S->d_chunk_off.as<uint32_t>(), d_best,
				S->d_csize.as<uint32_t>(), S->d_selbegin.as<uint32_t>(), S->d_terms.as<float>(), S->d_csum.as<float>());
			U26_TRY(after_launch(ctx, "chunk_sum_kernel"));
		}
		task_sum_kernel<<<div_up(32 * nt, 256), 256, 0, st>>>(nt, S->d_tasks.as<Task>(), S->d_seg.as<uint32_t>(), d_best, d_bestcov,
			S->d_csize.as<uint32_t>(), d_ncand, S->d_selbegin.as<uint32_t>(), S->d_terms.as<float>(), S->d_task_max.as<uint32_t>(),
			S->d_anchor_off.as<uint32_t>(), S->d_chunk_off.as<uint32_t>(), S->d_csum.as<float>(), S->d_out.as<TaskOut>());
		U26_TRY(after_launch(ctx, "task_sum_kernel"));
		ev.mark(5, st);
		U26_TRY(download(ctx, tout, S->d_out.ptr, nt));
		if (hits_out)
			U26_TRY(download(ctx, *hits_out, S->d_sel.ptr, nsel));
		ev.mark(6, st);
		U26_CUDA(ctx, cudaStreamSynchronize(st));
		if (trace)
			fprintf(stderr, "[u26 prp] %s tasks %u requests %u hits %u entries %u selected %u | raycast %.2f sort %.2f union %.2f entries %.2f select %.2f download %.2f ms\n",
				hits_out ? "materialize" : "level", nt, total_req, nh, ne_entries, nsel, ev.ms(0, 1), ev.ms(1, 2), ev.ms(2, 3), ev.ms(3, 4), ev.ms(4, 5),
				ev.ms(5, 6));
		for (int q = 0; q < 6; q++)
			out->gpu_ms[q] += ev.ms(q, q + 1);
		out->stage_ms[4] += ms_since(tl);
		return U26_OK;
	};

	// prp_select_response over a contour's results
	auto select_best = [&](const ContourRT& r) -> int
	{
		int sel = -1;
		for (size_t d = 0; d < r.res.size(); d++)
		{
			if (!valid_resp(r.res[d]))
				continue;
			if (sel < 0 || better_resp(r.res[d], uint32_t(d), r.res[sel], uint32_t(sel)))
				sel = int(d);
		}
		return sel;
	};
	// evaluate_current_runtime_directions_template for the listed contours: k from the
	// initial level, the active directions reset, levels until every active direction has
	// converged or been pruned
	auto run_levels = [&](std::vector<uint32_t> remaining) -> u26_status
	{
		for (uint32_t c : remaining)
		{
			ContourRT& r = R[c];
			r.k[0] = r.k0[0];
			r.k[1] = r.k0[1];
			r.finished = false;
			r.no_resp = false;
			for (size_t d = 0; d < r.dirs.size(); d++)
				if (r.active[d])
				{
					r.conv[d] = 0;
					r.pruned[d] = 0;
					r.present[d] = 0;
					r.res[d] = ComboState{};
				}
		}
		uint32_t level = 0;
		uint64_t captured = 0; // support hits gathered at this level (trace)
		for (; !remaining.empty() && level < 65; level++)
		{
			auto tl = std::chrono::steady_clock::now();
			std::vector<uint32_t> sids;
			for (uint32_t c : remaining)
				for (int sd = 0; sd < 2; sd++)
				{
					slots[2 * c + sd].k = R[c].k[sd];
					sids.push_back(2 * c + sd);
				}
			std::vector<uint32_t> counts;
			U26_TRY(build_candidates(sids, counts));
			if (trace)
				fprintf(stderr, "[u26 prp]   level candidates %.2f ms (%zu slots)\n", ms_since(tl), sids.size());
			out->stage_ms[2] += ms_since(tl);
			std::vector<Task> tasks;
			for (uint32_t c : remaining)
			{
				const ContourRT& r = R[c];
				for (uint32_t d = 0; d < r.dirs.size(); d++)
				{
					if (!r.active[d] || r.conv[d] || r.pruned[d])
						continue;
					Task t{};
					t.slot0 = 2 * c;
					t.slot1 = 2 * c + 1;
					t.contour_local = c;
					t.contour_global = c;
					t.combo = d;
					t.dir[0] = r.dirs[d].x;
					t.dir[1] = r.dirs[d].y;
					t.dir[2] = r.dirs[d].z;
					tasks.push_back(t);
				}
			}
			if (tasks.empty())
				break;
			std::vector<TaskOut> tout;
			U26_TRY(evaluate(tasks, counts, tout, nullptr));
			tl = std::chrono::steady_clock::now();
			// ---- k-ring control (evaluate_current_runtime_directions_template)
			for (size_t t = 0; t < tasks.size(); t++)
			{
				const Task& tk = tasks[t];
				ContourRT& r = R[tk.contour_local];
				const TaskOut& o = tout[t];
				ComboState cs;
				cs.present = true;
				cs.levels = level + 1;
				cs.eval_k_src = r.k[0];
				cs.eval_k_dst = r.k[1];
				cs.unculled = o.unculled;
				cs.anchors = o.anchors;
				if (o.best_root != kInfH)
				{
					cs.hit_count = o.hit_count;
					cs.covered = o.covered;
					cs.depth = o.depth;
					cs.volume = o.volume;
					cs.area = o.area;
					cs.cost = o.kappa;
					cs.objective = (o.area * o.depth) * o.depth;
					cs.coverage = o.anchors > 0 ? float(o.covered) / float(o.anchors) : 0.0f;
					cs.mfs = o.max_front_src;
					cs.mfd = o.max_front_dst;
				}
				cs.full_mesh = r.k[0] >= r.diam[0] && r.k[1] >= r.diam[1];
				const bool src_ok = cs.mfs < r.k[0] || r.k[0] >= r.diam[0];
				const bool dst_ok = cs.mfd < r.k[1] || r.k[1] >= r.diam[1];
				cs.eligible = usable(cs) && src_ok && dst_ok;
				r.conv[tk.combo] = (cs.eligible || cs.full_mesh) ? 1 : 0;
				r.present[tk.combo] = 1;
				r.res[tk.combo] = std::move(cs);
			}
			// the support of each contour's current best response, when this level produced it,
			// is gathered now while the level's hits are on the device, so that the final
			// winner needs no re-evaluation (materialize covers whatever is not captured)
			{
				constexpr uint64_t kCaptureCap = uint64_t(1) << 24;
				captured = 0;
				std::vector<int> task_of(size_t(nact) * 26, -1);
				for (size_t t = 0; t < tasks.size(); t++)
					if (tasks[t].combo < 26)
						task_of[size_t(tasks[t].contour_local) * 26 + tasks[t].combo] = int(t);
				std::vector<uint32_t> list, off(1, 0u);
				uint64_t total = 0;
				for (uint32_t c : remaining)
				{
					const int sel = select_best(R[c]);
					if (sel < 0 || sel >= 26)
						continue;
					const int t = task_of[size_t(c) * 26 + sel];
					const ComboState& cs = R[c].res[sel];
					if (t < 0 || cs.hits.size() == cs.hit_count || cs.in_store() || total + cs.hit_count > kCaptureCap)
						continue;
					list.push_back(uint32_t(t));
					total += cs.hit_count;
					off.push_back(uint32_t(total));
				}
				if (!list.empty() && total > 0)
				{
					// gathered into the pass's support store on the device; the winners' supports
					// are fetched once, after the levels (fetch_supports)
					U26_TRY(upload(ctx, S->d_cap_list, list));
					U26_TRY(upload(ctx, S->d_cap_off, off));
					const size_t need = sizeof(u26_prp_hit) * (S->store_used + total);
					if (need > S->d_store.bytes)
					{
						DevBuf grown;
						U26_CUDA(ctx, grown.reserve(need + need / 2));
						if (S->store_used)
							U26_CUDA(ctx, cudaMemcpyAsync(grown.ptr, S->d_store.ptr, sizeof(u26_prp_hit) * S->store_used, cudaMemcpyDeviceToDevice, st));
						std::swap(grown.ptr, S->d_store.ptr);
						std::swap(grown.bytes, S->d_store.bytes);
						grown.release(); // after the copy: cudaFree waits for the device
					}
					capture_kernel<<<uint32_t(list.size()), 256, 0, st>>>(S->d_cap_list.as<uint32_t>(), S->d_cap_off.as<uint32_t>(),
						S->d_keys.as<uint64_t>(), S->d_root.as<uint32_t>(), S->d_best.as<uint32_t>(), S->d_seg.as<uint32_t>(), S->d_pay.as<float>(),
						HitKeyCodec{ b }, S->d_edges.as<uint2>(), S->d_faces.as<uint32_t>(), S->d_store.as<u26_prp_hit>() + S->store_used);
					U26_TRY(after_launch(ctx, "capture_kernel"));
					for (size_t q = 0; q < list.size(); q++)
						R[tasks[list[q]].contour_local].res[tasks[list[q]].combo].store_off = S->store_used + off[q];
					S->store_used += total;
					captured = total;
				}
			}
			std::vector<uint32_t> next;
			for (uint32_t c : remaining)
			{
				ContourRT& r = R[c];
				r.levels = level + 1;
				bool has = false;
				float best = std::numeric_limits<float>::infinity();
				for (size_t d = 0; d < r.dirs.size(); d++)
					if (r.active[d] && valid_resp(r.res[d]))
					{
						has = true;
						best = std::fmin(best, resp_obj(r.res[d]));
					}
				if (has)
					for (size_t d = 0; d < r.dirs.size(); d++)
						if (r.active[d] && !r.conv[d] && r.present[d] && resp_obj(r.res[d]) >= best)
							r.pruned[d] = 1;
				bool pending = false, gs = false, gd = false;
				for (size_t d = 0; d < r.dirs.size(); d++)
				{
					if (!r.active[d] || r.conv[d] || r.pruned[d])
						continue;
					pending = true;
					const ComboState& cs = r.res[d];
					gs = gs || (r.k[0] < r.diam[0] && (!usable(cs) || cs.mfs >= r.k[0]));
					gd = gd || (r.k[1] < r.diam[1] && (!usable(cs) || cs.mfd >= r.k[1]));
				}
				if (!pending)
				{
					r.finished = true;
					r.no_resp = !has;
					continue;
				}
				const uint32_t ns = gs ? grow(r.k[0], r.diam[0]) : r.k[0];
				const uint32_t nd = gd ? grow(r.k[1], r.diam[1]) : r.k[1];
				if (ns <= r.k[0] && nd <= r.k[1])
				{
					r.finished = true;
					continue;
				}
				r.k[0] = ns;
				r.k[1] = nd;
				next.push_back(c);
			}
			remaining.swap(next);
			if (trace)
				fprintf(stderr, "[u26 prp]   level control %.2f ms (captured %llu support hits)\n", ms_since(tl), (unsigned long long)captured);
			out->stage_ms[5] += ms_since(tl);
		}
		out->levels = std::max(out->levels, level);
		return U26_OK;
	};
	{
		std::vector<uint32_t> all(nact);
		std::iota(all.begin(), all.end(), 0u);
		mark("distances, uploads, trees");
		U26_TRY(run_levels(all));
		mark("k-ring levels");
	}
	// ---- materialize: re-evaluate the listed (contour, direction) results once more with
	// the supports gathered (the evaluation is deterministic, so these are the hits the
	// stored metrics were computed on)
	auto materialize = [&](const std::vector<std::pair<uint32_t, uint32_t>>& cc) -> u26_status
	{
		if (cc.empty())
			return U26_OK;
		auto tl = std::chrono::steady_clock::now();
		std::vector<uint32_t> sids;
		std::vector<Task> tasks;
		for (const auto& [c, d] : cc)
		{
			const ContourRT& r = R[c];
			slots[2 * c].k = r.res[d].eval_k_src;
			slots[2 * c + 1].k = r.res[d].eval_k_dst;
			sids.push_back(2 * c);
			sids.push_back(2 * c + 1);
			Task t{};
			t.slot0 = 2 * c;
			t.slot1 = 2 * c + 1;
			t.contour_local = c;
			t.contour_global = c;
			t.combo = d;
			t.dir[0] = r.dirs[d].x;
			t.dir[1] = r.dirs[d].y;
			t.dir[2] = r.dirs[d].z;
			tasks.push_back(t);
		}
		std::vector<uint32_t> counts;
		U26_TRY(build_candidates(sids, counts));
		std::vector<TaskOut> tout;
		std::vector<u26_prp_hit> hits;
		U26_TRY(evaluate(tasks, counts, tout, &hits));
		for (size_t t = 0; t < tasks.size(); t++)
		{
			ComboState& cs = R[tasks[t].contour_local].res[tasks[t].combo];
			const TaskOut& o = tout[t];
			if (o.hit_count != cs.hit_count || o.area != cs.area || o.depth != cs.depth || o.covered != cs.covered)
				return set_error(ctx, U26_ERR_INVALID_INPUT, "PRP re-evaluation of contour %u direction %u differs", tasks[t].contour_local,
					tasks[t].combo);
			cs.hits.assign(hits.begin() + o.sel_offset, hits.begin() + o.sel_offset + o.hit_count);
		}
		out->stage_ms[6] += ms_since(tl);
		return U26_OK;
	};
	// the supports of the listed results that the levels captured on the device, fetched into
	// their hit lists with one gather and one copy back; the rest are left to materialize
	auto fetch_supports = [&](const std::vector<std::pair<uint32_t, uint32_t>>& cc) -> u26_status
	{
		std::vector<uint64_t> offs;
		std::vector<uint32_t> cnts, poss;
		std::vector<ComboState*> dst;
		uint64_t total = 0;
		for (const auto& [c, d] : cc)
		{
			ComboState& cs = R[c].res[d];
			if (!cs.in_store() || cs.hit_count == 0 || cs.hits.size() == cs.hit_count)
				continue;
			offs.push_back(cs.store_off);
			cnts.push_back(cs.hit_count);
			poss.push_back(uint32_t(total));
			total += cs.hit_count;
			dst.push_back(&cs);
		}
		if (dst.empty())
			return U26_OK;
		if (total > 0xFFFFFFFFull)
			return set_error(ctx, U26_ERR_CAPACITY, "PRP support fetch of %llu hits", (unsigned long long)total);
		U26_TRY(upload(ctx, S->d_fetch_off, offs));
		U26_TRY(upload(ctx, S->d_fetch_cnt, cnts));
		U26_TRY(upload(ctx, S->d_fetch_pos, poss));
		const size_t bytes = sizeof(u26_prp_hit) * total;
		U26_CUDA(ctx, S->d_capture.reserve(bytes));
		support_gather_kernel<<<uint32_t(dst.size()), 256, 0, st>>>(S->d_store.as<u26_prp_hit>(), S->d_fetch_off.as<uint64_t>(),
			S->d_fetch_cnt.as<uint32_t>(), S->d_fetch_pos.as<uint32_t>(), S->d_capture.as<u26_prp_hit>());
		U26_TRY(after_launch(ctx, "support_gather_kernel"));
		if (S->cap_host_bytes < bytes)
		{
			if (S->cap_host)
				cudaFreeHost(S->cap_host);
			S->cap_host = nullptr;
			S->cap_host_bytes = 0;
			U26_CUDA(ctx, cudaMallocHost(&S->cap_host, bytes + bytes / 2));
			g_alloc_count.fetch_add(1, std::memory_order_relaxed);
			S->cap_host_bytes = bytes + bytes / 2;
		}
		U26_CUDA(ctx, cudaMemcpyAsync(S->cap_host, S->d_capture.ptr, bytes, cudaMemcpyDeviceToHost, st));
		U26_CUDA(ctx, cudaStreamSynchronize(st));
		const u26_prp_hit* got = static_cast<const u26_prp_hit*>(S->cap_host);
		host_parallel_dynamic(uint32_t(dst.size()), [&](uint32_t q)
			{ dst[q]->hits.assign(got + poss[q], got + poss[q] + cnts[q]); });
		return U26_OK;
	};
	auto fetch_then_materialize = [&](const std::vector<std::pair<uint32_t, uint32_t>>& cc) -> u26_status
	{
		U26_TRY(fetch_supports(cc));
		std::vector<std::pair<uint32_t, uint32_t>> rest;
		for (const auto& e : cc)
		{
			const ComboState& cs = R[e.first].res[e.second];
			if (cs.hits.size() != cs.hit_count)
				rest.push_back(e);
		}
		return materialize(rest);
	};
	std::vector<int> chosen_idx(nc, -1);
	{
		std::vector<std::pair<uint32_t, uint32_t>> cc;
		for (uint32_t c = 0; c < nact; c++)
		{
			chosen_idx[c] = select_best(R[c]);
			if (chosen_idx[c] >= 0 && R[c].res[chosen_idx[c]].hits.size() != R[c].res[chosen_idx[c]].hit_count)
				cc.emplace_back(c, uint32_t(chosen_idx[c]));
		}
		U26_TRY(fetch_then_materialize(cc));
	}

	mark("materialize");
	// ---- S^2 direction refinement (prp_optimize_runtime_directions,
	// intersection_resolver2.cpp:1371-1486): per iteration, the steps of all open contours
	// in one launch, then every trial direction evaluated from the initial k-ring level in
	// the batched levels, accepted only when strictly better (trust radius x2 / x0.5)
	if (P->opt_iterations > 0 && nact > 0)
	{
		struct OptState
		{
			int combo = -1;
			uint32_t attempted = 0, accepted = 0;
			float trust = 0.3f;
			bool done = false;
		};
		std::vector<OptState> os(nact);
		for (uint32_t c = 0; c < nact; c++)
		{
			if (chosen_idx[c] < 0 || R[c].res[chosen_idx[c]].hits.empty())
				os[c].done = true;
			else
				os[c].combo = chosen_idx[c];
		}
		std::vector<ComboState> acc(nact);
		std::vector<V3h> acc_dir(nact);
		std::vector<float> pred(nact, 0.0f), gn(nact, 0.0f);
		for (uint32_t it = 0; it < P->opt_iterations; it++)
		{
			std::vector<uint32_t> open;
			std::vector<StepIn> sin;
			std::vector<u26_prp_hit> shits;
			for (uint32_t c = 0; c < nact; c++)
			{
				if (os[c].done)
					continue;
				const ContourRT& r = R[c];
				const ComboState& a = r.res[os[c].combo];
				StepIn si{};
				si.dir[0] = r.dirs[os[c].combo].x;
				si.dir[1] = r.dirs[os[c].combo].y;
				si.dir[2] = r.dirs[os[c].combo].z;
				si.trust = os[c].trust;
				si.hit_begin = uint32_t(shits.size());
				si.hit_count = uint32_t(a.hits.size());
				shits.insert(shits.end(), a.hits.begin(), a.hits.end());
				open.push_back(c);
				sin.push_back(si);
			}
			if (open.empty())
				break;
			const uint32_t no = uint32_t(open.size());
			U26_TRY(upload(ctx, S->d_step_in, sin));
			U26_TRY(upload(ctx, S->d_step_hits, shits));
			U26_CUDA(ctx, S->d_step_out.reserve(sizeof(StepOut) * no));
			dir_step_kernel<<<div_up(32 * no, 256), 256, 0, st>>>(no, S->d_step_in.as<StepIn>(), S->d_step_hits.as<u26_prp_hit>(), d_x,
				S->d_vmass.as<float>(), S->d_step_out.as<StepOut>());
			U26_TRY(after_launch(ctx, "dir_step_kernel"));
			std::vector<StepOut> so;
			U26_TRY(download(ctx, so, S->d_step_out.ptr, no));
			U26_CUDA(ctx, cudaStreamSynchronize(st));
			std::vector<uint32_t> trials;
			for (uint32_t i = 0; i < no; i++)
			{
				const uint32_t c = open[i];
				ContourRT& r = R[c];
				const uint32_t d = uint32_t(os[c].combo);
				if (!so[i].valid)
				{
					os[c].done = true;
					continue;
				}
				os[c].attempted++;
				acc[c] = r.res[d];
				acc_dir[c] = r.dirs[d];
				pred[c] = so[i].predicted;
				gn[c] = so[i].gnorm;
				r.dirs[d] = mkv(so[i].dir[0], so[i].dir[1], so[i].dir[2]);
				std::fill(r.active.begin(), r.active.end(), 0);
				r.active[d] = 1;
				trials.push_back(c);
			}
			if (trials.empty())
				break;
			U26_TRY(run_levels(trials));
			std::vector<std::pair<uint32_t, uint32_t>> taken;
			for (uint32_t c : trials)
			{
				ContourRT& r = R[c];
				OptState& o = os[c];
				const uint32_t d = uint32_t(o.combo);
				std::fill(r.active.begin(), r.active.end(), 1);
				ComboState& trial = r.res[d];
				const bool take = valid_resp(trial) && (!valid_resp(acc[c]) || better_resp(trial, d, acc[c], d));
				if (take)
				{
					o.accepted++;
					trial.opt_attempted = o.attempted;
					trial.opt_accepted = o.accepted;
					const float actual = resp_obj(acc[c]) - resp_obj(trial);
					if (pred[c] > 1e-20f && actual / pred[c] > 0.75f)
						o.trust = std::fmin(1.0f, o.trust * 2.0f);
					if (trial.hits.size() != trial.hit_count)
						taken.emplace_back(c, d);
				}
				else
				{
					r.res[d] = std::move(acc[c]);
					r.res[d].opt_attempted = o.attempted;
					r.res[d].opt_accepted = o.accepted;
					r.dirs[d] = acc_dir[c];
					o.trust = std::fmax(0.01f, o.trust * 0.5f);
					if (o.trust <= 0.01f || gn[c] < 1e-6f)
						o.done = true;
				}
				acc[c] = ComboState{};
			}
			// the accepted trials' supports feed the next step and the output
			U26_TRY(fetch_then_materialize(taken));
		}
		std::vector<std::pair<uint32_t, uint32_t>> cc;
		for (uint32_t c = 0; c < nact; c++)
		{
			chosen_idx[c] = select_best(R[c]);
			if (chosen_idx[c] >= 0 && R[c].res[chosen_idx[c]].hits.size() != R[c].res[chosen_idx[c]].hit_count)
				cc.emplace_back(c, uint32_t(chosen_idx[c]));
		}
		U26_TRY(fetch_then_materialize(cc));
	}

	mark("refinement");
	// ---- 4. selection, merge capture, suppression, output
	t0 = std::chrono::steady_clock::now();
	std::vector<ComboState> chosen(nc);
	std::vector<std::vector<uint32_t>> merge(nc);
	std::vector<float> pre_area(nc, 0.0f);
	// per contour (independent: each writes its own chosen / pre_area / merge entry)
	host_parallel_dynamic(nact, [&](uint32_t c)
	{
		const ContourRT& r = R[c];
		const int sel = chosen_idx[c];
		if (sel >= 0)
			chosen[c] = r.res[sel];
		pre_area[c] = chosen[c].area;
		std::set<uint32_t> adjc;
		auto flagged = [&](uint32_t v)
		{ return v == kInfH || G.vflag_off[v + 1] > G.vflag_off[v]; };
		// the boundary flags common to every listed vertex (sorted unique flag lists, intersected
		// in place of copies), without this contour's own two
		auto common = [&](const uint32_t* vs, int nvs, std::vector<uint32_t>& out)
		{
			out.clear();
			const uint32_t* b0 = G.vflags.data() + G.vflag_off[vs[0]];
			const uint32_t* e0 = G.vflags.data() + G.vflag_off[vs[0] + 1];
			for (const uint32_t* f = b0; f < e0; f++)
			{
				if (*f == 2 * c || *f == 2 * c + 1)
					continue;
				bool all = true;
				for (int j = 1; j < nvs && all; j++)
					all = std::binary_search(G.vflags.data() + G.vflag_off[vs[j]], G.vflags.data() + G.vflag_off[vs[j] + 1], *f);
				if (all)
					out.push_back(*f);
			}
		};
		std::vector<uint32_t> sf, df;
		for (const u26_prp_hit& h : chosen[c].hits)
		{
			// a hit links contours only through vertices that all carry boundary flags
			bool any_empty = false;
			for (int k = 0; k < 3; k++)
				any_empty = any_empty || !flagged(h.src_verts[k]) || !flagged(h.dst_verts[k]);
			if (any_empty)
				continue;
			uint32_t sv[3], dv[3];
			int ns = 0, nd = 0;
			for (int k = 0; k < 3; k++)
			{
				if (h.src_verts[k] != kInfH)
					sv[ns++] = h.src_verts[k];
				if (h.dst_verts[k] != kInfH)
					dv[nd++] = h.dst_verts[k];
			}
			common(sv, ns, sf);
			common(dv, nd, df);
			for (uint32_t a : sf)
				for (uint32_t bb : df)
					if (a == (bb ^ 1u))
					{
						const uint32_t o = a / 2;
						if (o != c && o < nact)
						{
							const ContourRT& ro = R[o];
							if (std::min(ro.obj[0], ro.obj[1]) == std::min(r.obj[0], r.obj[1]) && std::max(ro.obj[0], ro.obj[1]) == std::max(r.obj[0], r.obj[1]))
								adjc.insert(o);
						}
					}
		}
		merge[c].assign(adjc.begin(), adjc.end());
	});
	// the reference evaluates contours in batches: a contour only sees merge partners from
	// its own or earlier batches (later ones have no object ids yet)
	const uint32_t bsz = std::max(1u, P->batch_size);
	for (uint32_t c = 0; c < nact; c++)
	{
		const uint32_t batch_end = (c / bsz + 1) * bsz;
		auto& m = merge[c];
		m.erase(std::remove_if(m.begin(), m.end(), [&](uint32_t o)
					{ return o >= batch_end; }),
			m.end());
	}
	std::vector<uint32_t> conflicting;
	for (uint32_t c = 0; c < nact; c++)
		if (!merge[c].empty())
			conflicting.push_back(c);
	std::sort(conflicting.begin(), conflicting.end(), [&](uint32_t a, uint32_t bb)
		{
			if (pre_area[a] != pre_area[bb]) return pre_area[a] > pre_area[bb];
			return a < bb; });
	mark("selection, merge adjacency");
	std::vector<uint8_t> supp(nc, 0);
	for (uint32_t o : conflicting)
	{
		if (supp[o])
			continue;
		for (uint32_t a : merge[o])
			if (a != o && a < nact)
				supp[a] = 1;
	}
	// outputs
	out->pairs = G.ef;
	out->pair_idx.resize(2 * size_t(na));
	for (uint32_t p = 0; p < na; p++)
	{
		out->pair_idx[2 * p] = G.ee[p];
		out->pair_idx[2 * p + 1] = G.ff[p];
	}
	out->mesh_index = G.mesh_index;
	out->contour_index = G.contour_index;
	out->pair_length = G.len;
	out->contour_offsets.assign(nc + 1, 0u);
	for (uint32_t c = 0; c < nc; c++)
	{
		out->contour_offsets[c + 1] = out->contour_offsets[c] + uint32_t(G.contours[c].size());
		out->contour_pairs.insert(out->contour_pairs.end(), G.contours[c].begin(), G.contours[c].end());
	}
	out->results.assign(nc, u26_prp_result{});
	out->directions.assign(size_t(nc) * 26 * 3, 0.0f);
	out->hit_offsets.assign(nc + 1, 0u);
	for (uint32_t c = 0; c < nc; c++)
	{
		u26_prp_result& rr = out->results[c];
		rr.contour_idx = c;
		rr.contour_type = G.type[c];
		rr.num_pairs = uint32_t(G.contours[c].size());
		rr.combo_idx = kInfH;
		const bool processed = c < nact;
		static const ComboState kNoResponse{};
		const ComboState& cs = processed && !supp[c] ? chosen[c] : kNoResponse; // a reference, not a copy
		if (processed)
		{
			const ContourRT& r = R[c];
			rr.num_dirs = uint32_t(r.dirs.size());
			rr.object_id0 = r.obj[0];
			rr.object_id1 = r.obj[1];
			rr.init_k_src = r.k0[0];
			rr.init_k_dst = r.k0[1];
			rr.diam_src = r.diam[0];
			rr.diam_dst = r.diam[1];
			rr.num_boundary_src = uint32_t(r.bnd[0].size());
			rr.num_boundary_dst = uint32_t(r.bnd[1].size());
			for (size_t d = 0; d < r.dirs.size() && d < 26; d++)
			{
				out->directions[(size_t(c) * 26 + d) * 3] = r.dirs[d].x;
				out->directions[(size_t(c) * 26 + d) * 3 + 1] = r.dirs[d].y;
				out->directions[(size_t(c) * 26 + d) * 3 + 2] = r.dirs[d].z;
			}
			if (!supp[c] && chosen_idx[c] >= 0)
			{
				rr.combo_idx = uint32_t(chosen_idx[c]);
				const V3h dv = r.dirs[chosen_idx[c]];
				rr.dir[0] = dv.x;
				rr.dir[1] = dv.y;
				rr.dir[2] = dv.z;
			}
			rr.flags = (cs.eligible ? 1u : 0u) | (r.no_resp ? 2u : 0u) | (supp[c] ? 4u : 0u) | (cs.full_mesh ? 8u : 0u) | 16u;
		}
		rr.hit_count = uint32_t(cs.hits.size());
		rr.unculled_hit_count = cs.unculled;
		rr.covered_anchor_count = cs.covered;
		rr.boundary_anchor_count = cs.anchors;
		rr.eval_k_src = cs.eval_k_src;
		rr.eval_k_dst = cs.eval_k_dst;
		rr.max_frontier_hop_src = cs.mfs;
		rr.max_frontier_hop_dst = cs.mfd;
		rr.expansion_level_count = cs.levels;
		rr.depth = cs.depth;
		rr.volume = cs.volume;
		rr.objective = cs.objective;
		rr.area = cs.area;
		rr.displacement_cost = cs.cost;
		rr.coverage = cs.coverage;
		rr.normalized_objective = resp_obj(cs);
		rr.pre_finalize_area = processed ? pre_area[c] : 0.0f;
		rr.opt_attempted = cs.opt_attempted;
		rr.opt_accepted = cs.opt_accepted;
		out->hit_offsets[c + 1] = out->hit_offsets[c] + rr.hit_count;
	}
	// the supports, copied into place over the host threads
	out->hits.resize(out->hit_offsets[nc]);
	host_parallel_dynamic(nc, [&](uint32_t c)
	{
		if (out->hit_offsets[c + 1] > out->hit_offsets[c])
			std::copy(chosen[c].hits.begin(), chosen[c].hits.end(), out->hits.begin() + out->hit_offsets[c]);
	});
	mark("suppression, outputs");
	std::vector<unsigned long long> stats;
	U26_TRY(download(ctx, stats, S->d_stats.ptr, 16));
	U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, ctx->dev_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
	U26_CUDA(ctx, cudaStreamSynchronize(st));
	out->ray_tests = stats[0];
	out->ray_requests = stats[1];
	out->ray_pairs = alg_tests;
	out->ray_nodes = stats[2];
	out->ray_edge_tests = stats[3];
	out->ray_node_fetches = stats[4];
	out->ray_tri_fetches = stats[5];
	out->ray_edge_fetches = stats[6];
	out->ray_visits = stats[7];
	out->ray_candidate_tests = stats[8];
	out->fp64_rechecks = stats[9];
	out->fp64_flips = stats[10];
	out->dev_err = *ctx->host_word;
	if (P->fp64_recheck && P->form == 0 && !out->hits.empty())
		U26_TRY(fp64_metrics(S, d_x, out));
	if (tuning && out->tune_ms[0] > 0.0)
		S->tuned_cfg = int(std::min_element(out->tune_ms, out->tune_ms + kNumRaycastConfigs) - out->tune_ms);
	out->raycast_cfg = P->form != 0 ? -1 : forced ? cfg_now : S->tuned_cfg >= 0 ? S->tuned_cfg : kDefaultRaycastConfig;
	out->tuned = tuning ? 1u : 0u;
	mark("stats, FP64 metrics");
	if (trace_marks)
	{
		double prev = 0.0;
		for (const auto& [what, at] : marks)
		{
			fprintf(stderr, "[u26 prp] host %-32s %8.2f ms (+%.2f)\n", what, at, at - prev);
			prev = at;
		}
	}
	out->stage_ms[6] = ms_since(t0);
	out->stage_ms[7] = ms_since(t_total);
	if (out->dev_err & (U26_DEVERR_STACK_OVERFLOW | U26_DEVERR_ITERATION_CAP))
		return set_error(ctx, U26_ERR_ITERATION_CAP, "PRP device error flags 0x%x", out->dev_err);
	return U26_OK;
}

U26_API u26_status u26_prp_resolve(u26_scene* scene, u26_lbvh* face_tree, u26_lbvh* edge_tree, const float* x, const void* ef_pairs,
	const uint32_t* ef_indices, uint32_t num_pairs, const u26_prp_params* params, u26_prp_output** out)
{
	if (!scene || !out || !params)
		return U26_ERR_INVALID_INPUT;
	*out = nullptr;
	u26_ctx* ctx = scene->ctx;
	if (!face_tree || !edge_tree || face_tree->type != U26_TREE_FACE || edge_tree->type != U26_TREE_EDGE || !x)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_prp_resolve: need a face tree, an edge tree and positions");
	if (face_tree->n != scene->nf || edge_tree->n != scene->ne)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_prp_resolve: trees do not match the scene");
	if (num_pairs && (!ef_pairs || !ef_indices))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_prp_resolve: null EF list");
	std::unique_ptr<u26_prp_output> o(new u26_prp_output());
	const u26_status s = prp_run(scene, face_tree, edge_tree, x, ef_pairs, ef_indices, num_pairs, params, o.get());
	if (s != U26_OK)
		return s;
	o->scene = scene;
	o->pass = ++scene->passes;
	*out = o.release();
	return U26_OK;
}

U26_API u26_status u26_prp_make_response(u26_scene* scene, const u26_prp_output* o, const u26_prp_response_params* params,
	u26_collision_pair* narrow_list, uint32_t* narrow_indices, uint32_t first, uint32_t capacity, u26_prp_response_view* view)
{
	if (!scene || !o || !params || !view)
		return U26_ERR_INVALID_INPUT;
	u26_ctx* ctx = scene->ctx;
	if (o->scene != scene || o->pass != scene->passes)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_prp_make_response: the output is not this scene's latest pass");
	if ((narrow_list == nullptr) != (narrow_indices == nullptr))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_prp_make_response: give both narrow-phase arrays or neither");
	*view = u26_prp_response_view{};
	const uint32_t nh = uint32_t(o->hits.size());
	view->num_pairs = nh;
	if (narrow_list && (first > capacity || nh > capacity - first))
		return set_error(ctx, U26_ERR_CAPACITY, "u26_prp_make_response: narrow-phase list holds %u, needs %u", capacity, first + nh);
	ResponseInputs in{};
	in.hits = o->hits.data();
	in.hit_off = o->hit_offsets.data();
	in.results = o->results.data();
	in.pair_idx = o->pair_idx.data();
	in.mesh_index = o->mesh_index.data();
	in.contour_index = o->contour_index.data();
	in.nh = nh;
	in.nc = uint32_t(o->results.size());
	in.np = uint32_t(o->mesh_index.size());
	in.nv = scene->nv;
	in.ne = scene->ne;
	in.nf = scene->nf;
	in.fn = scene->d_fn.as<float>();
	in.en = scene->d_en.as<float>();
	in.vn = scene->d_vn.as<float>();
	in.va = scene->d_varea.as<float>();
	in.ea = scene->d_earea.as<float>();
	in.fa = scene->d_farea.as<float>();
	in.edges = scene->d_edges.as<uint2>();
	in.faces = scene->d_faces.as<uint32_t>();
	ResponseState& R = scene->resp;
	U26_TRY(response_run(ctx, in, params->depth_threshold, params->stiffness, R, narrow_list ? narrow_list + first : nullptr,
		narrow_indices ? narrow_indices + 2 * size_t(first) : nullptr));
	view->pairs = R.pairs.as<u26_collision_pair>();
	view->pair_info = R.info.as<uint32_t>();
	view->vert_regions = R.vcsr.as<uint32_t>();
	view->edge_regions = R.ecsr.as<uint32_t>();
	view->face_regions = R.fcsr.as<uint32_t>();
	view->vert_regions_len = R.vert_len;
	view->edge_regions_len = R.edge_len;
	view->face_regions_len = R.face_len;
	return U26_OK;
}

U26_API u26_status u26_prp_output_view_get(const u26_prp_output* o, u26_prp_output_view* v)
{
	if (!o || !v)
		return U26_ERR_INVALID_INPUT;
	v->num_pairs = uint32_t(o->pairs.size());
	v->num_orig_pairs = o->num_orig_pairs;
	v->num_contours = uint32_t(o->results.size());
	v->num_hits = uint32_t(o->hits.size());
	v->pairs = o->pairs.data();
	v->pair_indices = o->pair_idx.data();
	v->mesh_index = o->mesh_index.data();
	v->contour_index = o->contour_index.data();
	v->pair_length = o->pair_length.data();
	v->contour_offsets = o->contour_offsets.data();
	v->contour_pairs = o->contour_pairs.data();
	v->results = o->results.data();
	v->hit_offsets = o->hit_offsets.data();
	v->hits = o->hits.data();
	v->directions = o->directions.data();
	v->ray_tests = o->ray_tests;
	v->ray_requests = o->ray_requests;
	v->ray_pairs = o->ray_pairs;
	v->ray_nodes = o->ray_nodes;
	v->ray_edge_tests = o->ray_edge_tests;
	v->ray_node_fetches = o->ray_node_fetches;
	v->ray_tri_fetches = o->ray_tri_fetches;
	v->ray_edge_fetches = o->ray_edge_fetches;
	v->ray_visits = o->ray_visits;
	v->ray_candidate_tests = o->ray_candidate_tests;
	v->fp64_rechecks = o->fp64_rechecks;
	v->fp64_flips = o->fp64_flips;
	v->dc_tie_rechecks = o->dc_tie_rechecks;
	v->dc_tie_flips = o->dc_tie_flips;
	v->fp64_delta_rel_err = o->fp64_delta_rel_err;
	v->fp64_dc_rel_err = o->fp64_dc_rel_err;
	v->fp64_j_rel_err = o->fp64_j_rel_err;
	for (int i = 0; i < kNumRaycastConfigs; i++)
		v->tune_ms[i] = o->tune_ms[i];
	v->raycast_queue = o->raycast_cfg >= 0 && kRaycastConfigs[o->raycast_cfg].queue ? 1u : 0u;
	v->raycast_parts = o->raycast_cfg >= 0 ? kRaycastConfigs[o->raycast_cfg].split : 0u;
	v->raycast_blocks_per_sm = o->raycast_cfg >= 0 ? uint32_t(kRaycastConfigs[o->raycast_cfg].min_blocks) : 0u;
	v->tuned = o->tuned;
	for (int i = 0; i < 6; i++)
		v->gpu_ms[i] = o->gpu_ms[i];
	v->levels = o->levels;
	v->device_error_flags = o->dev_err;
	for (int i = 0; i < 8; i++)
		v->stage_ms[i] = o->stage_ms[i];
	return U26_OK;
}

U26_API void u26_prp_output_destroy(u26_prp_output* o) { delete o; }
