// EF (edge-face) intersection detection on sm_100a.
//
// Reference: Solver/CollisionDetector/intersection_resolver.cpp:86-197
// (fn_narrow_phase_ef_dcd_query) with distance::LineIntersection /
// RayTriangleIntersectionAndBary (intersection_resolver_helper.cpp:319-514), and the
// canonical (eid, fid) order of host_preprocess_ef_pairs (intersection_resolver.cpp:693-726).
//
// Two forms:
//  * u26_ef_narrow_phase: one thread per broad-phase pair (drop-in for the reference
//    kernel; the pair count is read on the device, no host round trip).
//  * u26_ef_detect: the broad phase and the segment-triangle test fused. Each edge
//    walks the face tree in the reference's visit order and tests the triangle as soon
//    as a leaf overlaps, so no broad-phase list is written or re-read.
#include "lbvh_internal.h"
#include "predicates.cuh"

namespace u26
{
	struct EfPairDev
	{
		uint32_t idx[5];
		float bary[3];
		float grad[3];
		float stiff;
	};
	static_assert(sizeof(EfPairDev) == 48, "EfPair is 48 bytes");

	// RayTriangleIntersectionAndBary (helper.cpp:335-380) under the canonical arithmetic.
	__device__ __forceinline__ bool ray_triangle(f3 start, f3 dir, float ray_len, f3 A, f3 B, f3 C, float& out_t, f3& out_bary)
	{
		const f3 AB = B - A;
		const f3 AC = C - A;
		const f3 N = cross(AB, AC);
		const f3 neg = -dir;
		const float nlen = length(N);
		const float den = dot(neg, N);
		if (fabsf(den) < nlen * 1e-6f)
			return false;
		const float inv_den = 1.0f / den;
		const f3 to_a = start - A;
		const float t = dot(to_a, N) * inv_den;
		if (t < 0.0f || t > ray_len)
			return false;
		const f3 cx = cross(neg, to_a);
		const float uu = dot(AC, cx) * inv_den;
		if (uu < 1e-6f || uu > (1.0f - 1e-6f))
			return false;
		const float vv = -dot(AB, cx) * inv_den;
		if (vv < 1e-6f || (vv + uu) > (1.0f - 1e-6f))
			return false;
		out_t = t;
		out_bary = mk3(1.0f - uu - vv, uu, vv);
		return true;
	}

	// LineIntersection (helper.cpp:452-482): segment p0->p1, time in [0, 1].
	__device__ __forceinline__ bool line_intersection(f3 p0, f3 p1, f3 A, f3 B, f3 C, f3& out_bary, float& out_time)
	{
		const f3 d = p1 - p0;
		const float len_sq = length_sq(d);
		if (len_sq < 1e-6f * 1e-6f)
			return false;
		const float len = sqrtf(len_sq);
		const float inv_len = 1.0f / len;
		const f3 ray = d * inv_len;
		if (ray_triangle(p0, ray, len, A, B, C, out_time, out_bary))
		{
			out_time = out_time * inv_len;
			return true;
		}
		return false;
	}

	// The pair filters of fn_narrow_phase_ef_dcd_query ahead of the geometric test: shared
	// vertices, vertex properties, zero contact distance (exact, no rounding involved).
	__device__ __forceinline__ bool ef_pair_eligible(uint32_t e0, uint32_t e1, uint32_t f0, uint32_t f1, uint32_t f2,
		const uint32_t* __restrict__ vprop, const float* __restrict__ d_hat)
	{
		if (e0 == f0 || e0 == f1 || e0 == f2 || e1 == f0 || e1 == f1 || e1 == f2)
			return false;
		const uint32_t lp = vprop ? __ldg(vprop + e0) : 0u;
		const uint32_t rp = vprop ? __ldg(vprop + f0) : 0u;
		if ((lp & 1u) && (rp & 1u))
			return false;
		if ((lp & 2u) && (rp & 2u) && ((lp >> 16) & 0x7FFFu) == ((rp >> 16) & 0x7FFFu))
			return false;
		return __ldg(d_hat + e0) + __ldg(d_hat + f0) != 0.0f;
	}

	// The FP64 recheck of one EF test (predicates.cuh): 0 when its FP32 decision (pass32) lies
	// outside the error band, else 1, plus 2 when the FP64 decision differs. Out of line: it
	// runs once per eligible leaf test and keeps its registers off the traversal loop.
	__device__ __noinline__ uint32_t ef_recheck(f3 pe0, f3 pe1, f3 A, f3 B, f3 C, bool pass32)
	{
		f3 fb = mk3(0.0f);
		float t = 0.0f;
		const bool seg32 = line_intersection(pe0, pe1, A, B, C, fb, t);
		Band bd;
		ef_pair_band(pe0, pe1, A, B, C, seg32, t, fb, bd);
		if (!bd.recheck())
			return 0u;
		const bool pass64 = ef_pair_f64(dd(pe0), dd(pe1), dd(A), dd(B), dd(C));
		return 1u | (pass64 != pass32 ? 2u : 0u);
	}

	// The per-pair body of fn_narrow_phase_ef_dcd_query.
	__device__ __forceinline__ bool ef_pair_test(uint32_t e0, uint32_t e1, uint32_t f0, uint32_t f1, uint32_t f2,
		const float* __restrict__ x, const uint32_t* __restrict__ vprop, const float* __restrict__ d_hat, EfPairDev& rec)
	{
		if (!ef_pair_eligible(e0, e1, f0, f1, f2, vprop, d_hat))
			return false;
		const f3 pe0 = ld3(x, e0), pe1 = ld3(x, e1);
		const f3 A = ld3(x, f0), B = ld3(x, f1), C = ld3(x, f2);
		f3 fb;
		float t;
		if (!line_intersection(pe0, pe1, A, B, C, fb, t))
			return false;
		const f3 n_un = cross(B - A, C - A);
		const float n_len = length(n_un);
		const float face_char = sqrtf(fmaxf(n_len, 1e-30f));
		const f3 n = n_un / fmaxf(n_len, 1e-30f);
		const float d0 = dot(pe0 - A, n);
		const float d1 = dot(pe1 - A, n);
		const float pen = fminf(fabsf(d0), fabsf(d1));
		if (pen < 1e-4f * face_char)
			return false;
		if (fminf(fminf(fb.x, fb.y), fb.z) < 1e-4f)
			return false;
		if (fminf(t, 1.0f - t) < 1e-4f)
			return false;
		rec.idx[0] = e0;
		rec.idx[1] = e1;
		rec.idx[2] = f0;
		rec.idx[3] = f1;
		rec.idx[4] = f2;
		rec.bary[0] = 1.0f - t;
		rec.bary[1] = fb.x;
		rec.bary[2] = fb.y;
		rec.grad[0] = rec.grad[1] = rec.grad[2] = 0.0f;
		rec.stiff = 0.0f;
		return true;
	}

	__device__ __forceinline__ void store_ef(EfPairDev* __restrict__ out, uint32_t* __restrict__ out_idx, uint32_t slot,
		const EfPairDev& rec, uint32_t eid, uint32_t fid)
	{
		uint4* dst = reinterpret_cast<uint4*>(out + slot);
		const uint4* src = reinterpret_cast<const uint4*>(&rec);
		dst[0] = src[0];
		dst[1] = src[1];
		dst[2] = src[2];
		reinterpret_cast<uint2*>(out_idx)[slot] = make_uint2(eid, fid);
	}

	namespace
	{
		__global__ void __launch_bounds__(256) ef_narrow_kernel(const uint2* __restrict__ broad, const uint32_t* __restrict__ broad_count,
			uint32_t max_broad, const float* __restrict__ x, const uint2* __restrict__ edges, const uint32_t* __restrict__ faces,
			const uint32_t* __restrict__ vprop, const float* __restrict__ d_hat, uint32_t* __restrict__ ef_count,
			EfPairDev* __restrict__ out, uint32_t* __restrict__ out_idx, uint32_t max_ef)
		{
			const uint32_t nb = min(*broad_count, max_broad);
			for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
			{
				const uint2 p = __ldg(broad + i);
				const uint2 e = __ldg(edges + p.x);
				const uint32_t f0 = __ldg(faces + 3 * p.y), f1 = __ldg(faces + 3 * p.y + 1), f2 = __ldg(faces + 3 * p.y + 2);
				EfPairDev rec;
				if (ef_pair_test(e.x, e.y, f0, f1, f2, x, vprop, d_hat, rec))
				{
					const uint32_t slot = atomicAdd(ef_count, 1u);
					if (slot < max_ef)
						store_ef(out, out_idx, slot, rec, p.x, p.y);
				}
			}
		}

		// Fused broad + narrow phase: the face-tree traversal of
		// fn_query_from_edges_unculled_v2 (query AABB = edge at x +- thickness + d_hat of its
		// first vertex, strict overlap, stack 32) with the EF test at each overlapping leaf.
		__global__ void __launch_bounds__(128) ef_detect_kernel(TreeView tv, const float* __restrict__ x, const uint2* __restrict__ edges,
			uint32_t num_edges, const uint32_t* __restrict__ faces, const uint32_t* __restrict__ vprop,
			const float* __restrict__ d_hat, const float* __restrict__ thickness, uint32_t* __restrict__ ef_count,
			EfPairDev* __restrict__ out, uint32_t* __restrict__ out_idx, uint32_t max_ef, unsigned long long* __restrict__ stats,
			const uint32_t* __restrict__ edge_order, uint32_t* __restrict__ dev_err)
		{
			const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
			if (tid >= num_edges)
				return;
			const uint32_t eid = edge_order ? __ldg(edge_order + tid) : tid;
			if (*tv.health == 0u)
				return;
			const uint2 e = __ldg(edges + eid);
			const f3 pa = ld3(x, e.x), pb = ld3(x, e.y);
			f3 mn = vmin(vmin(pa, pb), vmin(pa, pb));
			f3 mx = vmax(vmax(pa, pb), vmax(pa, pb));
			const float pad = __ldg(thickness + e.x) + __ldg(d_hat + e.x);
			mn = mn - mk3(pad);
			mx = mx + mk3(pad);
			uint32_t stack[32];
			int sp = 0;
			stack[sp++] = 0u;
			uint32_t loop = 0, visited = 0, tested = 0, rechecks = 0, flips = 0;
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
					visited++;
					if (overlap_strict(b, mn, mx))
					{
						const uint32_t fid = __ldg(tv.object_idx + cs);
						if (fid != kInvalid)
						{
							tested++;
							const uint32_t f0 = __ldg(faces + 3 * fid), f1 = __ldg(faces + 3 * fid + 1), f2 = __ldg(faces + 3 * fid + 2);
							EfPairDev rec;
							const bool pass32 = ef_pair_test(e.x, e.y, f0, f1, f2, x, vprop, d_hat, rec);
							if (pass32)
							{
								const uint32_t slot = atomicAdd(ef_count, 1u);
								if (slot < max_ef)
									store_ef(out, out_idx, slot, rec, eid, fid);
							}
							if (stats && ef_pair_eligible(e.x, e.y, f0, f1, f2, vprop, d_hat))
							{
								const uint32_t rc = ef_recheck(pa, pb, ld3(x, f0), ld3(x, f1), ld3(x, f2), pass32);
								rechecks += rc & 1u;
								flips += rc >> 1;
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
			if (stats)
			{
				// warp-aggregated counters: [0] node boxes tested, [1] leaf primitives tested,
				// [2] EF tests rechecked in FP64 (inside their FP32 error band), [3] FP32 / FP64 flips
				const uint32_t mask = __activemask();
				const uint32_t v = __reduce_add_sync(mask, visited);
				const uint32_t t = __reduce_add_sync(mask, tested);
				const uint32_t rc = __reduce_add_sync(mask, rechecks);
				const uint32_t fl = __reduce_add_sync(mask, flips);
				if ((threadIdx.x & 31) == uint32_t(__ffs(mask) - 1))
				{
					atomicAdd(stats + 0, (unsigned long long)v);
					atomicAdd(stats + 1, (unsigned long long)t);
					if (rc)
						atomicAdd(stats + 2, (unsigned long long)rc);
					if (fl)
						atomicAdd(stats + 3, (unsigned long long)fl);
				}
			}
		}

		__global__ void __launch_bounds__(256) ef_keys_kernel(const uint2* __restrict__ idx, uint32_t count, uint32_t num_faces,
			uint64_t* __restrict__ keys, uint32_t* __restrict__ vals)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= count)
				return;
			const uint2 p = idx[i];
			keys[i] = uint64_t(p.x) * uint64_t(num_faces) + uint64_t(p.y);
			vals[i] = i;
		}

		// 48-byte record a < b in memcmp order (bytes in memory order, unsigned)
		__device__ __forceinline__ bool rec_less(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b)
		{
#pragma unroll
			for (int w = 0; w < 12; w++)
			{
				const uint32_t x = __byte_perm(a[w], 0u, 0x0123u), y = __byte_perm(b[w], 0u, 0x0123u);
				if (x != y)
					return x < y;
			}
			return false;
		}

		// Equal (eid, fid) keys (duplicate pairs, e.g. from the proximity conversion) are put in
		// payload memcmp order, the tie-break of host_preprocess_ef_pairs' canonical sort
		// (intersection_resolver.cpp:700-716): each run head insertion-sorts its run of the
		// sorted permutation.
		__global__ void __launch_bounds__(256) ef_tiebreak_kernel(const uint64_t* __restrict__ keys, uint32_t* __restrict__ perm, uint32_t n,
			const uint32_t* __restrict__ recs)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i + 1 >= n || (i > 0 && keys[i] == keys[i - 1]) || keys[i + 1] != keys[i])
				return;
			uint32_t j = i + 1;
			while (j < n && keys[j] == keys[i])
				j++;
			for (uint32_t a = i + 1; a < j; a++)
			{
				const uint32_t v = perm[a];
				uint32_t b = a;
				while (b > i && rec_less(recs + 12 * size_t(v), recs + 12 * size_t(perm[b - 1])))
				{
					perm[b] = perm[b - 1];
					b--;
				}
				perm[b] = v;
			}
		}

		__global__ void __launch_bounds__(256) ef_gather_kernel(const uint32_t* __restrict__ perm, uint32_t count,
			const EfPairDev* __restrict__ src, const uint2* __restrict__ src_idx, EfPairDev* __restrict__ dst,
			uint2* __restrict__ dst_idx)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= count)
				return;
			const uint32_t j = perm[i];
			dst[i] = src[j];
			dst_idx[i] = src_idx[j];
		}
	} // namespace
} // namespace u26

namespace u26
{
	namespace
	{
		// fn_add_ef_from_proximity_pairs (intersection_resolver.cpp:199-363): a VF or EE proximity
		// pair at near-zero distance (|sum_k w_k x_k|^2 < 1e-10) becomes EF pairs of zero
		// stiffness. VF (v, f): (e, f) for every edge e at v, edge barycentre 1 at v, face
		// barycentres |w1|, |w2|. EE (e1, e2): (e1, g) for the faces g at e2 that share no vertex
		// with e1 and hold e2 (two matched corners), and (e2, g) for the faces at e1 likewise;
		// the corners of g on the shared edge take e1's barycentres in both (as the reference
		// writes them, intersection_resolver.cpp:289-300). Pairs are appended through *ef_count (order: the canonical sort's).
		__device__ __forceinline__ void emit_ef(uint32_t* __restrict__ ef_count, EfPairDev* __restrict__ out, uint32_t* __restrict__ out_idx,
			uint32_t max_ef, uint2 edge, uint3 face, float eb0, float fb0, float fb1, uint32_t eid, uint32_t fid)
		{
			const uint32_t slot = atomicAdd(ef_count, 1u);
			if (slot >= max_ef)
				return;
			EfPairDev r;
			r.idx[0] = edge.x;
			r.idx[1] = edge.y;
			r.idx[2] = face.x;
			r.idx[3] = face.y;
			r.idx[4] = face.z;
			r.bary[0] = eb0;
			r.bary[1] = fb0;
			r.bary[2] = fb1;
			r.grad[0] = r.grad[1] = r.grad[2] = 0.0f;
			r.stiff = 0.0f;
			out[slot] = r;
			reinterpret_cast<uint2*>(out_idx)[slot] = make_uint2(eid, fid);
		}

		__global__ void __launch_bounds__(256) ef_from_proximity_kernel(const u26_collision_pair* __restrict__ pairs,
			const uint2* __restrict__ pidx, const uint32_t* __restrict__ pair_count, uint32_t max_proximity, const float* __restrict__ x,
			const uint2* __restrict__ edges, const uint32_t* __restrict__ faces, const uint32_t* __restrict__ vae_csr,
			const uint32_t* __restrict__ eaf_csr, uint32_t* __restrict__ ef_count, EfPairDev* __restrict__ out, uint32_t* __restrict__ out_idx,
			uint32_t max_ef)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= min(*pair_count, max_proximity))
				return;
			const uint4 raw = *reinterpret_cast<const uint4*>(pairs[i].indices);
			const uint32_t type = (raw.x >> 31) + ((raw.y & 0x80000000u) >> 30) + ((raw.z & 0x80000000u) >> 29) + ((raw.w & 0x80000000u) >> 28);
			if (type != 4u && type != 8u)
				return;
			const float b2 = pairs[i].vec2[2], b3 = pairs[i].vec2[3];
			float w[4];
			if (type == 4u)
			{
				w[0] = 1.0f, w[1] = -b2, w[2] = -b3, w[3] = (b2 + b3) - 1.0f;
			}
			else
			{
				w[0] = b2, w[1] = 1.0f - b2, w[2] = -b3, w[3] = b3 - 1.0f;
			}
			const uint32_t id[4] = { raw.x & 0x7FFFFFFFu, raw.y & 0x7FFFFFFFu, raw.z & 0x7FFFFFFFu, raw.w & 0x7FFFFFFFu };
			const f3 d = ((w[0] * ld3(x, id[0]) + w[1] * ld3(x, id[1])) + w[2] * ld3(x, id[2])) + w[3] * ld3(x, id[3]);
			if (dot(d, d) >= 1e-10f)
				return;
			const uint2 q = pidx[i];
			if (type == 4u)
			{
				const uint32_t vid = id[0], fid = q.y;
				const uint3 face = make_uint3(faces[3 * fid], faces[3 * fid + 1], faces[3 * fid + 2]);
				const float fb0 = fabsf(w[1]), fb1 = fabsf(w[2]);
				for (uint32_t k = vae_csr[vid]; k < vae_csr[vid + 1]; k++)
				{
					const uint32_t ae = vae_csr[k];
					const uint2 e = edges[ae];
					emit_ef(ef_count, out, out_idx, max_ef, e, face, e.x == vid ? 1.0f : 0.0f, fb0, fb1, ae, fid);
				}
				return;
			}
			const uint32_t eid1 = q.x, eid2 = q.y;
			const uint2 e1 = edges[eid1], e2 = edges[eid2];
			const float e1b0 = fabsf(w[0]), e1b1 = fabsf(w[1]), e2b0 = fabsf(w[2]);
			// faces at e2 against e1, then faces at e1 against e2
			for (int side = 0; side < 2; side++)
			{
				const uint32_t at = side == 0 ? eid2 : eid1;
				const uint2 other = side == 0 ? e1 : e2; // the edge that must not touch the face
				const uint2 on = side == 0 ? e2 : e1;	  // the edge whose corners the face holds
				for (uint32_t k = eaf_csr[at]; k < eaf_csr[at + 1]; k++)
				{
					const uint32_t af = eaf_csr[k];
					const uint32_t fv[3] = { faces[3 * af], faces[3 * af + 1], faces[3 * af + 2] };
					bool shares = false;
					for (int c = 0; c < 3; c++)
						shares = shares || fv[c] == other.x || fv[c] == other.y;
					if (shares)
						continue;
					float fb[3] = { 0.0f, 0.0f, 0.0f };
					uint32_t matched = 0;
					for (int c = 0; c < 3; c++)
					{
						if (fv[c] == on.x)
						{
							fb[c] = e1b0;
							matched++;
						}
						else if (fv[c] == on.y)
						{
							fb[c] = e1b1;
							matched++;
						}
					}
					if (matched != 2u)
						continue;
					const uint3 face = make_uint3(fv[0], fv[1], fv[2]);
					if (side == 0)
						emit_ef(ef_count, out, out_idx, max_ef, e1, face, e1b0, fb[0], fb[1], eid1, af);
					else
						emit_ef(ef_count, out, out_idx, max_ef, e2, face, e2b0, fb[0], fb[1], eid2, af);
				}
			}
		}
	} // namespace
} // namespace u26

u26_status u26::ef_tiebreak(u26_ctx* ctx, const uint64_t* sorted_keys, uint32_t* perm, uint32_t count, const void* recs)
{
	ef_tiebreak_kernel<<<div_up(count, 256), 256, 0, ctx->stream>>>(sorted_keys, perm, count, static_cast<const uint32_t*>(recs));
	return after_launch(ctx, "ef_tiebreak_kernel");
}

using namespace u26;

namespace
{
	struct EfScratch
	{
		DevBuf keys, vals, pairs, idx;
		RadixSorter sorter;
	};
} // namespace

// Scratch for canonicalisation lives with the context (one per context).
#include <mutex>
#include <unordered_map>
static std::mutex g_ef_mutex;
static std::unordered_map<const u26_ctx*, EfScratch*> g_ef_scratch;

static EfScratch* ef_scratch(const u26_ctx* ctx)
{
	std::lock_guard<std::mutex> lock(g_ef_mutex);
	auto it = g_ef_scratch.find(ctx);
	if (it != g_ef_scratch.end())
		return it->second;
	EfScratch* s = new EfScratch();
	g_ef_scratch[ctx] = s;
	return s;
}

void u26_ef_release_ctx(const u26_ctx* ctx)
{
	std::lock_guard<std::mutex> lock(g_ef_mutex);
	auto it = g_ef_scratch.find(ctx);
	if (it == g_ef_scratch.end())
		return;
	it->second->keys.release();
	it->second->vals.release();
	it->second->pairs.release();
	it->second->idx.release();
	it->second->sorter.release();
	delete it->second;
	g_ef_scratch.erase(it);
}

U26_API u26_status u26_ef_narrow_phase(u26_ctx* ctx, const uint32_t* broad_pairs, const uint32_t* broad_count, uint32_t max_broad,
	const float* x, const uint32_t* edges, const uint32_t* faces, const uint32_t* vert_property, const float* d_hat,
	uint32_t* ef_count, void* ef_pairs, uint32_t* ef_indices, uint32_t max_ef)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (!broad_pairs || !broad_count || !x || !edges || !faces || !d_hat || !ef_count || (max_ef && (!ef_pairs || !ef_indices)))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_ef_narrow_phase: null input");
	if (max_broad == 0)
		return U26_OK;
	const uint32_t grid = std::min<uint32_t>(div_up(max_broad, 256), 148u * 16u);
	ef_narrow_kernel<<<grid, 256, 0, ctx->stream>>>(reinterpret_cast<const uint2*>(broad_pairs), broad_count, max_broad, x,
		reinterpret_cast<const uint2*>(edges), faces, vert_property, d_hat, ef_count, static_cast<EfPairDev*>(ef_pairs), ef_indices,
		max_ef);
	return after_launch(ctx, "ef_narrow_kernel");
}

U26_API u26_status u26_ef_detect(u26_lbvh* face_tree, const float* x, const uint32_t* edges, uint32_t num_edges,
	const uint32_t* faces, const uint32_t* vert_property, const float* d_hat, const float* thickness, const uint32_t* edge_order,
	uint32_t* ef_count, void* ef_pairs, uint32_t* ef_indices, uint32_t max_ef, uint64_t* stats)
{
	if (!face_tree)
		return U26_ERR_INVALID_INPUT;
	u26_ctx* ctx = face_tree->ctx;
	if (face_tree->type != U26_TREE_FACE)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_ef_detect: tree is not a face tree");
	if (!x || !edges || !faces || !d_hat || !thickness || !ef_count || (max_ef && (!ef_pairs || !ef_indices)))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_ef_detect: null input");
	if (num_edges == 0)
		return U26_OK;
	ef_detect_kernel<<<div_up(num_edges, 128), 128, 0, ctx->stream>>>(tree_view(face_tree), x, reinterpret_cast<const uint2*>(edges),
		num_edges, faces, vert_property, d_hat, thickness, ef_count, static_cast<EfPairDev*>(ef_pairs), ef_indices, max_ef,
		reinterpret_cast<unsigned long long*>(stats), edge_order, ctx->dev_err);
	return after_launch(ctx, "ef_detect_kernel");
}

U26_API u26_status u26_ef_add_from_proximity(u26_ctx* ctx, const u26_collision_pair* narrow_list, const uint32_t* narrow_indices,
	const uint32_t* narrow_count, uint32_t max_proximity, const float* x, const uint32_t* edges, const uint32_t* faces,
	const uint32_t* vert_adj_edges_csr, const uint32_t* edge_adj_faces_csr, uint32_t* ef_count, void* ef_pairs, uint32_t* ef_indices,
	uint32_t max_ef)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (max_proximity == 0)
		return U26_OK;
	if (!narrow_list || !narrow_indices || !narrow_count || !x || !edges || !faces || !vert_adj_edges_csr || !edge_adj_faces_csr ||
		!ef_count || (max_ef && (!ef_pairs || !ef_indices)))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_ef_add_from_proximity: null input");
	ef_from_proximity_kernel<<<div_up(max_proximity, 256), 256, 0, ctx->stream>>>(narrow_list, reinterpret_cast<const uint2*>(narrow_indices),
		narrow_count, max_proximity, x, reinterpret_cast<const uint2*>(edges), faces, vert_adj_edges_csr, edge_adj_faces_csr, ef_count,
		static_cast<EfPairDev*>(ef_pairs), ef_indices, max_ef);
	return after_launch(ctx, "ef_from_proximity_kernel");
}

U26_API u26_status u26_ef_canonicalize(u26_ctx* ctx, uint32_t count, void* ef_pairs, uint32_t* ef_indices, uint32_t num_edges,
	uint32_t num_faces)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (count <= 1)
		return U26_OK;
	if (!ef_pairs || !ef_indices || num_faces == 0 || num_edges == 0)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_ef_canonicalize: bad input");
	EfScratch* s = ef_scratch(ctx);
	U26_CUDA(ctx, s->keys.reserve(sizeof(uint64_t) * count));
	U26_CUDA(ctx, s->vals.reserve(sizeof(uint32_t) * count));
	U26_CUDA(ctx, s->pairs.reserve(sizeof(EfPairDev) * count));
	U26_CUDA(ctx, s->idx.reserve(sizeof(uint2) * count));
	ef_keys_kernel<<<div_up(count, 256), 256, 0, ctx->stream>>>(reinterpret_cast<const uint2*>(ef_indices), count, num_faces,
		s->keys.as<uint64_t>(), s->vals.as<uint32_t>());
	U26_TRY(after_launch(ctx, "ef_keys_kernel"));
	const uint64_t key_max = uint64_t(num_edges) * uint64_t(num_faces);
	int bits = 1;
	while (bits < 64 && (uint64_t(1) << bits) < key_max)
		bits++;
	U26_TRY(s->sorter.sort(ctx, s->keys.as<uint64_t>(), s->vals.as<uint32_t>(), count, 0, bits));
	U26_TRY(ef_tiebreak(ctx, s->keys.as<uint64_t>(), s->vals.as<uint32_t>(), count, ef_pairs));
	U26_CUDA(ctx, cudaMemcpyAsync(s->pairs.ptr, ef_pairs, sizeof(EfPairDev) * count, cudaMemcpyDeviceToDevice, ctx->stream));
	U26_CUDA(ctx, cudaMemcpyAsync(s->idx.ptr, ef_indices, sizeof(uint2) * count, cudaMemcpyDeviceToDevice, ctx->stream));
	ef_gather_kernel<<<div_up(count, 256), 256, 0, ctx->stream>>>(s->vals.as<uint32_t>(), count, s->pairs.as<EfPairDev>(),
		s->idx.as<uint2>(), static_cast<EfPairDev*>(ef_pairs), reinterpret_cast<uint2*>(ef_indices));
	return after_launch(ctx, "ef_gather_kernel");
}
