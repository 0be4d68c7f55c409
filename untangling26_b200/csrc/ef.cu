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

	// The per-pair body of fn_narrow_phase_ef_dcd_query.
	__device__ __forceinline__ bool ef_pair_test(uint32_t e0, uint32_t e1, uint32_t f0, uint32_t f1, uint32_t f2,
		const float* __restrict__ x, const uint32_t* __restrict__ vprop, const float* __restrict__ d_hat, EfPairDev& rec)
	{
		if (e0 == f0 || e0 == f1 || e0 == f2 || e1 == f0 || e1 == f1 || e1 == f2)
			return false;
		const uint32_t lp = vprop ? __ldg(vprop + e0) : 0u;
		const uint32_t rp = vprop ? __ldg(vprop + f0) : 0u;
		if ((lp & 1u) && (rp & 1u))
			return false;
		if ((lp & 2u) && (rp & 2u) && ((lp >> 16) & 0x7FFFu) == ((rp >> 16) & 0x7FFFu))
			return false;
		if (__ldg(d_hat + e0) + __ldg(d_hat + f0) == 0.0f)
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
			uint32_t loop = 0, visited = 0, tested = 0;
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
							if (ef_pair_test(e.x, e.y, f0, f1, f2, x, vprop, d_hat, rec))
							{
								const uint32_t slot = atomicAdd(ef_count, 1u);
								if (slot < max_ef)
									store_ef(out, out_idx, slot, rec, eid, fid);
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
				// warp-aggregated counters: [0] node boxes tested, [1] leaf primitives tested
				const uint32_t mask = __activemask();
				const uint32_t v = __reduce_add_sync(mask, visited);
				const uint32_t t = __reduce_add_sync(mask, tested);
				if ((threadIdx.x & 31) == uint32_t(__ffs(mask) - 1))
				{
					atomicAdd(stats + 0, (unsigned long long)v);
					atomicAdd(stats + 1, (unsigned long long)t);
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
	U26_CUDA(ctx, cudaMemcpyAsync(s->pairs.ptr, ef_pairs, sizeof(EfPairDev) * count, cudaMemcpyDeviceToDevice, ctx->stream));
	U26_CUDA(ctx, cudaMemcpyAsync(s->idx.ptr, ef_indices, sizeof(uint2) * count, cudaMemcpyDeviceToDevice, ctx->stream));
	ef_gather_kernel<<<div_up(count, 256), 256, 0, ctx->stream>>>(s->vals.as<uint32_t>(), count, s->pairs.as<EfPairDev>(),
		s->idx.as<uint2>(), static_cast<EfPairDev*>(ef_pairs), reinterpret_cast<uint2*>(ef_indices));
	return after_launch(ctx, "ef_gather_kernel");
}
