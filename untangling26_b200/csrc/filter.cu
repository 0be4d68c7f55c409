// Region-based pair filtering on sm_100a: the contour regions of a PRP pass switch off the
// proximity pairs and flag the CCD broad-phase pairs that would fight the untangling response.
//
//   fn_is_matched_invalid_region       intersection_resolver.cpp:2232-2337
//     0: neither primitive has a region; 1: some region of the left primitive is the
//     opposite side of some region of the right one (left == right ^ 1); 2: regions, no match.
//     VF pairs compare the vertex's row with the face's row, EE pairs the two edges' rows.
//   filter_invalid_pairs               intersection_resolver.cpp:2635-2676 (+ kernels 2344-2417)
//     over the proximity pairs [0, n) of the narrow-phase list: a pair whose weighted
//     distance |sum_k w_k x_k|^2 < (offset[i0] + offset[i2])^2 + 1e-10 marks its 4 vertices
//     invalid; then every pair touching an invalid vertex, or (with regions) whose region
//     match is 1, is disabled (k1 = k2 = 0).
//   filter_broad_phase_pairs           intersection_resolver.cpp:2586-2633 (+ kernels 2425-2540)
//     VF (vid, fid) and EE (eid1, eid2) broad-phase pairs get bit 31 on both ids when their
//     region match is 1 and bit 30 when one of their 4 vertices is invalid.
//
// The placeholder slot of a VV / VE template (index ~0, masked to 0x7fffffff) is out of
// range: the reference reads and writes vertex 0x7fffffff there; here slots with an index
// >= num_verts add nothing and mark nothing.
#include "u26_internal.h"

namespace u26
{
	namespace
	{
		constexpr uint32_t kMask = 0x7FFFFFFFu;
		constexpr uint32_t kFlagRegion = 1u << 31, kFlagNear = 1u << 30;

		struct Regions
		{
			const uint32_t *v, *e, *f; // upload_2d_csr_from arrays: [n + 1] absolute offsets, then data
		};

		// CollisionPairTemplate::get_collision_type (collision_data.h:72-79): the type bits of all four slots
		__device__ __forceinline__ uint32_t pair_type(const uint4 idx)
		{
			return (idx.x >> 31) + ((idx.y & 0x80000000u) >> 30) + ((idx.z & 0x80000000u) >> 29) + ((idx.w & 0x80000000u) >> 28);
		}

		// CollisionPairTemplate::get_weight (collision_data.h:131-147)
		__device__ __forceinline__ float4 pair_weight(uint32_t type, float b2, float b3)
		{
			if (type == 4u)
				return make_float4(1.0f, -b2, -b3, (b2 + b3) - 1.0f);
			if (type == 8u)
				return make_float4(b2, 1.0f - b2, -b3, b3 - 1.0f);
			if (type == 1u)
				return make_float4(1.0f, 0.0f, -1.0f, 0.0f);
			if (type == 2u)
				return make_float4(1.0f, 0.0f, -b2, -b3);
			return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		}

		// 0 no regions, 1 matched (left region == right region ^ 1), 2 regions without a match
		__device__ __forceinline__ uint32_t region_match(const uint32_t* __restrict__ lcsr, uint32_t l, const uint32_t* __restrict__ rcsr,
			uint32_t r)
		{
			const uint32_t l0 = lcsr[l], l1 = lcsr[l + 1], r0 = rcsr[r], r1 = rcsr[r + 1];
			if (l1 == l0 && r1 == r0)
				return 0u;
			for (uint32_t i = l0; i < l1; i++)
			{
				const uint32_t a = lcsr[i] ^ 1u;
				for (uint32_t j = r0; j < r1; j++)
					if (rcsr[j] == a)
						return 1u;
			}
			return 2u;
		}

		__global__ void __launch_bounds__(256) identify_invalid_kernel(const u26_collision_pair* __restrict__ pairs, uint32_t n,
			const float* __restrict__ x, const float* __restrict__ offset, uint32_t nv, uint32_t* __restrict__ invalid)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint4 raw = *reinterpret_cast<const uint4*>(pairs[i].indices);
			const float4 v2 = *reinterpret_cast<const float4*>(pairs[i].vec2);
			const float4 w = pair_weight(pair_type(raw), v2.z, v2.w);
			const uint32_t id[4] = { raw.x & kMask, raw.y & kMask, raw.z & kMask, raw.w & kMask };
			const float wk[4] = { w.x, w.y, w.z, w.w };
			f3 d = mk3(0.0f);
#pragma unroll
			for (int k = 0; k < 4; k++)
				if (id[k] < nv)
					d = d + wk[k] * ld3(x, id[k]);
			const float d2 = dot(d, d);
			const float th = (id[0] < nv ? offset[id[0]] : 0.0f) + (id[2] < nv ? offset[id[2]] : 0.0f);
			if (d2 < th * th + 1e-10f)
			{
#pragma unroll
				for (int k = 0; k < 4; k++)
					if (id[k] < nv)
						invalid[id[k]] = 1u;
			}
		}

		__global__ void __launch_bounds__(256) filter_pairs_kernel(u26_collision_pair* __restrict__ pairs, const uint2* __restrict__ pidx,
			uint32_t n, uint32_t nv, const uint32_t* __restrict__ invalid, Regions rg)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint4 raw = *reinterpret_cast<const uint4*>(pairs[i].indices);
			const uint32_t id[4] = { raw.x & kMask, raw.y & kMask, raw.z & kMask, raw.w & kMask };
			bool off = false;
#pragma unroll
			for (int k = 0; k < 4; k++)
				off = off || (id[k] < nv && invalid[id[k]] != 0u);
			if (!off && rg.v)
			{
				const uint32_t type = pair_type(raw);
				const uint2 q = pidx[i];
				if (type == 4u)
					off = region_match(rg.v, q.x, rg.f, q.y) == 1u;
				else if (type == 8u)
					off = region_match(rg.e, q.x, rg.e, q.y) == 1u;
			}
			if (off)
			{
				pairs[i].vec2[0] = 0.0f;
				pairs[i].vec2[1] = 0.0f;
			}
		}

		__global__ void __launch_bounds__(256) filter_broad_vf_kernel(uint32_t* __restrict__ list, uint32_t n, const uint32_t* __restrict__ invalid,
			Regions rg, const uint32_t* __restrict__ faces)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint2 p = reinterpret_cast<const uint2*>(list)[i];
			const uint32_t f0 = faces[3 * p.y], f1 = faces[3 * p.y + 1], f2 = faces[3 * p.y + 2];
			const bool near = invalid[p.x] != 0u || invalid[f0] != 0u || invalid[f1] != 0u || invalid[f2] != 0u;
			const bool region = region_match(rg.v, p.x, rg.f, p.y) == 1u;
			if (near || region)
			{
				const uint32_t fl = (region ? kFlagRegion : 0u) | (near ? kFlagNear : 0u);
				reinterpret_cast<uint2*>(list)[i] = make_uint2(p.x | fl, p.y | fl);
			}
		}

		__global__ void __launch_bounds__(256) filter_broad_ee_kernel(uint32_t* __restrict__ list, uint32_t n, const uint32_t* __restrict__ invalid,
			Regions rg, const uint2* __restrict__ edges)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const uint2 p = reinterpret_cast<const uint2*>(list)[i];
			const uint2 a = edges[p.x], b = edges[p.y];
			const bool near = invalid[a.x] != 0u || invalid[a.y] != 0u || invalid[b.x] != 0u || invalid[b.y] != 0u;
			const bool region = region_match(rg.e, p.x, rg.e, p.y) == 1u;
			if (near || region)
			{
				const uint32_t fl = (region ? kFlagRegion : 0u) | (near ? kFlagNear : 0u);
				reinterpret_cast<uint2*>(list)[i] = make_uint2(p.x | fl, p.y | fl);
			}
		}
	} // namespace
} // namespace u26

using namespace u26;

U26_API u26_status u26_filter_invalid_pairs(u26_ctx* ctx, u26_collision_pair* narrow_list, const uint32_t* narrow_indices,
	uint32_t num_proximity_pairs, uint32_t num_ef, const float* x, const float* vert_offset, uint32_t num_verts, uint32_t* vert_is_invalid,
	const uint32_t* vert_regions, const uint32_t* edge_regions, const uint32_t* face_regions)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (num_ef == 0 || num_proximity_pairs == 0)
		return U26_OK;
	if (!narrow_list || !narrow_indices || !x || !vert_offset || !vert_is_invalid)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_filter_invalid_pairs: null input");
	const bool with_regions = vert_regions != nullptr;
	if (with_regions && (!edge_regions || !face_regions))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_filter_invalid_pairs: give all three region arrays or none");
	const Regions rg{ vert_regions, edge_regions, face_regions };
	identify_invalid_kernel<<<div_up(num_proximity_pairs, 256), 256, 0, ctx->stream>>>(narrow_list, num_proximity_pairs, x, vert_offset,
		num_verts, vert_is_invalid);
	U26_TRY(after_launch(ctx, "identify_invalid_kernel"));
	filter_pairs_kernel<<<div_up(num_proximity_pairs, 256), 256, 0, ctx->stream>>>(narrow_list,
		reinterpret_cast<const uint2*>(narrow_indices), num_proximity_pairs, num_verts, vert_is_invalid, rg);
	return after_launch(ctx, "filter_pairs_kernel");
}

U26_API u26_status u26_filter_broad_phase_pairs(u26_ctx* ctx, uint32_t* vf_list, uint32_t num_vf, uint32_t* ee_list, uint32_t num_ee,
	uint32_t num_ef, const uint32_t* vert_is_invalid, const uint32_t* vert_regions, const uint32_t* edge_regions, const uint32_t* face_regions,
	const uint32_t* faces, const uint32_t* edges)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (num_ef == 0 || !vert_regions)
		return U26_OK;
	if (!vert_is_invalid || !edge_regions || !face_regions || (num_vf && (!vf_list || !faces)) || (num_ee && (!ee_list || !edges)))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_filter_broad_phase_pairs: null input");
	const Regions rg{ vert_regions, edge_regions, face_regions };
	if (num_vf)
	{
		filter_broad_vf_kernel<<<div_up(num_vf, 256), 256, 0, ctx->stream>>>(vf_list, num_vf, vert_is_invalid, rg, faces);
		U26_TRY(after_launch(ctx, "filter_broad_vf_kernel"));
	}
	if (num_ee)
	{
		filter_broad_ee_kernel<<<div_up(num_ee, 256), 256, 0, ctx->stream>>>(ee_list, num_ee, vert_is_invalid, rg,
			reinterpret_cast<const uint2*>(edges));
		U26_TRY(after_launch(ctx, "filter_broad_ee_kernel"));
	}
	return U26_OK;
}
