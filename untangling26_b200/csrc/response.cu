// Response assembly of a PRP pass on sm_100a: the selected supports S(r*) become collision
// pair templates for the Newton system, appended after the penalty pairs of the narrow-phase
// list, and every vertex / edge / face gets the sorted list of contour regions it belongs to.
//
//   make_response_from_min_hitinfo   intersection_resolver2.cpp:2105-2221
//     per hit: C = max(-depth - 3e-3, -depth_threshold), area = max(0.5 (A_src + A_dst), 3e-6),
//     k1 = area stiffness C, k2 = area stiffness; VF / FV enter as VF templates (FV with the
//     target vertex first and the normal reversed), EE as EE templates; region label
//     2 (256 contour + solution key) + source role (prp_classify_hit_solution and
//     prp_pack_response_region_label, intersection_resolver2.cpp:37-121)
//   upload_response_pairs_to_gpu    intersection_resolver2.cpp:2223-2294
//     templates at narrow_phase_list[first + i], (src, dst) at narrow_phase_list_indices
//   host_apply_untangling_constraint intersection_resolver2.cpp:2296-2427
//     vertex regions = sorted unique labels from the templates' vertices and the EF pairs'
//     edge / face vertices; edge and face regions = the union over their vertices; each as
//     one array of [n + 1] absolute offsets followed by the data (upload_2d_csr_from,
//     buffer_allocator.h:26-59)
//
// Kernels: one thread per hit (templates + 4 vertex labels), one per EF pair (5 labels), a
// radix sort of the (vertex, label) keys, a unique pass, then count / scan / fill passes of
// the k-way merges for edges (2 lists) and faces (3 lists). All of it is HBM-bound
// streaming work: the templates (64 B + 16 B info per hit) and the CSR arrays are the bytes.
#include "u26_internal.h"

namespace u26
{
	namespace
	{
		constexpr uint32_t kTypeBit = 0x80000000u;

		__device__ __forceinline__ uint32_t solution_code(float q)
		{
			if (!isfinite(q) || fabsf(q) <= 0.1f)
				return 1u;
			return q > 0.0f ? 2u : 0u;
		}

		__device__ __forceinline__ uint32_t solution_key(f3 ns, f3 nd, f3 r)
		{
			const float rl = length(r), sl = length(ns), dl = length(nd);
			const float sq = rl > 1e-12f && sl > 1e-12f ? dot(ns / sl, r / rl) : 0.0f;
			const float dq = rl > 1e-12f && dl > 1e-12f ? dot(nd / dl, r / rl) : 0.0f;
			return 3u * solution_code(sq) + solution_code(dq);
		}

		__global__ void __launch_bounds__(256) response_kernel(const u26_prp_hit* __restrict__ hits, uint32_t nh,
			const uint32_t* __restrict__ off, uint32_t nc, const float4* __restrict__ cinfo, const float* __restrict__ fn,
			const float* __restrict__ en, const float* __restrict__ vn, const float* __restrict__ va, const float* __restrict__ ea,
			const float* __restrict__ fa, float depth_threshold, float stiffness, int region_bits, u26_collision_pair* __restrict__ out,
			uint4* __restrict__ info, u26_collision_pair* __restrict__ narrow, uint2* __restrict__ narrow_idx, uint64_t* __restrict__ keys)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= nh)
				return;
			// contour of hit i: last c with off[c] <= i
			uint32_t lo = 0, hi = nc;
			while (hi - lo > 1)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if (off[mid] <= i)
					lo = mid;
				else
					hi = mid;
			}
			const uint32_t c = lo;
			const u26_prp_hit h = hits[i];
			const float4 ci = cinfo[c];
			const f3 r = mk3(ci.x, ci.y, ci.z);
			const float C = fmaxf(-ci.w - 3e-3f, -depth_threshold);
			f3 ns, nd, normal = r;
			float a_src, a_dst;
			uint32_t type;
			if (h.type == 0u)
			{
				ns = ld3(vn, h.src_id);
				nd = ld3(fn, h.dst_id);
				a_src = va[h.src_id];
				a_dst = fa[h.dst_id];
				type = 0u;
			}
			else if (h.type == 2u)
			{
				ns = ld3(fn, h.src_id);
				nd = ld3(vn, h.dst_id);
				a_src = fa[h.src_id];
				a_dst = va[h.dst_id];
				type = 1u;
			}
			else
			{
				ns = ld3(en, h.src_id);
				nd = ld3(en, h.dst_id);
				a_src = ea[h.src_id];
				a_dst = ea[h.dst_id];
				type = 2u;
			}
			const uint32_t region = 2u * (256u * c + (solution_key(ns, nd, r) & 255u)); // source role 0
			const float area = fmaxf(0.5f * (a_src + a_dst), 3e-6f);
			const float stiff = area * stiffness;
			float k1 = stiff * C, k2 = stiff;
			if (type == 0u && (!isfinite(k1) || !isfinite(k2)))
				k1 = k2 = 0.0f;
			u26_collision_pair t;
			if (type == 0u)
			{
				t.indices[0] = h.src_verts[0];
				t.indices[1] = h.dst_verts[0];
				t.indices[2] = h.dst_verts[1] | kTypeBit;
				t.indices[3] = h.dst_verts[2];
			}
			else if (type == 1u)
			{
				t.indices[0] = h.dst_verts[0];
				t.indices[1] = h.src_verts[0];
				t.indices[2] = h.src_verts[1] | kTypeBit;
				t.indices[3] = h.src_verts[2];
				normal = -1.0f * normal;
			}
			else
			{
				t.indices[0] = h.src_verts[0];
				t.indices[1] = h.src_verts[1];
				t.indices[2] = h.dst_verts[0];
				t.indices[3] = h.dst_verts[1] | kTypeBit;
			}
			t.vec1[0] = normal.x;
			t.vec1[1] = normal.y;
			t.vec1[2] = normal.z;
			t.vec1[3] = area;
			t.vec2[0] = k1;
			t.vec2[1] = k2;
			t.vec2[2] = h.bary[0];
			t.vec2[3] = h.bary[1];
			t.vec3[0] = t.vec3[1] = t.vec3[2] = t.vec3[3] = 0.0f;
			const uint32_t vid = h.type == 0u ? h.src_id : h.dst_id, fid = h.type == 0u ? h.dst_id : h.src_id;
			const uint4 inf = type == 2u ? make_uint4(h.src_id, h.dst_id, region, type) : make_uint4(vid, fid, region, type);
			out[i] = t;
			info[i] = inf;
			if (narrow)
			{
				narrow[i] = t;
				narrow_idx[i] = make_uint2(inf.x, inf.y);
			}
			// vertex labels: semantic region 2 contour + role on the source side, the other role on the target side
			const uint32_t s = 2u * c, o = s ^ 1u;
			const uint32_t lab[4] = { type == 1u ? o : s, type == 0u ? o : s, type == 1u ? s : o, type == 1u ? s : o };
#pragma unroll
			for (int k = 0; k < 4; k++)
				keys[4 * size_t(i) + k] = (uint64_t(t.indices[k] & ~kTypeBit) << region_bits) | lab[k];
		}

		// EF pair p: edge vertices take 2 contour + mesh role, face vertices the other role
		__global__ void ef_region_keys_kernel(const uint4* __restrict__ efp, uint32_t np, const uint2* __restrict__ edges,
			const uint32_t* __restrict__ faces, int region_bits, uint64_t* __restrict__ keys)
		{
			const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
			if (p >= np)
				return;
			const uint4 q = efp[p];
			const uint2 e = edges[q.x];
			const uint32_t er = q.z, fr = q.z ^ 1u;
			uint64_t* k = keys + 5 * size_t(p);
			k[0] = (uint64_t(e.x) << region_bits) | er;
			k[1] = (uint64_t(e.y) << region_bits) | er;
			k[2] = (uint64_t(faces[3 * q.y]) << region_bits) | fr;
			k[3] = (uint64_t(faces[3 * q.y + 1]) << region_bits) | fr;
			k[4] = (uint64_t(faces[3 * q.y + 2]) << region_bits) | fr;
		}

		__global__ void head_flags_kernel(const uint64_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ flag)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i > n)
				return;
			flag[i] = (i < n && (i == 0 || keys[i] != keys[i - 1])) ? 1u : 0u;
		}

		__global__ void compact_kernel(const uint64_t* __restrict__ keys, uint32_t n, const uint32_t* __restrict__ pos,
			uint64_t* __restrict__ ukeys)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			if (i == 0 || keys[i] != keys[i - 1])
				ukeys[pos[i]] = keys[i];
		}

		// vertex CSR: offsets by binary search of each vertex's first key; data = the labels
		__global__ void vert_csr_kernel(const uint64_t* __restrict__ ukeys, uint32_t nu, uint32_t nv, int region_bits,
			uint32_t* __restrict__ vcsr, uint32_t* __restrict__ voff)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i <= nv)
			{
				const uint64_t want = uint64_t(i) << region_bits;
				uint32_t lo = 0, hi = nu;
				while (lo < hi)
				{
					const uint32_t mid = (lo + hi) >> 1;
					if (ukeys[mid] < want)
						lo = mid + 1;
					else
						hi = mid;
				}
				voff[i] = lo;
				vcsr[i] = nv + 1 + lo;
			}
			if (i < nu)
				vcsr[nv + 1 + i] = uint32_t(ukeys[i] & ((uint64_t(1) << region_bits) - 1u));
		}

		// k-way sorted union of the vertex label lists of one edge (K = 2) or face (K = 3):
		// count (out == nullptr) or write
		template <int K>
		__device__ __forceinline__ uint32_t merge_lists(const uint32_t* __restrict__ vdata, const uint32_t* __restrict__ voff,
			const uint32_t (&v)[K], uint32_t* __restrict__ out)
		{
			uint32_t at[K], end[K];
#pragma unroll
			for (int k = 0; k < K; k++)
			{
				at[k] = voff[v[k]];
				end[k] = voff[v[k] + 1];
			}
			uint32_t n = 0;
			for (;;)
			{
				uint32_t m = 0xFFFFFFFFu;
				bool any = false;
#pragma unroll
				for (int k = 0; k < K; k++)
					if (at[k] < end[k])
					{
						m = min(m, vdata[at[k]]);
						any = true;
					}
				if (!any)
					break;
				if (out)
					out[n] = m;
				n++;
#pragma unroll
				for (int k = 0; k < K; k++)
					if (at[k] < end[k] && vdata[at[k]] == m)
						at[k]++;
			}
			return n;
		}

		template <int K>
		__global__ void prim_count_kernel(const uint32_t* __restrict__ prims, uint32_t n, const uint32_t* __restrict__ vdata,
			const uint32_t* __restrict__ voff, uint32_t* __restrict__ cnt)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i > n)
				return;
			if (i == n)
			{
				cnt[n] = 0u;
				return;
			}
			uint32_t v[K];
#pragma unroll
			for (int k = 0; k < K; k++)
				v[k] = prims[K * size_t(i) + k];
			cnt[i] = merge_lists<K>(vdata, voff, v, nullptr);
		}

		// pos: exclusive scan of the counts ([n + 1], pos[n] = total)
		template <int K>
		__global__ void prim_fill_kernel(const uint32_t* __restrict__ prims, uint32_t n, const uint32_t* __restrict__ vdata,
			const uint32_t* __restrict__ voff, const uint32_t* __restrict__ pos, uint32_t* __restrict__ csr)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i > n)
				return;
			csr[i] = n + 1 + pos[i];
			if (i == n)
				return;
			uint32_t v[K];
#pragma unroll
			for (int k = 0; k < K; k++)
				v[k] = prims[K * size_t(i) + k];
			merge_lists<K>(vdata, voff, v, csr + n + 1 + pos[i]);
		}

		int bits_for(uint32_t n) // bits to hold values 0 .. n - 1
		{
			int b = 1;
			while (b < 32 && (uint64_t(1) << b) < n)
				b++;
			return b;
		}
	} // namespace

	u26_status response_run(u26_ctx* ctx, const ResponseInputs& in, float depth_threshold, float stiffness, ResponseState& R,
		u26_collision_pair* narrow, uint32_t* narrow_idx)
	{
		cudaStream_t st = ctx->stream;
		const uint32_t nh = in.nh, np = in.np, nc = in.nc;
		R.num_pairs = nh;
		// host staging: hits, offsets, (dir, depth) per contour, (edge, face, region) per EF pair
		std::vector<float4> cinfo(std::max(nc, 1u));
		for (uint32_t c = 0; c < nc; c++)
			cinfo[c] = make_float4(in.results[c].dir[0], in.results[c].dir[1], in.results[c].dir[2], in.results[c].depth);
		std::vector<uint4> efp(std::max(np, 1u));
		for (uint32_t p = 0; p < np; p++)
			efp[p] = make_uint4(in.pair_idx[2 * p], in.pair_idx[2 * p + 1], 2u * in.contour_index[p] + (in.mesh_index[p] & 1u), 0u);
		const uint32_t nkeys = 4 * nh + 5 * np;
		U26_CUDA(ctx, R.hits.reserve(sizeof(u26_prp_hit) * std::max(nh, 1u)));
		U26_CUDA(ctx, R.off.reserve(sizeof(uint32_t) * (nc + 1)));
		U26_CUDA(ctx, R.cinfo.reserve(sizeof(float4) * cinfo.size()));
		U26_CUDA(ctx, R.efp.reserve(sizeof(uint4) * efp.size()));
		U26_CUDA(ctx, R.pairs.reserve(sizeof(u26_collision_pair) * std::max(nh, 1u)));
		U26_CUDA(ctx, R.info.reserve(sizeof(uint4) * std::max(nh, 1u)));
		U26_CUDA(ctx, R.keys.reserve(sizeof(uint64_t) * (nkeys + 1)));
		U26_CUDA(ctx, R.ukeys.reserve(sizeof(uint64_t) * (nkeys + 1)));
		U26_CUDA(ctx, R.vals.reserve(sizeof(uint32_t) * (nkeys + 1)));
		U26_CUDA(ctx, R.flags.reserve(sizeof(uint32_t) * (nkeys + 1)));
		U26_CUDA(ctx, R.voff.reserve(sizeof(uint32_t) * (in.nv + 1)));
		U26_CUDA(ctx, R.ecnt.reserve(sizeof(uint32_t) * (in.ne + 1)));
		U26_CUDA(ctx, R.fcnt.reserve(sizeof(uint32_t) * (in.nf + 1)));
		if (nh)
			U26_CUDA(ctx, cudaMemcpyAsync(R.hits.ptr, in.hits, sizeof(u26_prp_hit) * nh, cudaMemcpyHostToDevice, st));
		U26_CUDA(ctx, cudaMemcpyAsync(R.off.ptr, in.hit_off, sizeof(uint32_t) * (nc + 1), cudaMemcpyHostToDevice, st));
		U26_CUDA(ctx, cudaMemcpyAsync(R.cinfo.ptr, cinfo.data(), sizeof(float4) * cinfo.size(), cudaMemcpyHostToDevice, st));
		U26_CUDA(ctx, cudaMemcpyAsync(R.efp.ptr, efp.data(), sizeof(uint4) * efp.size(), cudaMemcpyHostToDevice, st));

		const int rb = bits_for(std::max(2u * nc, 2u));
		const int vb = bits_for(std::max(in.nv, 2u));
		if (rb + vb > 64)
			return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_prp_make_response: region keys exceed 64 bits");
		if (nh)
		{
			response_kernel<<<div_up(nh, 256), 256, 0, st>>>(R.hits.as<u26_prp_hit>(), nh, R.off.as<uint32_t>(), nc, R.cinfo.as<float4>(),
				in.fn, in.en, in.vn, in.va, in.ea, in.fa, depth_threshold, stiffness, rb, R.pairs.as<u26_collision_pair>(), R.info.as<uint4>(),
				narrow, reinterpret_cast<uint2*>(narrow_idx), R.keys.as<uint64_t>());
			U26_TRY(after_launch(ctx, "response_kernel"));
		}
		if (np)
		{
			ef_region_keys_kernel<<<div_up(np, 256), 256, 0, st>>>(R.efp.as<uint4>(), np, in.edges, in.faces, rb, R.keys.as<uint64_t>() + 4 * size_t(nh));
			U26_TRY(after_launch(ctx, "ef_region_keys_kernel"));
		}
		uint32_t nu = 0;
		if (nkeys)
		{
			U26_TRY(R.sorter.sort(ctx, R.keys.as<uint64_t>(), R.vals.as<uint32_t>(), nkeys, 0, rb + vb));
			head_flags_kernel<<<div_up(nkeys + 1, 256), 256, 0, st>>>(R.keys.as<uint64_t>(), nkeys, R.flags.as<uint32_t>());
			U26_TRY(after_launch(ctx, "head_flags_kernel"));
			U26_TRY(device_exclusive_scan(ctx, R.flags.as<uint32_t>(), nkeys + 1, R.scan_tmp));
			compact_kernel<<<div_up(nkeys, 256), 256, 0, st>>>(R.keys.as<uint64_t>(), nkeys, R.flags.as<uint32_t>(), R.ukeys.as<uint64_t>());
			U26_TRY(after_launch(ctx, "compact_kernel"));
			U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, R.flags.as<uint32_t>() + nkeys, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
			U26_CUDA(ctx, cudaStreamSynchronize(st));
			nu = *ctx->host_word;
		}
		R.vert_len = in.nv + 1 + nu;
		U26_CUDA(ctx, R.vcsr.reserve(sizeof(uint32_t) * R.vert_len));
		vert_csr_kernel<<<div_up(std::max(in.nv + 1, nu), 256), 256, 0, st>>>(R.ukeys.as<uint64_t>(), nu, in.nv, rb, R.vcsr.as<uint32_t>(),
			R.voff.as<uint32_t>());
		U26_TRY(after_launch(ctx, "vert_csr_kernel"));
		const uint32_t* vdata = R.vcsr.as<uint32_t>() + in.nv + 1;
		prim_count_kernel<2><<<div_up(in.ne + 1, 256), 256, 0, st>>>(reinterpret_cast<const uint32_t*>(in.edges), in.ne, vdata, R.voff.as<uint32_t>(),
			R.ecnt.as<uint32_t>());
		U26_TRY(after_launch(ctx, "prim_count_kernel<2>"));
		prim_count_kernel<3><<<div_up(in.nf + 1, 256), 256, 0, st>>>(in.faces, in.nf, vdata, R.voff.as<uint32_t>(), R.fcnt.as<uint32_t>());
		U26_TRY(after_launch(ctx, "prim_count_kernel<3>"));
		U26_TRY(device_exclusive_scan(ctx, R.ecnt.as<uint32_t>(), in.ne + 1, R.scan_tmp));
		U26_TRY(device_exclusive_scan(ctx, R.fcnt.as<uint32_t>(), in.nf + 1, R.scan_tmp));
		// both totals in one round trip (the context's pinned staging holds 16 words)
		uint32_t tot[2];
		U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, R.ecnt.as<uint32_t>() + in.ne, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
		U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word + 1, R.fcnt.as<uint32_t>() + in.nf, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
		U26_CUDA(ctx, cudaStreamSynchronize(st));
		tot[0] = ctx->host_word[0];
		tot[1] = ctx->host_word[1];
		R.edge_len = in.ne + 1 + tot[0];
		R.face_len = in.nf + 1 + tot[1];
		U26_CUDA(ctx, R.ecsr.reserve(sizeof(uint32_t) * R.edge_len));
		U26_CUDA(ctx, R.fcsr.reserve(sizeof(uint32_t) * R.face_len));
		prim_fill_kernel<2><<<div_up(in.ne + 1, 256), 256, 0, st>>>(reinterpret_cast<const uint32_t*>(in.edges), in.ne, vdata, R.voff.as<uint32_t>(),
			R.ecnt.as<uint32_t>(), R.ecsr.as<uint32_t>());
		U26_TRY(after_launch(ctx, "prim_fill_kernel<2>"));
		prim_fill_kernel<3><<<div_up(in.nf + 1, 256), 256, 0, st>>>(in.faces, in.nf, vdata, R.voff.as<uint32_t>(), R.fcnt.as<uint32_t>(),
			R.fcsr.as<uint32_t>());
		U26_TRY(after_launch(ctx, "prim_fill_kernel<3>"));
		U26_CUDA(ctx, cudaStreamSynchronize(st));
		return U26_OK;
	}
} // namespace u26

// ---- a fixed step along the assembled response -----------------------------------------
// Each response pair asks its two sides apart along its normal n by Delta = -k1 / k2 = -C =
// min(depth + 3e-3, depth_threshold): the pair's first primitive (the VF template's vertex, the
// EE template's first edge) moves +Delta / 2 n, the second -Delta / 2 n, shared among the
// primitive's vertices by its barycentric weights. A vertex moves by the weighted mean of the
// displacements its pairs ask for, times `scale`. The sums are accumulated in 2^-40 m and 2^-32
// fixed point (integer atomics), so the step does not depend on the order in which pairs land.
namespace u26
{
	namespace
	{
		constexpr double kStepScale = 1099511627776.0; // 2^40
		constexpr double kWeightScale = 4294967296.0;  // 2^32

		__device__ __forceinline__ void step_add(long long* __restrict__ acc, uint32_t v, uint32_t nv, f3 d, float w)
		{
			if (v >= nv || !(w > 0.0f))
				return;
			long long* a = acc + 4 * size_t(v);
			atomicAdd(reinterpret_cast<unsigned long long*>(a + 0), (unsigned long long)llrint(double(d.x * w) * kStepScale));
			atomicAdd(reinterpret_cast<unsigned long long*>(a + 1), (unsigned long long)llrint(double(d.y * w) * kStepScale));
			atomicAdd(reinterpret_cast<unsigned long long*>(a + 2), (unsigned long long)llrint(double(d.z * w) * kStepScale));
			atomicAdd(reinterpret_cast<unsigned long long*>(a + 3), (unsigned long long)llrint(double(w) * kWeightScale));
		}

		__global__ void __launch_bounds__(256) step_pairs_kernel(const u26_collision_pair* __restrict__ pairs, uint32_t n, uint32_t nv,
			long long* __restrict__ acc)
		{
			const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
			if (i >= n)
				return;
			const u26_collision_pair p = pairs[i];
			const float k1 = p.vec2[0], k2 = p.vec2[1];
			if (!(k2 > 0.0f) || !isfinite(k1))
				return;
			const float delta = -k1 / k2;
			const f3 half = mk3(p.vec1[0], p.vec1[1], p.vec1[2]) * (0.5f * delta);
			if (p.indices[2] & kTypeBit)
			{
				// VF template: vertex, face (f0 f1 f2), face barycentres b0 b1
				const float b0 = p.vec2[2], b1 = p.vec2[3], b2 = 1.0f - b0 - b1;
				step_add(acc, p.indices[0], nv, half, 1.0f);
				step_add(acc, p.indices[1], nv, -half, b0);
				step_add(acc, p.indices[2] & ~kTypeBit, nv, -half, b1);
				step_add(acc, p.indices[3], nv, -half, b2);
			}
			else if (p.indices[3] & kTypeBit)
			{
				// EE template: edge a0 a1, edge b0 b1, edge parameters
				const float ta = p.vec2[2], tb = p.vec2[3];
				step_add(acc, p.indices[0], nv, half, ta);
				step_add(acc, p.indices[1], nv, half, 1.0f - ta);
				step_add(acc, p.indices[2], nv, -half, tb);
				step_add(acc, p.indices[3] & ~kTypeBit, nv, -half, 1.0f - tb);
			}
		}

		__global__ void __launch_bounds__(256) step_apply_kernel(float* __restrict__ x, uint32_t nv, long long* __restrict__ acc, float scale,
			unsigned long long* __restrict__ moved)
		{
			const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
			if (v >= nv)
				return;
			long long* a = acc + 4 * size_t(v);
			const long long w = a[3];
			if (w > 0)
			{
				const double inv = kWeightScale / double(w) / kStepScale;
				for (int c = 0; c < 3; c++)
					x[3 * v + c] = float(double(x[3 * v + c]) + double(scale) * (double(a[c]) * inv));
				if (moved)
					atomicAdd(moved, 1ull);
			}
			a[0] = a[1] = a[2] = a[3] = 0; // ready for the next call
		}
	} // namespace
} // namespace u26

using namespace u26;

U26_API u26_status u26_response_step(u26_ctx* ctx, const u26_collision_pair* pairs, uint32_t num_pairs, float* x, uint32_t num_verts,
	float scale, long long* scratch, unsigned long long* moved)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (!x || !scratch || (num_pairs && !pairs))
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_response_step: null input");
	if (num_verts == 0)
		return U26_OK;
	if (moved)
		U26_CUDA(ctx, cudaMemsetAsync(moved, 0, sizeof(unsigned long long), ctx->stream));
	if (num_pairs)
	{
		step_pairs_kernel<<<div_up(num_pairs, 256), 256, 0, ctx->stream>>>(pairs, num_pairs, num_verts, scratch);
		U26_TRY(after_launch(ctx, "step_pairs_kernel"));
	}
	step_apply_kernel<<<div_up(num_verts, 256), 256, 0, ctx->stream>>>(x, num_verts, scratch, scale, moved);
	return after_launch(ctx, "step_apply_kernel");
}
