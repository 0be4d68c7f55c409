// Test infrastructure (oracle): CPU restatement of the reference's region-based pair
// filtering, the consumer of the PRP region labels. Loaded only by tests/ and bench.py's
// CPU legs.
//
// Followed (Solver/CollisionDetector/intersection_resolver.cpp):
//   fn_is_matched_invalid_region                 2232-2337
//   fn_identify_invalid_verts_from_proximity_pairs   2344-2365
//   fn_filter_invalid_proximity_pairs_from_invalid_verts 2366-2392
//   fn_filter_invalid_proximity_pairs_from_region_info   2394-2417
//   fn_filter_broadphase_vf_pairs / _ee_pairs    2425-2540
//   filter_broad_phase_pairs / filter_invalid_pairs  2586-2676
//   fn_add_ef_from_proximity_pairs               199-363 (near-zero-distance pairs as EF pairs)
// and CollisionPairTemplate::get_collision_type / get_weight (SimulationCore/collision_data.h:48-147).
//
// Deviation shared with the CUDA path: template slots whose masked index is >= num_verts (the
// ~0 placeholder of VV / VE pairs) are skipped; the reference reads and writes vertex
// 0x7fffffff there.
#include "oracle_common.h"

using u26o::uint;

namespace
{
	using namespace u26o;
	constexpr uint kMask = 0x7FFFFFFFu;

	struct PairT
	{
		uint idx[4];
		float vec1[4], vec2[4], vec3[4];
	};

	uint pair_type(const PairT& p)
	{
		const uint m = 0x80000000u;
		return ((p.idx[0] & m) >> 31) + ((p.idx[1] & m) >> 30) + ((p.idx[2] & m) >> 29) + ((p.idx[3] & m) >> 28);
	}

	void pair_weight(const PairT& p, float w[4])
	{
		const uint t = pair_type(p);
		const float b2 = p.vec2[2], b3 = p.vec2[3];
		if (t == 4u)
		{
			w[0] = 1.0f, w[1] = -b2, w[2] = -b3, w[3] = (b2 + b3) - 1.0f;
		}
		else if (t == 8u)
		{
			w[0] = b2, w[1] = 1.0f - b2, w[2] = -b3, w[3] = b3 - 1.0f;
		}
		else if (t == 1u)
		{
			w[0] = 1.0f, w[1] = 0.0f, w[2] = -1.0f, w[3] = 0.0f;
		}
		else if (t == 2u)
		{
			w[0] = 1.0f, w[1] = 0.0f, w[2] = -b2, w[3] = -b3;
		}
		else
			w[0] = w[1] = w[2] = w[3] = 0.0f;
	}

	uint region_match(const uint* lcsr, uint l, const uint* rcsr, uint r)
	{
		const uint lc = lcsr[l + 1] - lcsr[l], rc = rcsr[r + 1] - rcsr[r];
		if (lc == 0 && rc == 0)
			return 0;
		bool matched = false;
		for (uint i = 0; i < lc; i++)
			for (uint j = 0; j < rc; j++)
				if (lcsr[lcsr[l] + i] == (rcsr[rcsr[r] + j] ^ 1u))
				{
					matched = true;
					break;
				}
		return matched ? 1u : 2u;
	}
} // namespace

namespace
{
	struct EfRec // CollisionPair::EfPair (collision_data.h:150-220), 48 B
	{
		uint idx[5];
		float bary[3];
		float grad[3];
		float stiff;
	};
} // namespace

extern "C"
{
	// fn_add_ef_from_proximity_pairs over the proximity pairs [0, n), in pair order; csr arrays
	// in upload_2d_csr_from's layout. Returns the number of EF pairs produced (written up to max_out).
	uint oracle_ef_from_proximity(const void* pairs_v, const uint* pidx, uint n, const float* x, const uint* edges, const uint* faces,
		const uint* vae_csr, const uint* eaf_csr, void* out_v, uint* out_idx, uint max_out)
	{
		const PairT* pairs = static_cast<const PairT*>(pairs_v);
		EfRec* out = static_cast<EfRec*>(out_v);
		uint count = 0;
		auto emit = [&](uint e0, uint e1, uint f0, uint f1, uint f2, float eb, float fb0, float fb1, uint eid, uint fid)
		{
			if (count < max_out)
			{
				EfRec r{};
				r.idx[0] = e0, r.idx[1] = e1, r.idx[2] = f0, r.idx[3] = f1, r.idx[4] = f2;
				r.bary[0] = eb, r.bary[1] = fb0, r.bary[2] = fb1;
				out[count] = r;
				out_idx[2 * count] = eid;
				out_idx[2 * count + 1] = fid;
			}
			count++;
		};
		for (uint i = 0; i < n; i++)
		{
			const PairT& p = pairs[i];
			const uint t = pair_type(p);
			if (t != 4u && t != 8u)
				continue;
			float w[4];
			pair_weight(p, w);
			uint id[4];
			for (int k = 0; k < 4; k++)
				id[k] = p.idx[k] & kMask;
			const V3 d = ((w[0] * load3(x, id[0]) + w[1] * load3(x, id[1])) + w[2] * load3(x, id[2])) + w[3] * load3(x, id[3]);
			if (dot(d, d) >= 1e-10f)
				continue;
			if (t == 4u)
			{
				const uint v = id[0], f = pidx[2 * i + 1];
				for (uint k = vae_csr[v]; k < vae_csr[v + 1]; k++)
				{
					const uint ae = vae_csr[k];
					emit(edges[2 * ae], edges[2 * ae + 1], faces[3 * f], faces[3 * f + 1], faces[3 * f + 2], edges[2 * ae] == v ? 1.0f : 0.0f,
						std::fabs(w[1]), std::fabs(w[2]), ae, f);
				}
				continue;
			}
			const uint e1 = pidx[2 * i], e2 = pidx[2 * i + 1];
			const uint a0 = edges[2 * e1], a1 = edges[2 * e1 + 1], b0 = edges[2 * e2], b1 = edges[2 * e2 + 1];
			const float ab0 = std::fabs(w[0]), ab1 = std::fabs(w[1]), bb0 = std::fabs(w[2]);
			// faces at e2 that hold e2 and no vertex of e1: (e1, face)
			for (uint k = eaf_csr[e2]; k < eaf_csr[e2 + 1]; k++)
			{
				const uint g = eaf_csr[k];
				const uint* fv = faces + 3 * g;
				if (fv[0] == a0 || fv[1] == a0 || fv[2] == a0 || fv[0] == a1 || fv[1] == a1 || fv[2] == a1)
					continue;
				float fb[3] = { 0, 0, 0 };
				uint matched = 0;
				for (int c = 0; c < 3; c++)
					if (fv[c] == b0)
						fb[c] = ab0, matched++;
					else if (fv[c] == b1)
						fb[c] = ab1, matched++;
				if (matched == 2)
					emit(a0, a1, fv[0], fv[1], fv[2], ab0, fb[0], fb[1], e1, g);
			}
			// faces at e1 that hold e1 and no vertex of e2: (e2, face), corners with e1's barycentres
			for (uint k = eaf_csr[e1]; k < eaf_csr[e1 + 1]; k++)
			{
				const uint g = eaf_csr[k];
				const uint* fv = faces + 3 * g;
				if (fv[0] == b0 || fv[1] == b0 || fv[2] == b0 || fv[0] == b1 || fv[1] == b1 || fv[2] == b1)
					continue;
				float fb[3] = { 0, 0, 0 };
				uint matched = 0;
				for (int c = 0; c < 3; c++)
					if (fv[c] == a0)
						fb[c] = ab0, matched++;
					else if (fv[c] == a1)
						fb[c] = ab1, matched++;
				if (matched == 2)
					emit(b0, b1, fv[0], fv[1], fv[2], bb0, fb[0], fb[1], e2, g);
			}
		}
		return count;
	}

	uint oracle_region_match(const uint* lcsr, uint l, const uint* rcsr, uint r) { return region_match(lcsr, l, rcsr, r); }

	// filter_invalid_pairs: proximity pairs [0, n) of the narrow-phase list, in place
	void oracle_filter_invalid_pairs(void* pairs_v, const uint* pidx, uint n, uint num_ef, const float* x, const float* offset, uint nv,
		uint* invalid, const uint* vcsr, const uint* ecsr, const uint* fcsr)
	{
		if (num_ef == 0 || n == 0)
			return;
		PairT* pairs = static_cast<PairT*>(pairs_v);
		for (uint i = 0; i < n; i++)
		{
			const PairT& p = pairs[i];
			float w[4];
			pair_weight(p, w);
			V3 d = v3(0.0f);
			for (int k = 0; k < 4; k++)
			{
				const uint v = p.idx[k] & kMask;
				if (v < nv)
					d = d + w[k] * load3(x, v);
			}
			const float d2 = dot(d, d);
			const uint i0 = p.idx[0] & kMask, i2 = p.idx[2] & kMask;
			const float th = (i0 < nv ? offset[i0] : 0.0f) + (i2 < nv ? offset[i2] : 0.0f);
			if (d2 < th * th + 1e-10f)
				for (int k = 0; k < 4; k++)
				{
					const uint v = p.idx[k] & kMask;
					if (v < nv)
						invalid[v] = 1u;
				}
		}
		for (uint i = 0; i < n; i++)
		{
			PairT& p = pairs[i];
			bool off = false;
			for (int k = 0; k < 4; k++)
			{
				const uint v = p.idx[k] & kMask;
				if (v < nv && invalid[v] != 0u)
					off = true;
			}
			if (off)
			{
				p.vec2[0] = p.vec2[1] = 0.0f;
				continue;
			}
			if (!vcsr)
				continue;
			const uint t = pair_type(p);
			uint m = 0;
			if (t == 4u)
				m = region_match(vcsr, pidx[2 * i], fcsr, pidx[2 * i + 1]);
			else if (t == 8u)
				m = region_match(ecsr, pidx[2 * i], ecsr, pidx[2 * i + 1]);
			if (m == 1u)
				p.vec2[0] = p.vec2[1] = 0.0f;
		}
	}

	// filter_broad_phase_pairs: VF (vid, fid) and EE (eid1, eid2) lists, in place
	void oracle_filter_broad_phase(uint* vf, uint nvf, uint* ee, uint nee, uint num_ef, const uint* invalid, const uint* vcsr,
		const uint* ecsr, const uint* fcsr, const uint* faces, const uint* edges)
	{
		if (num_ef == 0 || !vcsr)
			return;
		for (uint i = 0; i < nvf; i++)
		{
			const uint v = vf[2 * i], f = vf[2 * i + 1];
			const bool near = invalid[v] || invalid[faces[3 * f]] || invalid[faces[3 * f + 1]] || invalid[faces[3 * f + 2]];
			const bool region = region_match(vcsr, v, fcsr, f) == 1u;
			const uint fl = (region ? 1u << 31 : 0u) | (near ? 1u << 30 : 0u);
			vf[2 * i] = v | fl;
			vf[2 * i + 1] = f | fl;
		}
		for (uint i = 0; i < nee; i++)
		{
			const uint a = ee[2 * i], b = ee[2 * i + 1];
			const bool near = invalid[edges[2 * a]] || invalid[edges[2 * a + 1]] || invalid[edges[2 * b]] || invalid[edges[2 * b + 1]];
			const bool region = region_match(ecsr, a, ecsr, b) == 1u;
			const uint fl = (region ? 1u << 31 : 0u) | (near ? 1u << 30 : 0u);
			ee[2 * i] = a | fl;
			ee[2 * i + 1] = b | fl;
		}
	}
}
