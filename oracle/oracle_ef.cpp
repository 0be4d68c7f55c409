// Test infrastructure (oracle): CPU restatement of EF (edge-face) intersection detection.
//   Solver/CollisionDetector/intersection_resolver.cpp:86-197  fn_narrow_phase_ef_dcd_query
//   Solver/CollisionDetector/intersection_resolver_helper.cpp:319-514  RayTriangleIntersectionAndBary,
//       LineIntersection
//   Solver/CollisionDetector/intersection_resolver.cpp:693-726  canonical EF sort
//   Solver/SimulationCore/collision_data.h:150-220  EfPair layout (48 bytes)
// Loaded only by tests/ and bench.py's cpu_baseline leg.
#include "oracle_common.h"
#include "oracle_fp64.h"

using namespace u26o;

namespace u26o
{
	// helper.cpp:335-380 (scalar form). Returns true on a hit, writes t (in [0, ray_len]),
	// barycentrics (1-u-v, u, v).
	bool ray_triangle(V3 start, V3 dir, float ray_len, V3 A, V3 B, V3 C, float& out_t, V3& out_bary)
	{
		const V3 AB = B - A;
		const V3 AC = C - A;
		const V3 N = cross(AB, AC);
		const V3 neg = -dir;
		const float nlen = length(N);
		const float den = dot(neg, N);
		if (std::fabs(den) < nlen * 1e-6f)
			return false;
		const float inv_den = 1.0f / den;
		const V3 to_a = start - A;
		const float t = dot(to_a, N) * inv_den;
		if (t < 0.0f || t > ray_len)
			return false;
		const V3 cx = cross(neg, to_a);
		const float uu = dot(AC, cx) * inv_den;
		if (uu < 1e-6f || uu > (1.0f - 1e-6f))
			return false;
		const float vv = -dot(AB, cx) * inv_den;
		if (vv < 1e-6f || (vv + uu) > (1.0f - 1e-6f))
			return false;
		out_t = t;
		out_bary = v3(1.0f - uu - vv, uu, vv);
		return true;
	}

	// helper.cpp:452-482: segment -> triangle, time normalised to [0, 1].
	bool line_intersection(V3 p0, V3 p1, V3 A, V3 B, V3 C, V3& out_bary, float& out_time)
	{
		const V3 d = p1 - p0;
		const float len_sq = length_sq(d);
		if (len_sq < 1e-6f * 1e-6f)
			return false;
		const float len = std::sqrt(len_sq);
		const float inv_len = 1.0f / len;
		const V3 ray = d * inv_len;
		if (ray_triangle(p0, ray, len, A, B, C, out_time, out_bary))
		{
			out_time = out_time * inv_len;
			return true;
		}
		return false;
	}
} // namespace u26o

namespace
{
	struct EfPairRec
	{
		uint idx[5];
		float bary[3];
		float grad[3];
		float stiff;
	};
	static_assert(sizeof(EfPairRec) == 48, "EfPair is 48 bytes");

	inline bool vprop_fixed(uint p) { return (p & 1u) != 0; }
	inline bool vprop_rigid(uint p) { return (p & 2u) != 0; }
	inline uint vprop_object(uint p) { return (p >> 16) & 0x7FFFu; }

	// One broad-phase (eid, fid) pair through the narrow-phase filters. Returns true and
	// fills rec when it produces an EF pair.
	bool ef_test(uint eid, uint fid, const float* x, const uint* edges, const uint* faces, const uint* vprop,
		const float* d_hat, EfPairRec& rec)
	{
		const uint e0 = edges[2 * eid], e1 = edges[2 * eid + 1];
		const uint f0 = faces[3 * fid], f1 = faces[3 * fid + 1], f2 = faces[3 * fid + 2];
		if (e0 == f0 || e0 == f1 || e0 == f2 || e1 == f0 || e1 == f1 || e1 == f2)
			return false;
		const uint lp = vprop ? vprop[e0] : 0u;
		const uint rp = vprop ? vprop[f0] : 0u;
		if (vprop_fixed(lp) && vprop_fixed(rp))
			return false;
		if (vprop_rigid(lp) && vprop_rigid(rp) && vprop_object(lp) == vprop_object(rp))
			return false;
		if (d_hat[e0] + d_hat[f0] == 0.0f)
			return false;
		const V3 pe0 = load3(x, e0), pe1 = load3(x, e1);
		const V3 A = load3(x, f0), B = load3(x, f1), C = load3(x, f2);
		V3 fb;
		float t;
		if (!line_intersection(pe0, pe1, A, B, C, fb, t))
			return false;
		const V3 n_un = cross(B - A, C - A);
		const float n_len = length(n_un);
		const float face_char = std::sqrt(std::fmax(n_len, 1e-30f));
		const V3 n = n_un / std::fmax(n_len, 1e-30f);
		const float d0 = dot(pe0 - A, n);
		const float d1 = dot(pe1 - A, n);
		const float pen = std::fmin(std::fabs(d0), std::fabs(d1));
		if (pen < 1e-4f * face_char)
			return false;
		const float bmin = std::fmin(std::fmin(fb.x, fb.y), fb.z);
		if (bmin < 1e-4f)
			return false;
		const float tmin = std::fmin(t, 1.0f - t);
		if (tmin < 1e-4f)
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
} // namespace

extern "C"
{
	int oracle_line_intersection(const float* p0, const float* p1, const float* a, const float* b, const float* c,
		float* out_bary3, float* out_t)
	{
		V3 bary;
		float t;
		const bool hit = line_intersection(load3(p0, 0), load3(p1, 0), load3(a, 0), load3(b, 0), load3(c, 0), bary, t);
		if (hit)
		{
			out_bary3[0] = bary.x;
			out_bary3[1] = bary.y;
			out_bary3[2] = bary.z;
			*out_t = t;
		}
		return hit ? 1 : 0;
	}

	// Narrow phase over broad-phase pairs (uint2 eid, fid). Writes EF pairs (48-byte
	// records) and (eid, fid) indices in canonical order: sorted by (eid, fid, payload
	// bytes), as host_preprocess_ef_pairs does (intersection_resolver.cpp:693-726).
	// Returns the number of EF pairs (output truncated at max_out).
	uint oracle_ef_narrow(const uint* broad_pairs, uint num_broad, const float* x, const uint* edges, const uint* faces,
		const uint* vprop, const float* d_hat, void* out_pairs, uint* out_indices, uint max_out)
	{
		std::vector<uint8_t> hit(num_broad, 0);
		std::vector<EfPairRec> recs(num_broad);
		parallel_for(num_broad, [&](uint i)
			{ hit[i] = ef_test(broad_pairs[2 * i], broad_pairs[2 * i + 1], x, edges, faces, vprop, d_hat, recs[i]) ? 1 : 0; });
		std::vector<uint> order;
		for (uint i = 0; i < num_broad; i++)
			if (hit[i])
				order.push_back(i);
		std::sort(order.begin(), order.end(), [&](uint a, uint b)
			{
				const uint ea = broad_pairs[2 * a], eb = broad_pairs[2 * b];
				if (ea != eb) return ea < eb;
				const uint fa = broad_pairs[2 * a + 1], fb = broad_pairs[2 * b + 1];
				if (fa != fb) return fa < fb;
				return std::memcmp(&recs[a], &recs[b], sizeof(EfPairRec)) < 0; });
		const uint count = uint(order.size());
		EfPairRec* out = static_cast<EfPairRec*>(out_pairs);
		for (uint k = 0; k < count && k < max_out; k++)
		{
			out[k] = recs[order[k]];
			out_indices[2 * k] = broad_pairs[2 * order[k]];
			out_indices[2 * k + 1] = broad_pairs[2 * order[k] + 1];
		}
		return count;
	}

	// The FP64 recheck of the EF tests over broad-phase pairs (u26_ef_detect's stats[2..3]):
	// out[0] tests rechecked (FP32 decision inside its error band), out[1] FP32 / FP64 flips.
	void oracle_ef_recheck(const uint* broad_pairs, uint num_broad, const float* x, const uint* edges, const uint* faces,
		const uint* vprop, const float* d_hat, uint64_t* out)
	{
		std::vector<uint8_t> rc(num_broad, 0);
		parallel_for(num_broad, [&](uint i)
			{
				const uint eid = broad_pairs[2 * i], fid = broad_pairs[2 * i + 1];
				const uint e0 = edges[2 * eid], e1 = edges[2 * eid + 1];
				const uint f0 = faces[3 * fid], f1 = faces[3 * fid + 1], f2 = faces[3 * fid + 2];
				if (e0 == f0 || e0 == f1 || e0 == f2 || e1 == f0 || e1 == f1 || e1 == f2)
					return;
				const uint lp = vprop ? vprop[e0] : 0u;
				const uint rp = vprop ? vprop[f0] : 0u;
				if ((vprop_fixed(lp) && vprop_fixed(rp)) || (vprop_rigid(lp) && vprop_rigid(rp) && vprop_object(lp) == vprop_object(rp)))
					return;
				if (d_hat[e0] + d_hat[f0] == 0.0f)
					return;
				EfPairRec rec;
				const bool pass32 = ef_test(eid, fid, x, edges, faces, vprop, d_hat, rec);
				const V3 pe0 = load3(x, e0), pe1 = load3(x, e1), A = load3(x, f0), B = load3(x, f1), C = load3(x, f2);
				V3 fb = v3(0.0f);
				float t = 0.0f;
				const bool seg32 = line_intersection(pe0, pe1, A, B, C, fb, t);
				rc[i] = uint8_t(recheck_ef(pe0, pe1, A, B, C, seg32, t, fb, pass32));
			});
		out[0] = out[1] = 0;
		for (uint i = 0; i < num_broad; i++)
		{
			out[0] += rc[i] & 1u;
			out[1] += rc[i] >> 1;
		}
	}
}
