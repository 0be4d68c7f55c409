// Filtered FP32 predicates with an FP64 recheck.
//
// The geometric tests of the path (the segment / ray - triangle test LineIntersection,
// intersection_resolver_helper.cpp:343-375 and 452-482; the EF grazing filters,
// intersection_resolver.cpp:86-197; the swept edge - edge test, cached_bvh.cpp:433-527) run
// in FP32 in the canonical expression order, and their FP32 decisions define the pair and hit
// sets (the reference's own sets). Each decision compares a quantity q computed in FP32 with a
// threshold. A static forward-error bound e on q (Higham's gamma_k times the same expression
// evaluated on magnitudes, here bounded through 1- and inf-norms of the difference vectors)
// says when the FP32 decision is certain: every condition is certain when |q - threshold| > e,
// and a test whose outcome is not fixed by a condition that certainly fails has a condition
// inside its band. Only those tests are re-evaluated in FP64 (same formula, double
// arithmetic, from the same float inputs); the recheck counts them and counts the flips
// (FP64 decision != FP32 decision). Set membership keeps the FP32 decision.
//
// gamma: the longest dependency chain of a decision quantity is 12 roundings (difference
// vectors, the ray direction's normalisation, cross and dot products, the comparison
// operand), and the bound is doubled for the evaluation of q itself: e = 24 u * magnitude,
// u = 2^-24.
#pragma once
#include "u26_common.cuh"

namespace u26
{
	constexpr float kBandGamma = 24.0f * 5.9604645e-08f;

	struct d3
	{
		double x, y, z;
	};
	__host__ __device__ __forceinline__ d3 dd(f3 a) { return d3{ double(a.x), double(a.y), double(a.z) }; }
	__host__ __device__ __forceinline__ d3 operator+(d3 a, d3 b) { return d3{ a.x + b.x, a.y + b.y, a.z + b.z }; }
	__host__ __device__ __forceinline__ d3 operator-(d3 a, d3 b) { return d3{ a.x - b.x, a.y - b.y, a.z - b.z }; }
	__host__ __device__ __forceinline__ d3 operator-(d3 a) { return d3{ -a.x, -a.y, -a.z }; }
	__host__ __device__ __forceinline__ d3 operator*(d3 a, double s) { return d3{ a.x * s, a.y * s, a.z * s }; }
	__host__ __device__ __forceinline__ double dot(d3 a, d3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
	__host__ __device__ __forceinline__ d3 cross(d3 a, d3 b)
	{
		return d3{ a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
	}

	__host__ __device__ __forceinline__ float norm1(f3 a) { return (fabsf(a.x) + fabsf(a.y)) + fabsf(a.z); }
	__host__ __device__ __forceinline__ float norm_inf(f3 a) { return fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fabsf(a.z)); }

	// one condition "q >= 0 passes" with error bound e: certainly fails / inside the band
	struct Band
	{
		bool fail = false, in = false;
		__host__ __device__ __forceinline__ void add(float q, float e)
		{
			fail = fail || q < -e;
			in = in || fabsf(q) <= e;
		}
		__host__ __device__ __forceinline__ bool recheck() const { return in && !fail; }
	};

	// FP32 numerators of ray_triangle and their error bounds
	struct TriTerms
	{
		float den, tnum, nu, nv, e_den, e_t, e_nu, e_nv;
	};

	// The band of ray_triangle(start, dir, ray_len, A, B, C): the parallel test, t in
	// [0, ray_len], uu and vv in [1e-6, 1 - 1e-6], uu + vv <= 1 - 1e-6, each written on the
	// FP32 numerators (t = tnum / den, uu = nu / den, vv = nv / den) so that no division
	// enters the bound.
	__host__ __device__ __forceinline__ void ray_triangle_band(f3 start, f3 dir, float ray_len, f3 A, f3 B, f3 C, Band& band, TriTerms& tt)
	{
		const f3 AB = B - A;
		const f3 AC = C - A;
		const f3 N = cross(AB, AC);
		const f3 neg = -dir;
		const float den = dot(neg, N);
		const f3 to_a = start - A;
		const float tnum = dot(to_a, N);
		const f3 cx = cross(neg, to_a);
		const float nu = dot(AC, cx), nv = -dot(AB, cx);
		const float nlen = length(N);
		const float sab = norm1(AB), sac = norm1(AC), sta = norm1(to_a), sd = norm_inf(neg), sd1 = norm1(neg);
		const float e_den = kBandGamma * ((sd * sab) * sac);
		const float e_nlen = kBandGamma * (sab * sac);
		const float e_t = kBandGamma * ((sta * sab) * sac);
		const float e_nu = kBandGamma * ((sac * sd1) * sta);
		const float e_nv = kBandGamma * ((sab * sd1) * sta);
		const float s = den >= 0.0f ? 1.0f : -1.0f;
		const float ad = fabsf(den);
		band.add(ad - 1e-6f * nlen, e_den + 1e-6f * e_nlen);							   // not parallel
		band.add(tnum * s, e_t);														   // t >= 0
		band.add(ray_len * ad - tnum * s, e_t + ray_len * e_den);						   // t <= ray_len
		band.add(nu * s - 1e-6f * ad, e_nu + 1e-6f * e_den);							   // uu >= 1e-6
		band.add((1.0f - 1e-6f) * ad - nu * s, e_nu + e_den);							   // uu <= 1 - 1e-6
		band.add(nv * s - 1e-6f * ad, e_nv + 1e-6f * e_den);							   // vv >= 1e-6
		band.add((1.0f - 1e-6f) * ad - (nu + nv) * s, (e_nu + e_nv) + e_den);			   // uu + vv <= 1 - 1e-6
		tt = TriTerms{ den, tnum, nu, nv, e_den, e_t, e_nu, e_nv };
	}

	// ray_triangle_band(...).recheck() for the ray-casting leaf tests, with the conditions
	// that need no square root first and an early exit when one of them certainly fails (the
	// common case); the same result as the full band, whatever the evaluation order.
	__host__ __device__ __forceinline__ bool tri_needs_recheck(f3 start, f3 dir, float ray_len, f3 A, f3 B, f3 C)
	{
		const f3 AB = B - A;
		const f3 AC = C - A;
		const f3 N = cross(AB, AC);
		const f3 neg = -dir;
		const float den = dot(neg, N);
		const f3 to_a = start - A;
		const float tnum = dot(to_a, N);
		const float sab = norm1(AB), sac = norm1(AC), sta = norm1(to_a);
		const float s = den >= 0.0f ? 1.0f : -1.0f;
		const float ad = fabsf(den);
		const float e_t = kBandGamma * ((sta * sab) * sac);
		const float e_den = kBandGamma * ((norm_inf(neg) * sab) * sac);
		Band bd;
		bd.add(tnum * s, e_t);
		bd.add(ray_len * ad - tnum * s, e_t + ray_len * e_den);
		if (bd.fail)
			return false;
		const f3 cx = cross(neg, to_a);
		const float nu = dot(AC, cx), nv = -dot(AB, cx);
		const float sd1 = norm1(neg);
		const float e_nu = kBandGamma * ((sac * sd1) * sta);
		const float e_nv = kBandGamma * ((sab * sd1) * sta);
		bd.add(nu * s - 1e-6f * ad, e_nu + 1e-6f * e_den);
		bd.add((1.0f - 1e-6f) * ad - nu * s, e_nu + e_den);
		bd.add(nv * s - 1e-6f * ad, e_nv + 1e-6f * e_den);
		bd.add((1.0f - 1e-6f) * ad - (nu + nv) * s, (e_nu + e_nv) + e_den);
		if (bd.fail)
			return false;
		bd.add(ad - 1e-6f * length(N), e_den + 1e-6f * (kBandGamma * (sab * sac)));
		return bd.recheck();
	}

	// ray_triangle in FP64 (same steps). Returns the hit, its t and barycentres.
	__host__ __device__ __forceinline__ bool ray_triangle_f64(d3 start, d3 dir, double ray_len, d3 A, d3 B, d3 C, double& out_t, d3& out_bary)
	{
		const d3 AB = B - A;
		const d3 AC = C - A;
		const d3 N = cross(AB, AC);
		const d3 neg = -dir;
		const double nlen = sqrt(dot(N, N));
		const double den = dot(neg, N);
		if (fabs(den) < nlen * double(1e-6f))
			return false;
		const d3 to_a = start - A;
		const double t = dot(to_a, N) / den;
		if (t < 0.0 || t > ray_len)
			return false;
		const d3 cx = cross(neg, to_a);
		const double uu = dot(AC, cx) / den;
		if (uu < double(1e-6f) || uu > 1.0 - double(1e-6f))
			return false;
		const double vv = -dot(AB, cx) / den;
		if (vv < double(1e-6f) || vv + uu > 1.0 - double(1e-6f))
			return false;
		out_t = t;
		out_bary = d3{ 1.0 - uu - vv, uu, vv };
		return true;
	}

	// LineIntersection in FP64: segment p0 -> p1, time in [0, 1].
	__host__ __device__ __forceinline__ bool line_intersection_f64(d3 p0, d3 p1, d3 A, d3 B, d3 C, d3& out_bary, double& out_time)
	{
		const d3 d = p1 - p0;
		const double len_sq = dot(d, d);
		if (len_sq < double(1e-6f) * double(1e-6f))
			return false;
		const double len = sqrt(len_sq);
		double t;
		if (!ray_triangle_f64(p0, d * (1.0 / len), len, A, B, C, t, out_bary))
			return false;
		out_time = t / len;
		return true;
	}

	// The swept edge - edge test's band: the separating plane of the swept edge (when it
	// has one), |det| >= 1e-10, s in [0, ray_max], t1 and t2 in [0, 1], on the numerators.
	// pn is the unit plane normal and pd its offset as the FP32 test computed them.
	__host__ __device__ __forceinline__ void edge_edge_band(f3 p0, f3 e1, f3 dir, float ray_max, bool plane, f3 pn, float pd, f3 q0,
		f3 q1, Band& band)
	{
		if (plane)
		{
			// d = dot(pn, q) - pd: magnitudes |q|, |p0| (pn is a unit vector)
			const float d0 = dot(pn, q0) - pd, d1 = dot(pn, q1) - pd;
			const float e0 = kBandGamma * (norm1(q0) + norm1(p0)), e1b = kBandGamma * (norm1(q1) + norm1(p0));
			// "not separated": not (both above 1e-6) and not (both below -1e-6)
			const bool above = (d0 - 1e-6f > e0) && (d1 - 1e-6f > e1b);
			const bool below = (-1e-6f - d0 > e0) && (-1e-6f - d1 > e1b);
			if (above || below)
				band.fail = true;
			else if (fabsf(d0 - 1e-6f) <= e0 || fabsf(d1 - 1e-6f) <= e1b || fabsf(d0 + 1e-6f) <= e0 || fabsf(d1 + 1e-6f) <= e1b)
				band.in = true;
		}
		if (band.fail)
			return; // certainly separated: the remaining conditions cannot change the outcome
		// the remaining conditions in turn, each numerator computed when it is needed and an
		// early return once one certainly fails (the common case: a miss): a failed condition
		// decides the band whatever the others give, so the result is the full band's
		const f3 e2v = q1 - q0;
		const f3 rr = q0 - p0;
		const f3 n = cross(e1, e2v);
		const float det = -dot(dir, n);
		const float s1 = norm1(e1), s2 = norm1(e2v), sd = norm_inf(dir);
		const float e_det = kBandGamma * ((sd * s1) * s2);
		const float s = det >= 0.0f ? 1.0f : -1.0f;
		const float ad = fabsf(det);
		band.add(ad - 1e-10f, e_det); // |det| >= 1e-10
		const float n_sv = -dot(rr, n);
		const float e_sv = kBandGamma * ((norm_inf(rr) * s1) * s2);
		band.add(n_sv * s, e_sv);								// s >= 0
		band.add(ray_max * ad - n_sv * s, e_sv + ray_max * e_det); // s <= ray_max
		if (band.fail)
			return;
		const float sr = norm1(rr);
		const float n_t1 = -dot(dir, cross(rr, e2v));
		const float e_t1 = kBandGamma * ((sd * sr) * s2);
		band.add(n_t1 * s, e_t1);			 // t1 >= 0
		band.add(ad - n_t1 * s, e_t1 + e_det); // t1 <= 1
		if (band.fail)
			return;
		const float n_t2 = dot(dir, cross(e1, rr));
		const float e_t2 = kBandGamma * ((sd * s1) * sr);
		band.add(n_t2 * s, e_t2);			 // t2 >= 0
		band.add(ad - n_t2 * s, e_t2 + e_det); // t2 <= 1
	}

	// The swept edge - edge test in FP64 (same steps as the FP32 test).
	__host__ __device__ __forceinline__ bool edge_edge_f64(d3 p0, d3 p1, d3 dir, double ray_max, d3 q0, d3 q1)
	{
		const d3 e1 = p1 - p0;
		d3 pn = cross(e1, dir);
		const double nl = sqrt(dot(pn, pn));
		if (nl >= double(1e-10f))
		{
			pn = pn * (1.0 / nl);
			const double pd = dot(pn, p0);
			const double d0 = dot(pn, q0) - pd, d1 = dot(pn, q1) - pd;
			const double eps = double(1e-6f);
			if ((d0 > eps && d1 > eps) || (d0 < -eps && d1 < -eps))
				return false;
		}
		const d3 e2v = q1 - q0;
		const d3 rr = q0 - p0;
		const d3 n = cross(e1, e2v);
		const double det = -dot(dir, n);
		if (fabs(det) < double(1e-10f))
			return false;
		const double sv = -dot(rr, n) / det;
		const double t1 = -dot(dir, cross(rr, e2v)) / det;
		const double t2 = dot(dir, cross(e1, rr)) / det;
		return sv >= 0.0 && sv <= ray_max && t1 >= 0.0 && t1 <= 1.0 && t2 >= 0.0 && t2 <= 1.0;
	}

	// The band of the EF test (fn_narrow_phase_ef_dcd_query's segment test and grazing
	// filters) of segment pe0 -> pe1 against triangle ABC. hit32: the FP32 segment test's
	// outcome; when it hit, t_seg and fb are its segment time and barycentres, and the three
	// filters (penetration >= 1e-4 sqrt|N|, every barycentre >= 1e-4, min(t, 1 - t) >= 1e-4)
	// join the band.
	__host__ __device__ __forceinline__ void ef_pair_band(f3 pe0, f3 pe1, f3 A, f3 B, f3 C, bool hit32, float t_seg, f3 fb, Band& band)
	{
		const f3 d = pe1 - pe0;
		const float len_sq = length_sq(d);
		if (len_sq < 1e-6f * 1e-6f)
		{
			band.fail = true; // degenerate segment: rejected on an exact zero-length test
			return;
		}
		const float len = sqrtf(len_sq);
		const float inv_len = 1.0f / len;
		const f3 ray = d * inv_len;
		TriTerms tt;
		ray_triangle_band(pe0, ray, len, A, B, C, band, tt);
		if (!hit32)
			return;
		const f3 n_un = cross(B - A, C - A);
		const float n_len = length(n_un);
		const float fc = sqrtf(fmaxf(n_len, 1e-30f));
		const f3 n = n_un / fmaxf(n_len, 1e-30f);
		const float pen = fminf(fabsf(dot(pe0 - A, n)), fabsf(dot(pe1 - A, n)));
		const float e_pen = kBandGamma * fmaxf(norm1(pe0 - A), norm1(pe1 - A));
		band.add(pen - 1e-4f * fc, e_pen + 1e-4f * (kBandGamma * fc));
		const float ad = fabsf(tt.den);
		const float uu = fb.y, vv = fb.z;
		const float e_uu = (tt.e_nu + fabsf(uu) * tt.e_den) / ad + kBandGamma * fabsf(uu);
		const float e_vv = (tt.e_nv + fabsf(vv) * tt.e_den) / ad + kBandGamma * fabsf(vv);
		band.add(fb.x - 1e-4f, e_uu + e_vv);
		band.add(uu - 1e-4f, e_uu);
		band.add(vv - 1e-4f, e_vv);
		const float t_ray = t_seg * len;
		const float e_ts = ((tt.e_t + fabsf(t_ray) * tt.e_den) / ad + kBandGamma * fabsf(t_ray)) * inv_len + kBandGamma * fabsf(t_seg);
		band.add(t_seg - 1e-4f, e_ts);
		band.add((1.0f - t_seg) - 1e-4f, e_ts);
	}

	// The EF test in FP64: the segment test and the three grazing filters.
	__host__ __device__ __forceinline__ bool ef_pair_f64(d3 pe0, d3 pe1, d3 A, d3 B, d3 C)
	{
		d3 fb;
		double t;
		if (!line_intersection_f64(pe0, pe1, A, B, C, fb, t))
			return false;
		const d3 n_un = cross(B - A, C - A);
		const double n_len = sqrt(dot(n_un, n_un));
		const double fc = sqrt(fmax(n_len, 1e-30));
		const d3 n = n_un * (1.0 / fmax(n_len, 1e-30));
		const double pen = fmin(fabs(dot(pe0 - A, n)), fabs(dot(pe1 - A, n)));
		const double lim = double(1e-4f);
		if (pen < lim * fc)
			return false;
		if (fmin(fmin(fb.x, fb.y), fb.z) < lim)
			return false;
		return fmin(t, 1.0 - t) >= lim;
	}
} // namespace u26
