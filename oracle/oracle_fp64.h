// Test infrastructure: the FP64 recheck of the filtered FP32 predicates, restated on the CPU
// for the oracle (the checker of the CUDA path's recheck counts and FP64 metrics).
//
// A geometric test's FP32 decision compares FP32 quantities with thresholds. With u = 2^-24
// and the error factor g = 24 u (12 roundings along the longest dependency chain, doubled),
// each quantity q gets the bound e = g * M, M a magnitude bound of the expression built from
// 1- and inf-norms of its difference vectors. A test is rechecked in FP64 when none of its
// conditions certainly fails (q < -e) and one lies inside its band (|q| <= e); its decision in
// FP64 (same steps in double from the same float inputs) is then compared with the FP32 one.
// The sets keep the FP32 decisions. Compile with -ffp-contract=off (as the rest of the oracle).
#pragma once
#include "oracle_common.h"

namespace u26o
{
	constexpr float kGamma = 24.0f * 5.9604645e-08f;

	struct D3
	{
		double x, y, z;
	};
	inline D3 d3(V3 a) { return D3{ double(a.x), double(a.y), double(a.z) }; }
	inline D3 operator-(D3 a, D3 b) { return D3{ a.x - b.x, a.y - b.y, a.z - b.z }; }
	inline D3 operator+(D3 a, D3 b) { return D3{ a.x + b.x, a.y + b.y, a.z + b.z }; }
	inline D3 operator*(D3 a, double s) { return D3{ a.x * s, a.y * s, a.z * s }; }
	inline D3 neg(D3 a) { return D3{ -a.x, -a.y, -a.z }; }
	inline double dotd(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
	inline D3 crossd(D3 a, D3 b) { return D3{ a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }

	inline float l1(V3 a) { return (std::fabs(a.x) + std::fabs(a.y)) + std::fabs(a.z); }
	inline float linf(V3 a) { return std::fmax(std::fmax(std::fabs(a.x), std::fabs(a.y)), std::fabs(a.z)); }

	struct BandAcc
	{
		bool fail = false, in = false;
		void cond(float q, float e)
		{
			if (q < -e)
				fail = true;
			if (std::fabs(q) <= e)
				in = true;
		}
		bool recheck() const { return in && !fail; }
	};

	struct TriErr
	{
		float den, tnum, nu, nv, e_den, e_t, e_nu, e_nv;
	};

	// all seven conditions of the ray - triangle test on its FP32 numerators
	inline void tri_band(V3 start, V3 dir, float ray_len, V3 A, V3 B, V3 C, BandAcc& b, TriErr& te)
	{
		const V3 AB = B - A, AC = C - A;
		const V3 N = cross(AB, AC);
		const V3 ng = -dir;
		const float den = dot(ng, N);
		const V3 to_a = start - A;
		const float tnum = dot(to_a, N);
		const V3 cx = cross(ng, to_a);
		const float nu = dot(AC, cx), nv = -dot(AB, cx);
		const float sab = l1(AB), sac = l1(AC), sta = l1(to_a), sd = linf(ng), sd1 = l1(ng);
		const float e_den = kGamma * ((sd * sab) * sac);
		const float e_t = kGamma * ((sta * sab) * sac);
		const float e_nu = kGamma * ((sac * sd1) * sta);
		const float e_nv = kGamma * ((sab * sd1) * sta);
		const float s = den >= 0.0f ? 1.0f : -1.0f;
		const float ad = std::fabs(den);
		b.cond(tnum * s, e_t);
		b.cond(ray_len * ad - tnum * s, e_t + ray_len * e_den);
		b.cond(nu * s - 1e-6f * ad, e_nu + 1e-6f * e_den);
		b.cond((1.0f - 1e-6f) * ad - nu * s, e_nu + e_den);
		b.cond(nv * s - 1e-6f * ad, e_nv + 1e-6f * e_den);
		b.cond((1.0f - 1e-6f) * ad - (nu + nv) * s, (e_nu + e_nv) + e_den);
		b.cond(ad - 1e-6f * length(N), e_den + 1e-6f * (kGamma * (sab * sac)));
		te = TriErr{ den, tnum, nu, nv, e_den, e_t, e_nu, e_nv };
	}

	inline bool tri_f64(D3 start, D3 dir, double ray_len, D3 A, D3 B, D3 C, double& t_out, D3& bary)
	{
		const D3 AB = B - A, AC = C - A;
		const D3 N = crossd(AB, AC);
		const D3 ng = neg(dir);
		const double nlen = std::sqrt(dotd(N, N));
		const double den = dotd(ng, N);
		if (std::fabs(den) < nlen * double(1e-6f))
			return false;
		const D3 to_a = start - A;
		const double t = dotd(to_a, N) / den;
		if (t < 0.0 || t > ray_len)
			return false;
		const D3 cx = crossd(ng, to_a);
		const double uu = dotd(AC, cx) / den;
		if (uu < double(1e-6f) || uu > 1.0 - double(1e-6f))
			return false;
		const double vv = -dotd(AB, cx) / den;
		if (vv < double(1e-6f) || vv + uu > 1.0 - double(1e-6f))
			return false;
		t_out = t;
		bary = D3{ 1.0 - uu - vv, uu, vv };
		return true;
	}

	inline bool seg_tri_f64(D3 p0, D3 p1, D3 A, D3 B, D3 C, D3& bary, double& time)
	{
		const D3 d = p1 - p0;
		const double len_sq = dotd(d, d);
		if (len_sq < double(1e-6f) * double(1e-6f))
			return false;
		const double len = std::sqrt(len_sq);
		double t;
		if (!tri_f64(p0, d * (1.0 / len), len, A, B, C, t, bary))
			return false;
		time = t / len;
		return true;
	}

	// the segment p0 -> p1 as line_intersection normalises it
	inline bool seg_band(V3 p0, V3 p1, V3 A, V3 B, V3 C, BandAcc& b, TriErr& te, float& len)
	{
		const V3 d = p1 - p0;
		const float len_sq = length_sq(d);
		if (len_sq < 1e-6f * 1e-6f)
		{
			b.fail = true;
			return false;
		}
		len = std::sqrt(len_sq);
		tri_band(p0, d * (1.0f / len), len, A, B, C, b, te);
		return true;
	}

	// VF / FV leaf test of the ray casts: 1 rechecked, +2 flipped
	inline uint recheck_vert_face(V3 orig, V3 end, V3 A, V3 B, V3 C, bool hit32)
	{
		BandAcc b;
		TriErr te;
		float len;
		if (!seg_band(orig, end, A, B, C, b, te, len) || !b.recheck())
			return 0;
		D3 bary;
		double t;
		const bool h64 = seg_tri_f64(d3(orig), d3(end), d3(A), d3(B), d3(C), bary, t) && t >= 0.0 && t <= 1.0;
		return 1u | (h64 != hit32 ? 2u : 0u);
	}

	// EF test (segment test + grazing filters): 1 rechecked, +2 flipped
	inline uint recheck_ef(V3 pe0, V3 pe1, V3 A, V3 B, V3 C, bool seg32, float t_seg, V3 fb, bool pass32)
	{
		BandAcc b;
		TriErr te;
		float len;
		if (!seg_band(pe0, pe1, A, B, C, b, te, len))
			return 0;
		if (seg32)
		{
			const V3 n_un = cross(B - A, C - A);
			const float n_len = length(n_un);
			const float fc = std::sqrt(std::fmax(n_len, 1e-30f));
			const V3 n = n_un / std::fmax(n_len, 1e-30f);
			const float pen = std::fmin(std::fabs(dot(pe0 - A, n)), std::fabs(dot(pe1 - A, n)));
			const float e_pen = kGamma * std::fmax(l1(pe0 - A), l1(pe1 - A));
			b.cond(pen - 1e-4f * fc, e_pen + 1e-4f * (kGamma * fc));
			const float ad = std::fabs(te.den);
			const float e_uu = (te.e_nu + std::fabs(fb.y) * te.e_den) / ad + kGamma * std::fabs(fb.y);
			const float e_vv = (te.e_nv + std::fabs(fb.z) * te.e_den) / ad + kGamma * std::fabs(fb.z);
			b.cond(fb.x - 1e-4f, e_uu + e_vv);
			b.cond(fb.y - 1e-4f, e_uu);
			b.cond(fb.z - 1e-4f, e_vv);
			const float t_ray = t_seg * len;
			const float e_ts = ((te.e_t + std::fabs(t_ray) * te.e_den) / ad + kGamma * std::fabs(t_ray)) * (1.0f / len) +
				kGamma * std::fabs(t_seg);
			b.cond(t_seg - 1e-4f, e_ts);
			b.cond((1.0f - t_seg) - 1e-4f, e_ts);
		}
		if (!b.recheck())
			return 0;
		D3 fb64;
		double t64;
		bool pass64 = seg_tri_f64(d3(pe0), d3(pe1), d3(A), d3(B), d3(C), fb64, t64);
		if (pass64)
		{
			const D3 dA = d3(A);
			const D3 n_un = crossd(d3(B) - dA, d3(C) - dA);
			const double n_len = std::sqrt(dotd(n_un, n_un));
			const double fc = std::sqrt(std::fmax(n_len, 1e-30));
			const D3 n = n_un * (1.0 / std::fmax(n_len, 1e-30));
			const double pen = std::fmin(std::fabs(dotd(d3(pe0) - dA, n)), std::fabs(dotd(d3(pe1) - dA, n)));
			const double lim = double(1e-4f);
			pass64 = !(pen < lim * fc) && !(std::fmin(std::fmin(fb64.x, fb64.y), fb64.z) < lim) && std::fmin(t64, 1.0 - t64) >= lim;
		}
		return 1u | (pass64 != pass32 ? 2u : 0u);
	}

	// swept edge - edge leaf test: 1 rechecked, +2 flipped. pn, pd: the FP32 separating plane
	// (unit normal of e1 x dir and its offset), used when `plane`.
	inline uint recheck_edge_edge(V3 p0, V3 p1, V3 dir, float ray_max, bool plane, V3 pn, float pd, V3 q0, V3 q1, bool hit32)
	{
		BandAcc b;
		const V3 e1 = p1 - p0;
		if (plane)
		{
			const float d0 = dot(pn, q0) - pd, d1 = dot(pn, q1) - pd;
			const float e0 = kGamma * (l1(q0) + l1(p0)), e1b = kGamma * (l1(q1) + l1(p0));
			const bool above = (d0 - 1e-6f > e0) && (d1 - 1e-6f > e1b);
			const bool below = (-1e-6f - d0 > e0) && (-1e-6f - d1 > e1b);
			if (above || below)
				return 0;
			if (std::fabs(d0 - 1e-6f) <= e0 || std::fabs(d1 - 1e-6f) <= e1b || std::fabs(d0 + 1e-6f) <= e0 || std::fabs(d1 + 1e-6f) <= e1b)
				b.in = true;
		}
		const V3 e2v = q1 - q0, rr = q0 - p0;
		const V3 n = cross(e1, e2v);
		const float det = -dot(dir, n);
		const float n_sv = -dot(rr, n);
		const float n_t1 = -dot(dir, cross(rr, e2v));
		const float n_t2 = dot(dir, cross(e1, rr));
		const float s1 = l1(e1), s2 = l1(e2v), sr = l1(rr), sd = linf(dir);
		const float e_det = kGamma * ((sd * s1) * s2);
		const float e_sv = kGamma * ((linf(rr) * s1) * s2);
		const float e_t1 = kGamma * ((sd * sr) * s2);
		const float e_t2 = kGamma * ((sd * s1) * sr);
		const float s = det >= 0.0f ? 1.0f : -1.0f;
		const float ad = std::fabs(det);
		b.cond(ad - 1e-10f, e_det);
		b.cond(n_sv * s, e_sv);
		b.cond(ray_max * ad - n_sv * s, e_sv + ray_max * e_det);
		b.cond(n_t1 * s, e_t1);
		b.cond(ad - n_t1 * s, e_t1 + e_det);
		b.cond(n_t2 * s, e_t2);
		b.cond(ad - n_t2 * s, e_t2 + e_det);
		if (!b.recheck())
			return 0;
		// FP64 test, same steps
		const D3 P0 = d3(p0), P1 = d3(p1), Q0 = d3(q0), Q1 = d3(q1), Dd = d3(dir);
		const D3 E1 = P1 - P0;
		bool h64 = true;
		D3 PN = crossd(E1, Dd);
		const double nl = std::sqrt(dotd(PN, PN));
		if (nl >= double(1e-10f))
		{
			PN = PN * (1.0 / nl);
			const double PD = dotd(PN, P0);
			const double a0 = dotd(PN, Q0) - PD, a1 = dotd(PN, Q1) - PD;
			const double eps = double(1e-6f);
			if ((a0 > eps && a1 > eps) || (a0 < -eps && a1 < -eps))
				h64 = false;
		}
		if (h64)
		{
			const D3 E2 = Q1 - Q0, RR = Q0 - P0;
			const D3 NN = crossd(E1, E2);
			const double DET = -dotd(Dd, NN);
			if (std::fabs(DET) < double(1e-10f))
				h64 = false;
			else
			{
				const double sv = -dotd(RR, NN) / DET;
				const double t1 = -dotd(Dd, crossd(RR, E2)) / DET;
				const double t2 = dotd(Dd, crossd(E1, RR)) / DET;
				h64 = sv >= 0.0 && sv <= double(ray_max) && t1 >= 0.0 && t1 <= 1.0 && t2 >= 0.0 && t2 <= 1.0;
			}
		}
		return 1u | (h64 != hit32 ? 2u : 0u);
	}
} // namespace u26o
