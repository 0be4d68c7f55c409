// Differentiation of the PRP objective over fixed supports S(r) on sm_100a.
//
// For each contour c with support S (the selected hits of u26_prp_resolve) and direction r:
//   delta_h(x, r) = (w_h . n_h) / (r . n_h)    (the ray distance of hit h)
//     VF: w = a - p, n = (b - a) x (c - a)   (vertex p along +r onto face abc)
//     FV: w = q - a, n = (b - a) x (c - a)   (vertex q along -r onto face abc)
//     EE: w = q0 - p0, n = (p1 - p0) x (q1 - q0)   (edge p0p1 swept along r onto q0q1)
//   J = (sum_h A_h) * D^2, D = max_h delta_h      (prp_eval_penetration_v2's objective,
//                                                   intersection_resolver2.cpp:1883-1954)
//   E = sum_h (delta_h + 3e-3)^2 / kappa_h         (its displacement cost; kappa_h the
//                                                   effective inverse mass, helper.cpp:611-645)
// The adjoint gives dJ/dr, dE/dr and dJ/dx, dE/dx: with g = 1 / (r . n), u = w - delta r,
//   d delta / dr = -delta n g
//   VF: d/dp = -n g, d/da = (n + u x (c - b)) g, d/db = ((c - a) x u) g, d/dc = (u x (b - a)) g
//   FV: d/dq =  n g, d/da = (-n + u x (c - b)) g, d/db, d/dc as VF
//   EE: d/dp0 = (-n - e2 x u) g, d/dp1 = (e2 x u) g, d/dq0 = (n - u x e1) g, d/dq1 = (u x e1) g
// (e1 = p1 - p0, e2 = q1 - q0). J's subgradient goes through the argmax hit (the first in
// key order among equal maxima); A_h and kappa_h are constants of the support (rest areas,
// masses and the stored barycentric coordinates). dE/dr is the gradient the reference's
// direction refinement builds (intersection_resolver2.cpp:1268-1320).
#include "u26_internal.h"

namespace u26
{
	namespace
	{
		struct HitGeo
		{
			f3 P[4];	   // the hit's vertices: VF p a b c, FV q a b c, EE p0 p1 q0 q1
			uint32_t V[4]; // their ids
			f3 n, w;
			float rn, delta;
		};

		__device__ __forceinline__ HitGeo hit_geo(const u26_prp_hit& h, const float* __restrict__ x, f3 r)
		{
			HitGeo G;
			if (h.type == 1u)
			{
				G.V[0] = h.src_verts[0];
				G.V[1] = h.src_verts[1];
				G.V[2] = h.dst_verts[0];
				G.V[3] = h.dst_verts[1];
			}
			else if (h.type == 0u)
			{
				G.V[0] = h.src_verts[0];
				G.V[1] = h.dst_verts[0];
				G.V[2] = h.dst_verts[1];
				G.V[3] = h.dst_verts[2];
			}
			else
			{
				G.V[0] = h.dst_verts[0];
				G.V[1] = h.src_verts[0];
				G.V[2] = h.src_verts[1];
				G.V[3] = h.src_verts[2];
			}
#pragma unroll
			for (int k = 0; k < 4; k++)
				G.P[k] = ld3(x, G.V[k]);
			if (h.type == 1u)
			{
				G.n = cross(G.P[1] - G.P[0], G.P[3] - G.P[2]);
				G.w = G.P[2] - G.P[0];
			}
			else
			{
				G.n = cross(G.P[2] - G.P[1], G.P[3] - G.P[1]);
				G.w = h.type == 0u ? G.P[1] - G.P[0] : G.P[0] - G.P[1];
			}
			G.rn = dot(r, G.n);
			G.delta = dot(G.w, G.n) / G.rn;
			return G;
		}

		// coefficient * d delta / d(vertex k), k = 0..3 in HitGeo order
		__device__ __forceinline__ void delta_vertex_grads(uint32_t type, const HitGeo& G, f3 r, float coef, f3 out[4])
		{
			const float g = coef / G.rn;
			const f3 u = G.w - r * G.delta;
			if (type == 1u)
			{
				const f3 e1 = G.P[1] - G.P[0], e2 = G.P[3] - G.P[2];
				const f3 e2u = cross(e2, u), ue1 = cross(u, e1);
				out[0] = (-G.n - e2u) * g;
				out[1] = e2u * g;
				out[2] = (G.n - ue1) * g;
				out[3] = ue1 * g;
				return;
			}
			const f3 A = G.P[1], B = G.P[2], C = G.P[3];
			const f3 sgn_n = type == 0u ? G.n : -G.n; // d w / d a: +1 for VF (w = a - p), -1 for FV (w = q - a)
			out[0] = (type == 0u ? -G.n : G.n) * g;
			out[1] = (sgn_n + cross(u, C - B)) * g;
			out[2] = cross(C - A, u) * g;
			out[3] = cross(u, B - A) * g;
		}

		__device__ __forceinline__ float hit_area(const u26_prp_hit& h, const float* __restrict__ va, const float* __restrict__ ea,
			const float* __restrict__ fa)
		{
			return h.type == 0u ? va[h.src_id] : (h.type == 1u ? ea[h.src_id] : fa[h.src_id]);
		}

		__device__ __forceinline__ float hit_kappa(const u26_prp_hit& h, const float* __restrict__ vert_mass)
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

		__device__ __forceinline__ void add3(float* __restrict__ gx, uint32_t v, f3 g)
		{
			atomicAdd(gx + 3 * size_t(v), g.x);
			atomicAdd(gx + 3 * size_t(v) + 1, g.y);
			atomicAdd(gx + 3 * size_t(v) + 2, g.z);
		}

		// One warp per contour: forward J, E (canonical 32-lane strided sums), then the
		// vector-Jacobian products for the upstream gradients gJ, gE (when given).
		__global__ void adjoint_kernel(const float* __restrict__ x, const u26_prp_hit* __restrict__ hits, const uint32_t* __restrict__ off,
			uint32_t nc, const float* __restrict__ dirs, const float* __restrict__ va, const float* __restrict__ ea, const float* __restrict__ fa,
			const float* __restrict__ vm, float* __restrict__ J_out, float* __restrict__ E_out, const float* __restrict__ gJ,
			const float* __restrict__ gE, float* __restrict__ grad_dirs, float* __restrict__ grad_x)
		{
			const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
			const int lane = threadIdx.x & 31;
			if (c >= nc)
				return;
			const uint32_t h0 = off[c], h1 = off[c + 1];
			const f3 r = mk3(dirs[3 * c], dirs[3 * c + 1], dirs[3 * c + 2]);
			float sA = 0.0f, sE = 0.0f, dmax = -INFINITY;
			uint32_t imax = kInvalid;
			for (uint32_t i = h0 + lane; i < h1; i += 32)
			{
				const u26_prp_hit h = hits[i];
				const HitGeo G = hit_geo(h, x, r);
				sA = sA + hit_area(h, va, ea, fa);
				const float kap = hit_kappa(h, vm);
				const float sd = G.delta + 3e-3f;
				sE = sE + (kap > 1e-8f ? (sd * sd) / kap : 0.0f);
				if (G.delta > dmax || imax == kInvalid)
				{
					dmax = G.delta;
					imax = i;
				}
			}
#pragma unroll
			for (int o = 16; o >= 1; o >>= 1)
			{
				sA = sA + __shfl_xor_sync(0xFFFFFFFFu, sA, o);
				sE = sE + __shfl_xor_sync(0xFFFFFFFFu, sE, o);
				const float od = __shfl_xor_sync(0xFFFFFFFFu, dmax, o);
				const uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, imax, o);
				if (oi != kInvalid && (imax == kInvalid || od > dmax || (od == dmax && oi < imax)))
				{
					dmax = od;
					imax = oi;
				}
			}
			const float D = h1 > h0 ? dmax : 0.0f;
			if (lane == 0)
			{
				if (J_out)
					J_out[c] = (sA * D) * D;
				if (E_out)
					E_out[c] = sE;
			}
			if (!grad_dirs && !grad_x)
				return;
			const float gj = gJ ? gJ[c] : 0.0f, ge = gE ? gE[c] : 0.0f;
			f3 gr = mk3(0.0f);
			for (uint32_t i = h0 + lane; i < h1; i += 32)
			{
				const u26_prp_hit h = hits[i];
				const HitGeo G = hit_geo(h, x, r);
				float coef = 0.0f;
				if (ge != 0.0f)
				{
					const float kap = hit_kappa(h, vm);
					if (kap > 1e-8f)
						coef = ge * (2.0f * (G.delta + 3e-3f) / kap);
				}
				if (i == imax && gj != 0.0f)
					coef = coef + gj * (2.0f * sA * D);
				if (coef == 0.0f)
					continue;
				gr = gr + G.n * (-G.delta * coef / G.rn);
				if (grad_x)
				{
					f3 gv[4];
					delta_vertex_grads(h.type, G, r, coef, gv);
#pragma unroll
					for (int k = 0; k < 4; k++)
						add3(grad_x, G.V[k], gv[k]);
				}
			}
#pragma unroll
			for (int o = 16; o >= 1; o >>= 1)
			{
				gr.x = gr.x + __shfl_xor_sync(0xFFFFFFFFu, gr.x, o);
				gr.y = gr.y + __shfl_xor_sync(0xFFFFFFFFu, gr.y, o);
				gr.z = gr.z + __shfl_xor_sync(0xFFFFFFFFu, gr.z, o);
			}
			if (lane == 0 && grad_dirs)
			{
				grad_dirs[3 * c] = gr.x;
				grad_dirs[3 * c + 1] = gr.y;
				grad_dirs[3 * c + 2] = gr.z;
			}
		}
	} // namespace
} // namespace u26

using namespace u26;

U26_API u26_status u26_prp_adjoint(u26_ctx* ctx, const float* x, const u26_prp_hit* hits, const uint32_t* hit_offsets, uint32_t num_contours,
	const float* dirs, const float* vert_area, const float* edge_area, const float* face_area, const float* vert_mass, float* J, float* E,
	const float* grad_J, const float* grad_E, float* grad_dirs, float* grad_x)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (num_contours == 0)
		return U26_OK;
	if (!x || !hits || !hit_offsets || !dirs || !vert_area || !edge_area || !face_area || !vert_mass)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_prp_adjoint: null input");
	adjoint_kernel<<<div_up(32 * num_contours, 256), 256, 0, ctx->stream>>>(x, hits, hit_offsets, num_contours, dirs, vert_area, edge_area,
		face_area, vert_mass, J, E, grad_J, grad_E, grad_dirs, grad_x);
	return after_launch(ctx, "adjoint_kernel");
}
