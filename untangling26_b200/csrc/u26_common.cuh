// Shared device helpers for the sm_100a kernels of libu26.
//
// Arithmetic follows one canonical expression order so that every geometric decision
// is reproducible bit for bit on the host (the library is compiled with --fmad=false,
// so a*b+c is two IEEE roundings; sqrtf and '/' are IEEE, no fast-math):
//   dot(a,b)     = (a.x*b.x + a.y*b.y) + a.z*b.z
//   cross(a,b)   = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
//   length(v)    = sqrtf(dot(v,v));  normalize(v) = v * (1/length(v))
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/u26.h"

namespace u26
{
	using uint = uint32_t;

	struct f3
	{
		float x, y, z;
	};

	__host__ __device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{ x, y, z }; }
	__host__ __device__ __forceinline__ f3 mk3(float s) { return f3{ s, s, s }; }
	__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
	__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
	__host__ __device__ __forceinline__ f3 operator-(f3 a) { return mk3(-a.x, -a.y, -a.z); }
	__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
	__host__ __device__ __forceinline__ f3 operator*(float s, f3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
	__host__ __device__ __forceinline__ f3 operator*(f3 a, f3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
	__host__ __device__ __forceinline__ f3 operator/(f3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
	__host__ __device__ __forceinline__ f3 vmin(f3 a, f3 b) { return mk3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
	__host__ __device__ __forceinline__ f3 vmax(f3 a, f3 b) { return mk3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
	__host__ __device__ __forceinline__ float dot(f3 a, f3 b)
	{
		float s = a.x * b.x;
		s = s + a.y * b.y;
		s = s + a.z * b.z;
		return s;
	}
	__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b)
	{
		return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
	}
	__host__ __device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
	__host__ __device__ __forceinline__ float length_sq(f3 a) { return dot(a, a); }
	__host__ __device__ __forceinline__ f3 normalize(f3 a) { return a * (1.0f / length(a)); }

	__device__ __forceinline__ f3 ld3(const float* __restrict__ p, uint i)
	{
		return mk3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
	}

	// Node AABB as the reference stores it: two float4 (min.xyz, flag) (max.xyz, flag).
	struct __align__(16) NodeBox
	{
		float4 mn;
		float4 mx;
	};

	// aabb.h:94-98: strict overlap on all three axes.
	__device__ __forceinline__ bool overlap_strict(const NodeBox& b, f3 qmn, f3 qmx)
	{
		return (b.mn.x < qmx.x) & (b.mn.y < qmx.y) & (b.mn.z < qmx.z) & (b.mx.x > qmn.x) & (b.mx.y > qmn.y) & (b.mx.z > qmn.z);
	}

	constexpr uint kInvalid = 0xFFFFFFFFu;

	inline uint div_up(uint a, uint b) { return (a + b - 1u) / b; }
	inline uint64_t div_up64(uint64_t a, uint64_t b) { return (a + b - 1u) / b; }
} // namespace u26

// Error-status word shared by kernels and read by the host (bit flags).
#define U26_DEVERR_UNHEALTHY 1u
#define U26_DEVERR_ITERATION_CAP 2u
#define U26_DEVERR_STACK_OVERFLOW 4u
