// Test infrastructure: CPU oracle for the Untangling26 collision/untangling hot path.
//
// This directory is the CHECKER, never the product. Only tests/, the smoke check in
// __graft_entry__.py and the cpu_baseline leg of bench.py may load it. The shipped
// path (untangling26_b200/libu26.so) does not link, include or call anything here.
//
// Arithmetic convention shared with the CUDA kernels (the canonical expression order):
//   dot(a,b)    = (a.x*b.x + a.y*b.y) + a.z*b.z        no FMA contraction
//   cross(a,b)  = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
//   length(v)   = sqrtf(dot(v,v))                       IEEE sqrt
//   normalize(v)= v * (1.0f / length(v))                IEEE divide
// The reference takes these from LuisaCompute, whose submodule is not checked out,
// so the expansion above is this build's definition ("parity unpinned" at the ulp
// level against the original binary; exact between oracle and CUDA path).
// Compile with -ffp-contract=off.
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <thread>
#include <vector>

namespace u26o
{
	using uint = uint32_t;

	struct V3
	{
		float x, y, z;
	};
	inline V3 v3(float x, float y, float z) { return V3{ x, y, z }; }
	inline V3 v3(float s) { return V3{ s, s, s }; }
	inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
	inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
	inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
	inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
	inline V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
	inline V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
	inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
	inline V3 vmin(V3 a, V3 b) { return v3(std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)); }
	inline V3 vmax(V3 a, V3 b) { return v3(std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)); }
	inline float dot(V3 a, V3 b)
	{
		float s = a.x * b.x;
		s = s + a.y * b.y;
		s = s + a.z * b.z;
		return s;
	}
	inline V3 cross(V3 a, V3 b)
	{
		return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
	}
	inline float length(V3 a) { return std::sqrt(dot(a, a)); }
	inline float length_sq(V3 a) { return dot(a, a); }
	inline V3 normalize(V3 a) { return a * (1.0f / length(a)); }
	inline float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

	inline V3 load3(const float* p, uint i) { return v3(p[3 * i + 0], p[3 * i + 1], p[3 * i + 2]); }

	// Fixed-size thread pool parallel_for over [0, n) in blocks of `block`
	// (the reference's fiber parallel_for uses block 256, cpu_parallel.h:481-605).
	int oracle_threads();
	void parallel_for(uint n, const std::function<void(uint)>& fn, uint block = 256);
} // namespace u26o
