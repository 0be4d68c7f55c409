// Host-side internals of libu26: the context object, grow-only device buffers and
// error plumbing shared by the .cu translation units.
#pragma once
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "u26_common.cuh"

struct u26_ctx
{
	int device = 0;
	cudaStream_t stream = nullptr;
	std::string last_error;
	uint64_t launches = 0;
	// device word the kernels OR error flags into (U26_DEVERR_*)
	uint32_t* dev_err = nullptr;
	// pinned host staging word for small readbacks
	uint32_t* host_word = nullptr;
	// device address of the allocation-free EF sort's static scratch, looked up by the first
	// u26_ef_canonicalize_noalloc call on this context
	unsigned char* noalloc_scratch = nullptr;
};

namespace u26
{
	// device and pinned-host allocations the library has made (u26_alloc_count)
	extern std::atomic<uint64_t> g_alloc_count;

	// Grow-only device allocation owned by a context-side object.
	struct DevBuf
	{
		void* ptr = nullptr;
		size_t bytes = 0;
		cudaError_t reserve(size_t want)
		{
			if (want <= bytes)
				return cudaSuccess;
			if (ptr)
				cudaFree(ptr);
			ptr = nullptr;
			bytes = 0;
			cudaError_t e = cudaMalloc(&ptr, want);
			if (e == cudaSuccess)
			{
				bytes = want;
				g_alloc_count.fetch_add(1, std::memory_order_relaxed);
			}
			return e;
		}
		void release()
		{
			if (ptr)
				cudaFree(ptr);
			ptr = nullptr;
			bytes = 0;
		}
		template <typename T>
		T* as() const { return static_cast<T*>(ptr); }
	};

	inline u26_status set_error(u26_ctx* ctx, u26_status st, const char* fmt, ...)
	{
		char buf[512];
		va_list ap;
		va_start(ap, fmt);
		vsnprintf(buf, sizeof(buf), fmt, ap);
		va_end(ap);
		if (ctx)
			ctx->last_error = buf;
		return st;
	}

	inline u26_status cuda_status(u26_ctx* ctx, cudaError_t e, const char* what)
	{
		if (e == cudaSuccess)
			return U26_OK;
		return set_error(ctx, U26_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
	}

	// Check the last launch; counts it.
	inline u26_status after_launch(u26_ctx* ctx, const char* what)
	{
		ctx->launches++;
		return cuda_status(ctx, cudaGetLastError(), what);
	}

	// Radix sort of (key64, value32) pairs over bits [bit_lo, bit_hi), stable.
	// keys/vals are sorted in place (ping-pong through internal scratch).
	// Exclusive scan of v[0, n) in place on ctx's stream; tmp is grown to the scratch it needs.
	u26_status device_exclusive_scan(u26_ctx* ctx, uint32_t* v, uint32_t n, DevBuf& tmp);

	struct RadixSorter
	{
		DevBuf keys_alt, vals_alt, counts, scan_tmp;
		u26_status sort(u26_ctx* ctx, uint64_t* keys, uint32_t* vals, uint32_t n, int bit_lo, int bit_hi);
		// Same passes over caller-provided scratch (allocates nothing): keys_alt/vals_alt hold
		// n entries, counts holds 256 * ceil(n / 2048) words. The result ends in keys/vals.
		static u26_status sort_into(u26_ctx* ctx, uint64_t* keys, uint32_t* vals, uint32_t n, int bit_lo, int bit_hi,
			uint64_t* keys_alt, uint32_t* vals_alt, uint32_t* counts);
		void release()
		{
			keys_alt.release();
			vals_alt.release();
			counts.release();
			scan_tmp.release();
		}
	};

	// Canonical EF order, ties: equal sorted keys put their permutation entries in memcmp order
	// of the 48-byte records recs[perm[i]] (ef.cu).
	u26_status ef_tiebreak(u26_ctx* ctx, const uint64_t* sorted_keys, uint32_t* perm, uint32_t count, const void* recs);

	// Response assembly of one PRP pass (response.cu): host-side results of the pass and the
	// scene's device tables.
	struct ResponseInputs
	{
		const u26_prp_hit* hits; // host [nh], contour order
		const uint32_t* hit_off; // host [nc + 1]
		const u26_prp_result* results; // host [nc]: dir, depth
		const uint32_t *pair_idx, *mesh_index, *contour_index; // host EF pairs [np]
		uint32_t nh, nc, np, nv, ne, nf;
		const float *fn, *en, *vn, *va, *ea, *fa; // device normals and rest areas
		const uint2* edges;
		const uint32_t* faces;
	};
	struct ResponseState
	{
		DevBuf hits, off, cinfo, efp, pairs, info, keys, ukeys, vals, flags, voff, ecnt, fcnt, vcsr, ecsr, fcsr, scan_tmp;
		RadixSorter sorter;
		uint32_t num_pairs = 0, vert_len = 0, edge_len = 0, face_len = 0;
		void release()
		{
			DevBuf* b[] = { &hits, &off, &cinfo, &efp, &pairs, &info, &keys, &ukeys, &vals, &flags, &voff, &ecnt, &fcnt, &vcsr, &ecsr, &fcsr, &scan_tmp };
			for (DevBuf* x : b)
				x->release();
			sorter.release();
		}
	};
	// narrow / narrow_idx: optional narrow-phase list slots (already offset to the first free one)
	u26_status response_run(u26_ctx* ctx, const ResponseInputs& in, float depth_threshold, float stiffness, ResponseState& R,
		u26_collision_pair* narrow, uint32_t* narrow_idx);
} // namespace u26

#define U26_TRY(expr)                   \
	do                                  \
	{                                   \
		u26_status _st = (expr);        \
		if (_st != U26_OK)              \
			return _st;                 \
	}                                   \
	while (0)

#define U26_CUDA(ctx, call) U26_TRY(::u26::cuda_status((ctx), (call), #call))
