// Allocation-free variant of the canonical EF sort (u26_ef_canonicalize).
//
// Some callers cannot let a library allocate device memory: a solver that owns all of
// its GPU memory in a fixed arena, or a host loop that must not run cudaMalloc/cudaFree
// because those calls can synchronise the whole device. For them this entry point does
// the same work as u26_ef_canonicalize with its scratch in a fixed-size array that lives
// in the library image (static device memory). Every GPU that loads libu26 holds this
// array (U26_NOALLOC_SCRATCH_BYTES, about 2.6 MB) until the process exits.
//
// The caller still passes the EF pairs and indices, which are sorted in place.
#include "u26_internal.h"

namespace
{
	constexpr uint32_t kMaxPairs = U26_NOALLOC_MAX_EF_PAIRS;
	constexpr uint32_t kTiles = (kMaxPairs + 2047u) / 2048u; // radix tiles of 2048 keys

	// scratch layout (bytes, each region 256-byte aligned)
	constexpr size_t kKeys = 0;
	constexpr size_t kKeysAlt = kKeys + sizeof(uint64_t) * kMaxPairs;
	constexpr size_t kVals = kKeysAlt + sizeof(uint64_t) * kMaxPairs;
	constexpr size_t kValsAlt = kVals + sizeof(uint32_t) * kMaxPairs;
	constexpr size_t kPairs = kValsAlt + sizeof(uint32_t) * kMaxPairs;
	constexpr size_t kIdx = kPairs + 48u * kMaxPairs;
	constexpr size_t kCounts = kIdx + sizeof(uint2) * kMaxPairs;
	constexpr size_t kTotal = kCounts + sizeof(uint32_t) * 256u * kTiles;
	static_assert(kTotal <= U26_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the declared size");
	static_assert(kKeysAlt % 256 == 0 && kVals % 256 == 0 && kValsAlt % 256 == 0 && kPairs % 256 == 0 && kIdx % 256 == 0 && kCounts % 256 == 0,
		"scratch regions must stay 256-byte aligned");

	// The scratch array. Host code must not use its name as an address: the device
	// address comes from cudaGetSymbolAddress, once per context, in scratch_for_context.
	static __device__ __align__(256) unsigned char g_ef_sort_scratch[U26_NOALLOC_SCRATCH_BYTES];

	struct EfRec
	{
		uint32_t w[12];
	};

	__global__ void noalloc_keys_kernel(const uint2* __restrict__ idx, uint32_t count, uint32_t num_faces, uint64_t* __restrict__ keys,
		uint32_t* __restrict__ vals, EfRec* __restrict__ pairs_copy, const EfRec* __restrict__ pairs, uint2* __restrict__ idx_copy)
	{
		const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
		if (i >= count)
			return;
		const uint2 p = idx[i];
		keys[i] = uint64_t(p.x) * uint64_t(num_faces) + uint64_t(p.y);
		vals[i] = i;
		pairs_copy[i] = pairs[i];
		idx_copy[i] = p;
	}

	__global__ void noalloc_gather_kernel(const uint32_t* __restrict__ perm, uint32_t count, const EfRec* __restrict__ src,
		const uint2* __restrict__ src_idx, EfRec* __restrict__ dst, uint2* __restrict__ dst_idx)
	{
		const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
		if (i >= count)
			return;
		const uint32_t j = perm[i];
		dst[i] = src[j];
		dst_idx[i] = src_idx[j];
	}

	// Device address of the scratch array for the context's device, looked up with that device
	// current by the first call on the context and kept on it. A context made after a device
	// reset looks it up anew.
	u26_status scratch_for_context(u26_ctx* ctx, unsigned char** out)
	{
		if (ctx->noalloc_scratch == nullptr)
		{
			int prev = 0;
			U26_CUDA(ctx, cudaGetDevice(&prev));
			U26_CUDA(ctx, cudaSetDevice(ctx->device));
			void* p = nullptr;
			const cudaError_t e = cudaGetSymbolAddress(&p, g_ef_sort_scratch);
			cudaSetDevice(prev);
			if (e != cudaSuccess || p == nullptr)
				return u26::set_error(ctx, U26_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
			ctx->noalloc_scratch = static_cast<unsigned char*>(p);
		}
		*out = ctx->noalloc_scratch;
		return U26_OK;
	}
} // namespace

using namespace u26;

U26_API u26_status u26_ef_canonicalize_noalloc(u26_ctx* ctx, uint32_t count, void* ef_pairs, uint32_t* ef_indices, uint32_t num_edges,
	uint32_t num_faces)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	if (count > kMaxPairs)
		return set_error(ctx, U26_ERR_CAPACITY, "u26_ef_canonicalize_noalloc: %u EF pairs exceed the fixed scratch limit of %u", count,
			kMaxPairs);
	if (count <= 1)
		return U26_OK;
	if (!ef_pairs || !ef_indices || num_faces == 0 || num_edges == 0)
		return set_error(ctx, U26_ERR_INVALID_INPUT, "u26_ef_canonicalize_noalloc: bad input");
	unsigned char* base = nullptr;
	U26_TRY(scratch_for_context(ctx, &base));
	uint64_t* keys = reinterpret_cast<uint64_t*>(base + kKeys);
	uint64_t* keys_alt = reinterpret_cast<uint64_t*>(base + kKeysAlt);
	uint32_t* vals = reinterpret_cast<uint32_t*>(base + kVals);
	uint32_t* vals_alt = reinterpret_cast<uint32_t*>(base + kValsAlt);
	EfRec* pairs_copy = reinterpret_cast<EfRec*>(base + kPairs);
	uint2* idx_copy = reinterpret_cast<uint2*>(base + kIdx);
	uint32_t* counts = reinterpret_cast<uint32_t*>(base + kCounts);
	// every scratch word the sort reads is written first in this call (keys, values and
	// copies by the keys kernel, the histogram table by each radix pass), so the previous
	// call's contents need no clearing
	noalloc_keys_kernel<<<div_up(count, 256), 256, 0, ctx->stream>>>(reinterpret_cast<const uint2*>(ef_indices), count, num_faces, keys,
		vals, pairs_copy, static_cast<const EfRec*>(ef_pairs), idx_copy);
	U26_TRY(after_launch(ctx, "noalloc_keys_kernel"));
	const uint64_t key_max = uint64_t(num_edges) * uint64_t(num_faces);
	int bits = 1;
	while (bits < 64 && (uint64_t(1) << bits) < key_max)
		bits++;
	U26_TRY(RadixSorter::sort_into(ctx, keys, vals, count, 0, bits, keys_alt, vals_alt, counts));
	U26_TRY(ef_tiebreak(ctx, keys, vals, count, pairs_copy));
	noalloc_gather_kernel<<<div_up(count, 256), 256, 0, ctx->stream>>>(vals, count, pairs_copy, idx_copy, static_cast<EfRec*>(ef_pairs),
		reinterpret_cast<uint2*>(ef_indices));
	return after_launch(ctx, "noalloc_gather_kernel");
}
