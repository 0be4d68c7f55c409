// Stable LSD radix sort of (uint64 key, uint32 value) pairs on the device.
//
// Replaces the host pdqsort + two PCIe copies of LBVH::construct_tree
// (lbvh.cpp:1037-1040). Only the live bits are sorted: for Morton keys
// (m32 << 32 | leaf id) with values starting as the identity, a stable sort of bits
// [32, 62) yields exactly the order of the full 64-bit key.
//
// Per 8-bit digit pass: (1) per-tile digit histogram, (2) exclusive scan of the
// digit-major count table (reduce / scan block sums / downsweep over 8192-word segments),
// (3) stable scatter: each tile is ranked in chunks of 256 with __match_any_sync peer
// masks and a per-warp digit table in shared memory.
#include "u26_internal.h"

namespace u26
{
	namespace
	{
		constexpr int kThreads = 256;
		constexpr int kChunks = 8;
		constexpr int kTile = kThreads * kChunks; // 2048 keys per tile
		constexpr int kWarps = kThreads / 32;

		__global__ void __launch_bounds__(kThreads) radix_hist_kernel(const uint64_t* __restrict__ keys, uint32_t n, int shift, uint32_t mask,
			uint32_t* __restrict__ counts, uint32_t num_tiles)
		{
			__shared__ uint32_t hist[256];
			hist[threadIdx.x] = 0;
			__syncthreads();
			const uint32_t base = blockIdx.x * kTile;
#pragma unroll
			for (int c = 0; c < kChunks; c++)
			{
				const uint32_t i = base + c * kThreads + threadIdx.x;
				if (i < n)
				{
					const uint32_t d = uint32_t(keys[i] >> shift) & mask;
					atomicAdd(&hist[d], 1u);
				}
			}
			__syncthreads();
			counts[threadIdx.x * num_tiles + blockIdx.x] = hist[threadIdx.x];
		}

		// Exclusive scan of counts[0, total) in place by one block of 1024 threads.
		__global__ void __launch_bounds__(1024) radix_scan_kernel(uint32_t* __restrict__ counts, uint32_t total)
		{
			__shared__ uint32_t warp_sums[32];
			const uint32_t per = (total + blockDim.x - 1) / blockDim.x;
			const uint32_t begin = threadIdx.x * per;
			const uint32_t end = min(total, begin + per);
			uint32_t local = 0;
			for (uint32_t i = begin; i < end; i++)
				local += counts[i];
			// block exclusive scan of `local`
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			uint32_t v = local;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1)
			{
				uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
				if (lane >= o)
					v += t;
			}
			if (lane == 31)
				warp_sums[warp] = v;
			__syncthreads();
			if (warp == 0)
			{
				uint32_t w = warp_sums[lane];
#pragma unroll
				for (int o = 1; o < 32; o <<= 1)
				{
					uint32_t t = __shfl_up_sync(0xFFFFFFFFu, w, o);
					if (lane >= o)
						w += t;
				}
				warp_sums[lane] = w;
			}
			__syncthreads();
			uint32_t run = v - local + (warp > 0 ? warp_sums[warp - 1] : 0u);
			for (uint32_t i = begin; i < end; i++)
			{
				const uint32_t c = counts[i];
				counts[i] = run;
				run += c;
			}
		}

		// ---- device-wide exclusive scan of uint32 words: segments of kScanSeg words, each
		// thread owning kScanPer consecutive words
		constexpr int kScanThreads = 1024;
		constexpr int kScanPer = 8;
		constexpr uint32_t kScanSeg = kScanThreads * kScanPer;

		__device__ __forceinline__ void load8(const uint32_t* __restrict__ v, uint32_t i, uint32_t n, uint32_t (&w)[kScanPer])
		{
			if (i + kScanPer <= n)
			{
				const uint4 a = *reinterpret_cast<const uint4*>(v + i);
				const uint4 b = *reinterpret_cast<const uint4*>(v + i + 4);
				w[0] = a.x, w[1] = a.y, w[2] = a.z, w[3] = a.w, w[4] = b.x, w[5] = b.y, w[6] = b.z, w[7] = b.w;
			}
			else
			{
#pragma unroll
				for (int j = 0; j < kScanPer; j++)
					w[j] = i + j < n ? v[i + j] : 0u;
			}
		}

		// block-wide exclusive scan of one value per thread; returns the exclusive prefix and
		// writes the block total to *total (all threads)
		__device__ __forceinline__ uint32_t block_exclusive(uint32_t x, uint32_t* total)
		{
			__shared__ uint32_t ws[32];
			__shared__ uint32_t tot;
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			uint32_t v = x;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1)
			{
				const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
				if (lane >= o)
					v += t;
			}
			if (lane == 31)
				ws[warp] = v;
			__syncthreads();
			if (warp == 0)
			{
				uint32_t w = lane < int(blockDim.x >> 5) ? ws[lane] : 0u;
#pragma unroll
				for (int o = 1; o < 32; o <<= 1)
				{
					const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, w, o);
					if (lane >= o)
						w += t;
				}
				ws[lane] = w;
				if (lane == 31)
					tot = w;
			}
			__syncthreads();
			const uint32_t r = v - x + (warp > 0 ? ws[warp - 1] : 0u);
			*total = tot;
			__syncthreads();
			return r;
		}

		__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* __restrict__ v, uint32_t n, uint32_t* __restrict__ seg_sums)
		{
			uint32_t w[kScanPer];
			load8(v, blockIdx.x * kScanSeg + threadIdx.x * kScanPer, n, w);
			uint32_t s = 0;
#pragma unroll
			for (int j = 0; j < kScanPer; j++)
				s += w[j];
			s = __reduce_add_sync(0xFFFFFFFFu, s);
			__shared__ uint32_t ws[32];
			if ((threadIdx.x & 31) == 0)
				ws[threadIdx.x >> 5] = s;
			__syncthreads();
			if (threadIdx.x < 32)
			{
				uint32_t t = ws[threadIdx.x];
				t = __reduce_add_sync(0xFFFFFFFFu, t);
				if (threadIdx.x == 0)
					seg_sums[blockIdx.x] = t;
			}
		}

		// exclusive scan in place of each segment, offset by offsets[segment] (or 0)
		__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(uint32_t* __restrict__ v, uint32_t n, const uint32_t* __restrict__ offsets)
		{
			uint32_t w[kScanPer];
			const uint32_t i = blockIdx.x * kScanSeg + threadIdx.x * kScanPer;
			load8(v, i, n, w);
			uint32_t s = 0;
#pragma unroll
			for (int j = 0; j < kScanPer; j++)
				s += w[j];
			uint32_t total;
			uint32_t run = block_exclusive(s, &total) + (offsets ? offsets[blockIdx.x] : 0u);
#pragma unroll
			for (int j = 0; j < kScanPer; j++)
			{
				const uint32_t c = w[j];
				w[j] = run;
				run += c;
			}
			if (i + kScanPer <= n)
			{
				*reinterpret_cast<uint4*>(v + i) = make_uint4(w[0], w[1], w[2], w[3]);
				*reinterpret_cast<uint4*>(v + i + 4) = make_uint4(w[4], w[5], w[6], w[7]);
			}
			else
			{
#pragma unroll
				for (int j = 0; j < kScanPer; j++)
					if (i + j < n)
						v[i + j] = w[j];
			}
		}

		__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
			uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n, int shift, uint32_t mask,
			const uint32_t* __restrict__ offsets, uint32_t num_tiles)
		{
			__shared__ uint32_t warp_cnt[kWarps][256];
			__shared__ uint32_t base_run[256];
			const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
			base_run[tid] = offsets[tid * num_tiles + blockIdx.x];
			const uint32_t lanemask_lt = (1u << lane) - 1u;
			const uint32_t tile_base = blockIdx.x * kTile;
			for (int c = 0; c < kChunks; c++)
			{
#pragma unroll
				for (int w = 0; w < kWarps; w++)
					warp_cnt[w][tid] = 0;
				__syncthreads();
				const uint32_t i = tile_base + c * kThreads + tid;
				const bool valid = i < n;
				uint64_t k = 0;
				uint32_t v = 0, d = 0x100u + lane; // invalid lanes get unique digits
				if (valid)
				{
					k = keys_in[i];
					v = vals_in[i];
					d = uint32_t(k >> shift) & mask;
				}
				const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
				const uint32_t rank = __popc(peers & lanemask_lt);
				const int leader = __ffs(peers) - 1;
				if (valid && lane == leader)
					warp_cnt[warp][d] = __popc(peers);
				__syncthreads();
				{
					uint32_t run = base_run[tid];
#pragma unroll
					for (int w = 0; w < kWarps; w++)
					{
						const uint32_t t = warp_cnt[w][tid];
						warp_cnt[w][tid] = run;
						run += t;
					}
					base_run[tid] = run;
				}
				__syncthreads();
				if (valid)
				{
					const uint32_t pos = warp_cnt[warp][d] + rank;
					keys_out[pos] = k;
					vals_out[pos] = v;
				}
				__syncthreads();
			}
		}
	} // namespace

	// Exclusive scan of v[0, n) in place; tmp holds ceil(n / 8192) + 1 words of scratch. The
	// segment sums are scanned recursively, so any n that fits the words works.
	u26_status device_exclusive_scan(u26_ctx* ctx, uint32_t* v, uint32_t n, DevBuf& tmp)
	{
		if (n == 0)
			return U26_OK;
		const uint32_t segs = div_up(n, kScanSeg);
		if (segs == 1)
		{
			scan_down_kernel<<<1, kScanThreads, 0, ctx->stream>>>(v, n, nullptr);
			return after_launch(ctx, "scan_down_kernel");
		}
		// scratch for every recursion level: segs + segs/8192 + ... words, 4-word aligned
		size_t words = 0;
		for (uint32_t m = segs; m > 1; m = div_up(m, kScanSeg))
			words += (m + 3u) & ~3u;
		U26_CUDA(ctx, tmp.reserve(sizeof(uint32_t) * (words + 4)));
		uint32_t* sums = tmp.as<uint32_t>();
		std::vector<std::pair<uint32_t*, uint32_t>> levels; // (array, length) from v upwards
		levels.emplace_back(v, n);
		uint32_t* cur = sums;
		for (uint32_t m = n; div_up(m, kScanSeg) > 1;)
		{
			const uint32_t k = div_up(m, kScanSeg);
			scan_reduce_kernel<<<k, kScanThreads, 0, ctx->stream>>>(levels.back().first, m, cur);
			U26_TRY(after_launch(ctx, "scan_reduce_kernel"));
			levels.emplace_back(cur, k);
			cur += (k + 3u) & ~3u;
			m = k;
		}
		// the top level fits one segment
		scan_down_kernel<<<1, kScanThreads, 0, ctx->stream>>>(levels.back().first, levels.back().second, nullptr);
		U26_TRY(after_launch(ctx, "scan_down_kernel"));
		for (size_t l = levels.size() - 1; l > 0; l--)
		{
			const uint32_t m = levels[l - 1].second;
			scan_down_kernel<<<div_up(m, kScanSeg), kScanThreads, 0, ctx->stream>>>(levels[l - 1].first, m, levels[l].first);
			U26_TRY(after_launch(ctx, "scan_down_kernel"));
		}
		return U26_OK;
	}

	u26_status RadixSorter::sort(u26_ctx* ctx, uint64_t* keys, uint32_t* vals, uint32_t n, int bit_lo, int bit_hi)
	{
		if (n <= 1 || bit_hi <= bit_lo)
			return U26_OK;
		const uint32_t num_tiles = div_up(n, kTile);
		U26_CUDA(ctx, keys_alt.reserve(sizeof(uint64_t) * n));
		U26_CUDA(ctx, vals_alt.reserve(sizeof(uint32_t) * n));
		U26_CUDA(ctx, counts.reserve(sizeof(uint32_t) * 256u * num_tiles));
		uint64_t* k_src = keys;
		uint32_t* v_src = vals;
		uint64_t* k_dst = keys_alt.as<uint64_t>();
		uint32_t* v_dst = vals_alt.as<uint32_t>();
		int passes = 0;
		for (int shift = bit_lo; shift < bit_hi; shift += 8)
		{
			const int bits = min(8, bit_hi - shift);
			const uint32_t mask = (1u << bits) - 1u;
			radix_hist_kernel<<<num_tiles, kThreads, 0, ctx->stream>>>(k_src, n, shift, mask, counts.as<uint32_t>(), num_tiles);
			U26_TRY(after_launch(ctx, "radix_hist_kernel"));
			U26_TRY(device_exclusive_scan(ctx, counts.as<uint32_t>(), 256u * num_tiles, scan_tmp));
			radix_scatter_kernel<<<num_tiles, kThreads, 0, ctx->stream>>>(k_src, v_src, k_dst, v_dst, n, shift, mask,
				counts.as<uint32_t>(), num_tiles);
			U26_TRY(after_launch(ctx, "radix_scatter_kernel"));
			std::swap(k_src, k_dst);
			std::swap(v_src, v_dst);
			passes++;
		}
		if (k_src != keys)
		{
			U26_CUDA(ctx, cudaMemcpyAsync(keys, k_src, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
			U26_CUDA(ctx, cudaMemcpyAsync(vals, v_src, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
		}
		return U26_OK;
	}

	u26_status RadixSorter::sort_into(u26_ctx* ctx, uint64_t* keys, uint32_t* vals, uint32_t n, int bit_lo, int bit_hi,
		uint64_t* keys_alt, uint32_t* vals_alt, uint32_t* counts)
	{
		if (n <= 1 || bit_hi <= bit_lo)
			return U26_OK;
		const uint32_t num_tiles = div_up(n, kTile);
		uint64_t* k_src = keys;
		uint32_t* v_src = vals;
		uint64_t* k_dst = keys_alt;
		uint32_t* v_dst = vals_alt;
		for (int shift = bit_lo; shift < bit_hi; shift += 8)
		{
			const int bits = min(8, bit_hi - shift);
			const uint32_t mask = (1u << bits) - 1u;
			radix_hist_kernel<<<num_tiles, kThreads, 0, ctx->stream>>>(k_src, n, shift, mask, counts, num_tiles);
			U26_TRY(after_launch(ctx, "radix_hist_kernel"));
			radix_scan_kernel<<<1, 1024, 0, ctx->stream>>>(counts, 256u * num_tiles);
			U26_TRY(after_launch(ctx, "radix_scan_kernel"));
			radix_scatter_kernel<<<num_tiles, kThreads, 0, ctx->stream>>>(k_src, v_src, k_dst, v_dst, n, shift, mask, counts, num_tiles);
			U26_TRY(after_launch(ctx, "radix_scatter_kernel"));
			std::swap(k_src, k_dst);
			std::swap(v_src, v_dst);
		}
		if (k_src != keys)
		{
			U26_CUDA(ctx, cudaMemcpyAsync(keys, k_src, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
			U26_CUDA(ctx, cudaMemcpyAsync(vals, v_src, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
		}
		return U26_OK;
	}
} // namespace u26
