// Context management of the libu26 C ABI.
#include "u26_internal.h"

void u26_ef_release_ctx(const u26_ctx* ctx);
void u26_prp_release_ctx(const u26_ctx* ctx);

namespace u26
{
	std::atomic<uint64_t> g_alloc_count{ 0 };
}

using namespace u26;

U26_API uint64_t u26_alloc_count(void) { return g_alloc_count.load(std::memory_order_relaxed); }

U26_API const char* u26_version(void) { return "u26-b200 0.1 (sm_100a)"; }

U26_API u26_status u26_ctx_create(int device, void* cuda_stream, u26_ctx** out)
{
	if (!out)
		return U26_ERR_INVALID_INPUT;
	*out = nullptr;
	int count = 0;
	if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
	{
		cudaGetLastError();
		return U26_ERR_NO_DEVICE;
	}
	if (device < 0 || device >= count)
		return U26_ERR_INVALID_INPUT;
	if (cudaSetDevice(device) != cudaSuccess)
		return U26_ERR_CUDA;
	u26_ctx* ctx = new u26_ctx();
	ctx->device = device;
	ctx->stream = static_cast<cudaStream_t>(cuda_stream);
	if (cudaMalloc(&ctx->dev_err, sizeof(uint32_t)) != cudaSuccess || cudaMallocHost(&ctx->host_word, sizeof(uint32_t) * 16) != cudaSuccess
		|| cudaMemset(ctx->dev_err, 0, sizeof(uint32_t)) != cudaSuccess)
	{
		u26_ctx_destroy(ctx);
		return U26_ERR_CUDA;
	}
	g_alloc_count.fetch_add(2, std::memory_order_relaxed);
	*out = ctx;
	return U26_OK;
}

U26_API void u26_ctx_destroy(u26_ctx* ctx)
{
	if (!ctx)
		return;
	u26_ef_release_ctx(ctx);
	u26_prp_release_ctx(ctx);
	if (ctx->dev_err)
		cudaFree(ctx->dev_err);
	if (ctx->host_word)
		cudaFreeHost(ctx->host_word);
	delete ctx;
}

U26_API u26_status u26_ctx_set_stream(u26_ctx* ctx, void* cuda_stream)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	ctx->stream = static_cast<cudaStream_t>(cuda_stream);
	return U26_OK;
}

U26_API u26_status u26_ctx_synchronize(u26_ctx* ctx)
{
	if (!ctx)
		return U26_ERR_INVALID_INPUT;
	return cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
}

U26_API const char* u26_ctx_last_error(const u26_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

U26_API uint64_t u26_ctx_launch_count(const u26_ctx* ctx) { return ctx ? ctx->launches : 0; }

/* Device error word: OR of U26_DEVERR_* flags raised by kernels since the last reset.
 * Synchronises. */
U26_API u26_status u26_ctx_device_errors(u26_ctx* ctx, uint32_t* flags, int reset)
{
	if (!ctx || !flags)
		return U26_ERR_INVALID_INPUT;
	U26_CUDA(ctx, cudaMemcpyAsync(ctx->host_word, ctx->dev_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
	if (reset)
		U26_CUDA(ctx, cudaMemsetAsync(ctx->dev_err, 0, sizeof(uint32_t), ctx->stream));
	U26_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	*flags = *ctx->host_word;
	return U26_OK;
}
