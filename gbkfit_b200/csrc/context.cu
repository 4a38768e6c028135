// Context (module object) management and error reporting of the C ABI.
#include "gbk_common.cuh"

#include <map>
#include <mutex>
#include <utility>

#include <new>

static thread_local cudaError_t g_last_cuda_error = cudaSuccess;

void gbk_set_last_cuda_error(cudaError_t e) { g_last_cuda_error = e; }

int gbk_finish(gbkb200_ctx* ctx)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_cuda_error = e;
        return GBKB200_ERR_CUDA;
    }
    if (!ctx->sync) return GBKB200_OK;
    return gbkb200_ctx_synchronize(ctx);
}

extern "C" int gbkb200_ctx_create(gbkb200_ctx** out, int device)
{
    if (!out) return GBKB200_ERR_INVALID_ARG;
    *out = nullptr;
    GBK_CUDA_TRY(cudaSetDevice(device));
    gbkb200_ctx* c = new (std::nothrow) gbkb200_ctx();
    if (!c) return GBKB200_ERR_OOM;
    c->device = device;
    if (cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&c->h_status, sizeof(int)) != cudaSuccess) {
        if (c->d_status) cudaFree(c->d_status);
        delete c;
        return GBKB200_ERR_OOM;
    }
    *c->h_status = 0;
    GBK_CUDA_TRY(cudaMemset(c->d_status, 0, sizeof(int)));
    *out = c;
    return GBKB200_OK;
}

extern "C" int gbkb200_ctx_destroy(gbkb200_ctx* ctx)
{
    if (!ctx) return GBKB200_OK;
    cudaStreamSynchronize(ctx->stream);
    gbk_fft_state_destroy(ctx);
    if (ctx->reduce_scratch) cudaFree(ctx->reduce_scratch);
    if (ctx->mc_scratch) cudaFree(ctx->mc_scratch);
    if (ctx->serve_scratch) cudaFree(ctx->serve_scratch);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    delete ctx;
    return GBKB200_OK;
}

extern "C" int gbkb200_ctx_set_stream(gbkb200_ctx* ctx, void* stream)
{
    if (!ctx) return GBKB200_ERR_INVALID_ARG;
    ctx->stream = static_cast<cudaStream_t>(stream);
    return GBKB200_OK;
}

extern "C" int gbkb200_ctx_set_sync(gbkb200_ctx* ctx, int sync)
{
    if (!ctx) return GBKB200_ERR_INVALID_ARG;
    ctx->sync = sync ? 1 : 0;
    return GBKB200_OK;
}

extern "C" int gbkb200_ctx_set_mcdisk(gbkb200_ctx* ctx, unsigned long long seed, int mode)
{
    if (!ctx || mode < 0 || mode > 3) return GBKB200_ERR_INVALID_ARG;
    ctx->seed = seed;
    ctx->mc_mode = mode;
    return GBKB200_OK;
}

extern "C" int gbkb200_ctx_reserve_scratch(gbkb200_ctx* ctx, size_t bytes)
{
    if (!ctx) return GBKB200_ERR_INVALID_ARG;
    if (ctx->mc_scratch_bytes >= bytes) return GBKB200_OK;
    GBK_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->mc_scratch) cudaFree(ctx->mc_scratch);
    ctx->mc_scratch = nullptr;
    ctx->mc_scratch_bytes = 0;
    if (cudaMalloc(&ctx->mc_scratch, bytes) != cudaSuccess) {
        (void)cudaGetLastError();
        return GBKB200_ERR_OOM;
    }
    ctx->mc_scratch_bytes = bytes;
    return GBKB200_OK;
}

extern "C" int gbkb200_ctx_synchronize(gbkb200_ctx* ctx)
{
    if (!ctx) return GBKB200_ERR_INVALID_ARG;
    GBK_CUDA_TRY(cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(int),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    GBK_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    int s = *ctx->h_status;
    if (s) {
        GBK_CUDA_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
        GBK_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        *ctx->h_status = 0;
        if (s & GBK_STATUS_BAD_TRAIT) return GBKB200_ERR_BAD_TRAIT;
        if (s & GBK_STATUS_TIMEOUT) return GBKB200_ERR_TIMEOUT;
        return GBKB200_ERR_INVALID_ARG;
    }
    return GBKB200_OK;
}

extern "C" const char* gbkb200_error_string(int code)
{
    switch (code) {
    case GBKB200_OK: return "ok";
    case GBKB200_ERR_INVALID_ARG: return "invalid argument";
    case GBKB200_ERR_UNSUPPORTED: return "unsupported size or configuration";
    case GBKB200_ERR_CUDA: return "CUDA runtime error";
    case GBKB200_ERR_BAD_TRAIT: return "unknown trait uid";
    case GBKB200_ERR_OOM: return "device allocation failed";
    case GBKB200_ERR_TIMEOUT: return "device-side wait timed out";
    case GBKB200_ERR_TOO_LARGE: return "size exceeds the documented maximum";
    default: return "unknown error";
    }
}

extern "C" const char* gbkb200_last_cuda_error(void)
{
    return cudaGetErrorString(g_last_cuda_error);
}

namespace {
std::mutex g_smem_mutex;
std::map<std::pair<int, const void*>, size_t> g_smem_limits;   // (device, kernel) -> bytes
}  // namespace

int gbk_raise_smem_limit(const void* fn, size_t bytes)
{
    if (bytes <= 48 * 1024) return GBKB200_OK;      // the default limit
    int dev = 0;
    GBK_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_smem_mutex);
    size_t& cur = g_smem_limits[{dev, fn}];
    if (bytes > cur) {
        GBK_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)bytes));
        cur = bytes;
    }
    return GBKB200_OK;
}
