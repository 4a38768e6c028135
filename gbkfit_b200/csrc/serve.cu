// One serving request in one call (no reference counterpart): the chain the
// serving loop runs per request, on the context's stream, composed from the
// library's own entry points: the request's packed parameters are copied
// from pinned host memory, the model cube is zeroed and evaluated (smdisk
// or mcdisk, gmodels.hpp), convolved with the dataset's resident PSF x LSF
// spectrum (fft.hpp:87-96), cropped (dmodels.hpp:7-46), its residual and
// sum of squares taken (objective.hpp:7-31, host/kernels.hpp:502-514), and
// chi^2 and the context's kernel status word are copied to pinned host
// memory, so that the caller sees the result without another CUDA call.
// The crop, residual and sum run as one fused kernel.
#include <algorithm>

#include "gbk_common.cuh"

namespace gbk {

constexpr int TAIL_BLOCKS = 296;   // 2 x 148 SMs
constexpr int TAIL_THREADS = 256;

// Crop of the convolved cube (dmodels.hpp:7-46 at scale 1: a copy), the
// residual (model - data) / error x mask x weight (objective.hpp:7-31) and its sum of
// squares, in one pass: fp32 within a block, one fp64 partial per block,
// and the last block to finish adds the partials in block order (a fixed
// order for a given size, so the sum does not depend on the schedule).
__global__ void __launch_bounds__(TAIL_THREADS)
    serve_tail_kernel(const float* __restrict__ scube, int px, int py, int ex, int ey, int ez,
                      int nx, int ny, int n, const float* __restrict__ obs,
                      const float* __restrict__ err, const float* __restrict__ msk, float weight,
                      float* __restrict__ crop,
                      double* part, unsigned* counter, float* chi2)
{
    __shared__ float ws[TAIL_THREADS / 32];
    __shared__ bool last;
    float acc = 0.f;
    const int nxy = nx * ny;
    for (int i = blockIdx.x * TAIL_THREADS + threadIdx.x; i < n; i += gridDim.x * TAIL_THREADS) {
        const int z = i / nxy, rem = i - z * nxy;
        const int y = rem / nx, x = rem - y * nx;
        const float m = scube[(long long)(ez + z) * px * py + (long long)(ey + y) * px + (ex + x)];
        if (crop) crop[i] = m;
        float r = m - obs[i];
        if (err) r /= err[i];
        if (msk) r *= msk[i];
        r *= weight;
        acc += r * r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int w = 0; w < TAIL_THREADS / 32; ++w) v += ws[w];
        part[blockIdx.x] = (double)v;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double s = 0;
        for (int b = 0; b < (int)gridDim.x; ++b) s += ((volatile double*)part)[b];
        chi2[0] = (float)s;
        *counter = 0u;   // ready for the next request on this context
    }
}

}  // namespace gbk

using namespace gbk;

// The packed parameters' copy, the zeroing of the cube (ncube floats at
// a->scube) and the model evaluation of one request.
static int serve_model(gbkb200_ctx* ctx, const gbkb200_serve_args* a, long long ncube)
{
    char* base = static_cast<char*>(a->blob_dev);
    auto at = [&](long long off) -> char* { return off < 0 ? nullptr : base + off; };
    const cudaStream_t st = ctx->stream;
    if (a->blob_bytes > 0) {
        if (!a->blob_host) return GBKB200_ERR_INVALID_ARG;
        GBK_CUDA_TRY(cudaMemcpyAsync(a->blob_dev, a->blob_host, (size_t)a->blob_bytes,
                                     cudaMemcpyHostToDevice, st));
    }
    GBK_CUDA_TRY(cudaMemsetAsync(a->scube, 0, (size_t)ncube * sizeof(float), st));
#define GBK_T(k)                                                                                 \
    reinterpret_cast<const int*>(at(a->off_uids[k])),                                            \
        reinterpret_cast<const float*>(at(a->off_cvalues[k])),                                   \
        reinterpret_cast<const int*>(at(a->off_ccounts[k])),                                     \
        reinterpret_cast<const float*>(at(a->off_pvalues[k])),                                   \
        reinterpret_cast<const int*>(at(a->off_pcounts[k]))
#define GBK_SERVE_DISK                                                                           \
    a->loose, a->tilted, a->nrnodes, reinterpret_cast<const float*>(at(a->off_rnodes)),          \
        reinterpret_cast<const float*>(at(a->off_vsys)),                                         \
        reinterpret_cast<const float*>(at(a->off_xpos)),                                         \
        reinterpret_cast<const float*>(at(a->off_ypos)),                                         \
        reinterpret_cast<const float*>(at(a->off_posa)),                                         \
        reinterpret_cast<const float*>(at(a->off_incl)), a->ntraits[0], GBK_T(0), GBK_T(1),    \
        a->ntraits[2], GBK_T(2), GBK_T(3), a->ntraits[4], GBK_T(4), GBK_T(5), a->ntraits[6],    \
        GBK_T(6), a->ntraits[7], GBK_T(7), a->ntraits[8], GBK_T(8), nullptr, a->spat_size[0],  \
        a->spat_size[1], a->spat_size[2], a->spat_step[0], a->spat_step[1], a->spat_step[2],    \
        a->spat_zero[0], a->spat_zero[1], a->spat_zero[2], a->spec_size, a->spec_step,          \
        a->spec_zero, nullptr, a->scube, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,  \
        nullptr, nullptr
    int rc;
    if (a->kind == 0)
        rc = gbkb200_gmodel_smdisk_evaluate_f32(ctx, GBK_SERVE_DISK);
    else
        rc = gbkb200_gmodel_mcdisk_evaluate_f32(
            ctx, a->cflux, a->nclouds, reinterpret_cast<const int*>(at(a->off_csum)), a->csum_len,
            reinterpret_cast<const unsigned char*>(at(a->off_hasordint)), GBK_SERVE_DISK);
#undef GBK_SERVE_DISK
#undef GBK_T
    return rc;
}

extern "C" int gbkb200_serve_model_f32(gbkb200_ctx* ctx, const gbkb200_serve_args* a)
{
    if (!ctx || !a || !a->blob_dev || !a->scube) return GBKB200_ERR_INVALID_ARG;
    if (a->kind != 0 && a->kind != 1) return GBKB200_ERR_INVALID_ARG;
    if (a->spat_size[0] < 1 || a->spat_size[1] < 1 || a->spat_size[2] < 1 || a->spec_size < 1)
        return GBKB200_ERR_INVALID_ARG;
    const long long n = (long long)a->spat_size[0] * a->spat_size[1] * a->spec_size;
    if (n >= (1ll << 31)) return GBKB200_ERR_TOO_LARGE;
    const int rc = serve_model(ctx, a, n);
    if (rc) return rc;
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}

extern "C" int gbkb200_serve_scube_chi2_f32(gbkb200_ctx* ctx, const gbkb200_serve_args* a)
{
    if (!ctx || !a || !a->blob_dev || !a->scube || !a->work || !a->spectrum || !a->obs ||
        !a->chi2_dev || !a->chi2_host || !a->status_host)
        return GBKB200_ERR_INVALID_ARG;
    if (a->kind != 0 && a->kind != 1) return GBKB200_ERR_INVALID_ARG;
    for (int k = 0; k < 3; ++k)
        if (a->size_hi[k] < 1 || a->size[k] < 1 || a->edge[k] < 0 ||
            a->edge[k] + a->size[k] > a->size_hi[k])
            return GBKB200_ERR_INVALID_ARG;
    // sizes are checked before anything is enqueued on the stream
    const long long vhi = (long long)a->size_hi[0] * a->size_hi[1] * a->size_hi[2];
    if ((long long)a->size[0] * a->size[1] * a->size[2] >= (1ll << 31) || vhi >= (1ll << 31))
        return GBKB200_ERR_TOO_LARGE;
    const cudaStream_t st = ctx->stream;
    int rc = serve_model(ctx, a, vhi);
    if (rc) return rc;
    if ((rc = gbkb200_fft_convolve_f32(ctx, a->size_hi, a->scube, a->work, a->spectrum))) return rc;
    if (!ctx->serve_scratch) {
        const size_t bytes = TAIL_BLOCKS * sizeof(double) + 256;
        if (cudaMalloc(&ctx->serve_scratch, bytes) != cudaSuccess) return GBKB200_ERR_OOM;
        GBK_CUDA_TRY(cudaMemsetAsync(ctx->serve_scratch, 0, bytes, st));
    }
    double* part = static_cast<double*>(ctx->serve_scratch);
    unsigned* counter = reinterpret_cast<unsigned*>(part + TAIL_BLOCKS);
    const long long n = (long long)a->size[0] * a->size[1] * a->size[2];
    int blocks = (int)std::min<long long>(TAIL_BLOCKS, (n + 4 * TAIL_THREADS - 1) / (4 * TAIL_THREADS));
    serve_tail_kernel<<<blocks, TAIL_THREADS, 0, st>>>(
        a->scube, a->size_hi[0], a->size_hi[1], a->edge[0], a->edge[1], a->edge[2], a->size[0],
        a->size[1], (int)n, a->obs, a->err, a->msk, a->weight, a->crop, part, counter, a->chi2_dev);
    GBK_CUDA_TRY(cudaMemcpyAsync(a->chi2_host, a->chi2_dev, sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
    GBK_CUDA_TRY(cudaMemcpyAsync(a->status_host, ctx->d_status, sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}
