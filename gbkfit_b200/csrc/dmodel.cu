// Data-model kernels: downscale/crop, mask, moment maps; objective kernels:
// residual and its (deterministic) sum.
//
// Reference: gbkfit/include/gbkfit/dmodel/dmodels.hpp:7-228,
// gbkfit/include/gbkfit/objective/objective.hpp:7-31 and the drivers
// gbkfit_host/include/gbkfit/host/kernels.hpp:55-135, 484-514.
#include "gbk_common.cuh"

#include <cmath>

namespace gbk {

// dmodels.hpp:7-46: box average of scale-sized blocks starting at offset
__global__ void downscale_kernel(int scx, int scy, int scz, int ofx, int ofy, int ofz, int srx,
                                 int sry, int dsx, int dsy, int dsz, const float* src, float* dst)
{
    const float nf = 1.0f / (scx * scy * scz);
    long long n = (long long)dsx * dsy * dsz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int x = (int)(i % dsx);
        int y = (int)((i / dsx) % dsy);
        int z = (int)(i / ((long long)dsx * dsy));
        int nx = ofx + x * scx, ny = ofy + y * scy, nz = ofz + z * scz;
        float sum = 0;
        for (int dz = 0; dz < scz; ++dz)
            for (int dy = 0; dy < scy; ++dy)
                for (int dx = 0; dx < scx; ++dx)
                    sum += src[idx3(nx + dx, ny + dy, nz + dz, srx, sry)];
        dst[i] = sum * nf;
    }
}

// dmodels.hpp:48-74
__global__ void mask_kernel(float cutoff, int apply, long long n, float* d, float* m)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float mv = 1.f;
        if (fabsf(d[i]) <= cutoff) {
            mv = 0.f;
            if (apply) d[i] = NAN;
        }
        if (m) m[i] = mv;
    }
}

// dmodels.hpp:76-228, one thread per (x, y) pixel; adjacent threads read
// adjacent x, so every spectral step is a coalesced row read, and orders 0-2
// (and the weight map) read the column once:
// * m0 = sum d dz in fp32, channel 0 upwards, as the reference sums it (the
//   mask |m0| > cutoff and the m0 map are the reference's, bit for bit);
// * fp64 running sums S0 = sum d dz, S1 = sum d v dz, S2 = sum d v^2 dz and
//   SW = sum w d dz give m1 = S1 / S0, m2 = sqrt(S2 / S0 - m1^2) (the centred
//   second moment, exact in fp64 for these magnitudes) and the weight map
//   SW / m0; the reference's fp32 sums round at ~1e-7 relative, these at
//   ~1e-16;
// * orders >= 3 take a second pass over the column with (v - m1)^k in fp64,
//   without dz, divided by m0, as the reference does.
// mm receives the mask map, mw the weight map.
__global__ void moments_kernel(int nx, int ny, int nz, float stz, float zz, const float* d,
                               const float* w, float cutoff, int norders, const int* orders,
                               float* md, float* mm, float* mw)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= nx) return;
    const long long i2 = x + (long long)nx * y, sxy = (long long)nx * ny;
    const int maxo = orders[norders - 1];
    float m0s = 0;
    double s0 = 0, s1 = 0, s2 = 0, sw = 0;
    const float* dp = d + i2;
    const float* wp = w ? w + i2 : nullptr;
#pragma unroll 4
    for (int z = 0; z < nz; ++z) {
        const float dv = dp[sxy * z];
        const float ddz = dv * stz;
        m0s += ddz;
        const double v = (double)(zz + z * stz);
        const double a = (double)ddz;
        s0 += a;
        s1 += a * v;
        s2 += a * v * v;
        if (wp) sw += (double)wp[sxy * z] * a;
    }
    const bool valid = fabsf(m0s) > cutoff;
    mm[i2] = valid ? 1.f : 0.f;
    const float m0 = valid ? m0s : NAN;
    if (w) mw[i2] = valid ? (float)(sw / (double)m0s) : NAN;
    int m = 0;
    if (orders[m] == 0) { md[i2 + sxy * m] = m0; m++; }
    if (maxo == 0) return;
    const double m1d = s1 / s0;
    const float m1 = valid ? (float)m1d : NAN;
    if (m < norders && orders[m] == 1) { md[i2 + sxy * m] = m1; m++; }
    if (maxo == 1) return;
    // a negative variance (negative cube values, e.g. convolution ringing)
    // gives NaN, as the reference's sqrt of its negative sum does
    const double var = s2 / s0 - m1d * m1d;
    const float m2 = valid ? (float)sqrt(var) : NAN;
    if (m < norders && orders[m] == 2) { md[i2 + sxy * m] = m2; m++; }
    for (; m < norders; ++m) {
        double mns = 0;
        const int k = orders[m];
        for (int z = 0; valid && z < nz; ++z) {
            const double t = (double)((zz + z * stz) - m1);
            double p = t;
            for (int e = 1; e < k; ++e) p *= t;
            mns += (double)dp[sxy * z] * p;
        }
        md[i2 + sxy * m] = valid ? (float)(mns / (double)m0s) : NAN;
    }
}

// objective.hpp:7-31
__global__ void residual_kernel(const float* od, const float* oe, const float* om,
                                const float* md, const float* mw, const float* mm, int n,
                                float weight, float* res)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float r = md[i] - od[i];
        if (oe) r /= oe[i];
        if (mw) r *= mw[i];
        if (om) r *= om[i];
        if (mm) r *= mm[i];
        res[i] = r * weight;
    }
}

// Deterministic sum of r^2 or |r|: fixed per-thread strides, warp shuffles,
// one partial per block (fp32 within a block, fp64 across blocks), final
// fp64 sum by a single block in index order.
constexpr int SUM_BLOCKS = 296;   // 2 x 148 SMs
constexpr int SUM_THREADS = 512;

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(SUM_THREADS) residual_sum_partial(const float* r, int n,
                                                                    int squared, double* part)
{
    __shared__ float ws[SUM_THREADS / 32];
    float acc = 0;
    const int n4 = n / 4;
    const float4* r4 = reinterpret_cast<const float4*>(r);
    const bool aligned = (reinterpret_cast<uintptr_t>(r) & 15) == 0;
    int start = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (aligned) {
        for (int i = start; i < n4; i += stride) {
            float4 v = r4[i];
            acc += squared ? v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w
                           : fabsf(v.x) + fabsf(v.y) + fabsf(v.z) + fabsf(v.w);
        }
        for (int i = 4 * n4 + start; i < n; i += stride)
            acc += squared ? r[i] * r[i] : fabsf(r[i]);
    } else {
        for (int i = start; i < n; i += stride) acc += squared ? r[i] * r[i] : fabsf(r[i]);
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < SUM_THREADS / 32 ? ws[threadIdx.x] : 0.f;
        v = warp_sum(v);
        if (threadIdx.x == 0) part[blockIdx.x] = (double)v;
    }
}

__global__ void residual_sum_final(const double* part, int nparts, float* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0;
        for (int i = 0; i < nparts; ++i) s += part[i];
        out[0] = (float)s;
    }
}

static int grid_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace gbk

using namespace gbk;

extern "C" int gbkb200_dmodel_dcube_downscale_f32(gbkb200_ctx* ctx, const int scale[3],
                                                  const int offset[3], const int src_size[3],
                                                  const int dst_size[3], const float* src,
                                                  float* dst)
{
    if (!ctx || !scale || !offset || !src_size || !dst_size || !src || !dst)
        return GBKB200_ERR_INVALID_ARG;
    for (int i = 0; i < 3; ++i) {
        if (scale[i] < 1 || offset[i] < 0 || dst_size[i] < 0) return GBKB200_ERR_INVALID_ARG;
        if (offset[i] + dst_size[i] * scale[i] > src_size[i]) return GBKB200_ERR_INVALID_ARG;
    }
    long long n = (long long)dst_size[0] * dst_size[1] * dst_size[2];
    if (n == 0) return gbk_finish(ctx);
    downscale_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(
        scale[0], scale[1], scale[2], offset[0], offset[1], offset[2], src_size[0], src_size[1],
        dst_size[0], dst_size[1], dst_size[2], src, dst);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}

extern "C" int gbkb200_dmodel_dcube_mask_f32(gbkb200_ctx* ctx, float cutoff, int apply,
                                             const int size[3], float* dcube_d, float* dcube_m,
                                             float* dcube_w)
{
    (void)dcube_w;   // dmodels.hpp:55-57: weights are not touched
    if (!ctx || !size || !dcube_d) return GBKB200_ERR_INVALID_ARG;
    long long n = (long long)size[0] * size[1] * size[2];
    if (n < 0) return GBKB200_ERR_INVALID_ARG;
    if (n == 0) return gbk_finish(ctx);
    mask_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(cutoff, apply, n, dcube_d, dcube_m);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}

extern "C" int gbkb200_dmodel_mmaps_moments_f32(gbkb200_ctx* ctx, const int size[3],
                                                const float step[3], const float zero[3],
                                                const float* dcube_d, const float* dcube_w,
                                                float cutoff, int norders, const int* orders,
                                                float* mmaps_d, float* mmaps_m, float* mmaps_w)
{
    if (!ctx || !size || !step || !zero || !dcube_d || norders < 1 || !orders || !mmaps_d)
        return GBKB200_ERR_INVALID_ARG;
    // the native module's mmaps_m slot holds the weight map and its mmaps_w
    // slot the mask map (host/kernels.hpp:124-131 swaps them back)
    float* mask = mmaps_w;
    float* wmap = mmaps_m;
    if (!mask || (dcube_w && !wmap)) return GBKB200_ERR_INVALID_ARG;
    if (size[0] < 1 || size[1] < 1 || size[2] < 1) return GBKB200_ERR_INVALID_ARG;
    dim3 grid((size[0] + 127) / 128, size[1]);
    moments_kernel<<<grid, 128, 0, ctx->stream>>>(size[0], size[1], size[2], step[2], zero[2],
                                                  dcube_d, dcube_w, cutoff, norders, orders,
                                                  mmaps_d, mask, wmap);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}

extern "C" int gbkb200_objective_residual_f32(gbkb200_ctx* ctx, const float* obs_d,
                                              const float* obs_e, const float* obs_m,
                                              const float* mdl_d, const float* mdl_w,
                                              const float* mdl_m, int size, float weight,
                                              float* residual)
{
    if (!ctx || !obs_d || !mdl_d || !residual || size < 0) return GBKB200_ERR_INVALID_ARG;
    if (size == 0) return gbk_finish(ctx);
    residual_kernel<<<grid_for(size, 256), 256, 0, ctx->stream>>>(obs_d, obs_e, obs_m, mdl_d,
                                                                  mdl_w, mdl_m, size, weight,
                                                                  residual);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}

extern "C" int gbkb200_objective_residual_sum_f32(gbkb200_ctx* ctx, const float* residual,
                                                  int size, int squared, float* sum)
{
    if (!ctx || !sum || size < 0 || (size > 0 && !residual)) return GBKB200_ERR_INVALID_ARG;
    size_t need = SUM_BLOCKS * sizeof(double);
    if (ctx->reduce_scratch_bytes < need) {
        if (ctx->reduce_scratch) cudaFree(ctx->reduce_scratch);
        ctx->reduce_scratch = nullptr;
        ctx->reduce_scratch_bytes = 0;
        if (cudaMalloc(&ctx->reduce_scratch, need) != cudaSuccess) return GBKB200_ERR_OOM;
        ctx->reduce_scratch_bytes = need;
    }
    double* part = static_cast<double*>(ctx->reduce_scratch);
    residual_sum_partial<<<SUM_BLOCKS, SUM_THREADS, 0, ctx->stream>>>(residual, size, squared, part);
    residual_sum_final<<<1, 32, 0, ctx->stream>>>(part, SUM_BLOCKS, sum);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}
