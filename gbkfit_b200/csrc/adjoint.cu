// Differentiable chi^2 of a thin smooth disk (no reference counterpart: the
// reference computes no gradients).  Forward: smdisk_evaluate on the padded
// grid (gmodels.hpp:645-958), fft_convolve_cached (fft.hpp:98-125), crop,
// residual and sum of squares (objective.hpp:7-31, host/kernels.hpp:502-514),
// with a multiplicative scale on the convolved model.  Adjoint:
//   1. chi2_adjoint_kernel: one pass over the padded cube; the crop voxels give
//      r = (scale conv - d) / e * mask * weight, chi^2 = sum r^2 and
//      g = d(chi^2)/d(conv) = 2 r mask weight / e * scale (0 outside the crop);
//   2. (host) g is convolved with the point-reflected PSF x LSF cube (the
//      adjoint of the circular convolution), giving G = d(chi^2)/d(model);
//   3. smdisk_nw_adjoint_kernel: every spaxel recomputes its ring position,
//      interpolation weights and line (nothing from the forward pass is
//      stored), sums G against the line's derivatives over its channel window
//      and chains them to the sub-node values and the geometry parameters.
#include "gbk_disk.cuh"

#include <climits>
#include <cmath>

namespace gbk {

constexpr int ADJ_BLOCKS = 296;     // 2 x 148 SMs, fixed: deterministic partials
constexpr int ADJ_THREADS = 256;

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Pass over the padded cube (pz, py, px); the crop [off, off + n) is compared
// with the data (nz, ny, nx).  part: (ADJ_BLOCKS, 2) fp64 partials of chi^2
// and d(chi^2)/d(scale).
__global__ void __launch_bounds__(ADJ_THREADS) chi2_adjoint_kernel(
    int px, int py, int pz, int ox, int oy, int oz, int nx, int ny, int nz, const float* conv,
    const float* od, const float* oe, const float* om, float weight, float scale, float* g,
    double* part)
{
    __shared__ double ws[2][ADJ_THREADS / 32];
    double c2 = 0.0, ds = 0.0;
    const long long total = (long long)px * py * pz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % px), y = (int)((i / px) % py), z = (int)(i / ((long long)px * py));
        const int cx = x - ox, cy = y - oy, cz = z - oz;
        float gv = 0.f;
        if (cx >= 0 && cx < nx && cy >= 0 && cy < ny && cz >= 0 && cz < nz) {
            const long long v = cx + (long long)nx * (cy + (long long)ny * cz);
            const float c = conv[i];
            float w = weight;
            if (om) w *= om[v];
            float r = scale * c - od[v];
            if (oe) {
                r /= oe[v];
                w /= oe[v];
            }
            if (om) r *= om[v];
            r *= weight;
            c2 += (double)(r * r);
            ds += 2.0 * (double)r * (double)w * (double)c;
            gv = 2.f * r * w * scale;
        }
        g[i] = gv;
    }
    c2 = warp_sum_d(c2);
    ds = warp_sum_d(ds);
    if ((threadIdx.x & 31) == 0) {
        ws[0][threadIdx.x >> 5] = c2;
        ws[1][threadIdx.x >> 5] = ds;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < ADJ_THREADS / 32; ++k) {
            a += ws[0][k];
            b += ws[1][k];
        }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

// sums nbins columns of (ADJ_BLOCKS, nbins) partials in block order
__global__ void sum_partials_kernel(const double* part, int nbins, double* out)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nbins; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < ADJ_BLOCKS; ++b) s += part[(long long)b * nbins + j];
        out[j] = s;
    }
}

struct NwArgs {
    int sx, sy, nz;
    float stx, sty, zx, zy, spec_step, spec_zero;
    int nsub;
    const float *rnodes, *vsys, *xpos, *ypos, *posa, *incl, *bsub, *vsub, *dsub;
};

// Gradient bins: [0, nsub) density sub-nodes, [nsub, 2 nsub) rotation,
// [2 nsub, 3 nsub) dispersion, then vsys, xpos, ypos, posa (deg), incl (deg).
__global__ void __launch_bounds__(ADJ_THREADS) smdisk_nw_adjoint_kernel(NwArgs a, const float* G,
                                                                        double* part)
{
    extern __shared__ double bins[];
    const int nb = 3 * a.nsub + 5;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) bins[j] = 0.0;
    __syncthreads();
    const float phi = a.posa[0] * GBK_D2R, inc = a.incl[0] * GBK_D2R;
    float sp, cp, si, ci;
    sincosf(phi, &sp, &cp);
    sincosf(inc, &si, &ci);
    const float ti = si / ci, vsys = a.vsys ? a.vsys[0] : 0.f;
    const long long plane = (long long)a.sx * a.sy;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % a.sx), y = (int)(i / a.sx);
        // sky -> disk (gmodels.hpp:143-157), as in the forward kernel
        const float xn = a.zx + x * a.stx - a.xpos[0], yn = a.zy + y * a.sty - a.ypos[0];
        float xr = xn, yr = yn;
        rot_lh_z(xr, yr, sp, cp);
        const float yd = yr / ci;
        const float r = sqrtf(xr * xr + yd * yd);
        int k;
        if (!disk_info(k, r, a.nsub, a.rnodes)) continue;
        const float s0 = a.rnodes[k - 1], s1 = a.rnodes[k], ds_ = s1 - s0;
        const float t = (r - s0) / ds_;
        const float b0 = a.bsub[k - 1], b1 = a.bsub[k];
        const float v0 = a.vsub[k - 1], v1 = a.vsub[k];
        const float d0 = a.dsub[k - 1], d1 = a.dsub[k];
        const float bl = b0 + t * (b1 - b0);
        if (bl == 0.f) continue;                       // the forward skips the spaxel
        const float rho = bl / ci;
        const float c = r > 0.f ? cosf(atan2f(yd, xr)) : 0.f;
        const float vrot = v0 + t * (v1 - v0);
        const float vv = (r > 0.f ? vrot * c * si : 0.f) + vsys;
        const float draw = d0 + t * (d1 - d0);
        const float sig = fabsf(draw), sgn = draw < 0.f ? -1.f : 1.f;
        int lo, hi;
        if (!line_window(vv, sig, a.nz, a.spec_step, a.spec_zero, lo, hi)) continue;
        // sums over the channel window of G times the line and its derivatives
        const float amp = 1 / (sig * sqrtf(2 * GBK_PI)), i2 = 2 * sig * sig;
        float S0 = 0.f, S1 = 0.f, S2 = 0.f;
        const float* col = G + x + (long long)a.sx * y;
        for (int z = lo; z <= hi; ++z) {
            const float zv = a.spec_zero + z * a.spec_step;
            const float d = zv - vv;
            const float L = amp * expf(-d * d / i2);
            const float gl = col[plane * z] * L;
            S0 += gl;
            S1 += gl * d;
            S2 += gl * d * d;
        }
        const float isg = 1 / sig;
        const float drho = S0;                                     // d chi2 / d rho
        const float dvv = rho * S1 * isg * isg;                    // d chi2 / d v
        const float dsig = rho * (S2 * isg * isg * isg - S0 * isg); // d chi2 / d sigma
        // sub-node values
        const float wb = drho / ci, wv = r > 0.f ? dvv * c * si : 0.f, wd = dsig * sgn;
        atomicAdd(&bins[k - 1], (double)((1 - t) * wb));
        atomicAdd(&bins[k], (double)(t * wb));
        atomicAdd(&bins[a.nsub + k - 1], (double)((1 - t) * wv));
        atomicAdd(&bins[a.nsub + k], (double)(t * wv));
        atomicAdd(&bins[2 * a.nsub + k - 1], (double)((1 - t) * wd));
        atomicAdd(&bins[2 * a.nsub + k], (double)(t * wd));
        // geometry: through r, cos(theta) and the inclination
        const float dr = wb * (b1 - b0) / ds_ + wv * (v1 - v0) / ds_ + wd * (d1 - d0) / ds_;
        const float dc = r > 0.f ? dvv * vrot * si : 0.f;
        float di = drho * rho * ti + (r > 0.f ? dvv * vrot * c * ci : 0.f);
        float dxr = 0.f, dyd = 0.f;
        if (r > 0.f) {
            const float ir = 1 / r, cs = xr * ir, sn = yd * ir;
            dxr = dr * cs + dc * sn * sn * ir;
            dyd = dr * sn - dc * cs * sn * ir;
        }
        const float dyr = dyd / ci;
        di += dyd * yd * ti;
        const float dxn = -dxr * sp - dyr * cp, dyn = dxr * cp - dyr * sp;
        const float dphi = dxr * yr - dyr * xr;
        const int g0 = 3 * a.nsub;
        atomicAdd(&bins[g0 + 0], (double)dvv);
        atomicAdd(&bins[g0 + 1], (double)-dxn);
        atomicAdd(&bins[g0 + 2], (double)-dyn);
        atomicAdd(&bins[g0 + 3], (double)(dphi * GBK_D2R));
        atomicAdd(&bins[g0 + 4], (double)(di * GBK_D2R));
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nb; j += blockDim.x) part[(long long)blockIdx.x * nb + j] = bins[j];
}

static int ctx_scratch(gbkb200_ctx* ctx, size_t need, double** out)
{
    if (ctx->reduce_scratch_bytes < need) {
        if (ctx->reduce_scratch) cudaFree(ctx->reduce_scratch);
        ctx->reduce_scratch = nullptr;
        ctx->reduce_scratch_bytes = 0;
        if (cudaMalloc(&ctx->reduce_scratch, need) != cudaSuccess) return GBKB200_ERR_OOM;
        ctx->reduce_scratch_bytes = need;
    }
    *out = static_cast<double*>(ctx->reduce_scratch);
    return GBKB200_OK;
}

}  // namespace gbk

using namespace gbk;

extern "C" int gbkb200_objective_chi2_adjoint_f32(gbkb200_ctx* ctx, const int size_p[3],
                                                  const int offset[3], const int size[3],
                                                  const float* conv_p, const float* obs_d,
                                                  const float* obs_e, const float* obs_m,
                                                  float weight, float scale, float* g_p,
                                                  double* out)
{
    if (!ctx || !size_p || !offset || !size || !conv_p || !obs_d || !g_p || !out)
        return GBKB200_ERR_INVALID_ARG;
    for (int k = 0; k < 3; ++k)
        if (size_p[k] < 1 || size[k] < 1 || offset[k] < 0 || offset[k] + size[k] > size_p[k])
            return GBKB200_ERR_INVALID_ARG;
    double* part;
    int rc = ctx_scratch(ctx, (size_t)ADJ_BLOCKS * 2 * sizeof(double), &part);
    if (rc) return rc;
    chi2_adjoint_kernel<<<ADJ_BLOCKS, ADJ_THREADS, 0, ctx->stream>>>(
        size_p[0], size_p[1], size_p[2], offset[0], offset[1], offset[2], size[0], size[1],
        size[2], conv_p, obs_d, obs_e, obs_m, weight, scale, g_p, part);
    sum_partials_kernel<<<1, 32, 0, ctx->stream>>>(part, 2, out);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}

extern "C" int gbkb200_gmodel_smdisk_nw_adjoint_f32(gbkb200_ctx* ctx,
                                                    const gbkb200_smdisk_nw_desc* d,
                                                    const float* g_cube, double* grad)
{
    if (!ctx || !d || !g_cube || !grad) return GBKB200_ERR_INVALID_ARG;
    if (d->spat_size[0] < 1 || d->spat_size[1] < 1 || d->spec_size < 1 || d->nsub < 2 ||
        !d->subrnodes || !d->xpos || !d->ypos || !d->posa || !d->incl || !d->bsub || !d->vsub ||
        !d->dsub)
        return GBKB200_ERR_INVALID_ARG;
    const int nb = 3 * d->nsub + 5;
    const size_t smem = (size_t)nb * sizeof(double);
    if (smem > 48 * 1024) return GBKB200_ERR_TOO_LARGE;
    double* part;
    int rc = ctx_scratch(ctx, (size_t)ADJ_BLOCKS * nb * sizeof(double), &part);
    if (rc) return rc;
    NwArgs a;
    a.sx = d->spat_size[0];
    a.sy = d->spat_size[1];
    a.nz = d->spec_size;
    a.stx = d->spat_step[0];
    a.sty = d->spat_step[1];
    a.zx = d->spat_zero[0];
    a.zy = d->spat_zero[1];
    a.spec_step = d->spec_step;
    a.spec_zero = d->spec_zero;
    a.nsub = d->nsub;
    a.rnodes = d->subrnodes;
    a.vsys = d->vsys;
    a.xpos = d->xpos;
    a.ypos = d->ypos;
    a.posa = d->posa;
    a.incl = d->incl;
    a.bsub = d->bsub;
    a.vsub = d->vsub;
    a.dsub = d->dsub;
    smdisk_nw_adjoint_kernel<<<ADJ_BLOCKS, ADJ_THREADS, smem, ctx->stream>>>(a, g_cube, part);
    sum_partials_kernel<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(part, nb, grad);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}
