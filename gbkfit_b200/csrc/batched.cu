// Batched smdisk -> PSF x LSF convolution -> chi^2 pipeline for many
// parameter sets of one thin disk (sampler walkers).
//
// No reference counterpart as one call: per set it computes what the
// reference computes with smdisk_evaluate (gmodels.hpp:645-958), DCube's
// fft_convolve_cached + crop (_dcube.py:245-289, fft.hpp:98-207,
// dmodels.hpp:7-46), Objective.residual and residual_sum (objective.hpp:7-31,
// host/kernels.hpp:502-514).
//
// Pruning: the crop window [e, e + N) of the convolution only reads model
// voxels in [0, W), W = N + K - 1 (no wrap-around, since P >= W), so the model
// is evaluated on the W window only and the FFT grid P is chosen freely
// (P >= W, factors 2, 3, 5, 7).  Per set:
//   K1  one block per (set, y < Wy): the spaxel row is evaluated once, its
//       lines are written into a shared-memory (z, x) slab in row groups,
//       each group gets its x-axis r2c in shared memory and is stored as
//       complex rows (z, y, kx);
//   K2  y-axis FFT of the (z < Wz, kx) columns (rows y >= Wy are zero);
//   K3  z-axis FFT of the (y, kx) columns, multiply by the PSF x LSF
//       spectrum and 1/(Px Py Pz), inverse z-axis FFT; only the crop rows
//       z in [ez, ez + Nz) are stored;
//   K4  inverse y-axis FFT of the (z < Nz, kx) columns; crop rows stored;
//   K5  x-axis c2r of the rows, crop, residual against the data and the
//       per-row fp32 partial of sum r^2 (warp shuffles);
//   K6  per set, the partials summed in a fixed order in fp64.
// Sets run in chunks whose intermediates (Wz x Py x hx complex each) stay in
// the 126 MB L2 between stages.
#include "gbk_batched.cuh"
#include "gbk_fft.cuh"

#include <climits>
#include <mutex>
#include <cmath>
#include <vector>

namespace gbk {

// per-voxel residual factor of the direct path: mask * weight / error
__global__ void k_iw(BatchKernelArgs P, float* iw, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float w = P.weight;
        if (P.msk) w *= P.msk[i];
        if (P.err) w /= P.err[i];
        iw[i] = w;
    }
}

// summed-area table of the zero-model residual^2 of each data plane, in fp64:
// T[y][x] = sum over y' < y, x' < x of ((0 - d) / e * m * weight)^2 (fp32 terms,
// as the residual kernels compute them)
__global__ void k_sat(BatchKernelArgs P, double* T)
{
    const int zo = blockIdx.x, ld = P.Nx + 1;
    double* t = T + (long long)zo * (P.Ny + 1) * ld;
    const long long base = (long long)zo * P.Ny * P.Nx;
    for (int x = threadIdx.x; x <= P.Nx; x += blockDim.x) t[x] = 0.0;
    for (int y = threadIdx.x; y < P.Ny; y += blockDim.x) {
        double s = 0.0;
        t[(long long)(y + 1) * ld] = 0.0;
        for (int x = 0; x < P.Nx; ++x) {
            const long long vi = base + (long long)y * P.Nx + x;
            float rr = 0.f - P.obs[vi];
            if (P.err) rr /= P.err[vi];
            if (P.msk) rr *= P.msk[vi];
            rr *= P.weight;
            s += (double)(rr * rr);
            t[(long long)(y + 1) * ld + x + 1] = s;
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < P.Nx; x += blockDim.x) {
        double s = 0.0;
        for (int y = 0; y < P.Ny; ++y) {
            s += t[(long long)(y + 1) * ld + x + 1];
            t[(long long)(y + 1) * ld + x + 1] = s;
        }
    }
}


// K1: model row + x-axis r2c.  Shared memory: two (rows_k1 x Px/2) complex
// buffers, the x twiddles, the post twiddles and 5 floats + 2 ints per spaxel.
__global__ void __launch_bounds__(512) k1_model_xfft(BatchKernelArgs P, int* status)
{
    extern __shared__ float2 sm[];
    const int M = P.Px / 2;
    const int G = P.rows_k1;
    float2* b0 = sm;
    float2* b1 = b0 + G * M;
    float2* s_tw = b1 + G * M;
    float2* s_post = s_tw + M;
    float* s_v = reinterpret_cast<float*>(s_post + P.hx);
    float* s_amp = s_v + P.Wx;
    float* s_i2 = s_amp + P.Wx;
    float* s_orv = s_i2 + P.Wx;
    int* s_lo = reinterpret_cast<int*>(s_orv + P.Wx);
    int* s_hi = s_lo + P.Wx;

    const int y = blockIdx.x;
    const int c = blockIdx.y;
    const int b = P.set0 + c;
    const DiskArgs a = set_disk(P, b);
    int bad = 0;
    for (int i = threadIdx.x; i < M; i += blockDim.x) s_tw[i] = P.ax.tw[i];
    for (int i = threadIdx.x; i < P.hx; i += blockDim.x) s_post[i] = P.post[i];
    const DiskConst kc = disk_const(a);
    for (int x = threadIdx.x; x < P.Wx; x += blockDim.x) {
        SpaxelOut o;
        int lo = INT_MAX, hi = -1;
        float amp = 0, i2 = 1;
        if (smdisk_spaxel(a, kc, x, y, 0, o, bad) &&
            line_window(o.vv, o.dv, P.Wz, a.spec_step, a.spec_zero, lo, hi)) {
            amp = 1 / (o.dv * sqrtf(2 * GBK_PI));
            i2 = 2 * o.dv * o.dv;
        } else {
            lo = INT_MAX;
            hi = -1;
        }
        s_v[x] = o.vv;
        s_amp[x] = amp;
        s_i2[x] = i2;
        s_orv[x] = o.orv;
        s_lo[x] = lo;
        s_hi[x] = hi;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    float* slab = reinterpret_cast<float*>(b0);   // (G, Px) reals = (G, M) complex
    for (int g0 = 0; g0 < P.Wz; g0 += G) {
        const int gn = min(G, P.Wz - g0);
        for (int i = threadIdx.x; i < G * M; i += blockDim.x) b0[i] = make_float2(0.f, 0.f);
        __syncthreads();
        // lines: a warp per spaxel, lanes along the channel window
        for (int x = warp; x < P.Wx; x += nwarps) {
            int lo = max(s_lo[x], g0), hi = min(s_hi[x], g0 + gn - 1);
            // empty windows carry lo = INT_MAX: skip them before adding the
            // lane offset (lo + lane would overflow)
            if (lo > hi) continue;
            float v = s_v[x], amp = s_amp[x], i2 = s_i2[x], orv = s_orv[x];
            for (int z = lo + lane; z <= hi; z += 32) {
                float zv = a.spec_zero + z * a.spec_step;
                float d = zv - v;
                const int si = (z - g0) * P.Px + x;
                if (GBK_OK_IDX(si, 2 * G * M, 1)) slab[si] = orv * (amp * expf(-d * d / i2));
            }
        }
        __syncthreads();
        float2* r = fft_smem(b0, b1, P.ax, G, 1, M, true, s_tw, false);
        // even/odd split into hx = M + 1 bins, stored as rows (z, y, kx)
        float2* out = P.work + (((long long)c * P.Wz + g0) * P.Py + y) * P.hx;
        const long long zs = (long long)P.Py * P.hx;
        const unsigned long long mhx = fdiv_magic(P.hx);
        for (int e = threadIdx.x; e < gn * P.hx; e += blockDim.x) {
            const int l = fdiv(e, mhx), k = e - l * P.hx;
            // k in [0, M]: k mod M and (M - k) mod M without a division
            float2 zk = r[l * M + (k == M ? 0 : k)];
            float2 zc = conjf2(r[l * M + (k == 0 ? 0 : M - k)]);
            float2 ev = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
            float2 od = make_float2(0.5f * (zk.x - zc.x), 0.5f * (zk.y - zc.y));
            float2 t = cmul(s_post[k], make_float2(od.y, -od.x));
            if (GBK_OK_IDX((out - P.work) + l * zs + k, P.lim_work, 2))
                out[l * zs + k] = cadd(ev, t);
        }
        __syncthreads();
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// K2/K3/K4: transforms of columns (o, i) of the chunk's complex cubes,
// element k at set * set_stride + o * so + i + k * sk.  Rows k >= nload are
// zero on input.  mode 0: one transform; mode 1: forward, multiply by
// spec[o * spec_so + i + k * spec_sk] * scale, inverse.  Output rows
// [s0, s0 + ns) are stored to rows [0, ns).
constexpr int BLT = 16;

__global__ void __launch_bounds__(256) k_lines(float2* data, long long set_stride, int inner,
                                                long long so, long long sk, AxisDev ax, int inv,
                                                int mode, const float2* spec, long long spec_so,
                                                long long spec_sk, float scale, int nload, int s0,
                                                int ns, long long lim_data, long long lim_spec)
{
    (void)lim_data;
    (void)lim_spec;
    extern __shared__ float2 sm[];
    const int n = ax.n;
    float2* b0 = sm;
    float2* b1 = b0 + BLT * n;
    float2* s_tw = b1 + BLT * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_tw[i] = ax.tw[i];
    const int tiles = (inner + BLT - 1) / BLT;
    const int o = blockIdx.x / tiles;
    const int i0 = (blockIdx.x % tiles) * BLT;
    const long long base = (long long)blockIdx.y * set_stride + (long long)o * so + i0;
    staged_copy<8>(
        BLT * n,
        [&](int e) {
            const int l = e % BLT, k = e / BLT;
            const long long gi = base + l + k * sk;
            return (i0 + l < inner && k < nload && GBK_OK_IDX(gi, lim_data, 10))
                       ? data[gi] : make_float2(0.f, 0.f);
        },
        [&](int e, float2 v) { b0[e] = v; });
    __syncthreads();
    float2* res = fft_smem(b0, b1, ax, BLT, BLT, 1, false, s_tw, mode == 0 ? inv != 0 : false);
    if (mode == 1) {
        const long long sbase = (long long)o * spec_so + i0;
        staged_copy<8>(
            BLT * n,
            [&](int e) {
                const int l = e % BLT, k = e / BLT;
                return (i0 + l < inner && GBK_OK_IDX(sbase + l + k * spec_sk, lim_spec, 11))
                           ? spec[sbase + l + k * spec_sk] : make_float2(0.f, 0.f);
            },
            [&](int e, float2 w) {
                if (i0 + e % BLT < inner) {
                    const float2 a = res[e];
                    res[e] = make_float2((a.x * w.x - a.y * w.y) * scale,
                                         (a.x * w.y + a.y * w.x) * scale);
                }
            });
        __syncthreads();
        res = fft_smem(res, res == b0 ? b1 : b0, ax, BLT, BLT, 1, false, s_tw, true);
    }
    for (int e = threadIdx.x; e < BLT * ns; e += blockDim.x) {
        int l = e % BLT, k = e / BLT;
        if (i0 + l < inner && GBK_OK_IDX(base + l + k * sk, lim_data, 12) &&
            GBK_OK_IDX((k + s0) * BLT + l, BLT * n, 13))
            data[base + l + k * sk] = res[(k + s0) * BLT + l];
    }
}

// K5: x-axis c2r of rows_k5 rows (z, y), crop, residual and r^2 partials.
__global__ void __launch_bounds__(256) k5_c2r_residual(BatchKernelArgs P)
{
    extern __shared__ float2 sm[];
    const int M = P.Px / 2;
    const int G = P.rows_k5;
    float2* b0 = sm;
    float2* b1 = b0 + G * M;
    float2* s_tw = b1 + G * M;
    float2* s_post = s_tw + M;
    __shared__ float warp_part[8];
    const int yg = blockIdx.x, z = blockIdx.y, c = blockIdx.z;
    const int b = P.set0 + c;
    const int y0 = yg * G;
    const int gn = min(G, P.Ny - y0);
    for (int i = threadIdx.x; i < M; i += blockDim.x) s_tw[i] = P.ax.tw[i];
    for (int i = threadIdx.x; i < P.hx; i += blockDim.x) s_post[i] = P.post[i];
    __syncthreads();
    const float2* rows = P.work + (((long long)c * P.Wz + z) * P.Py + y0) * P.hx;
    for (int e = threadIdx.x; e < G * M; e += blockDim.x) {
        const int l = fdiv(e, P.ax.mn), k = e - l * M;
        float2 v = make_float2(0.f, 0.f);
        if (l < gn && GBK_OK_IDX((rows - P.work) + (long long)l * P.hx + M, P.lim_work, 20)) {
            const float2* r = rows + (long long)l * P.hx;
            float2 a = r[k], bb = conjf2(r[M - k]);
            float2 s = cadd(a, bb), d = csub(a, bb);
            float2 t = cmul(conjf2(s_post[k]), d);
            v = make_float2(s.x - t.y, s.y + t.x);
        }
        b0[l * M + k] = v;
    }
    __syncthreads();
    float2* res = fft_smem(b0, b1, P.ax, G, 1, M, true, s_tw, true);
    const float* real = reinterpret_cast<const float*>(res);   // (G, Px) reals
    float acc = 0.f;
    const unsigned long long mnx = fdiv_magic(P.Nx);
    for (int e = threadIdx.x; e < gn * P.Nx; e += blockDim.x) {
        const int l = fdiv(e, mnx), x = e - l * P.Nx;
        if (!GBK_OK_IDX(l * P.Px + x + P.ex, 2 * G * M, 21)) continue;
        float m = real[l * P.Px + x + P.ex];
        long long vi = ((long long)z * P.Ny + (y0 + l)) * P.Nx + x;
        if (!GBK_OK_IDX(vi, P.lim_obs, 22)) continue;
        if (P.model && GBK_OK_IDX((long long)b * P.Nz * P.Ny * P.Nx + vi, P.lim_model, 23))
            P.model[(long long)b * P.Nz * P.Ny * P.Nx + vi] = m;
        // objective.hpp:7-31
        float r = m - P.obs[vi];
        if (P.err) r /= P.err[vi];
        if (P.msk) r *= P.msk[vi];
        r *= P.weight;
        acc += r * r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += warp_part[w];
        const int ngroups = (P.Ny + G - 1) / G;
        if (GBK_OK_IDX(((long long)b * P.Nz + z) * ngroups + yg, P.lim_part, 24))
            P.partials[((long long)b * P.Nz + z) * ngroups + yg] = (double)s;
    }
}

// K6: per set, fixed-order fp64 sum of its partials.
__global__ void __launch_bounds__(256) k6_sum(const double* partials, int nper, int set0,
                                               float* chi2)
{
    __shared__ double sh[256];
    const int b = set0 + blockIdx.x;
    double s = 0;
    for (int i = threadIdx.x; i < nper; i += blockDim.x) s += partials[(long long)b * nper + i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) chi2[b] = (float)sh[0];
}

}  // namespace gbk

using namespace gbk;

#ifdef GBK_CHECKED
// checked builds only: copies and clears the first violation recorded by the
// kernels of this file
extern "C" int gbkb200_debug_record(long long out[4])
{
    long long zero[4] = {0, 0, 0, 0};
    GBK_CUDA_TRY(cudaDeviceSynchronize());
    GBK_CUDA_TRY(cudaMemcpyFromSymbol(out, gbk_debug_record, sizeof(zero)));
    GBK_CUDA_TRY(cudaMemcpyToSymbol(gbk_debug_record, zero, sizeof(zero)));
    return GBKB200_OK;
}
#endif

struct gbkb200_batch {
    gbkb200_ctx* ctx = nullptr;
    BatchKernelArgs P{};
    int max_sets = 0, chunk = 0;
    size_t smem1 = 0, smem5 = 0, smem_y = 0, smem_z = 0;
    float2* tw[3] = {nullptr, nullptr, nullptr};
    float2* post = nullptr;
    float2* kspec = nullptr;
    float2* work = nullptr;
    double* partials = nullptr;
    int nper = 0;
    int direct = 0;
    int trim[3] = {0, 0, 0};          // direct mode: taps trimmed from each end (x, y, z)
    int ka_variant = 0;               // direct mode: the model kernel (model_variant)
    int kb_grid = 0;                  // persistent PSF kernel: blocks of a launch (else 0)
    int kb_threads = KB_THREADS;      // threads of a PSF-kernel block
    int* kb_work = nullptr;           // persistent PSF kernel: its item counter
    cudaEvent_t done = nullptr;       // recorded at the end of an asynchronous submission
    size_t smemB = 0;
    float* mplanes = nullptr;
    int* xrt = nullptr;
    double* sat = nullptr;
    float* iw = nullptr;
    void (*kb)(BatchKernelArgs) = nullptr;
    void (*ka)(BatchKernelArgs, int*) = nullptr;
    // per-stage timing: event pairs recorded around launches while enabled
    int timing = 0;
    int count = 0;                            // work counters on (timing mode 1)
    unsigned long long* counters = nullptr;   // device, GBK_CTR_N (direct mode, timing on)
    std::vector<cudaEvent_t> ev;      // 2 per record
    std::vector<int> ev_stage;
    size_t ev_used = 0;
    int ev_error = 0;
};

// records an event before (begin) or after (end) a launch of `stage`
static void stage_mark(gbkb200_batch* bt, int stage, bool begin)
{
    if (!bt->timing || bt->ev_error) return;
    const size_t i = begin ? 2 * bt->ev_used : 2 * bt->ev_used + 1;
    if (i >= bt->ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) {
            bt->ev_error = 1;
            return;
        }
        bt->ev.push_back(e);
    }
    cudaEventRecord(bt->ev[i], bt->ctx->stream);
    if (begin) {
        if (bt->ev_stage.size() <= bt->ev_used) bt->ev_stage.resize(bt->ev_used + 1);
        bt->ev_stage[bt->ev_used] = stage;
    } else {
        ++bt->ev_used;
    }
}

// the PSF kernel over cn sets: a block per (set, plane, band), or the
// persistent variant's resident wave over all of them
static void launch_kb(const gbkb200_batch* bt, BatchKernelArgs& P, int cn, cudaStream_t st)
{
    if (bt->kb_grid > 0) {
        P.kb_cn = cn;
        const long long items = (long long)cn * P.Nz * P.nbands;
        const int grid = (int)std::min<long long>(items, bt->kb_grid);
        cudaMemsetAsync(bt->kb_work, 0, sizeof(int), st);
        bt->kb<<<grid, bt->kb_threads, bt->smemB, st>>>(P);
    } else {
        bt->kb<<<dim3(cn, P.Nz * P.nbands), bt->kb_threads, bt->smemB, st>>>(P);
    }
}

static KaFn ka_fn(int Kz)
{
    static KaFn t[KA_KMAX / 2 + 1] = {};
    if (!t[0]) {
        ka_register_short(t);
        ka_register_long(t);
    }
    return t[Kz / 2];
}

// form 0: ballot masks, 1: transposed masks, 2: transposed masks and the scaled line
static KaFn ka_t_fn(int Kz, int form)
{
    static KaFn t[3][KA_KMAX / 2 + 1] = {};
    static std::once_flag once;
    std::call_once(once, [] {
        ka_t_register(t[0], false, false);
        ka_t_register(t[1], true, false);
        ka_t_register(t[2], true, true);
    });
    return t[form][Kz / 2];
}

static KaFn ka2_fn(int Kz)
{
    static KaFn t[KA_KMAX / 2 + 1] = {};
    static std::once_flag once;
    std::call_once(once, [] { ka2_register(t); });
    return t[Kz / 2];
}

static KcFn kc_fn(int Kz)
{
    static KcFn t[KA_KMAX / 2 + 1] = {};
    static std::once_flag once;
    std::call_once(once, [] { kc_register(t); });
    return t[Kz / 2];
}

static KbFn kb_fn(int K, int variant)
{
    static KbFn t[KB_VARIANTS][(KB_KMAX - KB_KMIN) / 2 + 1] = {};
    static std::once_flag once;
    std::call_once(once, [] {
        kb_register4(t);
        kb_register5(t + 3);
        kb_register_pf(t + 6);
        kb_register_wide(t + 7);
    });
    return t[variant][(K - KB_KMIN) / 2];
}

// Direct-mode setup: reversed FIR coefficients, plane buffers, the data's
// summed-area table and shared memory sizes.  Returns
// GBKB200_ERR_UNSUPPORTED when the direct path does not apply (PSF rank or
// size, cube size, shared memory).
static int setup_direct(gbkb200_batch* bt, const gbkb200_batch_desc* d)
{
    BatchKernelArgs& P = bt->P;
    if (d->psf_rank != 1 || !d->psf_u || !d->psf_v) return GBKB200_ERR_UNSUPPORTED;
    // Taps below 2^-35 of their factor's largest are dropped from both ends
    // (symmetrically, the centre stays): they change no output by more than
    // ~1e-10 of its peak, below fp32 resolution.  The evaluation window then
    // starts t taps later along each axis and is 2 t shorter, so every kept
    // tap meets the same model voxel as before.
    auto trim = [](const double* a, int n) {
        double m = 0;
        for (int i = 0; i < n; ++i) m = std::max(m, std::fabs(a[i]));
        const double thr = std::ldexp(m, -35);
        int t = 0;
        while (2 * t + 1 < n && std::fabs(a[t]) < thr && std::fabs(a[n - 1 - t]) < thr) ++t;
        return t;
    };
    const int tx = trim(d->psf_v, d->kernel_size[0]), ty = trim(d->psf_u, d->kernel_size[1]);
    const int tz = trim(d->lsf, d->kernel_size[2]);
    bt->trim[0] = tx; bt->trim[1] = ty; bt->trim[2] = tz;
    P.Kx = d->kernel_size[0] - 2 * tx;
    P.Ky = d->kernel_size[1] - 2 * ty;
    P.Kz = d->kernel_size[2] - 2 * tz;
    P.Wx = P.Nx + P.Kx - 1;
    P.Wy = P.Ny + P.Ky - 1;
    P.Wz = P.Nz + P.Kz - 1;
    P.disk.sx = P.Wx;
    P.disk.sy = P.Wy;
    P.disk.spec_size = P.Wz;
    P.disk.zx = d->spat_zero[0] + tx * d->spat_step[0];
    P.disk.zy = d->spat_zero[1] + ty * d->spat_step[1];
    P.disk.spec_zero = d->spec_zero + tz * d->spec_step;
    P.K = std::max(KB_KMIN, std::max(P.Kx, P.Ky) | 1);
    if (P.K > KB_KMAX || P.Kz > KA_KMAX || P.Nx > KB_NX_MAX || P.Wx > 1024 ||
        (long long)P.Nx * P.Ny * P.Nz >= (1LL << 31))
        return GBKB200_ERR_UNSUPPORTED;
    const int NW = (P.K + 7 + 3) / 4;
    P.pitch = (P.Wx + 31) / 32 * 32;
    P.nch = (P.Wx + 31) / 32;
    // the node-wise fast path of the spaxel evaluation: exactly one trait of
    // uid 101 for rpt, vpt, dpt and none of the other kinds
    {
        bool fast = !d->loose && !d->tilted;
        for (int k = 0; k < 9 && fast; ++k) {
            const bool want = k == 0 || k == 2 || k == 4;
            if (!want) {
                fast = d->ntraits[k] == 0;
                continue;
            }
            int uid = 0;
            fast = d->ntraits[k] == 1 && d->uids[k] &&
                   cudaMemcpy(&uid, d->uids[k], sizeof(int), cudaMemcpyDeviceToHost) ==
                       cudaSuccess &&
                   uid == 101;
        }
        P.nwfast = fast ? 1 : 0;
    }
    int band = d->psf_band > 0 ? std::min(d->psf_band, P.Ny) : P.Ny;
    P.nbands = (P.Ny + band - 1) / band;
    P.band = (P.Ny + P.nbands - 1) / P.nbands;
    // shared memory of a PSF block: rows of one pass at the widest box pitch;
    // at least K + 15 rows (8 output rows a pass), at most the whole band,
    // otherwise 54 KB (four blocks per SM)
    int bpmax = 4 * (2 * ((P.Nx + 7) / 8 - 1) + NW);
    bpmax += ((4 - bpmax % 32) + 32) % 32;
    // range entries of the band's input rows (the persistent variant 6: two
    // buffers, each rounded to 4 entries)
    const bool pf = d->psf_variant == 6;
    const long long xr_slot = ((long long)(P.band + P.K - 1) * P.nch + 3) & ~3LL;
    const long long xr_bytes = pf ? 2 * xr_slot * (long long)sizeof(int)
                                  : (long long)(P.band + P.K - 1) * P.nch * sizeof(int);
    const long long need_min = (long long)(P.K + 15) * bpmax;
    const long long need_all = (long long)(P.band + P.K + 7) * bpmax;
    // PSF kernel variant: 0-2 sized for 4 resident blocks per SM, 3-5 for 5,
    // epilogue (variant % 3) as in kb_psf_residual, 6 = 0 as a persistent
    // kernel; shared memory per block: 55 KB for 4 blocks per SM, 43 KB for 5
    if (d->psf_variant < 0 || d->psf_variant >= KB_VARIANTS) return GBKB200_ERR_INVALID_ARG;
    const bool wide = d->psf_variant == 7;
    const int blocks = (d->psf_variant >= 3 && d->psf_variant <= 5) ? 5 : 4;
    // variant 7: 256-thread blocks, two per SM, 110 KB each
    const long long budget = wide ? 110LL * 1024 : blocks == 5 ? 43LL * 1024 : 55LL * 1024;
    bt->kb_threads = wide ? 256 : KB_THREADS;
    const long long cap = std::max(need_min, std::min(need_all, (budget - xr_bytes) / 4));
    if (cap * (long long)sizeof(float) + xr_bytes > 227LL * 1024) return GBKB200_ERR_UNSUPPORTED;
    P.cap = (int)cap;
    P.xr_slot = pf ? (int)xr_slot : 0;
    bt->smemB = (size_t)cap * sizeof(float) + (size_t)xr_bytes;
    std::vector<float> vr(P.K, 0.f), ur(P.K, 0.f), lr(P.Kz);
    for (int s = 0; s < P.Kx; ++s) vr[s] = (float)d->psf_v[d->kernel_size[0] - 1 - tx - s];
    for (int t = 0; t < P.Ky; ++t) ur[t] = (float)d->psf_u[d->kernel_size[1] - 1 - ty - t];
    for (int t = 0; t < P.Kz; ++t) lr[t] = (float)d->lsf[d->kernel_size[2] - 1 - tz - t];
    const size_t nrows = (size_t)bt->chunk * P.Nz * P.Wy;
    for (int i = 0; i < 33; ++i) {
        P.vr[i] = i < P.K ? vr[i] : 0.f;
        P.ur[i] = i < P.K ? ur[i] : 0.f;
        P.lsfr[i] = i < P.Kz ? lr[i] : 0.f;
        P.ur2[i] = make_float2(P.ur[i], P.ur[i]);
    }
    if (cudaMalloc(&bt->mplanes, nrows * P.pitch * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&bt->xrt, nrows * P.nch * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&bt->sat, (size_t)P.Nz * (P.Ny + 1) * (P.Nx + 1) * sizeof(double)) !=
            cudaSuccess ||
        cudaMalloc(&bt->iw, (size_t)P.Nz * P.Ny * P.Nx * sizeof(float)) != cudaSuccess)
        return GBKB200_ERR_OOM;
    P.mplanes = bt->mplanes;
    P.xrt = bt->xrt;
    P.sat = bt->sat;
    P.iw = bt->iw;
    k_sat<<<P.Nz, 128, 0, bt->ctx->stream>>>(P, bt->sat);
    k_iw<<<592, 256, 0, bt->ctx->stream>>>(P, bt->iw, (long long)P.Nz * P.Ny * P.Nx);
    GBK_CUDA_TRY(cudaGetLastError());
    GBK_CUDA_TRY(cudaStreamSynchronize(bt->ctx->stream));
    if (d->model_variant < 0 || d->model_variant > 4) return GBKB200_ERR_INVALID_ARG;
    // variants 2-4 (4 x 8 tiles) keep a plane's entries of its 4 rows in
    // shared memory; 3 forms the masks by bit transposes; 4 is 3 with the
    // scaled line exponent
    const bool tiles = d->model_variant >= 2;
    if (tiles && (long long)P.Nz * 16 > 32 * 1024) return GBKB200_ERR_UNSUPPORTED;
    bt->ka = d->model_variant == 1 ? ka2_fn(P.Kz)
             : tiles               ? ka_t_fn(P.Kz, d->model_variant - 2)
                                   : ka_fn(P.Kz);
    bt->ka_variant = d->model_variant;
    bt->kb = kb_fn(P.K, d->psf_variant);
    {
        const int rc = gbk_raise_smem_limit(reinterpret_cast<const void*>(bt->kb), bt->smemB);
        if (rc) return rc;
    }
    if (pf) {
        // one resident wave of blocks
        int per_sm = 0, nsm = 0;
        GBK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, reinterpret_cast<const void*>(bt->kb), bt->kb_threads, bt->smemB));
        GBK_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, bt->ctx->device));
        bt->kb_grid = std::max(1, per_sm) * std::max(1, nsm);
        if (cudaMalloc(&bt->kb_work, sizeof(int)) != cudaSuccess) return GBKB200_ERR_OOM;
        P.kb_work = bt->kb_work;
    }
    bt->nper = P.Nz * P.nbands;
    if (cudaMalloc(&bt->partials, (size_t)bt->max_sets * bt->nper * sizeof(double)) != cudaSuccess)
        return GBKB200_ERR_OOM;
    P.partials = bt->partials;
    P.lim_part = (long long)bt->max_sets * bt->nper;
    P.lim_obs = (long long)P.Nx * P.Ny * P.Nz;
    bt->direct = 1;
    return GBKB200_OK;
}

static bool fft_factor_ok(int n)
{
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}

static int auto_fft_size(int w, bool even)
{
    for (int n = w;; ++n)
        if ((!even || n % 2 == 0) && fft_factor_ok(n)) return n;
}

static int make_axis_dev(AxisDev& a, float2*& tw, int n)
{
    a.n = n;
    if (n < 1 || n > (1 << 16)) return GBKB200_ERR_UNSUPPORTED;   // fdiv_magic's range
    int m = n, nr = 0;
    int r[FFT_MAX_PASSES];
    while (m % 8 == 0 && m > 8) { r[nr++] = 8; m /= 8; }
    while (m % 4 == 0) { r[nr++] = 4; m /= 4; }
    while (m % 2 == 0) { r[nr++] = 2; m /= 2; }
    for (int p = 3; p <= 7 && m > 1; p += 2)
        while (m % p == 0) { r[nr++] = p; m /= p; }
    if (m != 1) return GBKB200_ERR_UNSUPPORTED;
    a.nr = nr;
    for (int i = 0; i < nr; ++i) a.r[i] = r[i];
    axis_fill_magics(a);
    std::vector<float2> h(n);
    for (int k = 0; k < n; ++k) {
        double ang = -2.0 * M_PI * (double)k / (double)n;
        h[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    if (cudaMalloc(&tw, n * sizeof(float2)) != cudaSuccess) return GBKB200_ERR_OOM;
    GBK_CUDA_TRY(cudaMemcpy(tw, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    a.tw = tw;
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_destroy(gbkb200_batch* bt)
{
    if (!bt) return GBKB200_OK;
    if (bt->ctx) cudaStreamSynchronize(bt->ctx->stream);
    for (auto* p : bt->tw) cudaFree(p);
    cudaFree(bt->post);
    cudaFree(bt->kspec);
    cudaFree(bt->work);
    cudaFree(bt->partials);
    cudaFree(bt->mplanes);
    cudaFree(bt->xrt);
    cudaFree(bt->sat);
    cudaFree(bt->iw);
    cudaFree(bt->counters);
    for (cudaEvent_t e : bt->ev) cudaEventDestroy(e);
    if (bt->done) cudaEventDestroy(bt->done);
    cudaFree(bt->kb_work);
    delete bt;
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_create(gbkb200_ctx* ctx, const gbkb200_batch_desc* d,
                                    gbkb200_batch** out)
{
    if (!ctx || !d || !out) return GBKB200_ERR_INVALID_ARG;
    *out = nullptr;
    if (d->uids[1] || d->nrnodes < 2 || !d->rnodes || !d->obs_d || !d->psf || !d->lsf)
        return GBKB200_ERR_INVALID_ARG;   // thin disks only
    for (int i = 0; i < 3; ++i)
        if (d->size[i] < 1 || d->kernel_size[i] < 1 || d->kernel_size[i] % 2 == 0)
            return GBKB200_ERR_INVALID_ARG;
    if (d->max_sets < 1) return GBKB200_ERR_INVALID_ARG;
    auto* bt = new gbkb200_batch();
    bt->ctx = ctx;
    BatchKernelArgs& P = bt->P;
    P.Nx = d->size[0]; P.Ny = d->size[1]; P.Nz = d->size[2];
    P.Wx = P.Nx + d->kernel_size[0] - 1;
    P.Wy = P.Ny + d->kernel_size[1] - 1;
    P.Wz = P.Nz + d->kernel_size[2] - 1;
    P.ex = d->kernel_size[0] / 2; P.ey = d->kernel_size[1] / 2; P.ez = d->kernel_size[2] / 2;
    P.Px = d->fft_size[0] > 0 ? d->fft_size[0] : auto_fft_size(P.Wx, true);
    P.Py = d->fft_size[1] > 0 ? d->fft_size[1] : auto_fft_size(P.Wy, false);
    P.Pz = d->fft_size[2] > 0 ? d->fft_size[2] : auto_fft_size(P.Wz, false);
    if (P.Px < P.Wx || P.Py < P.Wy || P.Pz < P.Wz || P.Px % 2) {
        gbkb200_batch_destroy(bt);
        return GBKB200_ERR_INVALID_ARG;
    }
    P.hx = P.Px / 2 + 1;
    P.rows_k1 = d->rows_k1 > 0 ? d->rows_k1 : 16;
    P.rows_k5 = d->rows_k5 > 0 ? d->rows_k5 : 8;
    bt->max_sets = d->max_sets;
    bt->chunk = d->chunk > 0 ? std::min(d->chunk, d->max_sets) : std::min(8, d->max_sets);
    int rc;
    if ((rc = make_axis_dev(P.ax, bt->tw[0], P.Px / 2)) ||
        (rc = make_axis_dev(P.ay, bt->tw[1], P.Py)) ||
        (rc = make_axis_dev(P.az, bt->tw[2], P.Pz))) {
        gbkb200_batch_destroy(bt);
        return rc;
    }
    // disk tables (per-set pointers are offset in set_disk)
    DiskArgs& a = P.disk;
    a.loose = d->loose; a.tilted = d->tilted; a.nrnodes = d->nrnodes; a.rnodes = d->rnodes;
    TraitSet* ts[9] = {&a.rpt, &a.rht, &a.vpt, &a.vht, &a.dpt, &a.dht, &a.zpt, &a.spt, &a.wpt};
    for (int k = 0; k < 9; ++k) {
        ts[k]->n = d->ntraits[k];
        ts[k]->uids = d->uids[k];
        ts[k]->cv = d->cvalues[k];
        ts[k]->cc = d->ccounts[k];
        ts[k]->pc = d->pcounts[k];
        ts[k]->pv = nullptr;
        P.pstride[k] = d->npvalues[k];
        if (ts[k]->n < 0 || ts[k]->n > GBK_TRAIT_NUM_MAX) {
            gbkb200_batch_destroy(bt);
            return GBKB200_ERR_INVALID_ARG;
        }
    }
    a.opacity = nullptr;
    a.sx = P.Wx; a.sy = P.Wy; a.sz = 1;
    a.stx = d->spat_step[0]; a.sty = d->spat_step[1]; a.stz = 0;
    a.zx = d->spat_zero[0]; a.zy = d->spat_zero[1]; a.zz = 0;
    a.spec_size = P.Wz; a.spec_step = d->spec_step; a.spec_zero = d->spec_zero;
    a.image = a.scube = a.wdata = a.wdata_cmp = a.rdata = a.rdata_cmp = nullptr;
    a.ordata = a.ordata_cmp = a.vdata_cmp = a.ddata_cmp = nullptr;
    const int nv = d->loose ? d->nrnodes : 1, nt = d->tilted ? d->nrnodes : 1;
    P.vstride[0] = nv; P.vstride[1] = nv; P.vstride[2] = nv; P.vstride[3] = nt; P.vstride[4] = nt;
    P.obs = d->obs_d; P.err = d->obs_e; P.msk = d->obs_m; P.weight = d->weight;
    P.scale = 1.0f / (float)((long long)P.Px * P.Py * P.Pz);
    // direct separable convolution when requested or (automatic) when it applies
    if (d->conv_mode != 1) {
        const BatchKernelArgs saved = P;     // the direct set-up trims the window
        rc = setup_direct(bt, d);
        if (rc != GBKB200_OK) P = saved;
        if (rc == GBKB200_OK) {
            GBK_CUDA_TRY(cudaGetLastError());
            *out = bt;
            return GBKB200_OK;
        }
        if (d->conv_mode == 2 || rc != GBKB200_ERR_UNSUPPORTED) {
            gbkb200_batch_destroy(bt);
            return rc;
        }
    }
    // post twiddles of the x axis
    {
        std::vector<float2> h(P.hx);
        for (int k = 0; k < P.hx; ++k) {
            double ang = -2.0 * M_PI * (double)k / (double)P.Px;
            h[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        if (cudaMalloc(&bt->post, P.hx * sizeof(float2)) != cudaSuccess) {
            gbkb200_batch_destroy(bt);
            return GBKB200_ERR_OOM;
        }
        GBK_CUDA_TRY(cudaMemcpy(bt->post, h.data(), P.hx * sizeof(float2), cudaMemcpyHostToDevice));
        P.post = bt->post;
    }
    // PSF x LSF kernel cube on the FFT grid, centre rolled to the origin,
    // and its spectrum (the same r2c as the drop-in FFT path)
    {
        const int kx = d->kernel_size[0], ky = d->kernel_size[1], kz = d->kernel_size[2];
        std::vector<float> cube((size_t)P.Px * P.Py * P.Pz, 0.f);
        for (int z = 0; z < kz; ++z)
            for (int y = 0; y < ky; ++y)
                for (int x = 0; x < kx; ++x) {
                    int X = ((x - kx / 2) % P.Px + P.Px) % P.Px;
                    int Y = ((y - ky / 2) % P.Py + P.Py) % P.Py;
                    int Z = ((z - kz / 2) % P.Pz + P.Pz) % P.Pz;
                    // _dcube.py:205: (psf * lsf) in float64, then cast
                    cube[((size_t)Z * P.Py + Y) * P.Px + X] = (float)(d->psf[y * kx + x] * d->lsf[z]);
                }
        float* dcube = nullptr;
        size_t cbytes = (size_t)P.Pz * P.Py * P.hx * sizeof(float2);
        if (cudaMalloc(&dcube, cube.size() * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&bt->kspec, cbytes) != cudaSuccess) {
            cudaFree(dcube);
            gbkb200_batch_destroy(bt);
            return GBKB200_ERR_OOM;
        }
        GBK_CUDA_TRY(cudaMemcpy(dcube, cube.data(), cube.size() * sizeof(float),
                                cudaMemcpyHostToDevice));
        int size[3] = {P.Px, P.Py, P.Pz};
        int sync = ctx->sync;
        ctx->sync = 1;
        rc = gbkb200_fft_r2c_f32(ctx, size, dcube, bt->kspec);
        ctx->sync = sync;
        cudaFree(dcube);
        if (rc) {
            gbkb200_batch_destroy(bt);
            return rc;
        }
        P.kspec = bt->kspec;
    }
    // work space and partials
    size_t wbytes = (size_t)bt->chunk * P.Wz * P.Py * P.hx * sizeof(float2);
    bt->nper = P.Nz * ((P.Ny + P.rows_k5 - 1) / P.rows_k5);
    if (cudaMalloc(&bt->work, wbytes) != cudaSuccess ||
        cudaMalloc(&bt->partials, (size_t)bt->max_sets * bt->nper * sizeof(double)) != cudaSuccess) {
        gbkb200_batch_destroy(bt);
        return GBKB200_ERR_OOM;
    }
    P.work = bt->work;
    P.partials = bt->partials;
    P.lim_work = (long long)bt->chunk * P.Wz * P.Py * P.hx;
    P.lim_part = (long long)bt->max_sets * bt->nper;
    P.lim_obs = (long long)P.Nx * P.Ny * P.Nz;
    // shared memory sizes, set once here so evaluate() can be captured
    const int M = P.Px / 2;
    bt->smem1 = (size_t)(2 * P.rows_k1 * M + M + P.hx) * sizeof(float2) +
                (size_t)P.Wx * (4 * sizeof(float) + 2 * sizeof(int));
    bt->smem5 = (size_t)(2 * P.rows_k5 * M + M + P.hx) * sizeof(float2);
    bt->smem_y = (size_t)(2 * BLT * P.Py + P.Py) * sizeof(float2);
    bt->smem_z = (size_t)(2 * BLT * P.Pz + P.Pz) * sizeof(float2);
    const size_t lim = 227 * 1024;
    if (bt->smem1 > lim || bt->smem5 > lim || bt->smem_y > lim || bt->smem_z > lim) {
        gbkb200_batch_destroy(bt);
        return GBKB200_ERR_UNSUPPORTED;
    }
    if ((rc = gbk_raise_smem_limit(reinterpret_cast<const void*>(k1_model_xfft), bt->smem1)) ||
        (rc = gbk_raise_smem_limit(reinterpret_cast<const void*>(k5_c2r_residual), bt->smem5)) ||
        (rc = gbk_raise_smem_limit(reinterpret_cast<const void*>(k_lines),
                                   std::max(bt->smem_y, bt->smem_z)))) {
        gbkb200_batch_destroy(bt);
        return rc;
    }
    GBK_CUDA_TRY(cudaGetLastError());
    *out = bt;
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_info(const gbkb200_batch* bt, int fft_size[3], int* chunk,
                                  size_t* work_bytes, int* conv_mode)
{
    if (!bt) return GBKB200_ERR_INVALID_ARG;
    if (conv_mode) *conv_mode = bt->direct ? 2 : 1;
    if (fft_size) {
        fft_size[0] = bt->P.Px; fft_size[1] = bt->P.Py; fft_size[2] = bt->P.Pz;
    }
    if (chunk) *chunk = bt->chunk;
    if (work_bytes) {
        // device bytes the evaluator holds (its scratch, tables and partials)
        const BatchKernelArgs& P = bt->P;
        size_t b = (size_t)bt->max_sets * bt->nper * sizeof(double);
        if (bt->direct) {
            const size_t nrows = (size_t)bt->chunk * P.Nz * P.Wy;
            b += nrows * P.pitch * sizeof(float) + nrows * P.nch * sizeof(int) +
                 (size_t)P.Nz * (P.Ny + 1) * (P.Nx + 1) * sizeof(double) +
                 (size_t)P.Nz * P.Ny * P.Nx * sizeof(float);
        } else {
            b += (size_t)bt->chunk * P.Wz * P.Py * P.hx * sizeof(float2) +
                 (size_t)P.Pz * P.Py * P.hx * sizeof(float2) +
                 (size_t)(P.Px / 2 + P.Py + P.Pz + P.hx) * sizeof(float2);
        }
        *work_bytes = b;
    }
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_evaluate(gbkb200_batch* bt, int nsets, const float* vsys,
                                      const float* xpos, const float* ypos, const float* posa,
                                      const float* incl, const float* const pvalues[9],
                                      float* chi2, float* model)
{
    if (!bt || nsets < 0 || nsets > bt->max_sets || !xpos || !ypos || !posa || !incl || !chi2 ||
        !pvalues)
        return GBKB200_ERR_INVALID_ARG;
    BatchKernelArgs P = bt->P;
    cudaStream_t st = bt->ctx->stream;
    DiskArgs& a = P.disk;
    a.vsys = vsys; a.xpos = xpos; a.ypos = ypos; a.posa = posa; a.incl = incl;
    TraitSet* ts[9] = {&a.rpt, &a.rht, &a.vpt, &a.vht, &a.dpt, &a.dht, &a.zpt, &a.spt, &a.wpt};
    for (int k = 0; k < 9; ++k) {
        if (ts[k]->n > 0 && !pvalues[k] && P.pstride[k] > 0) return GBKB200_ERR_INVALID_ARG;
        ts[k]->pv = pvalues[k];
        if (ts[k]->n == 0) ts[k]->uids = nullptr;
    }
    P.model = model;
    P.lim_model = model ? (long long)nsets * P.Nz * P.Ny * P.Nx : 0;
    P.counters = bt->count ? bt->counters : nullptr;
    const long long set_stride = (long long)P.Wz * P.Py * P.hx;
    const long long lim_spec = (long long)P.Pz * P.Py * P.hx;
    const int tiles = (P.hx + BLT - 1) / BLT;
    if (bt->direct) {
        for (int s0 = 0; s0 < nsets; s0 += bt->chunk) {
            const int cn = std::min(bt->chunk, nsets - s0);
            P.set0 = s0;
            stage_mark(bt, 0, true);
            // variants 2 and 3: a block per (4 rows, chunk); otherwise a warp per item
            const bool tiles = bt->ka_variant >= 2;
            const int items = P.Wy * (bt->ka_variant == 1 ? (P.nch + 1) / 2 : P.nch);
            const int blocks = tiles ? (P.Wy + 3) / 4 * P.nch
                                     : (items + KA_THREADS / 32 - 1) / (KA_THREADS / 32);
            const size_t smem = tiles ? (size_t)P.Nz * 16 : 0;
            bt->ka<<<dim3(blocks, cn), KA_THREADS, smem, st>>>(P, bt->ctx->d_status);
            stage_mark(bt, 0, false);
            stage_mark(bt, 4, true);
            launch_kb(bt, P, cn, st);
            stage_mark(bt, 4, false);
        }
        stage_mark(bt, 5, true);
        if (nsets > 0) k6_sum<<<nsets, 256, 0, st>>>(P.partials, bt->nper, 0, chi2);
        stage_mark(bt, 5, false);
        GBK_CUDA_TRY(cudaGetLastError());
        return gbk_finish(bt->ctx);
    }
    for (int s0 = 0; s0 < nsets; s0 += bt->chunk) {
        const int cn = std::min(bt->chunk, nsets - s0);
        P.set0 = s0;
        stage_mark(bt, 0, true);
        k1_model_xfft<<<dim3(P.Wy, cn), 512, bt->smem1, st>>>(P, bt->ctx->d_status);
        stage_mark(bt, 0, false);
        stage_mark(bt, 1, true);
        // K2: y forward over (z < Wz, kx); columns stride hx, outer stride Py * hx
        k_lines<<<dim3(tiles * P.Wz, cn), 256, bt->smem_y, st>>>(
            P.work, set_stride, P.hx, (long long)P.Py * P.hx, P.hx, P.ay, 0, 0, nullptr, 0, 0,
            1.f, P.Wy, 0, P.Py, P.lim_work, lim_spec);
        stage_mark(bt, 1, false);
        stage_mark(bt, 2, true);
        // K3: z conv over (y < Py, kx); element stride Py * hx
        k_lines<<<dim3(tiles * P.Py, cn), 256, bt->smem_z, st>>>(
            P.work, set_stride, P.hx, P.hx, (long long)P.Py * P.hx, P.az, 0, 1, P.kspec, P.hx,
            (long long)P.Py * P.hx, P.scale, P.Wz, P.ez, P.Nz, P.lim_work, lim_spec);
        stage_mark(bt, 2, false);
        stage_mark(bt, 3, true);
        // K4: y inverse over (z < Nz, kx)
        k_lines<<<dim3(tiles * P.Nz, cn), 256, bt->smem_y, st>>>(
            P.work, set_stride, P.hx, (long long)P.Py * P.hx, P.hx, P.ay, 1, 0, nullptr, 0, 0,
            1.f, P.Py, P.ey, P.Ny, P.lim_work, lim_spec);
        stage_mark(bt, 3, false);
        stage_mark(bt, 4, true);
        k5_c2r_residual<<<dim3((P.Ny + P.rows_k5 - 1) / P.rows_k5, P.Nz, cn), 256, bt->smem5,
                          st>>>(P);
        stage_mark(bt, 4, false);
    }
    stage_mark(bt, 5, true);
    if (nsets > 0) k6_sum<<<nsets, 256, 0, st>>>(P.partials, bt->nper, 0, chi2);
    stage_mark(bt, 5, false);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(bt->ctx);
}

extern "C" int gbkb200_batch_window(const gbkb200_batch* bt, int offset[3], int size[3])
{
    if (!bt || !offset || !size) return GBKB200_ERR_INVALID_ARG;
    if (!bt->direct) return GBKB200_ERR_UNSUPPORTED;
    const BatchKernelArgs& P = bt->P;
    // the window starts t trimmed taps into the untrimmed one, whose first
    // voxel is the high-resolution grid's first voxel
    offset[0] = bt->trim[0]; offset[1] = bt->trim[1]; offset[2] = bt->trim[2];
    size[0] = P.Wx; size[1] = P.Wy; size[2] = P.Wz;
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_evaluate_cubes(gbkb200_batch* bt, int nsets, const float* cubes,
                                            float* chi2, float* model)
{
    if (!bt || nsets < 0 || nsets > bt->max_sets || !cubes || !chi2)
        return GBKB200_ERR_INVALID_ARG;
    if (!bt->direct) return GBKB200_ERR_UNSUPPORTED;
    BatchKernelArgs P = bt->P;
    cudaStream_t st = bt->ctx->stream;
    P.model = model;
    P.lim_model = model ? (long long)nsets * P.Nz * P.Ny * P.Nx : 0;
    P.counters = bt->count ? bt->counters : nullptr;
    const KcFn kc = kc_fn(P.Kz);
    for (int s0 = 0; s0 < nsets; s0 += bt->chunk) {
        const int cn = std::min(bt->chunk, nsets - s0);
        P.set0 = s0;
        stage_mark(bt, 0, true);
        kc<<<dim3((P.Wy * P.nch + KA_THREADS / 32 - 1) / (KA_THREADS / 32), cn), KA_THREADS, 0,
             st>>>(P, cubes);
        stage_mark(bt, 0, false);
        stage_mark(bt, 4, true);
        launch_kb(bt, P, cn, st);
        stage_mark(bt, 4, false);
    }
    stage_mark(bt, 5, true);
    if (nsets > 0) k6_sum<<<nsets, 256, 0, st>>>(P.partials, bt->nper, 0, chi2);
    stage_mark(bt, 5, false);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(bt->ctx);
}

// chi^2 of nsets sets to pinned host memory and the submission's event
static int submit_tail(gbkb200_batch* bt, int nsets, const float* chi2_dev, float* chi2_host)
{
    cudaStream_t st = bt->ctx->stream;
    if (nsets > 0 && chi2_host)
        GBK_CUDA_TRY(cudaMemcpyAsync(chi2_host, chi2_dev, (size_t)nsets * sizeof(float),
                                     cudaMemcpyDeviceToHost, st));
    // the kernels' status word, read by gbkb200_batch_take_status once done
    GBK_CUDA_TRY(cudaMemcpyAsync(bt->ctx->h_status, bt->ctx->d_status, sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
    if (!bt->done) GBK_CUDA_TRY(cudaEventCreateWithFlags(&bt->done, cudaEventDisableTiming));
    GBK_CUDA_TRY(cudaEventRecord(bt->done, st));
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_take_status(gbkb200_batch* bt)
{
    if (!bt) return GBKB200_ERR_INVALID_ARG;
    const int s = *bt->ctx->h_status;
    if (!s) return GBKB200_OK;
    // cleared for the next submission (enqueued after the completed one)
    *bt->ctx->h_status = 0;
    GBK_CUDA_TRY(cudaMemsetAsync(bt->ctx->d_status, 0, sizeof(int), bt->ctx->stream));
    if (s & GBK_STATUS_BAD_TRAIT) return GBKB200_ERR_BAD_TRAIT;
    if (s & GBK_STATUS_TIMEOUT) return GBKB200_ERR_TIMEOUT;
    return GBKB200_ERR_INVALID_ARG;
}

extern "C" int gbkb200_batch_submit(gbkb200_batch* bt, int nsets, const void* in_host,
                                    void* in_dev, size_t in_bytes, const float* vsys,
                                    const float* xpos, const float* ypos, const float* posa,
                                    const float* incl, const float* const pvalues[9],
                                    float* chi2_dev, float* chi2_host)
{
    if (!bt || (in_bytes > 0 && (!in_host || !in_dev))) return GBKB200_ERR_INVALID_ARG;
    if (in_bytes > 0)
        GBK_CUDA_TRY(cudaMemcpyAsync(in_dev, in_host, in_bytes, cudaMemcpyHostToDevice,
                                     bt->ctx->stream));
    int rc = gbkb200_batch_evaluate(bt, nsets, vsys, xpos, ypos, posa, incl, pvalues, chi2_dev,
                                    nullptr);
    if (rc) return rc;
    return submit_tail(bt, nsets, chi2_dev, chi2_host);
}

extern "C" int gbkb200_batch_submit_cubes(gbkb200_batch* bt, int nsets, const float* cubes,
                                          float* chi2_dev, float* chi2_host)
{
    int rc = gbkb200_batch_evaluate_cubes(bt, nsets, cubes, chi2_dev, nullptr);
    if (rc) return rc;
    return submit_tail(bt, nsets, chi2_dev, chi2_host);
}

extern "C" int gbkb200_batch_query(const gbkb200_batch* bt, int* done)
{
    if (!bt || !done) return GBKB200_ERR_INVALID_ARG;
    if (!bt->done) {
        *done = 1;
        return GBKB200_OK;
    }
    const cudaError_t e = cudaEventQuery(bt->done);
    if (e == cudaSuccess) {
        *done = 1;
        return GBKB200_OK;
    }
    if (e == cudaErrorNotReady) {
        (void)cudaGetLastError();
        *done = 0;
        return GBKB200_OK;
    }
    GBK_CUDA_TRY(e);
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_set_timing(gbkb200_batch* bt, int enable)
{
    if (!bt) return GBKB200_ERR_INVALID_ARG;
    if (enable < 0 || enable > 2) return GBKB200_ERR_INVALID_ARG;
    if (enable == 1 && !bt->counters) {
        if (cudaMalloc(&bt->counters, GBK_CTR_N * sizeof(unsigned long long)) != cudaSuccess)
            return GBKB200_ERR_OOM;
        GBK_CUDA_TRY(cudaMemset(bt->counters, 0, GBK_CTR_N * sizeof(unsigned long long)));
    }
    bt->timing = enable ? 1 : 0;
    bt->count = enable == 1 ? 1 : 0;
    bt->ev_used = 0;
    bt->ev_error = 0;
    return GBKB200_OK;
}

extern "C" int gbkb200_batch_timing(gbkb200_batch* bt, double ms[GBKB200_BATCH_STAGES],
                                    int launches[GBKB200_BATCH_STAGES])
{
    if (!bt || !ms || !launches) return GBKB200_ERR_INVALID_ARG;
    for (int s = 0; s < GBKB200_BATCH_STAGES; ++s) {
        ms[s] = 0.0;
        launches[s] = 0;
    }
    GBK_CUDA_TRY(cudaStreamSynchronize(bt->ctx->stream));
    const int failed = bt->ev_error;
    for (size_t i = 0; i < bt->ev_used && !failed; ++i) {
        float t = 0.f;
        GBK_CUDA_TRY(cudaEventElapsedTime(&t, bt->ev[2 * i], bt->ev[2 * i + 1]));
        ms[bt->ev_stage[i]] += t;
        launches[bt->ev_stage[i]] += 1;
    }
    bt->ev_used = 0;
    bt->ev_error = 0;
    return failed ? GBKB200_ERR_OOM : GBKB200_OK;
}

extern "C" int gbkb200_batch_counters(gbkb200_batch* bt, unsigned long long out[GBKB200_BATCH_COUNTERS])
{
    if (!bt || !out) return GBKB200_ERR_INVALID_ARG;
    static_assert(GBK_CTR_N == GBKB200_BATCH_COUNTERS, "counter slots");
    for (int i = 0; i < GBKB200_BATCH_COUNTERS; ++i) out[i] = 0;
    if (!bt->counters) return GBKB200_OK;
    GBK_CUDA_TRY(cudaStreamSynchronize(bt->ctx->stream));
    GBK_CUDA_TRY(cudaMemcpy(out, bt->counters, GBK_CTR_N * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost));
    GBK_CUDA_TRY(cudaMemset(bt->counters, 0, GBK_CTR_N * sizeof(unsigned long long)));
    return GBKB200_OK;
}
