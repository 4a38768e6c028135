// Hand-written 3-D real FFT convolution for the GBKFIT data cube.
//
// Replaces the reference's FFTW3 (gbkfit_host/include/gbkfit/host/fft.hpp) and
// cuFFT (gbkfit_cuda/include/gbkfit/cuda/fft.hpp) plans: r2c of the padded
// model cube, complex multiply by the cached PSF x LSF spectrum scaled by 1/N
// (gbkfit_host/include/gbkfit/host/kernels.hpp:32-53), c2r back in place.
//
// Layout: real cube (nz, ny, nx) C-order, x fastest; spectrum (nz, ny, hx)
// with hx = nx/2 + 1, as FFTW/cuFFT lay out a 3-D r2c of (n0=nz, n1=ny, n2=nx).
//
// Kernels (all passes in shared memory, self-sorting mixed-radix Stockham with
// radices 8/4/2/3/5/7 and a generic odd-prime butterfly up to 61; twiddles
// are computed on the host in double precision):
//   x_r2c   rows of the real cube, as nx/2-point complex FFTs plus the
//           even/odd split (nx even) or full complex FFTs (nx odd);
//   lines   tiles of 16 adjacent columns along y or z, one 128-byte
//           coalesced row of the tile per element index;
//   conv_z  the z pass fused with the pointwise multiply and the inverse z
//           pass: a column is read once and written once;
//   x_c2r   the inverse of x_r2c.
#include "gbk_fft.cuh"

#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

namespace gbk {

// ---- x axis: rows of the real cube --------------------------------------------
// ax: the complex transform of length M = nx/2 (nx even) or nx (nx odd).
// post: exp(-2 pi i k / nx) for k in [0, nx/2].  Shared memory:
// 2 * L * M complex + M twiddles + (nx/2 + 1) post twiddles.
__global__ void __launch_bounds__(FFT_THREADS) x_r2c_kernel(const float* in, float2* out, int rows,
                                                            int nx, AxisDev ax, const float2* post)
{
    extern __shared__ float2 sm[];
    const int M = ax.n;
    const int hx = nx / 2 + 1;
    const int L = max(1, min(16, 8192 / M));
    float2* b0 = sm;
    float2* b1 = b0 + L * M;
    float2* s_tw = b1 + L * M;
    float2* s_post = s_tw + M;
    load_twiddles(s_tw, ax.tw, M);
    const bool even = (nx & 1) == 0;
    if (even) load_twiddles(s_post, post, hx);
    const long long row0 = (long long)blockIdx.x * L;
    staged_copy<8>(
        L * M,
        [&](int e) {
            const int l = fdiv(e, ax.mn), m = e - l * M;
            const long long row = row0 + l;
            float2 v = make_float2(0.f, 0.f);
            if (row < rows) {
                if (even) v = reinterpret_cast<const float2*>(in + row * nx)[m];
                else v = make_float2(in[row * nx + m], 0.f);
            }
            return v;
        },
        [&](int e, float2 v) { b0[e] = v; });
    __syncthreads();
    float2* z = fft_smem(b0, b1, ax, L, 1, M, true, s_tw, false);
    const unsigned long long mhx = fdiv_magic(hx);
    for (int e = threadIdx.x; e < L * hx; e += blockDim.x) {
        const int l = fdiv(e, mhx), k = e - l * hx;
        long long row = row0 + l;
        if (row >= rows) continue;
        float2 X;
        if (even) {
            // k in [0, M]: k mod M and (M - k) mod M without a division
            float2 zk = z[l * M + (k == M ? 0 : k)];
            float2 zc = conjf2(z[l * M + (k == 0 ? 0 : M - k)]);
            float2 ev = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
            float2 od = make_float2(0.5f * (zk.x - zc.x), 0.5f * (zk.y - zc.y));
            // X = E + W^k * (-i) * O
            float2 t = cmul(s_post[k], make_float2(od.y, -od.x));
            X = cadd(ev, t);
        } else {
            X = z[l * M + k];
        }
        out[row * hx + k] = X;
    }
}

// Inverse of x_r2c (unnormalised, like FFTW's c2r).
__global__ void __launch_bounds__(FFT_THREADS) x_c2r_kernel(const float2* in, float* out, int rows,
                                                            int nx, AxisDev ax, const float2* post)
{
    extern __shared__ float2 sm[];
    const int M = ax.n;
    const int hx = nx / 2 + 1;
    const int L = max(1, min(16, 8192 / M));
    float2* b0 = sm;
    float2* b1 = b0 + L * M;
    float2* s_tw = b1 + L * M;
    float2* s_post = s_tw + M;
    load_twiddles(s_tw, ax.tw, M);
    const bool even = (nx & 1) == 0;
    if (even) load_twiddles(s_post, post, hx);
    __syncthreads();
    const long long row0 = (long long)blockIdx.x * L;
    if (even) {
        // Z[k] = (X[k] + conj X[M-k]) + i W^-k (X[k] - conj X[M-k]): the two
        // halves are staged first (b0: X[k], b1: X[M-k]), then combined
        staged_copy<8>(
            L * M,
            [&](int e) {
                const int l = fdiv(e, ax.mn), k = e - l * M;
                const long long row = row0 + l;
                return row < rows ? in[row * hx + k] : make_float2(0.f, 0.f);
            },
            [&](int e, float2 v) { b0[e] = v; });
        staged_copy<8>(
            L * M,
            [&](int e) {
                const int l = fdiv(e, ax.mn), k = e - l * M;
                const long long row = row0 + l;
                return row < rows ? in[row * hx + M - k] : make_float2(0.f, 0.f);
            },
            [&](int e, float2 v) { b1[e] = v; });
        __syncthreads();
        for (int e = threadIdx.x; e < L * M; e += blockDim.x) {
            const int k = e - fdiv(e, ax.mn) * M;
            const float2 a = b0[e], b = conjf2(b1[e]);
            const float2 s = cadd(a, b), d = csub(a, b);
            const float2 w = conjf2(s_post[k]);
            const float2 t = cmul(w, d);
            b0[e] = make_float2(s.x - t.y, s.y + t.x);
        }
    } else {
        // full Hermitian extension
        staged_copy<8>(
            L * M,
            [&](int e) {
                const int l = fdiv(e, ax.mn), k = e - l * M;
                const long long row = row0 + l;
                if (row >= rows) return make_float2(0.f, 0.f);
                const float2* r = in + row * hx;
                return k < hx ? r[k] : conjf2(r[nx - k]);
            },
            [&](int e, float2 v) { b0[e] = v; });
    }
    __syncthreads();
    float2* z = fft_smem(b0, b1, ax, L, 1, M, true, s_tw, true);
    for (int e = threadIdx.x; e < L * M; e += blockDim.x) {
        const int l = fdiv(e, ax.mn), m = e - l * M;
        long long row = row0 + l;
        if (row >= rows) continue;
        float2 v = z[l * M + m];
        if (even) reinterpret_cast<float2*>(out + row * nx)[m] = v;
        else out[row * nx + m] = v.x;
    }
}

// ---- y / z axes: strided columns -------------------------------------------------
// Column (o, i) of the complex cube: element k at o * so + i + k * sk, for
// i in [0, inner).  A block holds LT adjacent columns (16, or 8 for long
// lines, whose 16-column blocks would leave two resident blocks per SM).
// mode 0: one transform (dir inv); mode 1: forward, multiply by spec (same
// layout) times scale, inverse.
template<int LT>
__global__ void __launch_bounds__(FFT_THREADS) lines_kernel(float2* data, int inner, long long so,
                                                            long long sk, AxisDev ax, int inv,
                                                            int mode, const float2* spec,
                                                            float scale)
{
    extern __shared__ float2 sm[];
    const int n = ax.n;
    float2* b0 = sm;
    float2* b1 = b0 + LT * n;
    float2* s_tw = b1 + LT * n;
    load_twiddles(s_tw, ax.tw, n);
    const int tiles = (inner + LT - 1) / LT;
    const int o = blockIdx.x / tiles;
    const int i0 = (blockIdx.x % tiles) * LT;
    const long long base = (long long)o * so + i0;
    staged_copy<8>(
        LT * n,
        [&](int e) {
            const int l = e % LT, k = e / LT;
            return (i0 + l < inner) ? data[base + l + k * sk] : make_float2(0.f, 0.f);
        },
        [&](int e, float2 v) { b0[e] = v; });
    __syncthreads();
    float2* res = fft_smem(b0, b1, ax, LT, LT, 1, false, s_tw, mode == 0 ? inv != 0 : false);
    if (mode == 1) {
        staged_copy<8>(
            LT * n,
            [&](int e) {
                const int l = e % LT, k = e / LT;
                return (i0 + l < inner) ? spec[base + l + k * sk] : make_float2(0.f, 0.f);
            },
            [&](int e, float2 b) {
                const int l = e % LT;
                if (i0 + l < inner) {
                    const float2 a = res[e];
                    res[e] = make_float2((a.x * b.x - a.y * b.y) * scale,
                                         (a.x * b.y + a.y * b.x) * scale);
                }
            });
        __syncthreads();
        float2* other = (res == b0) ? b1 : b0;
        res = fft_smem(res, other, ax, LT, LT, 1, false, s_tw, true);
    }
    for (int e = threadIdx.x; e < LT * n; e += blockDim.x) {
        int l = e % LT, k = e / LT;
        if (i0 + l < inner) data[base + l + k * sk] = res[k * LT + l];
    }
}

// pointwise (a * b) * scale over the spectrum (used when nz == 1)
__global__ void cmul_scale_kernel(float2* a, const float2* b, long long n, float scale)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float2 x = a[i], y = b[i];
        a[i] = make_float2((x.x * y.x - x.y * y.y) * scale, (x.x * y.y + x.y * y.x) * scale);
    }
}

// ---- host-side plans and caches -------------------------------------------------

struct Axis {
    AxisDev dev{};
    float2* tw = nullptr;
};

struct Plan {
    int nx = 0, ny = 0, nz = 0, hx = 0;
    Axis ax, ay, az;
    float2* post = nullptr;   // exp(-2 pi i k / nx), k in [0, nx/2]
};

using Size3 = std::array<int, 3>;

struct FftState {
    std::map<Size3, Plan> plans;
    std::map<std::pair<Size3, const void*>, float2*> spectra;   // cached data2 spectra
    std::map<Size3, float2*> work;                              // data1 spectra
};

static bool factorize(int n, int* r, int& nr)
{
    nr = 0;
    while (n % 8 == 0 && n > 8) { r[nr++] = 8; n /= 8; }
    while (n % 4 == 0) { r[nr++] = 4; n /= 4; }
    while (n % 2 == 0) { r[nr++] = 2; n /= 2; }
    for (int p = 3; p <= FFT_MAX_PRIME && n > 1; p += 2) {
        while (n % p == 0) {
            if (nr >= FFT_MAX_PASSES) return false;
            r[nr++] = p;
            n /= p;
        }
    }
    if (n == 8) r[nr++] = 8, n = 1;
    return n == 1;
}

static int make_axis(Axis& a, int n)
{
    a.dev.n = n;
    if (n < 1 || n > (1 << 16)) return GBKB200_ERR_UNSUPPORTED;   // fdiv_magic's range
    if (!factorize(n, a.dev.r, a.dev.nr)) return GBKB200_ERR_UNSUPPORTED;
    axis_fill_magics(a.dev);
    std::vector<float2> h(n);
    for (int k = 0; k < n; ++k) {
        double ang = -2.0 * M_PI * (double)k / (double)n;
        h[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    GBK_CUDA_TRY(cudaMalloc(&a.tw, n * sizeof(float2)));
    GBK_CUDA_TRY(cudaMemcpy(a.tw, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    a.dev.tw = a.tw;
    return GBKB200_OK;
}

static size_t lines_smem(int n, int lt) { return (size_t)(2 * lt * n + n) * sizeof(float2); }
// columns per lines_kernel block: 16 while a block needs at most 60 KB
static int lines_tile(int n) { return lines_smem(n, 16) <= 60 * 1024 ? 16 : 8; }
static size_t rows_smem(int M, int nx)
{
    int L = std::max(1, std::min(16, 8192 / M));
    return (size_t)(2 * L * M + M + nx / 2 + 1) * sizeof(float2);
}
static constexpr size_t SMEM_LIMIT = 227 * 1024;

static int get_plan(FftState* st, const Size3& s, Plan** out)
{
    auto it = st->plans.find(s);
    if (it != st->plans.end()) { *out = &it->second; return GBKB200_OK; }
    Plan p;
    p.nx = s[0]; p.ny = s[1]; p.nz = s[2]; p.hx = p.nx / 2 + 1;
    if (p.nx < 1 || p.ny < 1 || p.nz < 1) return GBKB200_ERR_INVALID_ARG;
    const int M = (p.nx % 2 == 0 && p.nx > 1) ? p.nx / 2 : p.nx;
    if (rows_smem(M, p.nx) > SMEM_LIMIT || lines_smem(p.ny, lines_tile(p.ny)) > SMEM_LIMIT ||
        lines_smem(p.nz, lines_tile(p.nz)) > SMEM_LIMIT)
        return GBKB200_ERR_UNSUPPORTED;
    int rc;
    if ((rc = make_axis(p.ax, M))) return rc;
    if ((rc = make_axis(p.ay, p.ny))) return rc;
    if ((rc = make_axis(p.az, p.nz))) return rc;
    std::vector<float2> post(p.hx);
    for (int k = 0; k < p.hx; ++k) {
        double ang = -2.0 * M_PI * (double)k / (double)p.nx;
        post[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    GBK_CUDA_TRY(cudaMalloc(&p.post, p.hx * sizeof(float2)));
    GBK_CUDA_TRY(cudaMemcpy(p.post, post.data(), p.hx * sizeof(float2), cudaMemcpyHostToDevice));
    auto res = st->plans.emplace(s, p);
    *out = &res.first->second;
    return GBKB200_OK;
}

static int set_smem(const void* fn, size_t bytes)
{
    return gbk_raise_smem_limit(fn, bytes);
}

// x-pass launch helpers
static int launch_r2c(const Plan& p, const float* in, float2* out, cudaStream_t st)
{
    if ((reinterpret_cast<uintptr_t>(in) & 7) || (reinterpret_cast<uintptr_t>(out) & 7))
        return GBKB200_ERR_INVALID_ARG;   // rows are read as float2 pairs
    const int rows = p.ny * p.nz;
    const int M = p.ax.dev.n;
    const int L = std::max(1, std::min(16, 8192 / M));
    size_t smem = rows_smem(M, p.nx);
    int rc = set_smem((const void*)x_r2c_kernel, smem);
    if (rc) return rc;
    x_r2c_kernel<<<(rows + L - 1) / L, FFT_THREADS, smem, st>>>(in, out, rows, p.nx, p.ax.dev, p.post);
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}

static int launch_c2r(const Plan& p, const float2* in, float* out, cudaStream_t st)
{
    if ((reinterpret_cast<uintptr_t>(in) & 7) || (reinterpret_cast<uintptr_t>(out) & 7))
        return GBKB200_ERR_INVALID_ARG;
    const int rows = p.ny * p.nz;
    const int M = p.ax.dev.n;
    const int L = std::max(1, std::min(16, 8192 / M));
    size_t smem = rows_smem(M, p.nx);
    int rc = set_smem((const void*)x_c2r_kernel, smem);
    if (rc) return rc;
    x_c2r_kernel<<<(rows + L - 1) / L, FFT_THREADS, smem, st>>>(in, out, rows, p.nx, p.ax.dev, p.post);
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}

// y or z pass over the complex cube (mode 0: single transform; mode 1: conv)
static int launch_lines(const Plan& p, float2* data, int axis, int inv, int mode,
                        const float2* spec, float scale, cudaStream_t st)
{
    const Axis& a = axis == 1 ? p.ay : p.az;
    if (a.dev.n == 1 && mode == 0) return GBKB200_OK;
    const int lt = lines_tile(a.dev.n);
    const int tiles = (p.hx + lt - 1) / lt;
    long long so, sk;
    int outer;
    if (axis == 1) { outer = p.nz; so = (long long)p.ny * p.hx; sk = p.hx; }
    else { outer = p.ny; so = p.hx; sk = (long long)p.ny * p.hx; }
    size_t smem = lines_smem(a.dev.n, lt);
    auto kern = lt == 16 ? lines_kernel<16> : lines_kernel<8>;
    int rc = set_smem((const void*)kern, smem);
    if (rc) return rc;
    kern<<<outer * tiles, FFT_THREADS, smem, st>>>(data, p.hx, so, sk, a.dev, inv, mode, spec,
                                                   scale);
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}

// x and y passes of the forward transform (the z pass is fused with the
// spectrum multiply in convolve_tail)
static int forward_xy(const Plan& p, const float* r, float2* c, cudaStream_t st)
{
    int rc;
    if ((rc = launch_r2c(p, r, c, st))) return rc;
    return launch_lines(p, c, 1, 0, 0, nullptr, 1.f, st);
}

static int forward(const Plan& p, const float* r, float2* c, cudaStream_t st)
{
    int rc;
    if ((rc = forward_xy(p, r, c, st))) return rc;
    return launch_lines(p, c, 2, 0, 0, nullptr, 1.f, st);
}

// c holds the x/y-transformed cube: forward z, multiply by spec * scale,
// inverse z (one fused pass), then inverse y and c2r into r
static int convolve_tail(const Plan& p, float2* c, const float2* spec, float* r, cudaStream_t st)
{
    int rc;
    // fft.hpp:185-197: nfactor = T{1} / (n0 * n1 * n2) in T
    const float scale = 1.0f / (float)(p.nx * p.ny * p.nz);
    if (p.nz > 1) {
        if ((rc = launch_lines(p, c, 2, 0, 1, spec, scale, st))) return rc;
    } else {
        long long n = (long long)p.nz * p.ny * p.hx;
        cmul_scale_kernel<<<(int)std::min<long long>((n + 255) / 256, 148 * 32), 256, 0, st>>>(
            c, spec, n, scale);
        GBK_CUDA_TRY(cudaGetLastError());
    }
    if ((rc = launch_lines(p, c, 1, 1, 0, nullptr, 1.f, st))) return rc;
    return launch_c2r(p, c, r, st);
}

static FftState* state(gbkb200_ctx* ctx)
{
    if (!ctx->fft_state) ctx->fft_state = new FftState();
    return static_cast<FftState*>(ctx->fft_state);
}

static int get_size(const int size[3], Size3& s)
{
    if (!size) return GBKB200_ERR_INVALID_ARG;
    s = {size[0], size[1], size[2]};
    if (s[0] < 1 || s[1] < 1 || s[2] < 1) return GBKB200_ERR_INVALID_ARG;
    return GBKB200_OK;
}

}  // namespace gbk

using namespace gbk;

int gbk_fft_state_destroy(gbkb200_ctx* ctx)
{
    if (!ctx || !ctx->fft_state) return GBKB200_OK;
    FftState* st = static_cast<FftState*>(ctx->fft_state);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : st->spectra) cudaFree(kv.second);
    for (auto& kv : st->work) cudaFree(kv.second);
    for (auto& kv : st->plans) {
        cudaFree(kv.second.ax.tw);
        cudaFree(kv.second.ay.tw);
        cudaFree(kv.second.az.tw);
        cudaFree(kv.second.post);
    }
    delete st;
    ctx->fft_state = nullptr;
    return GBKB200_OK;
}

extern "C" int gbkb200_fft_clear_cache(gbkb200_ctx* ctx)
{
    if (!ctx) return GBKB200_ERR_INVALID_ARG;
    return gbk_fft_state_destroy(ctx);
}

extern "C" int gbkb200_fft_r2c_f32(gbkb200_ctx* ctx, const int size[3], const float* data_r,
                                   void* data_c)
{
    Size3 s;
    int rc;
    if (!ctx || !data_r || !data_c) return GBKB200_ERR_INVALID_ARG;
    if ((rc = get_size(size, s))) return rc;
    Plan* p;
    if ((rc = get_plan(state(ctx), s, &p))) return rc;
    if ((rc = forward(*p, data_r, static_cast<float2*>(data_c), ctx->stream))) return rc;
    return gbk_finish(ctx);
}

extern "C" int gbkb200_fft_c2r_f32(gbkb200_ctx* ctx, const int size[3], const void* data_c,
                                   float* data_r)
{
    Size3 s;
    int rc;
    if (!ctx || !data_r || !data_c) return GBKB200_ERR_INVALID_ARG;
    if ((rc = get_size(size, s))) return rc;
    FftState* st = state(ctx);
    Plan* p;
    if ((rc = get_plan(st, s, &p))) return rc;
    // work on a copy so that data_c is preserved
    float2*& w = st->work[s];
    size_t bytes = (size_t)p->nz * p->ny * p->hx * sizeof(float2);
    if (!w) GBK_CUDA_TRY(cudaMalloc(&w, bytes));
    GBK_CUDA_TRY(cudaMemcpyAsync(w, data_c, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    if ((rc = launch_lines(*p, w, 2, 1, 0, nullptr, 1.f, ctx->stream))) return rc;
    if ((rc = launch_lines(*p, w, 1, 1, 0, nullptr, 1.f, ctx->stream))) return rc;
    if ((rc = launch_c2r(*p, w, data_r, ctx->stream))) return rc;
    return gbk_finish(ctx);
}

extern "C" int gbkb200_fft_convolve_f32(gbkb200_ctx* ctx, const int size[3], float* data1_r,
                                        void* data1_c, const void* data2_c)
{
    Size3 s;
    int rc;
    if (!ctx || !data1_r || !data1_c || !data2_c) return GBKB200_ERR_INVALID_ARG;
    if ((rc = get_size(size, s))) return rc;
    Plan* p;
    if ((rc = get_plan(state(ctx), s, &p))) return rc;
    // data1_c is work space: the reference multiplies in place and runs
    // FFTW's multi-dimensional c2r on it, which destroys it (fft.hpp:199-207)
    float2* c = static_cast<float2*>(data1_c);
    if ((rc = forward_xy(*p, data1_r, c, ctx->stream))) return rc;
    if ((rc = convolve_tail(*p, c, static_cast<const float2*>(data2_c), data1_r, ctx->stream)))
        return rc;
    return gbk_finish(ctx);
}

extern "C" int gbkb200_fft_convolve_cached_f32(gbkb200_ctx* ctx, const int size[3],
                                               float* data1_r, const float* data2_r)
{
    Size3 s;
    int rc;
    if (!ctx || !data1_r || !data2_r) return GBKB200_ERR_INVALID_ARG;
    if ((rc = get_size(size, s))) return rc;
    FftState* st = state(ctx);
    Plan* p;
    if ((rc = get_plan(st, s, &p))) return rc;
    size_t bytes = (size_t)p->nz * p->ny * p->hx * sizeof(float2);
    auto key = std::make_pair(s, (const void*)data2_r);
    auto it = st->spectra.find(key);
    float2* spec;
    if (it == st->spectra.end()) {
        if (cudaMalloc(&spec, bytes) != cudaSuccess) return GBKB200_ERR_OOM;
        st->spectra[key] = spec;
        if ((rc = forward(*p, data2_r, spec, ctx->stream))) return rc;
    } else {
        spec = it->second;
    }
    float2*& w = st->work[s];
    if (!w && cudaMalloc(&w, bytes) != cudaSuccess) return GBKB200_ERR_OOM;
    if ((rc = forward_xy(*p, data1_r, w, ctx->stream))) return rc;
    if ((rc = convolve_tail(*p, w, spec, data1_r, ctx->stream))) return rc;
    return gbk_finish(ctx);
}
