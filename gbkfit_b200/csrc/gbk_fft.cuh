// Shared-memory mixed-radix Stockham FFT passes (device side), used by the
// drop-in FFT convolution (fft.cu) and the batched pipeline (batched.cu).
#pragma once

#include "gbk_common.cuh"

namespace gbk {

constexpr int FFT_MAX_PASSES = 24;
constexpr int FFT_MAX_PRIME = 61;
constexpr int FFT_THREADS = 256;

// Division by a run-time divisor as a multiply and a shift: for 0 <= x < 2^24
// and 1 <= d <= 2^16, x / d = (x * m) >> 40 with m = ceil(2^40 / d) (exact: with
// x = q d + r the product is q + r / d + x (m - 2^40 / d) / 2^40, and
// r / d + x / 2^40 < 1 because x d < 2^40).
__host__ __device__ inline unsigned long long fdiv_magic(int d)
{
    return ((1ull << 40) + (unsigned long long)d - 1) / (unsigned long long)d;
}
__device__ __forceinline__ int fdiv(int x, unsigned long long m)
{
    return (int)(((unsigned long long)(unsigned)x * m) >> 40);
}

struct AxisDev {
    int n;
    int nr;
    int r[FFT_MAX_PASSES];
    const float2* tw;   // tw[k] = exp(-2 pi i k / n), k in [0, n)
    // division multipliers (fdiv_magic): of n, and per pass of n / r[p] (the
    // butterflies of the pass) and of Ns (the product of the earlier radices)
    unsigned long long mn;
    unsigned long long mnb[FFT_MAX_PASSES];
    unsigned long long mns[FFT_MAX_PASSES];
};

// fills the division multipliers of an axis whose n, nr and r[] are set
inline void axis_fill_magics(AxisDev& a)
{
    a.mn = fdiv_magic(a.n);
    int ns = 1;
    for (int p = 0; p < a.nr; ++p) {
        a.mnb[p] = fdiv_magic(a.n / a.r[p]);
        a.mns[p] = fdiv_magic(ns);
        ns *= a.r[p];
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{ return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 mul_mi(float2 a, bool inv)
{ return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }

template<int R>
__device__ __forceinline__ void dft_small(float2* v, bool inv, const float2* tw, int n)
{
    if (R == 2) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        float2 s13 = cadd(v[1], v[3]), d13 = mul_mi(csub(v[1], v[3]), inv);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    } else if (R == 8) {
        float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<4>(e, inv, tw, n);
        dft_small<4>(o, inv, tw, n);
        const float h = 0.70710678118654752f;
        // o[m] *= W8^m
        float2 o1 = inv ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                        : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
        float2 o2 = mul_mi(o[2], inv);
        float2 o3 = inv ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                        : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
        v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
    } else if (R == 3) {
        const float c = -0.5f, s = 0.86602540378443865f;
        float2 a = v[0], b = v[1], d = v[2];
        float2 t = cadd(b, d);
        float2 m = make_float2(a.x + c * t.x, a.y + c * t.y);
        float2 q = csub(b, d);
        // forward: -i s q ; inverse: +i s q
        float2 iq = inv ? make_float2(-s * q.y, s * q.x) : make_float2(s * q.y, -s * q.x);
        v[0] = cadd(a, t);
        v[1] = cadd(m, iq);
        v[2] = csub(m, iq);
    } else {
        // generic odd R (5, 7): out[m] = sum_r v[r] W_R^(r m), W_R^q = tw[q n / R]
        float2 out[R];
        const int step = n / R;
#pragma unroll
        for (int m = 0; m < R; ++m) {
            float2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tw[((r * m) % R) * step];
                if (inv) w = conjf2(w);
                acc = cadd(acc, cmul(v[r], w));
            }
            out[m] = acc;
        }
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = out[m];
    }
}

// One Stockham pass of radix R over L lines held in shared memory; element
// (k, l) of the lines sits at k * sk + l * sl.
template<int R>
__device__ __forceinline__ void pass_r(const float2* src, float2* dst, int n, int Ns, int L, int sk,
                                       int sl, bool rows, const float2* tw, bool inv,
                                       unsigned long long m_nb, unsigned long long m_ns,
                                       unsigned long long m_L)
{
    const int nb = n / R;
    const int twstep = n / (Ns * R);
    const int total = nb * L;
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        int j, l;
        if (rows) { l = fdiv(u, m_nb); j = u - l * nb; }
        else { j = fdiv(u, m_L); l = u - j * L; }
        const int jq = fdiv(j, m_ns);          // j / Ns
        const int k = j - jq * Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int si = (j + r * nb) * sk + l * sl;
            float2 x = GBK_OK_IDX(si, n * L, 101) ? src[si] : make_float2(0.f, 0.f);
            if (r > 0 && k > 0) {
                const int ti = r * k * twstep;
                float2 w = GBK_OK_IDX(ti, n, 103) ? tw[ti] : make_float2(1.f, 0.f);
                if (inv) w = conjf2(w);
                x = cmul(x, w);
            }
            v[r] = x;
        }
        dft_small<R>(v, inv, tw, n);
        const int d0 = jq * Ns * R + k;
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const int di = (d0 + m * Ns) * sk + l * sl;
            if (GBK_OK_IDX(di, n * L, 102)) dst[di] = v[m];
        }
    }
}

// generic prime radix (11..61): inputs re-read from shared memory
static __device__ void pass_generic(const float2* src, float2* dst, int n, int R, int Ns, int L, int sk,
                             int sl, bool rows, const float2* tw, bool inv,
                             unsigned long long m_nb, unsigned long long m_ns,
                             unsigned long long m_L)
{
    const int nb = n / R;
    const int twstep = n / (Ns * R);
    const int step = n / R;
    const int total = nb * L * R;
    const unsigned long long m_R = fdiv_magic(R);
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        const int w = fdiv(u, m_R);
        const int m = u - w * R;
        int j, l;
        if (rows) { l = fdiv(w, m_nb); j = w - l * nb; }
        else { j = fdiv(w, m_L); l = w - j * L; }
        const int jq = fdiv(j, m_ns);          // j / Ns
        const int k = j - jq * Ns;
        float2 acc = make_float2(0.f, 0.f);
        for (int r = 0; r < R; ++r) {
            float2 x = src[(j + r * nb) * sk + l * sl];
            int e = (r * k * twstep + ((r * m) % R) * step) % n;
            float2 t = tw[e];
            if (inv) t = conjf2(t);
            acc = cadd(acc, cmul(x, t));
        }
        const int d0 = jq * Ns * R + k;
        dst[(d0 + m * Ns) * sk + l * sl] = acc;
    }
}

// All passes of one transform; returns the buffer holding the result.  The
// direction and the line layout are template parameters, so the
// butterflies' direction selects and the index mapping's branch fold away.
template<bool INV, bool ROWS>
static __device__ float2* fft_smem_t(float2* b0, float2* b1, const AxisDev& ax, int L, int sk,
                                     int sl, const float2* tw)
{
    constexpr bool inv = INV, rows = ROWS;
    float2* src = b0;
    float2* dst = b1;
    int Ns = 1;
    const unsigned long long m_L = rows ? 0ull : fdiv_magic(L);
    for (int p = 0; p < ax.nr; ++p) {
        const int R = ax.r[p];
        const unsigned long long mb = ax.mnb[p], ms = ax.mns[p];
        switch (R) {
        case 2: pass_r<2>(src, dst, ax.n, Ns, L, sk, sl, rows, tw, inv, mb, ms, m_L); break;
        case 3: pass_r<3>(src, dst, ax.n, Ns, L, sk, sl, rows, tw, inv, mb, ms, m_L); break;
        case 4: pass_r<4>(src, dst, ax.n, Ns, L, sk, sl, rows, tw, inv, mb, ms, m_L); break;
        case 5: pass_r<5>(src, dst, ax.n, Ns, L, sk, sl, rows, tw, inv, mb, ms, m_L); break;
        case 7: pass_r<7>(src, dst, ax.n, Ns, L, sk, sl, rows, tw, inv, mb, ms, m_L); break;
        case 8: pass_r<8>(src, dst, ax.n, Ns, L, sk, sl, rows, tw, inv, mb, ms, m_L); break;
        default: pass_generic(src, dst, ax.n, R, Ns, L, sk, sl, rows, tw, inv, mb, ms, m_L); break;
        }
        __syncthreads();
        float2* t = src;
        src = dst;
        dst = t;
        Ns *= R;
    }
    return src;
}

static __device__ __forceinline__ float2* fft_smem(float2* b0, float2* b1, const AxisDev& ax,
                                                   int L, int sk, int sl, bool rows,
                                                   const float2* tw, bool inv)
{
    if (rows)
        return inv ? fft_smem_t<true, true>(b0, b1, ax, L, sk, sl, tw)
                   : fft_smem_t<false, true>(b0, b1, ax, L, sk, sl, tw);
    return inv ? fft_smem_t<true, false>(b0, b1, ax, L, sk, sl, tw)
               : fft_smem_t<false, false>(b0, b1, ax, L, sk, sl, tw);
}

__device__ __forceinline__ void load_twiddles(float2* s_tw, const float2* g_tw, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_tw[i] = g_tw[i];
}

// Element-wise copy of count elements in rounds of U per thread: the U global
// loads of a round are issued before any of their results is used, so each
// thread keeps U loads in flight (load(e) reads element e, store(e, v) writes
// it; elements e >= count are neither read nor written).
template<int U, typename Load, typename Store>
__device__ __forceinline__ void staged_copy(int count, Load load, Store store)
{
    for (int e0 = threadIdx.x; e0 < count; e0 += U * (int)blockDim.x) {
        float2 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * (int)blockDim.x;
            v[u] = e < count ? load(e) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * (int)blockDim.x;
            if (e < count) store(e, v[u]);
        }
    }
}

}  // namespace gbk
