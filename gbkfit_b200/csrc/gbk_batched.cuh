// Batched evaluator: kernel arguments and the direct-convolution kernels
// (templates on the LSF and PSF FIR lengths, instantiated in their own
// translation units so that they compile in parallel).
#pragma once

#include "gbk_disk.cuh"
#include "gbk_fft.cuh"

#include <climits>

namespace gbk {

struct BatchKernelArgs {
    int Nx, Ny, Nz, Wx, Wy, Wz, Px, Py, Pz, hx, ex, ey, ez;
    int rows_k1;     // z rows per shared-memory group in K1
    int rows_k5;     // y rows per block in K5
    DiskArgs disk;   // per-set pointers are offset from set 0 by the strides
    int vstride[5];  // vsys, xpos, ypos, posa, incl values per set
    int pstride[9];  // trait parameter values per set, per kind
    AxisDev ax, ay, az;
    const float2* post;   // exp(-2 pi i k / Px), k in [0, Px/2]
    const float2* kspec;  // PSF x LSF spectrum (Pz, Py, hx)
    float scale;          // 1 / (Px Py Pz)
    const float *obs, *err, *msk;
    const float* iw;      // direct mode: mask * weight / error per voxel
    float weight;
    float2* work;         // (chunk, Wz, Py, hx)
    float* model;         // optional (nsets, Nz, Ny, Nx)
    double* partials;     // (nsets, Nz, ceil(Ny / rows_k5))
    int set0;
    // element counts of the buffers (bounds of the checked build)
    long long lim_work, lim_model, lim_part, lim_obs, lim_smem1, lim_smem5;
    // direct (separable) convolution
    int Kx, Ky, Kz;       // PSF (x, y) and LSF box sizes
    int K;                // FIR length of the PSF kernel (odd, >= Kx, Ky; zero-padded taps)
    int pitch;            // row pitch of the LSF-convolved planes in HBM (floats, % 4 == 0)
    int tpitch;           // row pitch of the model kernel's shared tile (odd: no bank conflicts)
    int tile_floats;      // Nz * tpitch rounded up to 4
    int sp;               // row pitch of the PSF kernel's shared rows (floats, % 32 == 4)
    int band, nbands;     // output rows per PSF block, bands per plane
    const float* vr;      // (K): PSF x factor, reversed
    const float* ur;      // (K): PSF y factor, reversed
    const float* lsfr;    // (Kz): LSF reversed
    float* mplanes;       // (chunk, Nz, Wy, pitch): only the xr segments are written
    int* xr;              // (chunk, Nz, Wy): nonzero x range of each plane row, or -1
    const double* sat;    // (Nz, Ny + 1, Nx + 1): summed-area table of the zero-model r^2
};

// set b's per-set inputs: pointers offset from set 0 by the strides
__device__ __forceinline__ DiskArgs set_disk(const BatchKernelArgs& P, int b)
{
    DiskArgs a = P.disk;
    if (a.vsys) a.vsys += (long long)b * P.vstride[0];
    a.xpos += (long long)b * P.vstride[1];
    a.ypos += (long long)b * P.vstride[2];
    a.posa += (long long)b * P.vstride[3];
    a.incl += (long long)b * P.vstride[4];
    TraitSet* ts[9] = {&a.rpt, &a.rht, &a.vpt, &a.vht, &a.dpt, &a.dht, &a.zpt, &a.spt, &a.wpt};
#pragma unroll
    for (int k = 0; k < 9; ++k)
        if (ts[k]->pv) ts[k]->pv += (long long)b * P.pstride[k];
    return a;
}

// ---- direct convolution: LSF FIR per column, separable PSF FIR per plane ----
//
// Crop output (zo, yo, xo) of the reference's FFT convolution equals
//   sum_t sum_sy sum_sx  lsf[Kz-1-t] psf[Ky-1-sy][Kx-1-sx] model(zo+t, yo+sy, xo+sx)
// in window coordinates (the padded grid's first W indices): the kernel is
// PSF(x, y) x LSF(z), and PSF = u(y) v(x) (rank 1: a circular Gaussian's
// 8-sigma truncation corners are ~1e-14 of the peak).
//
// Sparsity: a line is exactly zero outside its +-5 sigma channel window and
// off the disk, so each LSF-convolved plane is nonzero only in a band of
// rows and columns.  The model kernel records each plane row's nonzero x
// range; the PSF kernel convolves only the bounding box of its plane (sums
// of exact zeros are exact zeros, so results do not change) and takes the
// residual outside the box, where the model is exactly 0, from a summed-area
// table of ((0 - data) / error * mask * weight)^2 built once per data cube.

// KA: one block per (set, window row y): the row's spaxel lines, each spectral
// column convolved with the LSF (a warp per spaxel, KZ taps unrolled with the
// coefficients in registers), then per output plane the nonzero x segment of
// the row (aligned to 4) and its range.
constexpr int KA_THREADS = 256;

template<int KZ>
__global__ void __launch_bounds__(KA_THREADS, 3) ka_lines_lsf(BatchKernelArgs P, int* status)
{
    extern __shared__ float4 sm4[];
    const int tp = P.tpitch, lb = P.Wz + 2 * (KZ - 1);
    float* tile = reinterpret_cast<float*>(sm4);          // (Nz, tp)
    float* lbuf = tile + P.tile_floats;                    // (nwarps, lb)
    float* s_v = lbuf + (KA_THREADS / 32) * lb;
    float* s_amp = s_v + P.Wx;
    float* s_i2 = s_amp + P.Wx;
    float* s_orv = s_i2 + P.Wx;
    int* s_lo = reinterpret_cast<int*>(s_orv + P.Wx);
    int* s_hi = s_lo + P.Wx;
    int* s_xmin = s_hi + P.Wx;                             // (Nz)
    int* s_xmax = s_xmin + P.Nz;
    const int y = blockIdx.x, c = blockIdx.y, b = P.set0 + c;
    const DiskArgs a = set_disk(P, b);
    int bad = 0;
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
    float4* t4 = reinterpret_cast<float4*>(tile);
    for (int i = threadIdx.x; i < P.tile_floats / 4; i += blockDim.x)
        t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = threadIdx.x; i < P.Nz; i += blockDim.x) {
        s_xmin[i] = INT_MAX;
        s_xmax[i] = -1;
    }
    float lz[KZ];
#pragma unroll
    for (int t = 0; t < KZ; ++t) lz[t] = P.lsfr[t];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    // L[j], j = z - lo + KZ - 1: the line with KZ - 1 zeros on both sides
    float* L = lbuf + warp * lb;
    for (int x = warp; x < P.Wx; x += nwarps) {
        const int lo = s_lo[x], hi = s_hi[x];
        if (lo > hi) continue;
        const float v = s_v[x], amp = s_amp[x], i2 = s_i2[x], orv = s_orv[x];
        const int n = hi - lo + 1;
        for (int j = lane; j < KZ - 1; j += 32) {
            L[j] = 0.f;
            L[n + KZ - 1 + j] = 0.f;
        }
        // gmodels.hpp:109-115: the line, channel by channel (window coordinates)
        for (int z = lo + lane; z <= hi; z += 32) {
            float zv = a.spec_zero + z * a.spec_step;
            float d = zv - v;
            L[z - lo + KZ - 1] = orv * (amp * expf(-d * d / i2));
        }
        __syncwarp();
        const int zo0 = max(0, lo - KZ + 1), zo1 = min(P.Nz - 1, hi);
        for (int zo = zo0 + lane; zo <= zo1; zo += 32) {
            const float* l = L + (zo - lo + KZ - 1);
            float acc = 0.f;
#pragma unroll
            for (int t = 0; t < KZ; ++t) acc += lz[t] * l[t];
            tile[zo * tp + x] = acc;
            atomicMin(&s_xmin[zo], x);
            atomicMax(&s_xmax[zo], x);
        }
        __syncwarp();
    }
    __syncthreads();
    // per output plane: the row's nonzero x range and its 4-aligned segment
    for (int zo = warp; zo < P.Nz; zo += nwarps) {
        const int xmin = s_xmin[zo], xmax = s_xmax[zo];
        const long long row = ((long long)c * P.Nz + zo) * P.Wy + y;
        if (xmax < 0) {
            if (lane == 0) P.xr[row] = -1;
            continue;
        }
        if (lane == 0) P.xr[row] = xmin | (xmax << 16);
        float* dst = P.mplanes + row * P.pitch;
        const float* srow = tile + zo * tp;
        for (int x = (xmin & ~3) + lane; x <= (xmax | 3); x += 32) dst[x] = srow[x];
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// sum of the summed-area table over rows [y0, y1) and columns [x0, x1)
__device__ __forceinline__ double sat_box(const double* T, int ld, int y0, int y1, int x0, int x1)
{
    return T[(long long)y1 * ld + x1] - T[(long long)y0 * ld + x1] - T[(long long)y1 * ld + x0] +
           T[(long long)y0 * ld + x0];
}

// KB: one block per (set, output plane zo, band of output rows): the bounding
// box of the band's nonzero input rows is loaded (cp.async) and convolved in
// x in place (a warp per 1, 2 or 4 rows, 8 outputs per lane and window), then
// in y in place (8 x 4 outputs per item, ascending rounds of whole row groups:
// an output row only overwrites an input row that no later output reads),
// then the crop, residual (objective.hpp:7-31) and r^2 stream over the box
// from shared memory against the data; the zero-model residual outside the
// box comes from the summed-area table.
constexpr int KB_THREADS = 256;
constexpr int KB_IT = 2;        // y items per thread and round

template<int K>
__global__ void __launch_bounds__(KB_THREADS, 2) kb_psf_residual(BatchKernelArgs P)
{
    constexpr int NW = (K + 7 + 3) / 4;     // float4 slots of one 8-output x window
    extern __shared__ float4 sm4[];
    float* S = reinterpret_cast<float*>(sm4);                   // (band + K - 1, sp)
    __shared__ float warp_part[KB_THREADS / 32];
    const int zo = blockIdx.x / P.nbands, band = blockIdx.x % P.nbands;
    const int c = blockIdx.y, b = P.set0 + c;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ob0 = band * P.band, ob1 = min(P.Ny, ob0 + P.band);  // output rows [ob0, ob1)
    const int in1 = min(P.Wy, ob1 + K - 1);                        // input rows [ob0, in1)
    const long long prow = ((long long)c * P.Nz + zo) * P.Wy;
    const int* xr = P.xr + prow;
    const int ld = P.Nx + 1;
    const double* T = P.sat + (long long)zo * (P.Ny + 1) * ld;
    // bounding box of the nonzero input rows (every warp, no barrier)
    int y0 = INT_MAX, y1 = -1, x0 = INT_MAX, x1 = -1;
    for (int y = ob0 + lane; y < in1; y += 32) {
        const int v = xr[y];
        if (v >= 0) {
            y0 = min(y0, y);
            y1 = max(y1, y);
            x0 = min(x0, v & 0xffff);
            x1 = max(x1, v >> 16);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, o));
        x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, o));
    }
    const long long plane = (long long)P.Ny * P.Nx;
    float* model = P.model ? P.model + ((long long)b * P.Nz + zo) * plane : nullptr;
    const long long part = ((long long)b * P.Nz + zo) * P.nbands + band;
    if (y1 < 0) {   // nothing reaches this band: the model is 0 on it
        if (model)
            for (long long i = (long long)ob0 * P.Nx + threadIdx.x; i < (long long)ob1 * P.Nx;
                 i += blockDim.x)
                model[i] = 0.f;
        if (threadIdx.x == 0) P.partials[part] = sat_box(T, ld, ob0, ob1, 0, P.Nx);
        return;
    }
    // output box: x in 8-column strips [g_lo, g_hi], y rows [yo_lo, yo_hi]
    const int g_lo = max(0, x0 - K + 1) >> 3, g_hi = min(P.Nx - 1, x1) >> 3;
    const int ns8 = g_hi - g_lo + 1;
    const int yo_lo = max(ob0, y0 - K + 1), yo_hi = min(ob1 - 1, y1);
    // load rows [y0, y1], float4 slots [2 g_lo, 2 g_hi + NW): the row's
    // segment from HBM, zeros elsewhere
    {
        const int nsl = 2 * (ns8 - 1) + NW, sl0 = 2 * g_lo;
        const int nrows = y1 - y0 + 1;
        const float4* src = reinterpret_cast<const float4*>(P.mplanes + prow * P.pitch);
        for (int i = threadIdx.x; i < nrows * nsl; i += blockDim.x) {
            const int y = y0 + i / nsl, sl = sl0 + i % nsl;
            const int v = xr[y];
            float4* d = reinterpret_cast<float4*>(S + (long long)(y - ob0) * P.sp) + sl;
            if (v >= 0 && sl >= (v & 0xffff) >> 2 && sl <= (v >> 16) >> 2)
                cp_async16(d, src + (long long)y * (P.pitch / 4) + sl);
            else
                *d = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        cp_async_wait_all();
    }
    __syncthreads();
    // x FIR in place: S[y][xo] = sum_s vr[s] S[y][xo + s] over the strips; a
    // warp owns rw whole rows (lane = strip * rw + row), loads before __syncwarp
    {
        float vr[K];
#pragma unroll
        for (int s = 0; s < K; ++s) vr[s] = P.vr[s];
        const int rw = ns8 <= 8 ? 4 : (ns8 <= 16 ? 2 : 1);
        const int spw = 32 / rw;                    // strips per warp pass
        const int r = lane % rw, sidx = lane / rw;
        for (int ry = y0 + warp * rw; ry <= y1; ry += (KB_THREADS / 32) * rw) {
            const int y = ry + r;
            float4* row = reinterpret_cast<float4*>(S + (long long)(y - ob0) * P.sp);
            for (int gs = g_lo; gs <= g_hi; gs += spw) {
                const int g = gs + sidx;
                const bool act = g <= g_hi && y <= y1;
                float w[4 * NW];
                if (act) {
#pragma unroll
                    for (int m = 0; m < NW; ++m) {
                        const float4 f = row[2 * g + m];
                        w[4 * m] = f.x; w[4 * m + 1] = f.y; w[4 * m + 2] = f.z; w[4 * m + 3] = f.w;
                    }
                }
                __syncwarp();
                if (act) {
                    float o[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        float acc = 0.f;
#pragma unroll
                        for (int s = 0; s < K; ++s) acc += vr[s] * w[q + s];
                        o[q] = acc;
                    }
                    row[2 * g] = make_float4(o[0], o[1], o[2], o[3]);
                    row[2 * g + 1] = make_float4(o[4], o[5], o[6], o[7]);
                }
                __syncwarp();
            }
        }
    }
    __syncthreads();
    // y FIR in place: model(yo, xo) = sum_t ur[t] S[yo + t][xo] (rows outside
    // [y0, y1] are zero), written to S row yo; items of 8 rows x 4 columns in
    // ascending rounds of whole 8-row groups
    const int ngy = (yo_hi - yo_lo + 8) / 8, s4_lo = 2 * g_lo, ns4 = 2 * ns8;
    {
        float ur[K];
#pragma unroll
        for (int t = 0; t < K; ++t) ur[t] = P.ur[t];
        const int gpr = max(1, KB_THREADS * KB_IT / ns4);   // row groups per round
        for (int gr0 = 0; gr0 < ngy; gr0 += gpr) {
            const int nitems = min(gpr, ngy - gr0) * ns4;
            float acc[KB_IT][8][4];
#pragma unroll
            for (int it = 0; it < KB_IT; ++it) {
                const int item = threadIdx.x + it * KB_THREADS;
#pragma unroll
                for (int q = 0; q < 8; ++q)
#pragma unroll
                    for (int k = 0; k < 4; ++k) acc[it][q][k] = 0.f;
                if (item < nitems) {
                    const int yb = yo_lo + 8 * (gr0 + item / ns4), s4 = s4_lo + item % ns4;
#pragma unroll
                    for (int m = 0; m < K + 7; ++m) {
                        const int y = yb + m;
                        const float4 p = (y >= y0 && y <= y1)
                            ? reinterpret_cast<const float4*>(S + (long long)(y - ob0) * P.sp)[s4]
                            : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int t = m - q;
                            if (t >= 0 && t < K) {
                                acc[it][q][0] += ur[t] * p.x;
                                acc[it][q][1] += ur[t] * p.y;
                                acc[it][q][2] += ur[t] * p.z;
                                acc[it][q][3] += ur[t] * p.w;
                            }
                        }
                    }
                }
            }
            __syncthreads();
#pragma unroll
            for (int it = 0; it < KB_IT; ++it) {
                const int item = threadIdx.x + it * KB_THREADS;
                if (item < nitems) {
                    const int yb = yo_lo + 8 * (gr0 + item / ns4), s4 = s4_lo + item % ns4;
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        if (yb + q < ob1)
                            reinterpret_cast<float4*>(S + (long long)(yb + q - ob0) * P.sp)[s4] =
                                make_float4(acc[it][q][0], acc[it][q][1], acc[it][q][2],
                                            acc[it][q][3]);
                }
            }
            __syncthreads();
        }
    }
    // crop + residual over the box: rows [yo_lo, yb_end), columns [xb0, xb_end)
    const int yb_end = min(ob1, yo_lo + 8 * ngy), xb0 = 8 * g_lo, xb_end = min(P.Nx, 8 * g_hi + 8);
    float sum = 0.f;
    const long long pbase = (long long)zo * plane;
    if ((P.Nx & 3) == 0) {
        const int nv = (xb_end - xb0) >> 2;        // xb0 and xb_end are multiples of 4
        const int n = (yb_end - yo_lo) * nv;
#pragma unroll 4
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int yo = yo_lo + i / nv, xo = xb0 + 4 * (i % nv);
            const float4 m = *reinterpret_cast<const float4*>(S + (long long)(yo - ob0) * P.sp + xo);
            const long long vi = pbase + (long long)yo * P.Nx + xo;
            const float4 o = *reinterpret_cast<const float4*>(P.obs + vi);
            const float4 w = *reinterpret_cast<const float4*>(P.iw + vi);
            const float r0 = (m.x - o.x) * w.x, r1 = (m.y - o.y) * w.y;
            const float r2 = (m.z - o.z) * w.z, r3 = (m.w - o.w) * w.w;
            sum += r0 * r0 + r1 * r1 + r2 * r2 + r3 * r3;
            if (model) *reinterpret_cast<float4*>(model + (long long)yo * P.Nx + xo) = m;
        }
    } else {
        const int nw = xb_end - xb0, n = (yb_end - yo_lo) * nw;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int yo = yo_lo + i / nw, xo = xb0 + i % nw;
            const float m = S[(long long)(yo - ob0) * P.sp + xo];
            const long long vi = pbase + (long long)yo * P.Nx + xo;
            const float r0 = (m - P.obs[vi]) * P.iw[vi];
            sum += r0 * r0;
            if (model) model[(long long)yo * P.Nx + xo] = m;
        }
    }
    if (model) {
        const int bw = P.Nx;
        for (long long i = (long long)ob0 * bw + threadIdx.x; i < (long long)ob1 * bw;
             i += blockDim.x) {
            const int yo = (int)(i / bw), xo = (int)(i % bw);
            if (yo < yo_lo || yo >= yb_end || xo < xb0 || xo >= xb_end) model[i] = 0.f;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) warp_part[warp] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < KB_THREADS / 32; ++w) s += warp_part[w];
        const double outside = sat_box(T, ld, ob0, ob1, 0, P.Nx) -
                               sat_box(T, ld, yo_lo, yb_end, xb0, xb_end);
        P.partials[part] = (double)s + outside;
    }
}

typedef void (*KaFn)(BatchKernelArgs, int*);
typedef void (*KbFn)(BatchKernelArgs);
constexpr int KA_KMAX = 33;                 // longest LSF of the direct path
constexpr int KB_KMIN = 5, KB_KMAX = 33;    // PSF FIR lengths (odd)
// fill t[Kz / 2] (model kernel) and t[(K - KB_KMIN) / 2] (PSF kernel)
void ka_register_short(KaFn* t);
void ka_register_long(KaFn* t);
void kb_register(KbFn* t);

}  // namespace gbk
