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
    int pitch;            // row pitch of the LSF-convolved planes in HBM (floats, % 32 == 0)
    int cap;              // shared-memory floats of a PSF block (rows of one pass)
    int band, nbands;     // output rows per PSF block, bands per plane
    int xr_slot;          // persistent PSF kernel: ints per range-entry buffer (% 4 == 0)
    int kb_cn;            // persistent PSF kernel: sets of the launch
    int* kb_work;         // persistent PSF kernel: item counter (zeroed before each launch)
    // FIR coefficients in the parameter block (constant bank, uniform loads)
    float vr[33];         // (K): PSF x factor, reversed, zero-padded
    float ur[33];         // (K): PSF y factor, reversed, zero-padded
    float lsfr[33];       // (Kz): LSF reversed
    float2 ur2[33];       // (K): ur duplicated into packed pairs (FFMA2 operands)
    float* mplanes;       // (chunk, Nz, Wy, pitch): written where xr is not empty
    int nch;              // 32-column chunks per window row, ceil(Wx / 32)
    int nwfast;           // the disk's traits are exactly rpt/vpt/dpt uid 101 (smdisk_spaxel_nw)
    int* xrt;             // (chunk, Nz, Wy, nch): the nonzero columns of each plane row
                          // chunk as a 32-bit mask (bit j: column 32 chunk + j; 0: the
                          // chunk is zero).  Every column of a 4-column group with a set
                          // bit is written; written by the model kernel, read by the
                          // PSF kernel
    const double* sat;    // (Nz, Ny + 1, Nx + 1): summed-area table of the zero-model r^2
    // executed-work counters (null unless enabled): what the direct-mode kernels
    // actually compute, for the roofline of the measured launches
    unsigned long long* counters;   // [GBK_CTR_*]
};

// counters[] slots (FMA = one fused multiply-add of one lane)
enum {
    GBK_CTR_KA_FMA = 0,     // LSF FIR taps of the model kernel
    GBK_CTR_KA_LINE = 1,    // line values (one exp each) of the model kernel
    GBK_CTR_KB_XFMA = 2,    // PSF x FIR taps
    GBK_CTR_KB_YFMA = 3,    // PSF y FIR taps
    GBK_CTR_KB_VOX = 4,     // residual voxels computed from the model box
    GBK_CTR_KA_SPAXEL = 5,  // spaxel evaluations
    GBK_CTR_N = 8
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

constexpr int KA_THREADS = 128;        // 4 independent (row, chunk) warps per block

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
// rows and columns.  The model kernel records each plane row chunk's nonzero
// columns; the PSF kernel convolves only the bounding box of its plane (sums
// of exact zeros are exact zeros, so results do not change) and takes the
// residual outside the box, where the model is exactly 0, from a summed-area
// table of ((0 - data) / error * mask * weight)^2 built once per data cube.

// KA: a warp per (set, window row y, 32-spaxel chunk of the row), no block
// synchronisation.  A lane evaluates its spaxel and then streams its
// LSF-convolved spectral column over the warp's output channel range: a
// sliding window of KZ line values in registers (compile-time rotation, KZ
// taps per output), each output plane row chunk stored as one coalesced
// 128-byte segment.  Per plane the chunk's nonzero-column mask is stored.
// Warp-wide transpose of a 32 x 32 bit matrix: lane i holds row i (bit j =
// column j) and receives column i (bit j = row j of lane j).  Five butterfly
// stages, each exchanging the off-diagonal blocks of the 2s x 2s sub-blocks
// (s = 16, 8, 4, 2, 1) with the partner lane i ^ s.
__device__ __forceinline__ unsigned warp_transpose32(unsigned v, int lane)
{
    constexpr unsigned M[5] = {0x0000ffffu, 0x00ff00ffu, 0x0f0f0f0fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int s = 16 >> k;
        const unsigned y = __shfl_xor_sync(0xffffffffu, v, s);
        v = (lane & s) ? ((v & ~M[k]) | ((y >> s) & M[k])) : ((v & M[k]) | ((y << s) & ~M[k]));
    }
    return v;
}

// The nonzero-lane masks of output planes [mz, mz + 32): lane j receives the
// mask of plane mz + j, bit l set when lane l's output range [olo, ohi]
// holds that plane (the per-plane ballots of the range test, for 32 planes
// at once).  A lane without a line passes olo > ohi.
__device__ __forceinline__ unsigned plane_masks32(int olo, int ohi, int mz, int lane)
{
    const int a = max(olo - mz, 0), e = min(ohi - mz, 31);
    const unsigned row = a <= e ? ((0xffffffffu >> (31 - e)) & (0xffffffffu << a)) : 0u;
    return warp_transpose32(row, lane);
}

template<int KZ>
__global__ void __launch_bounds__(KA_THREADS, (KZ <= 15 ? 8 : 4)) ka_lines_lsf(BatchKernelArgs P, int* status)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int item = blockIdx.x * (KA_THREADS / 32) + warp;
    if (item >= P.Wy * P.nch) return;                    // whole warp
    const int y = item / P.nch, chunk = item % P.nch;
    const int c = blockIdx.y, b = P.set0 + c;
    const DiskArgs a = set_disk(P, b);
    const DiskConst kc = disk_const(a);
    int bad = 0;
    const int x = chunk * 32 + lane;
    SpaxelOut o{};
    int lo = INT_MAX, hi = -1;
    float amp = 0.f, rinv = 0.f;
    const bool on = x < P.Wx && (P.nwfast ? smdisk_spaxel_nw(a, kc, x, y, o)
                                           : smdisk_spaxel(a, kc, x, y, 0, o, bad));
    if (on && line_window(o.vv, o.dv, P.Wz, a.spec_step, a.spec_zero, lo, hi)) {
        amp = o.orv * (1 / (o.dv * sqrtf(2 * GBK_PI)));
        // exp(-d^2 / (2 sigma^2)) as exp2(-d^2 * log2(e) / (2 sigma^2))
        rinv = 1.4426950408889634f / (2 * o.dv * o.dv);
    } else {
        lo = INT_MAX;
        hi = -1;
    }
    const float v = o.vv, z0 = a.spec_zero, dz = a.spec_step;
    // gmodels.hpp:109-115: the line at window channel z (0 outside [lo, hi]);
    // 2^x by the PTX ex2.approx instruction (relative error ~2^-22; the
    // argument is >= -18.1 inside the +-5 sigma window, far from underflow)
    // (one unsigned compare for z in [lo, hi]; a lane without a line has
    // amp = 0 and rinv = 0, so its value is 0 whatever the compare says)
    // zf: z as a float (exact: channel indices are far below 2^24)
    const unsigned wlen = (unsigned)hi - (unsigned)lo;
    auto line_f = [&](int z, float zf) {
        const float d = (z0 + zf * dz) - v;
        float e;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-(d * d) * rinv));
        return (unsigned)z - (unsigned)lo <= wlen ? amp * e : 0.f;
    };
    auto line = [&](int z) { return line_f(z, (float)z); };
    // the lane's and the warp's output channel ranges
    const bool lit = lo <= hi;
    const int olo = lit ? max(0, lo - KZ + 1) : INT_MAX, ohi = lit ? min(P.Nz - 1, hi) : -1;
    const unsigned olen = lit ? (unsigned)(ohi - olo) : 0u;
    int zlo = olo, zhi = ohi;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        zlo = min(zlo, __shfl_xor_sync(0xffffffffu, zlo, s));
        zhi = max(zhi, __shfl_xor_sync(0xffffffffu, zhi, s));
    }
    // the range table, plane-major (set, plane, row, chunk) as the PSF kernel
    // reads it: this warp's entry of plane z at xr[z * xs]
    const long long xs = (long long)P.Wy * P.nch;
    int* xr = P.xrt + ((long long)c * P.Nz * P.Wy + y) * P.nch + chunk;
    // planes outside [zlo, zhi] are empty for this chunk
    for (int zo = lane; zo < P.Nz; zo += 32)
        if (zo < zlo || zo > zhi) xr[zo * xs] = 0;
    if (zlo <= zhi) {
        float lz[KZ];
#pragma unroll
        for (int t = 0; t < KZ; ++t) lz[t] = P.lsfr[t];
        float w[KZ];
#pragma unroll
        for (int t = 0; t < KZ - 1; ++t) w[t] = line(zlo + t);
        const long long zstride = (long long)P.Wy * P.pitch;
        float* dp = P.mplanes + ((long long)c * P.Nz * P.Wy + y) * P.pitch + x + zlo * zstride;
        unsigned mm = 0u;
        // lane (zo - mz) keeps the ballot of plane zo; flushed at plane fl, every
        // 32 planes and at the last one
        int mz = zlo, own = zlo + lane, fl = min(zlo + 31, zhi);
        float zf = (float)(zlo + KZ - 1);       // the newest window channel, counted in float
        for (int zb = zlo; zb <= zhi; zb += KZ) {
#pragma unroll
            for (int k = 0; k < KZ; ++k) {
                const int zo = zb + k;
                if (zo > zhi) break;
                w[(k + KZ - 1) % KZ] = line_f(zo + KZ - 1, zf);
                zf += 1.f;
                // two independent accumulation chains (even and odd taps)
                float acc0 = 0.f, acc1 = 0.f;
#pragma unroll
                for (int t = 0; t < KZ; t += 2) acc0 += lz[t] * w[(k + t) % KZ];
#pragma unroll
                for (int t = 1; t < KZ; t += 2) acc1 += lz[t] * w[(k + t) % KZ];
                *dp = acc0 + acc1;      // plane zo
                dp += zstride;
                // zo in [olo, ohi] (false for a lane without a line: olo = INT_MAX, ohi = -1)
                const unsigned m = __ballot_sync(0xffffffffu,
                                                 (unsigned)zo - (unsigned)olo <= olen);
                if (zo == own) mm = m;
                if (zo == fl) {
                    if (own <= zo) xr[own * xs] = (int)mm;
                    mz = zo + 1;
                    own = mz + lane;
                    fl = min(mz + 31, zhi);
                }
            }
        }
    }
    if (P.counters && lane == 0) {
        atomicAdd(&P.counters[GBK_CTR_KA_SPAXEL], 32ull);
        if (zlo <= zhi) {
            const unsigned long long n = (unsigned long long)(zhi - zlo + 1) * 32;
            atomicAdd(&P.counters[GBK_CTR_KA_FMA], n * KZ);
            atomicAdd(&P.counters[GBK_CTR_KA_LINE], n + (KZ - 1) * 32ull);
        }
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// KA on compact spaxel tiles: a block per (set, 4 window rows, 32-column
// chunk), its warp w on the 4 x 8 tile of columns [32 chunk + 8 w, + 8); lane
// l takes spaxel (32 chunk + 8 w + (l & 7), 4 rg + (l >> 3)).  The lines of
// nearby spaxels have close channel windows, and a 4 x 8 tile spans fewer
// velocities than a 32-spaxel row, so the warp's channel range (the union of
// its lanes' output ranges) is shorter: ~1.57 instead of ~2.11 times the
// lanes' own ranges for the 128 x 128 x 96 batch workload.  Each plane row
// store is a 32-byte segment.  A warp's ballot of plane zo holds four rows'
// 8-column masks; each goes into byte w of that row chunk's entry (columns
// 8 w .. 8 w + 7) in shared memory (Nz x 4 entries, zero where no warp
// writes), and the block stores whole entries once all four warps are done.
// The lines, the LSF FIR and its order of operations are those of
// ka_lines_lsf (identical values).
// TM (transposed masks): no ballot in the channel loop; after it, each group
// of 32 planes gets its masks at once, every lane forming its output range
// as a 32-bit row and the warp transposing the 32 rows (plane_masks32): the
// same masks for a few instructions per group instead of several per plane.
// SL (scaled line): the exponent as -t^2 with t = zf (dz s) + (z0 - v) s and
// s = sqrt(log2(e) / (2 sigma^2)), one multiply-add and one multiply per
// channel instead of a multiply-add, an add and two multiplies; the same line
// up to fp32 rounding (not bit-identical to the other forms).
template<int KZ, bool TM, bool SL = false>
__global__ void __launch_bounds__(KA_THREADS, (KZ <= 15 ? 8 : 4)) ka_lines_lsf_t(BatchKernelArgs P, int* status)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rg = blockIdx.x / P.nch, chunk = blockIdx.x % P.nch;   // grid: ceil(Wy / 4) nch
    extern __shared__ unsigned s_ent[];                               // (Nz, 4 rows)
    for (int i = threadIdx.x; i < 4 * P.Nz; i += KA_THREADS) s_ent[i] = 0u;
    __syncthreads();
    const int y = 4 * rg + (lane >> 3), x = chunk * 32 + 8 * warp + (lane & 7);
    const bool row_ok = y < P.Wy;
    const int c = blockIdx.y, b = P.set0 + c;
    const DiskArgs a = set_disk(P, b);
    const DiskConst kc = disk_const(a);
    int bad = 0;
    SpaxelOut o{};
    int lo = INT_MAX, hi = -1;
    float amp = 0.f, rinv = 0.f;
    const bool on = row_ok && x < P.Wx &&
                    (P.nwfast ? smdisk_spaxel_nw(a, kc, x, y, o) : smdisk_spaxel(a, kc, x, y, 0, o, bad));
    if (on && line_window(o.vv, o.dv, P.Wz, a.spec_step, a.spec_zero, lo, hi)) {
        amp = o.orv * (1 / (o.dv * sqrtf(2 * GBK_PI)));
        rinv = 1.4426950408889634f / (2 * o.dv * o.dv);
    } else {
        lo = INT_MAX;
        hi = -1;
    }
    const float v = o.vv, z0 = a.spec_zero, dz = a.spec_step;
    const unsigned wlen = (unsigned)hi - (unsigned)lo;
    const float sc = SL ? sqrtf(rinv) : 0.f;
    const float dzs = dz * sc, cs = (z0 - v) * sc;
    auto line_f = [&](int z, float zf) {
        float e;
        if constexpr (SL) {
            const float t = fmaf(zf, dzs, cs);
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-(t * t)));
        } else {
            const float d = (z0 + zf * dz) - v;
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-(d * d) * rinv));
        }
        return (unsigned)z - (unsigned)lo <= wlen ? amp * e : 0.f;
    };
    auto line = [&](int z) { return line_f(z, (float)z); };
    const bool lit = lo <= hi;
    const int olo = lit ? max(0, lo - KZ + 1) : INT_MAX, ohi = lit ? min(P.Nz - 1, hi) : -1;
    const unsigned olen = lit ? (unsigned)(ohi - olo) : 0u;
    int zlo = olo, zhi = ohi;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        zlo = min(zlo, __shfl_xor_sync(0xffffffffu, zlo, s));
        zhi = max(zhi, __shfl_xor_sync(0xffffffffu, zhi, s));
    }
    // byte `warp` of the entries of plane z, rows 4 rg + r (r < 4)
    auto put = [&](int z, unsigned m) {
        unsigned char* e = reinterpret_cast<unsigned char*>(s_ent + 4 * z) + warp;
#pragma unroll
        for (int r = 0; r < 4; ++r) e[4 * r] = (unsigned char)(m >> (8 * r));
    };
    if (zlo <= zhi) {
        float lz[KZ];
#pragma unroll
        for (int t = 0; t < KZ; ++t) lz[t] = P.lsfr[t];
        float w[KZ];
#pragma unroll
        for (int t = 0; t < KZ - 1; ++t) w[t] = line(zlo + t);
        const long long zstride = (long long)P.Wy * P.pitch;
        float* dp = P.mplanes + ((long long)c * P.Nz * P.Wy + (row_ok ? y : 0)) * P.pitch + x +
                    zlo * zstride;
        unsigned mm = 0u;
        int mz = zlo, own = zlo + lane, fl = min(zlo + 31, zhi);
        float zf = (float)(zlo + KZ - 1);
        for (int zb = zlo; zb <= zhi; zb += KZ) {
#pragma unroll
            for (int k = 0; k < KZ; ++k) {
                const int zo = zb + k;
                if (zo > zhi) break;
                w[(k + KZ - 1) % KZ] = line_f(zo + KZ - 1, zf);
                zf += 1.f;
                float acc0 = 0.f, acc1 = 0.f;
#pragma unroll
                for (int t = 0; t < KZ; t += 2) acc0 += lz[t] * w[(k + t) % KZ];
#pragma unroll
                for (int t = 1; t < KZ; t += 2) acc1 += lz[t] * w[(k + t) % KZ];
                if (row_ok) *dp = acc0 + acc1;      // plane zo
                dp += zstride;
                if constexpr (!TM) {
                    const unsigned m = __ballot_sync(0xffffffffu,
                                                     (unsigned)zo - (unsigned)olo <= olen);
                    if (zo == own) mm = m;
                    if (zo == fl) {
                        if (own <= zo) put(own, mm);
                        mz = zo + 1;
                        own = mz + lane;
                        fl = min(mz + 31, zhi);
                    }
                }
            }
        }
        if constexpr (TM) {
            // lanes without a line: olo = INT_MAX, ohi = -1 (an empty row)
            for (int g = zlo; g <= zhi; g += 32) {
                const unsigned m = plane_masks32(olo, ohi, g, lane);
                if (g + lane <= zhi) put(g + lane, m);
            }
        }
    }
    // the block's entries: every plane of its rows in the window
    __syncthreads();
    const int nrow = min(4, P.Wy - 4 * rg);
    const long long xs = (long long)P.Wy * P.nch;
    int* xr = P.xrt + ((long long)c * P.Nz * P.Wy + 4 * rg) * P.nch + chunk;
    for (int i = threadIdx.x; i < nrow * P.Nz; i += KA_THREADS) {
        const int z = i / nrow, r = i - z * nrow;
        xr[z * xs + r * P.nch] = (int)s_ent[4 * z + r];
    }
    if (P.counters && lane == 0) {
        atomicAdd(&P.counters[GBK_CTR_KA_SPAXEL], 32ull);
        if (zlo <= zhi) {
            const unsigned long long n = (unsigned long long)(zhi - zlo + 1) * 32;
            atomicAdd(&P.counters[GBK_CTR_KA_FMA], n * KZ);
            atomicAdd(&P.counters[GBK_CTR_KA_LINE], n + (KZ - 1) * 32ull);
        }
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
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

// KB: one block per (set, output plane zo, band of output rows), sets fastest.  The block
// finds the bounding box of the band's nonzero input row chunks and works
// through its output rows in passes whose input rows fit the block's shared
// memory (box-relative row pitch; usually one pass):
//   - the rows' nonzero 4-column groups are loaded from HBM (cp.async), the rest of
//     the rows that the y FIR reads is zeroed;
//   - x FIR in place, a warp per row, its lanes on consecutive (row, strip)
//     pairs of its rows, 8 outputs per lane window;
//   - y FIR, 8 x 4 outputs per (8-row group, column) item in registers, and
//     in the same item the crop, residual (objective.hpp:7-31) and r^2
//     against the data.
// The zero-model residual outside the box comes from the summed-area table.
constexpr int KB_THREADS = 128;
constexpr int KB_NX_MAX = 512;  // widest data cube of the direct mode

// MINB: resident blocks per SM the registers are sized for (4: up to 128
// registers a thread; 5: up to 102, with the shared memory per block sized to
// match, see setup_direct)
// EPI: how the y FIR meets the residual.  0: y FIR in place in rounds of
// items with a barrier between loads and stores, then a residual pass over the
// pass's rows reading shared memory; 1: the residual in each y-FIR item's
// epilogue (no write-back, no barriers between items), its data loaded after
// the item's FIR; 2: as 1, with the item's data requested before its FIR.
template<int K, int MINB, int EPI, bool PF, int NT>
__global__ void __launch_bounds__(NT, MINB) kb_psf_residual(BatchKernelArgs P)
{
    constexpr int NW = (K + 7 + 3) / 4;     // float4 slots of one 8-output x window
    constexpr int NWARPS = NT / 32;
    extern __shared__ float4 sm4[];
    float* S = reinterpret_cast<float*>(sm4);                   // (rows of a pass, bp)
    // (in1 - ob0, nch) range entries of an item; PF: two buffers of xr_slot ints
    int* const s_xr0 = reinterpret_cast<int*>(S + P.cap);
    __shared__ float warp_part[NWARPS];
    __shared__ int s_box[4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ld = P.Nx + 1;
    // PF (persistent): the blocks take items of cn x Nz x nbands (sets fastest)
    // from a work counter, one ahead: the next item's range entries are copied
    // into the other buffer (cp.async) while this item runs.  Otherwise one
    // item per block:
    // blockIdx.x the set, blockIdx.y the (plane, band) - sets vary fastest, so
    // the blocks in flight share a few planes of the data.
    const int nit = PF ? P.kb_cn * P.Nz * P.nbands : 1;
    auto entries = [&](int it, const int*& src, int& n, int& ob0_) {
        const int c_ = PF ? it % P.kb_cn : blockIdx.x;
        const int yi = PF ? it / P.kb_cn : blockIdx.y;
        const int zo_ = yi / P.nbands, band_ = yi % P.nbands;
        ob0_ = band_ * P.band;
        const int ob1_ = min(P.Ny, ob0_ + P.band), in1_ = min(P.Wy, ob1_ + K - 1);
        src = P.xrt + (((long long)c_ * P.Nz + zo_) * P.Wy + ob0_) * P.nch;
        n = (in1_ - ob0_) * P.nch;
    };
    auto prefetch = [&](int it, int* dst) {
        const int* src;
        int n, o;
        entries(it, src, n, o);
        for (int i = threadIdx.x; i < n; i += NT) cp_async4(dst + i, src + i);
    };
    __shared__ int s_next;
    int buf = 0, it = 0;
    if (PF) {
        if (threadIdx.x == 0) s_next = atomicAdd(P.kb_work, 1);
        __syncthreads();
        it = s_next;
        __syncthreads();      // every thread has read s_next before it is rewritten
        if (it < nit) prefetch(it, s_xr0);
    }
    while (it < nit) {
    int* const s_xr = s_xr0 + buf * P.xr_slot;
    const int c = PF ? it % P.kb_cn : (int)blockIdx.x, b = P.set0 + c;
    const int yi = PF ? it / P.kb_cn : (int)blockIdx.y;
    const int zo = yi / P.nbands, band = yi % P.nbands;
    const int ob0 = band * P.band, ob1 = min(P.Ny, ob0 + P.band);  // output rows [ob0, ob1)
    const int in1 = min(P.Wy, ob1 + K - 1);                        // input rows [ob0, in1)
    const long long prow = ((long long)c * P.Nz + zo) * P.Wy;
    const int* xr = P.xrt + prow * P.nch;                          // (y, chunk) at [y nch + chunk]
    const double* T = P.sat + (long long)zo * (P.Ny + 1) * ld;
    if (PF) cp_async_wait_all();          // this item's entries (this thread's copies)
    if (threadIdx.x == 0) {
        s_box[0] = INT_MAX; s_box[1] = -1; s_box[2] = INT_MAX; s_box[3] = -1;
        if (PF) s_next = atomicAdd(P.kb_work, 1);
    }
    __syncthreads();
    // the next item's entries, into the other buffer (its last reader, the
    // item before this one, has finished)
    const int next = PF ? s_next : nit;
    if (PF && next < nit) prefetch(next, s_xr0 + (buf ^ 1) * P.xr_slot);
    do {
    // bounding box of the nonzero input row chunks
    {
        int y0 = INT_MAX, y1 = -1, x0 = INT_MAX, x1 = -1;
        // the entries of rows [ob0, in1), eight loads in flight per thread
        // (PF: already in s_xr)
        const int* src = xr + ob0 * P.nch;
        const int n = (in1 - ob0) * P.nch;
        for (int i0 = 0; i0 < n; i0 += 8 * NT) {
            int v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = i0 + u * NT + threadIdx.x;
                if (PF) {
                    v[u] = i < n ? s_xr[i] : 0;
                } else {
                    v[u] = i < n ? src[i] : 0;
                    if (i < n) s_xr[i] = v[u];
                }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (v[u] != 0) {
                    const int i = i0 + u * NT + (int)threadIdx.x;
                    const int r = i / P.nch, ch = i - r * P.nch;
                    y0 = min(y0, ob0 + r);
                    y1 = max(y1, ob0 + r);
                    x0 = min(x0, ch * 32 + __ffs(v[u]) - 1);
                    x1 = max(x1, ch * 32 + 31 - __clz(v[u]));
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, o));
            y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, o));
            x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, o));
            x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        }
        if (lane == 0 && y1 >= 0) {
            atomicMin(&s_box[0], y0);
            atomicMax(&s_box[1], y1);
            atomicMin(&s_box[2], x0);
            atomicMax(&s_box[3], x1);
        }
    }
    __syncthreads();
    const int y0 = s_box[0], y1 = s_box[1], x0 = s_box[2], x1 = s_box[3];
    const long long plane = (long long)P.Ny * P.Nx;
    float* model = P.model ? P.model + ((long long)b * P.Nz + zo) * plane : nullptr;
    const long long part = ((long long)b * P.Nz + zo) * P.nbands + band;
    if (y1 < 0) {   // nothing reaches this band: the model is 0 on it
        if (model)
            for (long long i = (long long)ob0 * P.Nx + threadIdx.x; i < (long long)ob1 * P.Nx;
                 i += NT)
                model[i] = 0.f;
        if (threadIdx.x == 0) P.partials[part] = sat_box(T, ld, ob0, ob1, 0, P.Nx);
        break;
    }
    // output box: x in 8-column strips [g_lo, g_hi], rows [yo_lo, yb_end) in 8-row groups
    const int g_lo = max(0, x0 - K + 1) >> 3, g_hi = min(P.Nx - 1, x1) >> 3;
    const int ns8 = g_hi - g_lo + 1, ns4 = 2 * ns8, sl0 = 2 * g_lo;
    const int yo_lo = max(ob0, y0 - K + 1), yo_hi = min(ob1 - 1, y1);
    const int yb_end = min(ob1, yo_lo + 8 * ((yo_hi - yo_lo + 8) / 8));
    const int xb0 = 8 * g_lo, xb_end = min(P.Nx, 8 * g_hi + 8);
    // the zero-model part, issued now so that its loads overlap the passes
    double outside = 0.0;
    if (threadIdx.x == 0)
        outside = sat_box(T, ld, ob0, ob1, 0, P.Nx) - sat_box(T, ld, yo_lo, yb_end, xb0, xb_end);
    // box-relative rows: float4 slots [sl0, sl0 + nsl), pitch bp (% 32 == 4)
    const int nsl = 2 * (ns8 - 1) + NW;
    int bp = 4 * nsl;
    bp += ((4 - bp % 32) + 32) % 32;
    const int bp4 = bp / 4;
    const int bo = ((P.cap / bp - (K + 7)) / 8) * 8;        // output rows per pass (>= 8)
    const float4* src = reinterpret_cast<const float4*>(P.mplanes + prow * P.pitch);
    const int pbase = zo * P.Ny * P.Nx;       // the data cube has < 2^31 voxels
    float sum = 0.f;
    unsigned long long c_x = 0, c_y = 0, c_v = 0;    // executed work (thread 0)
    for (int ys = yo_lo; ys < yb_end; ys += bo) {
        const int ye = min(yb_end, ys + bo);                 // outputs [ys, ye)
        const int ng = (ye - ys + 7) / 8;
        const int rend = ys + 8 * ng + K - 1;                // rows [ys, rend) are read
        const int ly0 = max(y0, ys), ly1 = min(y1, rend - 1);
        if (P.counters && threadIdx.x == 0) {
            if (ly0 <= ly1) c_x += (unsigned long long)(ly1 - ly0 + 1) * ns8 * 8 * K;
            c_y += (unsigned long long)ng * ns4 * 32 * K;
            c_v += (unsigned long long)(ye - ys) * (xb_end - xb0);
        }
        // load rows [ly0, ly1]: the 4-column groups that hold a nonzero value, zeros elsewhere
        if (ly0 <= ly1) {
            const int tc = min(nsl, NT), tr = NT / tc;
            const int ti = threadIdx.x % tc, ty = threadIdx.x / tc;
            if (ty < tr) {
                for (int y = ly0 + ty; y <= ly1; y += tr) {
                    const int* vrow = s_xr + (y - ob0) * P.nch;
                    float4* d = reinterpret_cast<float4*>(S) + (y - ys) * bp4;
                    const float4* g = src + (long long)y * (P.pitch / 4);
                    for (int j = ti; j < nsl; j += tc) {
                        // the slot's 4 columns hold a nonzero value: load them
                        // (all written), else they are zeros
                        const int sl = sl0 + j, ch = sl >> 3;
                        const unsigned v = ch < P.nch ? (unsigned)vrow[ch] : 0u;
                        if ((v >> (4 * (sl & 7))) & 0xfu)
                            cp_async16(d + j, g + sl);
                        else
                            d[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
            }
        }
        // the other rows that the y FIR reads: zeros in its strips
        {
            const int tc = min(ns4, NT), tr = NT / tc;
            const int ti = threadIdx.x % tc, ty = threadIdx.x / tc;
            if (ty < tr) {
                for (int y = ys + ty; y < rend; y += tr) {
                    if (y >= ly0 && y <= ly1) continue;
                    float4* d = reinterpret_cast<float4*>(S) + (y - ys) * bp4;
                    for (int j = ti; j < ns4; j += tc) d[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
        // x FIR in place: S[y][xo] = sum_s vr[s] S[y][xo + s].  A warp owns whole
        // rows (ly0 + warp, + NWARPS, ...); its lanes take consecutive (row,
        // strip) pairs of those rows, 32 per pass.  Strip g writes columns
        // [8g, 8g + 8) and reads columns >= 8g, so a row's strips in increasing
        // order across passes, with loads before __syncwarp, never read a
        // column that an earlier store of the row has overwritten.
        if (ly0 <= ly1) {
            float vr[K];
#pragma unroll
            for (int s = 0; s < K; ++s) vr[s] = P.vr[s];
            const int nr = ly1 - ly0 + 1;
            const int nri = warp < nr ? (nr - 1 - warp) / NWARPS + 1 : 0;   // rows of this warp
            const int npairs = nri * ns8;
            const int di = 32 / ns8, dg = 32 % ns8;
            int ri = lane / ns8, gi = lane % ns8;       // the lane's pair: row index, strip
            for (int q0 = 0; q0 < npairs; q0 += 32) {
                const bool act = q0 + lane < npairs;
                float4* row = reinterpret_cast<float4*>(S) + (ly0 + warp + NWARPS * ri - ys) * bp4;
                float w[4 * NW];
                if (act) {
#pragma unroll
                    for (int m = 0; m < NW; ++m) {
                        const float4 f = row[2 * gi + m];
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
                    row[2 * gi] = make_float4(o[0], o[1], o[2], o[3]);
                    row[2 * gi + 1] = make_float4(o[4], o[5], o[6], o[7]);
                }
                __syncwarp();
                ri += di;
                gi += dg;
                if (gi >= ns8) {
                    gi -= ns8;
                    ++ri;
                }
            }
        }
        __syncthreads();
        if constexpr (EPI == 0) {
            constexpr int kIt = 1;     // y items per thread and round
            // y FIR in place: model(yo, xo) = sum_t ur[t] S[yo + t][xo], written to S row yo.
            // Packed FP32 pairs (FFMA2: two lanes of fma, each rounded as fmaf),
            // columns (x, x+1) and (x+2, x+3) of a float4 per instruction.  Items
            // (8-row group, float4 column) in ascending order, NT x kIt
            // per round, loads before the round's barrier and stores after it: a
            // column's group is written only after every lower group of that
            // column, the only readers of its rows, has loaded them.
            {
                float2 u2[K];
    #pragma unroll
                for (int t = 0; t < K; ++t) u2[t] = make_float2(P.ur[t], P.ur[t]);
                const int nitems = ng * ns4;
                for (int gr0 = 0; gr0 < nitems; gr0 += NT * kIt) {
                    float2 acc[kIt][8][2];
    #pragma unroll
                    for (int it = 0; it < kIt; ++it) {
                        const int item = gr0 + threadIdx.x + it * NT;
    #pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            acc[it][q][0] = make_float2(0.f, 0.f);
                            acc[it][q][1] = make_float2(0.f, 0.f);
                        }
                        if (item < nitems) {
                            const int rb = 8 * (item / ns4), s4 = item % ns4;
                            const float4* colp = reinterpret_cast<const float4*>(S) + rb * bp4 + s4;
    #pragma unroll
                            for (int m = 0; m < K + 7; ++m) {
                                const float4 p = colp[m * bp4];
                                const float2 pxy = make_float2(p.x, p.y), pzw = make_float2(p.z, p.w);
    #pragma unroll
                                for (int q = 0; q < 8; ++q) {
                                    const int t = m - q;
                                    if (t >= 0 && t < K) {
                                        acc[it][q][0] = __ffma2_rn(u2[t], pxy, acc[it][q][0]);
                                        acc[it][q][1] = __ffma2_rn(u2[t], pzw, acc[it][q][1]);
                                    }
                                }
                            }
                        }
                    }
                    __syncthreads();
    #pragma unroll
                    for (int it = 0; it < kIt; ++it) {
                        const int item = gr0 + threadIdx.x + it * NT;
                        if (item < nitems) {
                            const int rb = 8 * (item / ns4), s4 = item % ns4;
    #pragma unroll
                            for (int q = 0; q < 8; ++q)
                                if (ys + rb + q < ye)
                                    reinterpret_cast<float4*>(S)[(rb + q) * bp4 + s4] =
                                        make_float4(acc[it][q][0].x, acc[it][q][0].y,
                                                    acc[it][q][1].x, acc[it][q][1].y);
                        }
                    }
                    __syncthreads();
                }
            }
            // crop + residual over rows [ys, ye), columns [xb0, xb_end)
            if ((P.Nx & 3) == 0) {
                // flat float4 index over the pass, stepped without divisions
                const int nv = (xb_end - xb0) >> 2;        // xb0 and xb_end are multiples of 4
                const int n = (ye - ys) * nv;
                const int dq = NT / nv, dr = NT % nv;
                int row = threadIdx.x / nv, col = threadIdx.x % nv;
                // running offsets: si in S (float4), vi in the data plane (float)
                int si = row * bp4 + col, vi = pbase + (ys + row) * P.Nx + xb0 + 4 * col;
                const int dsi = dq * bp4 + dr, dvi = dq * P.Nx + 4 * dr;
                float2 s2 = make_float2(0.f, 0.f);
    #pragma unroll 4
                for (int i = threadIdx.x; i < n; i += NT) {
                    const float4 m = reinterpret_cast<const float4*>(S)[si];
                    const float4 o = *reinterpret_cast<const float4*>(P.obs + vi);
                    const float4 w = *reinterpret_cast<const float4*>(P.iw + vi);
                    // packed pairs: r = (m - o) w, s2 += r^2
                    const float2 r01 = __fmul2_rn(__fadd2_rn(make_float2(m.x, m.y),
                                                             make_float2(-o.x, -o.y)),
                                                  make_float2(w.x, w.y));
                    const float2 r23 = __fmul2_rn(__fadd2_rn(make_float2(m.z, m.w),
                                                             make_float2(-o.z, -o.w)),
                                                  make_float2(w.z, w.w));
                    s2 = __ffma2_rn(r01, r01, s2);
                    s2 = __ffma2_rn(r23, r23, s2);
                    if (model) *reinterpret_cast<float4*>(model + (vi - pbase)) = m;
                    col += dr;
                    si += dsi;
                    vi += dvi;
                    if (col >= nv) {
                        col -= nv;
                        si += bp4 - nv;
                        vi += P.Nx - 4 * nv;
                    }
                }
                sum += s2.x + s2.y;
            } else {
                const int nw = xb_end - xb0, n = (ye - ys) * nw;
                for (int i = threadIdx.x; i < n; i += NT) {
                    const int row = i / nw, col = i % nw;
                    const int yo = ys + row, xo = xb0 + col;
                    const float m = S[row * bp + col];
                    const int vi = pbase + yo * P.Nx + xo;
                    const float r0 = (m - P.obs[vi]) * P.iw[vi];
                    sum += r0 * r0;
                    if (model) model[yo * P.Nx + xo] = m;
                }
            }
        } else {
            // y FIR with the residual in its epilogue: item (8-row group rb, float4
            // column s4) computes model(ys + rb + q, xb0 + 4 s4 + j) = sum_t ur[t]
            // S[rb + q + t][4 s4 + j] for q < 8, j < 4 in registers, on packed FP32
            // pairs (FFMA2: two lanes of fma, each rounded as fmaf), then compares
            // them with the data (crop + residual, objective.hpp:7-31) and adds
            // r^2.  S is only read here, so items need no barriers between them.
            {
                const int nitems = ng * ns4;
                const bool vec = (P.Nx & 3) == 0;
                float2 s2 = make_float2(0.f, 0.f);
                for (int item = threadIdx.x; item < nitems; item += NT) {
                    const int rb = 8 * (item / ns4), s4 = item % ns4;
                    float2 acc[8][2];
    #pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        acc[q][0] = make_float2(0.f, 0.f);
                        acc[q][1] = make_float2(0.f, 0.f);
                    }
                    const int xo = xb0 + 4 * s4;
                    const bool inside = xo < xb_end;
                    // the item's data and weights, requested before its FIR so that
                    // their loads are in flight while the multiply-adds run
                    // (Nx % 4 == 0: a float4 column lies wholly inside or outside the crop)
                    float4 ov[8], wv[8];
                    if (EPI == 2 && vec) {
    #pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int yo = ys + rb + q;
                            if (inside && yo < ye) {
                                const int vi = pbase + yo * P.Nx + xo;
                                ov[q] = __ldg(reinterpret_cast<const float4*>(P.obs + vi));
                                wv[q] = __ldg(reinterpret_cast<const float4*>(P.iw + vi));
                            } else {
                                ov[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                                wv[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                            }
                        }
                    }
                    const float4* colp = reinterpret_cast<const float4*>(S) + rb * bp4 + s4;
    #pragma unroll
                    for (int m = 0; m < K + 7; ++m) {
                        const float4 p = colp[m * bp4];
                        const float2 pxy = make_float2(p.x, p.y), pzw = make_float2(p.z, p.w);
    #pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int t = m - q;
                            if (t >= 0 && t < K) {
                                acc[q][0] = __ffma2_rn(P.ur2[t], pxy, acc[q][0]);
                                acc[q][1] = __ffma2_rn(P.ur2[t], pzw, acc[q][1]);
                            }
                        }
                    }
                    if (!inside) continue;
                    if (vec) {
    #pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int yo = ys + rb + q;
                            if (yo >= ye) break;
                            const int vi = pbase + yo * P.Nx + xo;
                            float4 o, w;
                            if constexpr (EPI == 2) {
                                o = ov[q];
                                w = wv[q];
                            } else {
                                o = __ldg(reinterpret_cast<const float4*>(P.obs + vi));
                                w = __ldg(reinterpret_cast<const float4*>(P.iw + vi));
                            }
                            const float2 r01 = __fmul2_rn(__fadd2_rn(acc[q][0], make_float2(-o.x, -o.y)),
                                                          make_float2(w.x, w.y));
                            const float2 r23 = __fmul2_rn(__fadd2_rn(acc[q][1], make_float2(-o.z, -o.w)),
                                                          make_float2(w.z, w.w));
                            s2 = __ffma2_rn(r01, r01, s2);
                            s2 = __ffma2_rn(r23, r23, s2);
                            if (model)
                                *reinterpret_cast<float4*>(model + (vi - pbase)) =
                                    make_float4(acc[q][0].x, acc[q][0].y, acc[q][1].x, acc[q][1].y);
                        }
                    } else {
    #pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int yo = ys + rb + q;
                            if (yo >= ye) break;
                            const float mv[4] = {acc[q][0].x, acc[q][0].y, acc[q][1].x, acc[q][1].y};
    #pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                if (xo + j >= xb_end) break;
                                const int vi = pbase + yo * P.Nx + xo + j;
                                const float r0 = (mv[j] - P.obs[vi]) * P.iw[vi];
                                s2.x = fmaf(r0, r0, s2.x);
                                if (model) model[yo * P.Nx + xo + j] = mv[j];
                            }
                        }
                    }
                }
                sum += s2.x + s2.y;
            }
        }
        __syncthreads();    // S is reloaded by the next pass
    }
    if (model) {
        const int bw = P.Nx;
        for (long long i = (long long)ob0 * bw + threadIdx.x; i < (long long)ob1 * bw;
             i += NT) {
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
        for (int w = 0; w < NWARPS; ++w) s += warp_part[w];
        P.partials[part] = (double)s + outside;
        if (P.counters) {
            atomicAdd(&P.counters[GBK_CTR_KB_XFMA], c_x);
            atomicAdd(&P.counters[GBK_CTR_KB_YFMA], c_y);
            atomicAdd(&P.counters[GBK_CTR_KB_VOX], c_v);
        }
    }
    } while (0);
    if (PF) __syncthreads();   // before the next item reuses the shared memory
    buf ^= 1;
    it = next;
    }
}

// ka_lines_lsf on two 32-column chunks per warp: lane l evaluates columns
// 64 q + l and 64 q + 32 + l (chunks 2 q and 2 q + 1) and runs both LSF FIRs
// as packed FP32 pairs (FFMA2: two lanes of fma, each rounded as fmaf, so
// every value is the one ka_lines_lsf computes); each chunk keeps its own
// range-table entries.  Half the multiply-add instructions per spaxel.
template<int KZ>
__global__ void __launch_bounds__(KA_THREADS, (KZ <= 15 ? 5 : 4)) ka_lines_lsf2(BatchKernelArgs P, int* status)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int npair = (P.nch + 1) >> 1;
    const int item = blockIdx.x * (KA_THREADS / 32) + warp;
    if (item >= P.Wy * npair) return;                    // whole warp
    const int y = item / npair, c0 = 2 * (item % npair), c1 = c0 + 1;
    const bool has1 = c1 < P.nch;                        // warp-uniform
    const int c = blockIdx.y, b = P.set0 + c;
    const DiskArgs a = set_disk(P, b);
    const DiskConst kc = disk_const(a);
    int bad = 0;
    float amp[2], rinv[2], vv[2];
    int lo[2], hi[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int x = (c0 + h) * 32 + lane;
        SpaxelOut o{};
        lo[h] = INT_MAX;
        hi[h] = -1;
        amp[h] = 0.f;
        rinv[h] = 0.f;
        const bool on = x < P.Wx && (P.nwfast ? smdisk_spaxel_nw(a, kc, x, y, o)
                                               : smdisk_spaxel(a, kc, x, y, 0, o, bad));
        if (on && line_window(o.vv, o.dv, P.Wz, a.spec_step, a.spec_zero, lo[h], hi[h])) {
            amp[h] = o.orv * (1 / (o.dv * sqrtf(2 * GBK_PI)));
            rinv[h] = 1.4426950408889634f / (2 * o.dv * o.dv);
        } else {
            lo[h] = INT_MAX;
            hi[h] = -1;
        }
        vv[h] = o.vv;
    }
    const float z0 = a.spec_zero, dz = a.spec_step;
    const unsigned wlen0 = (unsigned)hi[0] - (unsigned)lo[0];
    const unsigned wlen1 = (unsigned)hi[1] - (unsigned)lo[1];
    // the lines of both columns at window channel z (as line_f of ka_lines_lsf)
    auto line2 = [&](int z, float zf) {
        const float zv = z0 + zf * dz;
        const float d0 = zv - vv[0], d1 = zv - vv[1];
        float e0, e1;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e0) : "f"(-(d0 * d0) * rinv[0]));
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e1) : "f"(-(d1 * d1) * rinv[1]));
        return make_float2((unsigned)z - (unsigned)lo[0] <= wlen0 ? amp[0] * e0 : 0.f,
                           (unsigned)z - (unsigned)lo[1] <= wlen1 ? amp[1] * e1 : 0.f);
    };
    int olo[2], ohi[2];
    unsigned olen[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const bool lit = lo[h] <= hi[h];
        olo[h] = lit ? max(0, lo[h] - KZ + 1) : INT_MAX;
        ohi[h] = lit ? min(P.Nz - 1, hi[h]) : -1;
        olen[h] = lit ? (unsigned)(ohi[h] - olo[h]) : 0u;
    }
    int zlo = min(olo[0], olo[1]), zhi = max(ohi[0], ohi[1]);
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        zlo = min(zlo, __shfl_xor_sync(0xffffffffu, zlo, s));
        zhi = max(zhi, __shfl_xor_sync(0xffffffffu, zhi, s));
    }
    // the range table, plane-major: the chunks' entries of plane z at [z * xs]
    const long long xs = (long long)P.Wy * P.nch;
    int* xr0 = P.xrt + ((long long)c * P.Nz * P.Wy + y) * P.nch + c0;
    int* xr1 = xr0 + 1;                                   // chunk c1 (used when has1)
    for (int zo = lane; zo < P.Nz; zo += 32)
        if (zo < zlo || zo > zhi) {
            xr0[zo * xs] = 0;
            if (has1) xr1[zo * xs] = 0;
        }
    if (zlo <= zhi) {
        float2 lz[KZ];
#pragma unroll
        for (int t = 0; t < KZ; ++t) lz[t] = make_float2(P.lsfr[t], P.lsfr[t]);
        float2 w[KZ];
#pragma unroll
        for (int t = 0; t < KZ - 1; ++t) w[t] = line2(zlo + t, (float)(zlo + t));
        const long long zstride = (long long)P.Wy * P.pitch;
        float* dp = P.mplanes + ((long long)c * P.Nz * P.Wy + y) * P.pitch + c0 * 32 + lane +
                    zlo * zstride;
        unsigned mm0 = 0u, mm1 = 0u;
        int mz = zlo, own = zlo + lane, fl = min(zlo + 31, zhi);
        float zf = (float)(zlo + KZ - 1);
        for (int zb = zlo; zb <= zhi; zb += KZ) {
#pragma unroll
            for (int k = 0; k < KZ; ++k) {
                const int zo = zb + k;
                if (zo > zhi) break;
                w[(k + KZ - 1) % KZ] = line2(zo + KZ - 1, zf);
                zf += 1.f;
                float2 acc0 = make_float2(0.f, 0.f), acc1 = make_float2(0.f, 0.f);
#pragma unroll
                for (int t = 0; t < KZ; t += 2) acc0 = __ffma2_rn(lz[t], w[(k + t) % KZ], acc0);
#pragma unroll
                for (int t = 1; t < KZ; t += 2) acc1 = __ffma2_rn(lz[t], w[(k + t) % KZ], acc1);
                const float2 r = __fadd2_rn(acc0, acc1);
                dp[0] = r.x;
                if (has1) dp[32] = r.y;
                dp += zstride;
                const unsigned m0 = __ballot_sync(0xffffffffu,
                                                  (unsigned)zo - (unsigned)olo[0] <= olen[0]);
                const unsigned m1 = __ballot_sync(0xffffffffu,
                                                  (unsigned)zo - (unsigned)olo[1] <= olen[1]);
                if (zo == own) {
                    mm0 = m0;
                    mm1 = m1;
                }
                if (zo == fl) {
                    if (own <= zo) {
                        xr0[own * xs] = (int)mm0;
                        if (has1) xr1[own * xs] = (int)mm1;
                    }
                    mz = zo + 1;
                    own = mz + lane;
                    fl = min(mz + 31, zhi);
                }
            }
        }
    }
    if (P.counters && lane == 0) {
        const unsigned long long nc = has1 ? 2 : 1;
        atomicAdd(&P.counters[GBK_CTR_KA_SPAXEL], 32ull * nc);
        if (zlo <= zhi) {
            const unsigned long long n = (unsigned long long)(zhi - zlo + 1) * 32 * nc;
            atomicAdd(&P.counters[GBK_CTR_KA_FMA], n * KZ);
            atomicAdd(&P.counters[GBK_CTR_KA_LINE], n + (KZ - 1) * 32ull * nc);
        }
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// The LSF FIR of given model cubes (any gmodel's output on the evaluation
// window, e.g. mcdisk's clouds) into the PSF kernel's input: the same
// planes and range table as ka_lines_lsf, so that the PSF FIR, residual and
// sum run unchanged.  cubes: (sets, Wz, Wy, Wx), set b = P.set0 + slot;
// one warp per (window row y, 32-column chunk), a lane per column, the
// channel axis walked with a KZ-deep register window (each cube value is
// read once).  A plane row chunk's mask marks its nonzero outputs (all
// outputs are written), so the PSF kernel skips exactly the zero ones.
template<int KZ>
__global__ void __launch_bounds__(KA_THREADS) kc_cube_lsf(BatchKernelArgs P,
                                                          const float* __restrict__ cubes)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int item = blockIdx.x * (KA_THREADS / 32) + warp;
    if (item >= P.Wy * P.nch) return;                    // whole warp
    const int y = item / P.nch, chunk = item % P.nch;
    const int c = blockIdx.y, b = P.set0 + c;
    const int x = chunk * 32 + lane;
    const bool in = x < P.Wx;
    const long long plane = (long long)P.Wy * P.Wx;
    const float* col = cubes + (long long)b * P.Wz * plane + (long long)y * P.Wx + (in ? x : 0);
    auto ld = [&](int z) { return in ? __ldg(col + z * plane) : 0.f; };
    float lz[KZ];
#pragma unroll
    for (int t = 0; t < KZ; ++t) lz[t] = P.lsfr[t];
    float w[KZ];
#pragma unroll
    for (int t = 0; t < KZ - 1; ++t) w[t] = ld(t);
    // the range table, plane-major: this warp's entry of plane z at xr[z * xs]
    const long long xs = (long long)P.Wy * P.nch;
    int* xr = P.xrt + ((long long)c * P.Nz * P.Wy + y) * P.nch + chunk;
    const long long zstride = (long long)P.Wy * P.pitch;
    float* dp = P.mplanes + ((long long)c * P.Nz * P.Wy + y) * P.pitch + x;
    unsigned mm = 0u;
    for (int zb = 0; zb < P.Nz; zb += KZ) {
#pragma unroll
        for (int k = 0; k < KZ; ++k) {
            const int zo = zb + k;
            if (zo >= P.Nz) break;
            w[(k + KZ - 1) % KZ] = ld(zo + KZ - 1);
            float acc0 = 0.f, acc1 = 0.f;
#pragma unroll
            for (int t = 0; t < KZ; t += 2) acc0 += lz[t] * w[(k + t) % KZ];
#pragma unroll
            for (int t = 1; t < KZ; t += 2) acc1 += lz[t] * w[(k + t) % KZ];
            const float v = acc0 + acc1;
            *dp = v;        // plane zo
            dp += zstride;
            // lane (zo % 32) keeps the ballot of plane zo; written every 32
            // planes and at the last one
            const unsigned m = __ballot_sync(0xffffffffu, v != 0.f);
            if ((zo & 31) == lane) mm = m;
            if ((zo & 31) == 31 || zo == P.Nz - 1) {
                const int own = (zo & ~31) + lane;
                if (own <= zo) xr[own * xs] = (int)mm;
            }
        }
    }
    if (P.counters && lane == 0)
        atomicAdd(&P.counters[GBK_CTR_KA_FMA], (unsigned long long)P.Nz * 32 * KZ);
}

typedef void (*KaFn)(BatchKernelArgs, int*);
typedef void (*KbFn)(BatchKernelArgs);
constexpr int KA_KMAX = 33;                 // longest LSF of the direct path
constexpr int KB_KMIN = 5, KB_KMAX = 33;    // PSF FIR lengths (odd)
static_assert(KA_KMAX <= 33 && KB_KMAX <= 33, "coefficient arrays of BatchKernelArgs");
// fill t[Kz / 2] (model kernel) and t[(K - KB_KMIN) / 2] (PSF kernel)
void ka_register_short(KaFn* t);
void ka_register_long(KaFn* t);
// t[Kz / 2]: the two-chunk model kernel (ka_lines_lsf2)
void ka2_register(KaFn* t);
// t[Kz / 2]: the model kernel on 4 x 8 spaxel tiles (ka_lines_lsf_t)
void ka_t_register(KaFn* t, bool tm, bool sl);
// t[Kz / 2]: the LSF FIR of given model cubes
typedef void (*KcFn)(BatchKernelArgs, const float*);
void kc_register(KcFn* t);
// t[v][(K - KB_KMIN) / 2] for the PSF kernel variant v = 3 * (MINB == 5) + EPI
// (v = 6: MINB 4, EPI 0, persistent with prefetched range entries; v = 7:
// 256-thread blocks, MINB 2, EPI 0)
constexpr int KB_VARIANTS = 8;
void kb_register4(KbFn (*t)[(KB_KMAX - KB_KMIN) / 2 + 1]);   // MINB 4, EPI 0-2
void kb_register5(KbFn (*t)[(KB_KMAX - KB_KMIN) / 2 + 1]);   // MINB 5, EPI 0-2
void kb_register_pf(KbFn (*t)[(KB_KMAX - KB_KMIN) / 2 + 1]); // MINB 4, EPI 0, persistent
void kb_register_wide(KbFn (*t)[(KB_KMAX - KB_KMIN) / 2 + 1]); // 256 threads, MINB 2, EPI 0

}  // namespace gbk
