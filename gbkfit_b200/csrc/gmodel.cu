// smdisk / mcdisk / wcube evaluation kernels and their C-ABI entry points.
//
// Reference: gbkfit/include/gbkfit/gmodel/gmodels.hpp (per-spaxel and
// per-cloud arithmetic, restated in gbk_traits.cuh and below) and the drivers
// gbkfit_host/include/gbkfit/host/kernels.hpp:160-423 (OpenMP) and
// gbkfit_cuda/src/wrapper.cu:82-324 (one thread per item, global atomics).
//
// Design:
//  * thin disks (spatial z = 1): one thread per spaxel; a warp (32 adjacent x)
//    walks the union of its lanes' channel windows so every channel step is one
//    coalesced 128-byte row update; each voxel has a single writer, so the
//    accumulation needs no atomics;
//  * thick disks: a block owns a 32-spaxel row segment, its warps walk the
//    spatial z axis and accumulate the spectral columns in shared memory
//    (shared atomics), then add each column to HBM once;
//  * mcdisk: one thread per cloud, Philox counter-based random numbers keyed by
//    (seed, cloud), red.global.add into the cube (mode 0) or an ordered
//    two-pass fixed-point accumulation (mode 1, deterministic).
#include "gbk_disk.cuh"

#include <climits>

namespace gbk {

// Thin disk: one thread per spaxel (spatial z = 1).  Block (32, 8): a warp is
// a run of 32 adjacent x at one y.
__global__ void __launch_bounds__(256) smdisk_thin_kernel(DiskArgs a, int* status)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const bool inside = x < a.sx && y < a.sy;
    int bad = 0;
    DiskConst kc = disk_const(a);
    SpaxelOut o;
    bool on = inside && smdisk_spaxel(a, kc, x, y, 0, o, bad);
    int zlo = INT_MAX, zhi = -1;
    float amp = 0, inv2c2 = 0;
    if (on) {
        if (a.image) a.image[x + (long long)a.sx * y] += o.orv;
        smdisk_side_outputs(a, x, y, 0, o);
        if (a.scube && line_window(o.vv, o.dv, a.spec_size, a.spec_step, a.spec_zero, zlo, zhi)) {
            amp = 1 / (o.dv * sqrtf(2 * GBK_PI));
            inv2c2 = 2 * o.dv * o.dv;
        } else {
            zlo = INT_MAX;
            zhi = -1;
        }
    }
    // channel loop over the union of the warp's windows: coalesced rows
    const unsigned full = 0xffffffffu;
    int wlo = __reduce_min_sync(full, zlo);
    int whi = __reduce_max_sync(full, zhi);
    if (a.scube) {
        const long long plane = (long long)a.sx * a.sy;
        float* col = a.scube + (x + (long long)a.sx * y);
        for (int z = wlo; z <= whi; ++z) {
            if (z >= zlo && z <= zhi) {
                float zv = a.spec_zero + z * a.spec_step;
                float d = zv - o.vv;
                col[plane * z] += o.orv * (amp * expf(-d * d / inv2c2));
            }
        }
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// Thick disk (or thin with spatial z > 1): block (32, 8) owns 32 adjacent
// spaxel columns of one row; each warp takes every 8th spatial z and adds its
// lines into a shared (spec_size x 32) column tile; the tile is then added to
// the cube.  With USE_SMEM = false (spectra too long for shared memory) the
// lines go straight to HBM with atomics.
template<bool USE_SMEM>
__global__ void __launch_bounds__(256) smdisk_thick_kernel(DiskArgs a, int* status)
{
    extern __shared__ float tile[];
    const int tx = threadIdx.x, tz = threadIdx.y;
    const int x = blockIdx.x * 32 + tx;
    const int y = blockIdx.y;
    const long long plane = (long long)a.sx * a.sy;
    int bad = 0;
    if (USE_SMEM && a.scube) {
        for (int i = tz * 32 + tx; i < a.spec_size * 32; i += 256) tile[i] = 0.f;
        __syncthreads();
    }
    DiskConst kc = disk_const(a);
    if (x < a.sx) {
        for (int z = tz; z < a.sz; z += 8) {
            SpaxelOut o;
            if (!smdisk_spaxel(a, kc, x, y, z, o, bad)) continue;
            if (a.image) atomicAdd(&a.image[x + (long long)a.sx * y], o.orv);
            smdisk_side_outputs(a, x, y, z, o);
            int zlo, zhi;
            if (a.scube && line_window(o.vv, o.dv, a.spec_size, a.spec_step, a.spec_zero, zlo, zhi)) {
                float amp = 1 / (o.dv * sqrtf(2 * GBK_PI));
                float inv2c2 = 2 * o.dv * o.dv;
                for (int zs = zlo; zs <= zhi; ++zs) {
                    float zv = a.spec_zero + zs * a.spec_step;
                    float d = zv - o.vv;
                    float f = o.orv * (amp * expf(-d * d / inv2c2));
                    if (USE_SMEM) atomicAdd(&tile[zs * 32 + tx], f);
                    else atomicAdd(&a.scube[x + (long long)a.sx * y + plane * zs], f);
                }
            }
        }
    }
    if (USE_SMEM && a.scube) {
        __syncthreads();
        if (x < a.sx) {
            float* col = a.scube + (x + (long long)a.sx * y);
            for (int zs = tz; zs < a.spec_size; zs += 8) {
                float v = tile[zs * 32 + tx];
                if (v != 0.f) col[plane * zs] += v;
            }
        }
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// ---- mcdisk ------------------------------------------------------------------

// The cloud's line at distance d from its centre without the amplitude:
// exp(-d^2 / (2 sigma^2)) as 2^(-d^2 rinv) with rinv = log2(e) / (2 sigma^2),
// by the PTX ex2.approx instruction (relative error ~2^-22; inside the +-5
// sigma window the argument is >= -18.1, far from the flush to zero)
__device__ __forceinline__ float line_e2(float d, float rinv)
{
    float e;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-(d * d) * rinv));
    return e;
}

// Philox-4x32-10 (Salmon et al., SC'11), counter {ci, k/4, 0, 0}, key = seed
struct Philox {
    unsigned ci, k0, k1, k, w0, w1, w2, w3;   // the current block in registers
    __device__ void block(unsigned j)
    {
        unsigned c0 = ci, c1 = j, c2 = 0, c3 = 0, a = k0, b = k1;
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            unsigned hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
            unsigned hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
            unsigned n0 = hi1 ^ c1 ^ a, n2 = hi0 ^ c3 ^ b;
            c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
            a += 0x9E3779B9u;
            b += 0xBB67AE85u;
        }
        w0 = c0; w1 = c1; w2 = c2; w3 = c3;
    }
    __device__ float next()
    {
        const unsigned j = k & 3u;
        if (j == 0) block(k >> 2);
        const unsigned v = j == 0 ? w0 : j == 1 ? w1 : j == 2 ? w2 : w3;
        ++k;
        // ((v >> 8) + 0.5) / 2^24 rounded to float: the odd integer
        // 2 (v >> 8) + 1 < 2^25 rounded to float, times 2^-25 (exact), is the
        // same single rounding
        return __uint2float_rn(((v >> 8) << 1) | 1u) * 0x1p-25f;
    }
};

// traits.hpp:310-326
__device__ __forceinline__ void sample_polar(float& r, float& t, Philox& rng, float rmin, float rmax)
{
    float u1 = rng.next();
    r = sqrtf(rmax * rmax + (rmin * rmin - rmax * rmax) * u1);
    float u2 = rng.next();
    t = 2 * GBK_PI * u2;
}

// math.hpp:207-217 (rejection sampling of ggauss; the moffat pdf is a stub 0
// in the reference, so its loop always accepts the first x)
__device__ __forceinline__ float rejection(int kind, Philox& rng, float trunc, float c, float d)
{
    // bounded: after 4096 rejections the last proposal is kept (the reference
    // loops without a limit; its acceptance rate here is >= 1/10)
    float x = 0;
    for (int it = 0; it < 4096; ++it) {
        x = (0 - trunc) + rng.next() * ((0 + trunc) - (0 - trunc));
        float u = rng.next();
        float y = (kind == 4 ? ggauss_pdf(0, 0, c, d) : 0.f) * u;
        float z = kind == 4 ? ggauss_pdf(x, 0, c, d) : 0.f;
        if (!(y > z)) break;
    }
    return x;
}

// math.hpp:152-498 samplers as selected by traits.hpp:596-631, 1516-1590
__device__ __forceinline__ float rh_trait_rnd(Philox& rng, int uid, const float* c, const float* p,
                                              const Ring& g, int& bad)
{
    int off = uid >= 1000 ? 1 : 0;
    int kind = uid - 1000 * off;
    if (kind < 1 || kind > 7) { bad = 1; return NAN; }
    bool use_rn = c[1] != 0;
    float p1 = use_rn ? nw(g, p, off * g.nrnodes) : p[off];
    float p2 = 0;
    if (kind == 4 || kind == 6) p2 = use_rn ? nw(g, p, (off + 1) * g.nrnodes) : p[off + 1];
    float u;
    switch (kind) {
    case 1: return (0 - p1) + rng.next() * ((0 + p1) - (0 - p1));
    case 2: u = rng.next() * 2 - 1.f; return 0 - p1 * sgn(u) * logf(1 - 2 * fabsf(u));
    case 3: { float u1 = rng.next(); float u2 = rng.next();
              return 0 + p1 * sqrtf(-2 * logf(u1)) * cosf(2 * GBK_PI * u2); }
    case 4: return rejection(4, rng, 5 * p1, p1, p2);
    case 5: u = rng.next() * 2 - 1.f; return 0 + p1 * tanf(GBK_PI * 0.5f * u);
    case 6: return rejection(6, rng, 5 * p1, p1, p2);
    default: u = rng.next() * 2 - 1.f; return 0 + p1 * atanhf(u);
    }
}

// The projection values that are the same for every cloud of a call: centre
// and systemic velocity of a disk that is not loose, angles of a disk that is
// not tilted (evaluated once per thread, with the expressions of the
// per-cloud path)
struct McConst {
    float vsys, xpos, ypos;
    float s_i, c_i, s_p, c_p;      // sincos(-incl), sincos(-posa)
    float sin_incl, cos_incl;
    float ix, iy, iz, ispec;       // 1 / the grid steps
};

// 1 / (sigma sqrt(2 pi)) and log2(e) / (2 sigma^2) of a cloud's line from
// one reciprocal of sigma
__device__ __forceinline__ void mc_line_consts(float dv, float& amp, float& rinv)
{
    const float r = 1.f / dv;
    amp = r * 0.3989422804014327f;
    rinv = 0.7213475204444817f * r * r;
}

// line_window with the reciprocal of the channel width
__device__ __forceinline__ bool mc_line_window(float v, float d, int nz, float istep, float zero,
                                               int& zlo, int& zhi)
{
    if (!isfinite(v) || !isfinite(d)) return false;
    const float zmin = v - d * GBK_LINE_WIDTH, zmax = v + d * GBK_LINE_WIDTH;
    float a = rintf((zmin - zero) * istep), b = rintf((zmax - zero) * istep);
    a = a < 0.f ? 0.f : a;
    b = (float)(nz - 1) < b ? (float)(nz - 1) : b;
    zlo = (int)a;
    zhi = (int)b;
    return zlo <= zhi;
}

__device__ __forceinline__ McConst mc_const(const DiskArgs& a)
{
    McConst k{};
    k.ix = 1.f / a.stx;
    k.iy = 1.f / a.sty;
    k.iz = 1.f / a.stz;
    k.ispec = 1.f / a.spec_step;
    if (!a.loose) {
        k.vsys = a.vsys ? a.vsys[0] : 0.f;
        k.xpos = a.xpos[0];
        k.ypos = a.ypos[0];
    }
    if (!a.tilted) {
        const float posai = a.posa[0] * GBK_D2R, incli = a.incl[0] * GBK_D2R;
        sincosf(-incli, &k.s_i, &k.c_i);
        sincosf(-posai, &k.s_p, &k.c_p);
        k.sin_incl = sinf(incli);
        k.cos_incl = cosf(incli);
    }
    return k;
}

// gmodels.hpp:325-608 up to the splat: sample one cloud and return its
// voxel and line.  false if the cloud is discarded.
__device__ __forceinline__ bool mcdisk_cloud(const DiskArgs& a, const McArgs& m,
                                             const McConst& mk, int ci, int& xo, int& yo,
                                             int& zo, SpaxelOut& o, int& bad)
{
    Philox rng;
    rng.ci = (unsigned)ci;
    rng.k0 = (unsigned)m.seed;
    rng.k1 = (unsigned)(m.seed >> 32);
    rng.k = 0;
    const float* rnodes = a.rnodes;
    const int nrn = a.nrnodes;
    // cumulative cloud counts -> trait and ring (gmodels.hpp:400-416)
    int lo = 0, hi = m.csum_len - 1;
    while (lo < hi) {   // first index with ci < csum[index]
        int mid = (lo + hi) >> 1;
        if (ci < m.csum[mid]) hi = mid;
        else lo = mid + 1;
    }
    int rnidx = lo, tidx = 0;
    const float *rpc = a.rpt.cv, *rpp = a.rpt.pv, *rhc = a.rht.cv, *rhp = a.rht.pv;
    for (tidx = 0; tidx < a.rpt.n; ++tidx) {
        int size = m.hasordint[tidx] ? 1 : nrn - 2;
        if (rnidx < size) break;
        rnidx -= size;
        rpc += a.rpt.cc[tidx];
        rpp += a.rpt.pc[tidx];
        rhc += a.rht.cc[tidx];
        rhp += a.rht.pc[tidx];
    }
    if (tidx >= a.rpt.n) return false;   // cloud index beyond the budget
    float rv = m.cflux / a.stz;
    float sign = 1, rd = 0, theta = 0;
    // traits.hpp:1333-1435
    {
        int uid = a.rpt.uids[tidx];
        int kind = uid >= 1000 ? uid - 1000 : uid;
        int rn = rnidx + 1;
        if (kind == 1) {
            sample_polar(rd, theta, rng, rnodes[0], rnodes[nrn - 1]);
        } else if ((kind >= 2 && kind <= 7) || kind == 101 || kind == 102) {
            float hw = rnodes[1] - rnodes[0];
            sample_polar(rd, theta, rng, rnodes[rn] - hw, rnodes[rn] + hw);
            if (kind == 102) {
                int k = (int)rintf(rpc[0]);
                float amp = rpp[rn];
                float ph = rpp[nrn + rn] * GBK_D2R;
                float vr = amp * (rng.next() * 2 - 1.f);
                float vf = amp * cosf(k * (theta - ph));
                sign = vr > vf ? 1.f : -1.f;
            }
        } else if (kind >= 51 && kind <= 54) {
            // not implemented in the reference: position stays at the origin
        } else if (kind == 103) {
        } else {
            bad = 1;
            return false;
        }
    }
    if (sign < 0) rv = -rv;
    rv *= a.stz;
    rv /= a.stx * a.sty;
    float xd = rd * cosf(theta), yd = rd * sinf(theta);
    Ring g;
    g.rnodes = rnodes;
    g.nrnodes = nrn;
    g.r = rd;
    g.theta = theta;
    if (!disk_info(g.rnidx, rd, nrn, rnodes)) return false;
    TraitVals pt = {0, 0, 0, 0}, ht = {0, 0, 0, 0};
    if (a.spt.uids) {
        eval_set_r<K_SP>(pt, a.spt, g, 0, 0, 0, bad);
        const float sv = tv_sum(pt, a.spt.n);
        if (!sv) return false;
    }
    float zd = rh_trait_rnd(rng, a.rht.uids[tidx], rhc, rhp, g, bad);
    if (a.zpt.uids) {
        eval_set_r<K_ZP>(pt, a.zpt, g, 0, 0, 0, bad);
        const float zv = tv_sum(pt, a.zpt.n);
        zd += zv;
    }
    float vsysi = mk.vsys, xposi = mk.xpos, yposi = mk.ypos;
    if (a.loose) {
        vsysi = a.vsys ? lerp(rd, g.rnidx, rnodes, a.vsys, 0) : 0.f;
        xposi = lerp(rd, g.rnidx, rnodes, a.xpos, 0);
        yposi = lerp(rd, g.rnidx, rnodes, a.ypos, 0);
    }
    float s_i = mk.s_i, c_i = mk.c_i, s_p = mk.s_p, c_p = mk.c_p;
    float sin_incl = mk.sin_incl, cos_incl = mk.cos_incl;
    if (a.tilted) {
        const float posai = lerp(rd, g.rnidx, rnodes, a.posa, 0) * GBK_D2R;
        const float incli = lerp(rd, g.rnidx, rnodes, a.incl, 0) * GBK_D2R;
        sincosf(-incli, &s_i, &c_i);
        sincosf(-posai, &s_p, &c_p);
        sin_incl = sinf(incli);
        cos_incl = cosf(incli);
    }
    // disk -> world (gmodels.hpp:159-165 with negated parameters, :495-496)
    float xn = xd, yn = yd, zn = zd;
    rot_lh_x(yn, zn, s_i, c_i);
    rot_lh_z(xn, yn, s_p, c_p);
    xn -= -xposi;
    yn -= -yposi;
    float fx = rintf((xn - a.zx) * mk.ix), fy = rintf((yn - a.zy) * mk.iy);
    float fz = rintf((zn - a.zz) * mk.iz);
    if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) return false;
    if (fx < 0 || fx >= a.sx || fy < 0 || fy >= a.sy || fz < 0 || fz >= a.sz) return false;
    int x = (int)fx, y = (int)fy, z = (int)fz;
    float vv = 0, dv = 0, wv = 1;
    if (a.vpt.uids) eval_set_r<K_VP>(pt, a.vpt, g, sin_incl, cos_incl, 0, bad);
    if (a.vht.uids) eval_set_r<K_VH>(ht, a.vht, g, 0, 0, fabsf(zd), bad);
    vv += tv_dot(pt, &ht, a.vpt.n);
    vv += vsysi;
    if (a.dpt.uids) eval_set_r<K_DP>(pt, a.dpt, g, 0, 0, 0, bad);
    if (a.dht.uids) eval_set_r<K_DH>(ht, a.dht, g, 0, 0, fabsf(zd), bad);
    dv += tv_dot(pt, &ht, a.dpt.n);
    dv = fabsf(dv);
    if (a.wpt.uids && a.wdata) {
        eval_set_r<K_WP>(pt, a.wpt, g, 0, 0, 0, bad);
        wv *= tv_prod(pt, a.wpt.n);
    }
    float orv = rv;
    if (a.opacity) {
        long long sxy = (long long)a.sx * a.sy;
        for (int oz = z + 1; oz < a.sz; ++oz)
            orv -= orv * a.opacity[x + (long long)a.sx * y + sxy * oz];
    }
    xo = x;
    yo = y;
    zo = z;
    o.rv = rv;
    o.vv = vv;
    o.dv = dv;
    o.wv = wv;
    o.orv = orv;
    return true;
}

// Fast mode: one thread per cloud; every contribution is a red.global.add.
__global__ void __launch_bounds__(256) mcdisk_kernel(DiskArgs a, McArgs m, int* status)
{
    int bad = 0;
    const McConst mk = mc_const(a);
    for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < m.nclouds;
         ci += gridDim.x * blockDim.x) {
        int x, y, z;
        SpaxelOut o;
        if (!mcdisk_cloud(a, m, mk, ci, x, y, z, o, bad)) continue;
        if (a.image) atomicAdd(&a.image[x + (long long)a.sx * y], o.orv);
        int zlo, zhi;
        if (a.scube &&
            mc_line_window(o.vv, o.dv, a.spec_size, mk.ispec, a.spec_zero, zlo, zhi)) {
            float amp, rinv;
            mc_line_consts(o.dv, amp, rinv);
            float* col = a.scube + (x + (long long)a.sx * y);
            long long plane = (long long)a.sx * a.sy;
            for (int zs = zlo; zs <= zhi; ++zs) {
                float zv = a.spec_zero + zs * a.spec_step;
                float d = zv - o.vv;
                atomicAdd(&col[plane * zs], o.orv * (amp * line_e2(d, rinv)));
            }
        }
        long long idx = idx3(x, y, z, a.sx, a.sy);
        // last-writer-wins assignments, racy as in the reference
        if (a.wdata) a.wdata[idx] = o.wv;
        if (a.wdata_cmp) a.wdata_cmp[idx] = o.wv;
        if (a.rdata) atomicAdd(&a.rdata[idx], o.rv);
        if (a.rdata_cmp) atomicAdd(&a.rdata_cmp[idx], o.rv);
        if (a.ordata) atomicAdd(&a.ordata[idx], o.orv);
        if (a.ordata_cmp) atomicAdd(&a.ordata_cmp[idx], o.orv);
        if (a.vdata_cmp) a.vdata_cmp[idx] = o.vv;
        if (a.ddata_cmp) a.ddata_cmp[idx] = o.dv;
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// ---- mcdisk mode 2: channel-contiguous lines, 16-byte vector atomics ---------
// The cube lines go to a scratch cube laid out spaxel-major with the channels
// contiguous (a column of nzp = spec_size rounded up to 4 floats per spaxel),
// four channels per red.global.add.v4.f32 (about spectral window / 4 + 1
// atomics per cloud instead of one per channel); a tiled transpose then adds
// the scratch cube to scube in the reference's (channel, y, x) layout.  The
// other outputs are accumulated as in mode 0.
__global__ void __launch_bounds__(256) mcdisk_v4_kernel(DiskArgs a, McArgs m, float* lines,
                                                        int nzp, int copies, int* status)
{
    // block b adds into copy b % copies of the scratch cube (copies of nsp x
    // nzp floats): reductions to the same element from many blocks spread
    // over the copies' L2 lines
    if (lines) lines += (long long)(blockIdx.x % copies) * a.sx * a.sy * nzp;
    int bad = 0;
    const McConst mk = mc_const(a);
    for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < m.nclouds;
         ci += gridDim.x * blockDim.x) {
        int x, y, z;
        SpaxelOut o;
        if (!mcdisk_cloud(a, m, mk, ci, x, y, z, o, bad)) continue;
        if (a.image) atomicAdd(&a.image[x + (long long)a.sx * y], o.orv);
        int zlo, zhi;
        if (lines && mc_line_window(o.vv, o.dv, a.spec_size, mk.ispec, a.spec_zero, zlo, zhi)) {
            float amp, rinv;
            mc_line_consts(o.dv, amp, rinv);
            float* col = lines + (x + (long long)a.sx * y) * nzp;
            for (int z4 = zlo & ~3; z4 <= zhi; z4 += 4) {
                float v[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int zs = z4 + j;
                    const float d = (a.spec_zero + zs * a.spec_step) - o.vv;
                    v[j] = (zs >= zlo && zs <= zhi) ? o.orv * (amp * line_e2(d, rinv)) : 0.f;
                }
                atomicAdd(reinterpret_cast<float4*>(col + z4), make_float4(v[0], v[1], v[2], v[3]));
            }
        }
        long long idx = idx3(x, y, z, a.sx, a.sy);
        if (a.wdata) a.wdata[idx] = o.wv;
        if (a.wdata_cmp) a.wdata_cmp[idx] = o.wv;
        if (a.rdata) atomicAdd(&a.rdata[idx], o.rv);
        if (a.rdata_cmp) atomicAdd(&a.rdata_cmp[idx], o.rv);
        if (a.ordata) atomicAdd(&a.ordata[idx], o.orv);
        if (a.ordata_cmp) atomicAdd(&a.ordata_cmp[idx], o.orv);
        if (a.vdata_cmp) a.vdata_cmp[idx] = o.vv;
        if (a.ddata_cmp) a.ddata_cmp[idx] = o.dv;
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// scube[z][s] += sum over the copies c of lines[c][s][z] (in copy order) for
// spaxels s < nsp, channels z < nz (32 x 32 tiles)
__global__ void __launch_bounds__(256) mc_lines_add_kernel(const float* __restrict__ lines,
                                                           float* __restrict__ scube,
                                                           long long nsp, int nzp, int nz,
                                                           int copies)
{
    __shared__ float tile[32][33];
    const long long s0 = (long long)blockIdx.x * 32;
    const int z0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const long long cstride = nsp * nzp;
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const long long s = s0 + ty + k;
        const int z = z0 + tx;
        float v = 0.f;
        if (s < nsp && z < nz)
            for (int c = 0; c < copies; ++c) v += lines[c * cstride + s * nzp + z];
        tile[ty + k][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int z = z0 + ty + k;
        const long long s = s0 + tx;
        if (s < nsp && z < nz) scube[(long long)z * nsp + s] += tile[tx][ty + k];
    }
}

// Copies of the channel-contiguous line scratch for a call: 1 up to 256
// clouds per spaxel, doubling per doubling of the density up to 8, and no
// more than fit in 64 MB (reductions to one element from many blocks queue
// in its L2 slice; small cubes with many clouds are where that happens)
static int mc_line_copies(long long nclouds, long long nsp, int nzp)
{
    const long long per = nclouds / (nsp > 0 ? nsp : 1);
    int c = per < 256 ? 1 : per < 512 ? 2 : per < 1024 ? 4 : 8;
    const long long one = nsp * nzp * (long long)sizeof(float);
    while (c > 1 && c * one > (64LL << 20)) c >>= 1;
    return c;
}

extern "C" size_t gbkb200_mcdisk_scratch_bytes(int nclouds, int spat_size_x, int spat_size_y,
                                               int spec_size)
{
    const long long nsp = (long long)spat_size_x * spat_size_y;
    const int nzp = (spec_size + 3) & ~3;
    return (size_t)mc_line_copies(nclouds, nsp, nzp) * nsp * nzp * sizeof(float);
}

// ---- deterministic mcdisk: 64-bit fixed-point accumulation ------------------
// Integer addition is associative, so the sums do not depend on the order in
// which clouds land.  A bound pass finds the largest contribution M of the
// call (the line peak |orv| / (sigma sqrt(2 pi)) for the cube, |orv| and |rv|
// for the maps); contributions are scaled by 2^k with nclouds * M * 2^k <
// 2^62 (no overflow whatever the cloud positions), rounded to integers and
// added with 64-bit atomics; the sums are then added to the float outputs.

__device__ __forceinline__ void atomic_max_abs(unsigned* m, float v)
{
    // non-negative floats order as their bit patterns
    v = fabsf(v);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(m, __float_as_uint(v));
}

// exponent k of the fixed-point scale 2^k for the bound M (bit pattern)
__device__ __forceinline__ int fixed_shift(unsigned mbits, int nclouds)
{
    const float M = __uint_as_float(mbits);
    int e = 0;
    frexpf(M > 0.f ? M : 1.f, &e);            // M < 2^e
    const int cb = 32 - __clz(nclouds);       // nclouds < 2^cb
    return 62 - cb - e;
}

__device__ __forceinline__ void fixed_add(long long* acc, float v, int k)
{
    const long long q = llrint((double)v * ldexp(1.0, k));
    atomicAdd(reinterpret_cast<unsigned long long*>(acc), (unsigned long long)q);
}

// bound[0]: cube contributions, bound[1]: map contributions
__global__ void __launch_bounds__(256) mcdisk_bound_kernel(DiskArgs a, McArgs m, unsigned* bound)
{
    int bad = 0;
    const McConst mk = mc_const(a);
    for (int base = blockIdx.x * blockDim.x; base < m.nclouds; base += gridDim.x * blockDim.x) {
        const int ci = base + threadIdx.x;
        float vc = 0.f, vm = 0.f;
        int x, y, z;
        SpaxelOut o;
        if (ci < m.nclouds && mcdisk_cloud(a, m, mk, ci, x, y, z, o, bad)) {
            int zlo, zhi;
            float amp, rinv;
            mc_line_consts(o.dv, amp, rinv);
            if (a.scube &&
                mc_line_window(o.vv, o.dv, a.spec_size, mk.ispec, a.spec_zero, zlo, zhi))
                vc = o.orv * amp;
            vm = fmaxf(fabsf(o.orv), fabsf(o.rv));
        }
        atomic_max_abs(&bound[0], vc);
        atomic_max_abs(&bound[1], vm);
    }
}

struct McFixed {
    long long *scube, *image, *rdata, *rdata_cmp, *ordata, *ordata_cmp;
    const unsigned* bound;
};

__global__ void __launch_bounds__(256) mcdisk_fixed_kernel(DiskArgs a, McArgs m, McFixed f,
                                                           int* status)
{
    int bad = 0;
    const McConst mk = mc_const(a);
    const int kc = fixed_shift(f.bound[0], m.nclouds), km = fixed_shift(f.bound[1], m.nclouds);
    for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < m.nclouds;
         ci += gridDim.x * blockDim.x) {
        int x, y, z;
        SpaxelOut o;
        if (!mcdisk_cloud(a, m, mk, ci, x, y, z, o, bad)) continue;
        const long long sp = x + (long long)a.sx * y;
        if (f.image) fixed_add(&f.image[sp], o.orv, km);
        int zlo, zhi;
        if (f.scube && mc_line_window(o.vv, o.dv, a.spec_size, mk.ispec, a.spec_zero, zlo, zhi)) {
            float amp, rinv;
            mc_line_consts(o.dv, amp, rinv);
            const long long plane = (long long)a.sx * a.sy;
            for (int zs = zlo; zs <= zhi; ++zs) {
                const float zv = a.spec_zero + zs * a.spec_step;
                const float d = zv - o.vv;
                fixed_add(&f.scube[sp + plane * zs], o.orv * (amp * line_e2(d, rinv)), kc);
            }
        }
        const long long idx = idx3(x, y, z, a.sx, a.sy);
        // last-writer-wins assignments, racy as in the reference
        if (a.wdata) a.wdata[idx] = o.wv;
        if (a.wdata_cmp) a.wdata_cmp[idx] = o.wv;
        if (f.rdata) fixed_add(&f.rdata[idx], o.rv, km);
        if (f.rdata_cmp) fixed_add(&f.rdata_cmp[idx], o.rv, km);
        if (f.ordata) fixed_add(&f.ordata[idx], o.orv, km);
        if (f.ordata_cmp) fixed_add(&f.ordata_cmp[idx], o.orv, km);
        if (a.vdata_cmp) a.vdata_cmp[idx] = o.vv;
        if (a.ddata_cmp) a.ddata_cmp[idx] = o.dv;
    }
    if (bad) atomicOr(status, GBK_STATUS_BAD_TRAIT);
}

// out[i] += acc[i] / 2^k
__global__ void fixed_to_float_kernel(const long long* acc, float* out, long long n,
                                      const unsigned* bound, int which, int nclouds)
{
    const int k = fixed_shift(bound[which], nclouds);
    const double inv = ldexp(1.0, -k);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (acc[i]) out[i] += (float)((double)acc[i] * inv);
}

// ---- wcube (gmodels.hpp:52-82) -----------------------------------------------
__global__ void wcube_kernel(int sx, int sy, int sz, int spec_z, const float* spat, float* spec)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= sx) return;
    float sum = 0, mx = 0;
    for (int z = 0; z < sz; ++z) {
        float v = spat[idx3(x, y, z, sx, sy)];
        sum += v;
        mx = mx < v ? v : mx;
    }
    float mean = sum / sz;
    float w = mx > 0 ? mean / mx : 0.f;
    for (int z = 0; z < spec_z; ++z) spec[idx3(x, y, z, sx, sy)] = w;
}

}  // namespace gbk

using namespace gbk;

static void fill_set(TraitSet& s, int n, const int* u, const float* cv, const int* cc,
                     const float* pv, const int* pc)
{
    s.n = n; s.uids = u; s.cv = cv; s.cc = cc; s.pv = pv; s.pc = pc;
}

#define GBK_FILL_DISK(a)                                                                   \
    a.loose = loose; a.tilted = tilted; a.nrnodes = nrnodes; a.rnodes = rnodes;          \
    a.vsys = vsys; a.xpos = xpos; a.ypos = ypos; a.posa = posa; a.incl = incl;            \
    fill_set(a.rpt, nrt, rpt_uids, rpt_cvalues, rpt_ccounts, rpt_pvalues, rpt_pcounts);    \
    fill_set(a.rht, nrt, rht_uids, rht_cvalues, rht_ccounts, rht_pvalues, rht_pcounts);    \
    fill_set(a.vpt, nvt, vpt_uids, vpt_cvalues, vpt_ccounts, vpt_pvalues, vpt_pcounts);    \
    fill_set(a.vht, nvt, vht_uids, vht_cvalues, vht_ccounts, vht_pvalues, vht_pcounts);    \
    fill_set(a.dpt, ndt, dpt_uids, dpt_cvalues, dpt_ccounts, dpt_pvalues, dpt_pcounts);    \
    fill_set(a.dht, ndt, dht_uids, dht_cvalues, dht_ccounts, dht_pvalues, dht_pcounts);    \
    fill_set(a.zpt, nzt, zpt_uids, zpt_cvalues, zpt_ccounts, zpt_pvalues, zpt_pcounts);    \
    fill_set(a.spt, nst, spt_uids, spt_cvalues, spt_ccounts, spt_pvalues, spt_pcounts);    \
    fill_set(a.wpt, nwt, wpt_uids, wpt_cvalues, wpt_ccounts, wpt_pvalues, wpt_pcounts);    \
    a.opacity = opacity; a.sx = spat_size_x; a.sy = spat_size_y; a.sz = spat_size_z;      \
    a.stx = spat_step_x; a.sty = spat_step_y; a.stz = spat_step_z;                        \
    a.zx = spat_zero_x; a.zy = spat_zero_y; a.zz = spat_zero_z;                           \
    a.spec_size = spec_size; a.spec_step = spec_step; a.spec_zero = spec_zero;            \
    a.image = image; a.scube = scube; a.wdata = wdata; a.wdata_cmp = wdata_cmp;           \
    a.rdata = rdata; a.rdata_cmp = rdata_cmp; a.ordata = ordata;                          \
    a.ordata_cmp = ordata_cmp; a.vdata_cmp = vdata_cmp; a.ddata_cmp = ddata_cmp

static int check_disk(const DiskArgs& a)
{
    if (a.nrnodes < 2 || !a.rnodes || !a.xpos || !a.ypos || !a.posa || !a.incl)
        return GBKB200_ERR_INVALID_ARG;
    if (a.sx <= 0 || a.sy <= 0 || a.sz <= 0) return GBKB200_ERR_INVALID_ARG;
    if (a.scube && a.spec_size <= 0) return GBKB200_ERR_INVALID_ARG;
    const TraitSet* sets[] = {&a.rpt, &a.vpt, &a.dpt, &a.zpt, &a.spt, &a.wpt};
    for (const TraitSet* s : sets)
        if (s->n < 0 || s->n > GBK_TRAIT_NUM_MAX) return GBKB200_ERR_INVALID_ARG;
    return GBKB200_OK;
}

// Shared launch helper of the smdisk entry point (also used by the batched
// driver for its per-set fallback).
int gbk_launch_smdisk(const DiskArgs& a, cudaStream_t stream, int* status)
{
    const bool thin = a.rht.uids == nullptr;
    if (thin && a.sz == 1) {
        dim3 block(32, 8), grid((a.sx + 31) / 32, (a.sy + 7) / 8);
        smdisk_thin_kernel<<<grid, block, 0, stream>>>(a, status);
    } else {
        dim3 block(32, 8), grid((a.sx + 31) / 32, a.sy);
        size_t smem = a.scube ? (size_t)a.spec_size * 32 * sizeof(float) : 0;
        if (smem <= 200 * 1024) {
            const int rc = gbk_raise_smem_limit(
                reinterpret_cast<const void*>(smdisk_thick_kernel<true>), smem);
            if (rc) return rc;
            smdisk_thick_kernel<true><<<grid, block, smem, stream>>>(a, status);
        } else {
            smdisk_thick_kernel<false><<<grid, block, 0, stream>>>(a, status);
        }
    }
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}

extern "C" int gbkb200_gmodel_smdisk_evaluate_f32(gbkb200_ctx* ctx, GBKB200_DISK_ARGS)
{
    if (!ctx) return GBKB200_ERR_INVALID_ARG;
    DiskArgs a;
    GBK_FILL_DISK(a);
    int rc = check_disk(a);
    if (rc) return rc;
    rc = gbk_launch_smdisk(a, ctx->stream, ctx->d_status);
    if (rc) return rc;
    return gbk_finish(ctx);
}

extern "C" int gbkb200_gmodel_mcdisk_evaluate_f32(gbkb200_ctx* ctx, float cflux, int nclouds,
                                                  const int* ncloudscsum, int ncloudscsum_len,
                                                  const unsigned char* hasordint,
                                                  GBKB200_DISK_ARGS)
{
    if (!ctx) return GBKB200_ERR_INVALID_ARG;
    DiskArgs a;
    GBK_FILL_DISK(a);
    int rc = check_disk(a);
    if (rc) return rc;
    if (nclouds < 0 || (nclouds > 0 && (!ncloudscsum || ncloudscsum_len <= 0 || !hasordint)))
        return GBKB200_ERR_INVALID_ARG;
    if (!a.rpt.uids || !a.rht.uids) return GBKB200_ERR_INVALID_ARG;
    if (nclouds == 0) return gbk_finish(ctx);
    McArgs m;
    m.cflux = cflux;
    m.nclouds = nclouds;
    m.csum = ncloudscsum;
    m.csum_len = ncloudscsum_len;
    m.hasordint = hasordint;
    m.seed = ctx->seed;
    int blocks = (nclouds + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    // modes 0 and 2: the lines channel-contiguous in the context's scratch with
    // vector atomics when the spectral cube is requested (mode 0 falls back to
    // one atomic per channel if the scratch cannot be had); mode 3 and the
    // other outputs: one fp32 atomic per channel and element
    bool vec = (ctx->mc_mode == 0 || ctx->mc_mode == 2) && a.scube;
    const int copies = mc_line_copies(nclouds, (long long)a.sx * a.sy, (a.spec_size + 3) & ~3);
    if (vec) {
        const long long nsp = (long long)a.sx * a.sy;
        const int nzp = (a.spec_size + 3) & ~3;
        const size_t need = (size_t)copies * nsp * nzp * sizeof(float);
        if (ctx->mc_scratch_bytes < need) {
            if (ctx->mc_scratch) cudaFree(ctx->mc_scratch);
            ctx->mc_scratch = nullptr;
            ctx->mc_scratch_bytes = 0;
            if (cudaMalloc(&ctx->mc_scratch, need) == cudaSuccess) {
                ctx->mc_scratch_bytes = need;
            } else {
                (void)cudaGetLastError();      // the failed allocation is not sticky
                if (ctx->mc_mode == 2) return GBKB200_ERR_OOM;
                vec = false;
            }
        }
    }
    if (ctx->mc_mode == 3 || ((ctx->mc_mode == 0 || ctx->mc_mode == 2) && !vec)) {
        mcdisk_kernel<<<blocks, 256, 0, ctx->stream>>>(a, m, ctx->d_status);
        GBK_CUDA_TRY(cudaGetLastError());
        return gbk_finish(ctx);
    }
    if (vec) {
        const long long nsp = (long long)a.sx * a.sy;
        const int nzp = (a.spec_size + 3) & ~3;
        const size_t need = (size_t)copies * nsp * nzp * sizeof(float);
        float* lines = static_cast<float*>(ctx->mc_scratch);
        GBK_CUDA_TRY(cudaMemsetAsync(lines, 0, need, ctx->stream));
        mcdisk_v4_kernel<<<blocks, 256, 0, ctx->stream>>>(a, m, lines, nzp, copies,
                                                          ctx->d_status);
        const dim3 tg((unsigned)((nsp + 31) / 32), (unsigned)((a.spec_size + 31) / 32));
        mc_lines_add_kernel<<<tg, 256, 0, ctx->stream>>>(lines, a.scube, nsp, nzp, a.spec_size,
                                                         copies);
        GBK_CUDA_TRY(cudaGetLastError());
        return gbk_finish(ctx);
    }
    // deterministic: fixed-point accumulators in the context's scratch
    const long long nsp = (long long)a.sx * a.sy, nsv = nsp * a.sz;
    const long long ncube = a.scube ? nsp * a.spec_size : 0;
    float* outs[6] = {a.scube, a.image, a.rdata, a.rdata_cmp, a.ordata, a.ordata_cmp};
    const long long lens[6] = {ncube, a.image ? nsp : 0, a.rdata ? nsv : 0,
                               a.rdata_cmp ? nsv : 0, a.ordata ? nsv : 0, a.ordata_cmp ? nsv : 0};
    long long total = 2;    // the two bounds, as one 8-byte slot
    for (long long l : lens) total += l;
    const size_t need = (size_t)total * sizeof(long long);
    if (ctx->mc_scratch_bytes < need) {
        if (ctx->mc_scratch) cudaFree(ctx->mc_scratch);
        ctx->mc_scratch = nullptr;
        ctx->mc_scratch_bytes = 0;
        if (cudaMalloc(&ctx->mc_scratch, need) != cudaSuccess) return GBKB200_ERR_OOM;
        ctx->mc_scratch_bytes = need;
    }
    GBK_CUDA_TRY(cudaMemsetAsync(ctx->mc_scratch, 0, need, ctx->stream));
    unsigned* bound = static_cast<unsigned*>(ctx->mc_scratch);
    long long* acc = static_cast<long long*>(ctx->mc_scratch) + 2;
    long long* ptrs[6];
    long long off = 0;
    for (int i = 0; i < 6; ++i) {
        ptrs[i] = lens[i] ? acc + off : nullptr;
        off += lens[i];
    }
    McFixed f;
    f.scube = ptrs[0]; f.image = ptrs[1]; f.rdata = ptrs[2]; f.rdata_cmp = ptrs[3];
    f.ordata = ptrs[4]; f.ordata_cmp = ptrs[5];
    f.bound = bound;
    mcdisk_bound_kernel<<<blocks, 256, 0, ctx->stream>>>(a, m, bound);
    mcdisk_fixed_kernel<<<blocks, 256, 0, ctx->stream>>>(a, m, f, ctx->d_status);
    for (int i = 0; i < 6; ++i) {
        if (!lens[i]) continue;
        long long g = (lens[i] + 255) / 256;
        if (g > 148 * 8) g = 148 * 8;
        fixed_to_float_kernel<<<(int)g, 256, 0, ctx->stream>>>(ptrs[i], outs[i], lens[i], bound,
                                                             i == 0 ? 0 : 1, nclouds);
    }
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}

extern "C" int gbkb200_gmodel_wcube_evaluate_f32(gbkb200_ctx* ctx, int spat_size_x,
                                                 int spat_size_y, int spat_size_z,
                                                 int spec_size_z, const float* spat_data,
                                                 float* spec_data)
{
    if (!ctx || !spat_data || !spec_data || spat_size_x <= 0 || spat_size_y <= 0 ||
        spat_size_z <= 0 || spec_size_z < 0)
        return GBKB200_ERR_INVALID_ARG;
    dim3 grid((spat_size_x + 127) / 128, spat_size_y);
    wcube_kernel<<<grid, 128, 0, ctx->stream>>>(spat_size_x, spat_size_y, spat_size_z,
                                                spec_size_z, spat_data, spec_data);
    GBK_CUDA_TRY(cudaGetLastError());
    return gbk_finish(ctx);
}
