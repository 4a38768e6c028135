// Device-side trait catalogue and disk geometry of the GBKFIT model.
//
// Restates, in float, the arithmetic of the reference's shared templates
// (paths relative to src/gbkfit/driver/native/gbkfit/include/gbkfit/):
// gmodel/traits.hpp (traits), math/math.hpp (profiles) and the geometry of
// gmodel/gmodels.hpp.  The operation order of each expression follows the
// reference so that fp32 results agree to within a few ulp; CUDA's own
// sinf/cosf/expf/... (not the fast intrinsics) are used throughout.
#pragma once

#include "gbk_common.cuh"

namespace gbk {

// ---- math.hpp ------------------------------------------------------------

__device__ __forceinline__ float wrap_angle(float a)       // math.hpp:28-36
{
    while (a < -GBK_PI) a += 2 * GBK_PI;
    while (a > +GBK_PI) a -= 2 * GBK_PI;
    return a;
}

__device__ __forceinline__ int sgn(float x) { return (0.f < x) - (x < 0.f); }

// math.hpp:44-51
__device__ __forceinline__ void rot_lh_x(float& y, float& z, float s, float c)
{
    float ny = y * c + z * s;
    float nz = -y * s + z * c;
    y = ny;
    z = nz;
}

// math.hpp:62-71 (the reference's non-standard convention)
__device__ __forceinline__ void rot_lh_z(float& x, float& y, float s, float c)
{
    float nx = -x * s + y * c;
    float ny = -x * c - y * s;
    x = nx;
    y = ny;
}

__device__ __forceinline__ float uniform_fun(float x, float a, float b, float c)
{ return x >= b && x <= c ? a : 0.f; }
__device__ __forceinline__ float uniform_cdf(float x, float b, float c)
{ return x < b ? 0.f : (x > c ? 1.f : ((x - b) / (c - b))); }
__device__ __forceinline__ float uniform_pdf(float x, float b, float c)
{ float a = 1 / (c - b); return uniform_fun(x, a, b, c); }

__device__ __forceinline__ float expon_fun(float x, float a, float b, float c)
{ return a * expf(-fabsf(x - b) / c); }
__device__ __forceinline__ float expon_cdf(float x, float b, float c)
{ return 0.5f + 0.5f * sgn(x - b) * (1 - expf(-fabsf(x - b) / c)); }
__device__ __forceinline__ float expon_pdf(float x, float b, float c)
{ float a = 1 / (2 * c); return expon_fun(x, a, b, c); }

__device__ __forceinline__ float gauss_fun(float x, float a, float b, float c)
{ return a * expf(-(x - b) * (x - b) / (2 * c * c)); }
__device__ __forceinline__ float gauss_cdf(float x, float b, float c)
{ return (float)(0.5 * (1 + erf((double)(x - b) / ((double)c * 1.4142135623730951)))); }
__device__ __forceinline__ float gauss_pdf(float x, float b, float c)
{ float a = 1 / (c * sqrtf(2 * GBK_PI)); return gauss_fun(x, a, b, c); }

__device__ __forceinline__ float ggauss_fun(float x, float a, float b, float c, float d)
{ return a * expf(-powf(fabsf(x - b) / c, d)); }
__device__ __forceinline__ float ggauss_pdf(float x, float b, float c, float d)
{ float a = d / (2 * c * tgammaf(1 / d)); return ggauss_fun(x, a, b, c, d); }

__device__ __forceinline__ float lorentz_fun(float x, float a, float b, float c)
{ return a * c * c / ((x - b) * (x - b) + c * c); }
__device__ __forceinline__ float lorentz_cdf(float x, float b, float c)
{ return 0.5f + atanf((x - b) / c) / GBK_PI; }
__device__ __forceinline__ float lorentz_pdf(float x, float b, float c)
{ float a = 1 / (GBK_PI * c); return lorentz_fun(x, a, b, c); }

__device__ __forceinline__ float moffat_fun(float x, float a, float b, float c, float d)
{ return a / powf(1 + ((x - b) / c) * ((x - b) / c), d); }

// math.hpp:455-471: std::pow(float, 2) is evaluated in double there
__device__ __forceinline__ float sech2_fun(float x, float a, float b, float c)
{ float q = 1 / coshf((x - b) / c); return (float)(a * ((double)q * (double)q)); }
__device__ __forceinline__ float sech2_cdf(float x, float b, float c)
{ return 0.5f * (1 + tanhf((x - b) / c)); }
__device__ __forceinline__ float sech2_pdf(float x, float b, float c)
{ float a = 1 / (2 * c); return sech2_fun(x, a, b, c); }

// math.hpp:500-511
__device__ __forceinline__ float lerp(float x, int i, const float* xd, const float* yd, int off)
{
    float x1 = xd[i - 1], x2 = xd[i];
    float y1 = yd[off + i - 1], y2 = yd[off + i];
    float t = (x - x1) / (x2 - x1);
    return y1 + t * (y2 - y1);
}

// ---- traits.hpp ----------------------------------------------------------

struct Ring {            // position of a spaxel/cloud on the disk
    int rnidx;           // sub-node index (first node with r < node)
    const float* rnodes;
    int nrnodes;
    float r, theta;
};

__device__ __forceinline__ float nw(const Ring& g, const float* p, int off)
{ return lerp(g.r, g.rnidx, g.rnodes, p, off); }

// traits.hpp:199-246 (blob mixtures; np = 1: 6 params per blob, 2: 7)
static __device__ float p_mixture(int kind, int np, float r, float theta, const float* c, const float* p)
{
    float res = 0;
    int nb = (int)rintf(c[0]);
    for (int i = 0; i < nb; ++i) {
        float br = p[i], bt = p[nb + i], ba = p[2 * nb + i], bs = p[3 * nb + i];
        float bb = np == 2 ? p[4 * nb + i] : 0.f;
        float bq = p[(np == 2 ? 5 : 4) * nb + i];
        float bp = p[(np == 2 ? 6 : 5) * nb + i];
        bt *= GBK_D2R;
        bp *= GBK_D2R;
        float xn = r * cosf(theta) - br * cosf(bt);
        float yn = r * sinf(theta) - br * sinf(bt);
        float s, co;
        sincosf(bt + bp, &s, &co);
        rot_lh_z(xn, yn, s, co);
        float rn = sqrtf(xn * xn + (yn * yn) / (bq * bq));
        switch (kind) {
        case 51: res += expon_fun(rn, ba, 0, bs); break;
        case 52: res += gauss_fun(rn, ba, 0, bs); break;
        case 53: res += ggauss_fun(rn, ba, 0, bs, bb); break;
        default: res += moffat_fun(rn, ba, 0, bs, bb); break;
        }
    }
    return res;
}

// traits.hpp:285-295
__device__ __forceinline__ float p_nw_harmonic(const Ring& g, const float* c, const float* p)
{
    int k = (int)rintf(c[0]);
    float a = nw(g, p, 0);
    float ph = k ? nw(g, p, g.nrnodes) * GBK_D2R : 0.f;
    return a * cosf(k * (g.theta - ph));
}

// traits.hpp:297-308
__device__ __forceinline__ float p_nw_distortion(const Ring& g, const float* p)
{
    float a = nw(g, p, 0);
    float ph = nw(g, p, g.nrnodes) * GBK_D2R;
    float s = nw(g, p, 2 * g.nrnodes);
    float t = wrap_angle(g.theta - ph);
    return a * expf(-(t * t * g.r * g.r) / (2 * s * s));
}

// Density (traits.hpp:1242-1331, uid and 1000 + uid) and dispersion
// (traits.hpp:1702-1775) polar profiles share their catalogue.
static __device__ float p_profile(int kind, const float* c, const float* p, const Ring& g, int& bad)
{
    float r = g.r;
    switch (kind) {
    case 1: return p[0];
    case 2: return expon_fun(r, p[0], 0, p[1]);
    case 3: return gauss_fun(r, p[0], 0, p[1]);
    case 4: return ggauss_fun(r, p[0], 0, p[1], p[2]);
    case 5: return lorentz_fun(r, p[0], 0, p[1]);
    case 6: return moffat_fun(r, p[0], 0, p[1], p[2]);
    case 7: return sech2_fun(r, p[0], 0, p[1]);
    case 51: return p_mixture(51, 1, r, g.theta, c, p);
    case 52: return p_mixture(52, 1, r, g.theta, c, p);
    case 53: return p_mixture(53, 2, r, g.theta, c, p);
    case 54: return p_mixture(54, 2, r, g.theta, c, p);
    case 101: return nw(g, p, 0);
    case 102: return p_nw_harmonic(g, c, p);
    case 103: return p_nw_distortion(g, p);
    default: bad = 1; return NAN;
    }
}

// traits.hpp:898-1078, 1592-1673
static __device__ float vp_trait(int uid, const float* c, const float* p, const Ring& g, float sin_incl,
                          float cos_incl, int& bad)
{
    float r = g.r;
    float mtan = cosf(g.theta) * sin_incl;
    float out;
    switch (uid) {
    case 1: out = p[0]; return out * mtan;
    case 2: out = p[1] * (2 / GBK_PI) * atanf(r / p[0]); return out * mtan;
    case 3: out = p[1] * (1 - expf(-r / p[0])); return out * mtan;
    case 4: out = p[1] * powf(r / p[0], p[3]) / (1 + powf(r / p[0], p[2])); return out * mtan;
    case 5: out = r < p[0] ? p[1] * r / p[0] : p[1]; return out * mtan;
    case 6: out = p[1] * tanhf(r / p[0]); return out * mtan;
    case 7: out = p[1] * (1 - expf(-r / p[0])) * (1 + p[2] * r / p[0]); return out * mtan;
    case 8: out = p[1] * powf(1 + r / p[0], p[2]) * powf(1 + powf(r / p[0], -p[3]), -1 / p[3]);
            return out * mtan;
    case 101: if (r == 0) return 0.f; out = nw(g, p, 0); return out * mtan;
    case 102: if (r == 0) return 0.f; out = p_nw_harmonic(g, c, p); return out * mtan;
    case 103: if (r == 0) return 0.f; out = nw(g, p, 0); return out * (sinf(g.theta) * sin_incl);
    case 104: if (r == 0) return 0.f; out = p_nw_harmonic(g, c, p);
              return out * (sinf(g.theta) * sin_incl);
    case 105: out = nw(g, p, 0); return out * cos_incl;
    case 106: out = p_nw_harmonic(g, c, p); return out * cos_incl;
    case 107: return nw(g, p, 0);
    case 108: return p_nw_harmonic(g, c, p);
    default: bad = 1; return NAN;
    }
}

// traits.hpp:1195-1208
__device__ __forceinline__ float azrange(float theta, float ph, float s)
{
    float pmin = wrap_angle(ph - s * 0.5f);
    float pmax = wrap_angle(ph + s * 0.5f);
    if (pmin < pmax) return (theta > pmin && theta < pmax) ? 1.f : 0.f;
    return (theta < pmin && theta > pmax) ? 0.f : 1.f;
}

// traits.hpp:561-594, 633-896, 1437-1514 (height traits)
static __device__ float rh_trait(int uid, const float* c, const float* p, const Ring& g, float z, int& bad)
{
    float trunc = c[0];
    bool use_rn = c[1] != 0;
    float p1 = use_rn ? nw(g, p, 0) : p[0];
    if (uid >= 1 && uid <= 7) {
        float lo = -trunc * p1, hi = trunc * p1;
        bool in = z >= lo && z <= hi;
        switch (uid) {
        case 1: {
            float v = uniform_pdf(z, 0 - p1, 0 + p1);
            if (trunc == 0) return v;
            return in ? v / (uniform_cdf(hi, -p1, p1) - uniform_cdf(lo, -p1, p1)) : 0.f;
        }
        case 2: {
            float v = expon_pdf(z, 0, p1);
            if (trunc == 0) return v;
            return in ? v / (expon_cdf(hi, 0, p1) - expon_cdf(lo, 0, p1)) : 0.f;
        }
        case 3: {
            float v = gauss_pdf(z, 0, p1);
            if (trunc == 0) return v;
            return in ? v / (gauss_cdf(hi, 0, p1) - gauss_cdf(lo, 0, p1)) : 0.f;
        }
        case 4: {
            float p2 = use_rn ? nw(g, p, g.nrnodes) : p[1];
            float v = ggauss_pdf(z, 0, p1, p2);
            if (trunc == 0) return v;
            return in ? v / (0.f - 0.f) : 0.f;   // the reference's ggauss cdf is a stub (0)
        }
        case 5: {
            float v = lorentz_pdf(z, 0, p1);
            if (trunc == 0) return v;
            return in ? v / (lorentz_cdf(hi, 0, p1) - lorentz_cdf(lo, 0, p1)) : 0.f;
        }
        case 6: {   // the reference's moffat pdf and cdf are stubs (0)
            if (trunc == 0) return 0.f;
            return in ? 0.f / (0.f - 0.f) : 0.f;
        }
        default: {
            float v = sech2_pdf(z, 0, p1);
            if (trunc == 0) return v;
            return in ? v / (sech2_cdf(hi, 0, p1) - sech2_cdf(lo, 0, p1)) : 0.f;
        }
        }
    }
    if (uid >= 1001 && uid <= 1007) {
        // opacity: unnormalised, amplitude first; the 3-parameter form reads
        // p[1] for its third smooth parameter (traits.hpp:652-672)
        float p2 = use_rn ? nw(g, p, g.nrnodes) : p[1];
        float p3 = use_rn ? nw(g, p, 2 * g.nrnodes) : p[1];
        float v;
        switch (uid - 1000) {
        case 1: v = uniform_fun(z, p1, 0 - p2, 0 + p2); break;
        case 2: v = expon_fun(z, p1, 0, p2); break;
        case 3: v = gauss_fun(z, p1, 0, p2); break;
        case 4: v = ggauss_fun(z, p1, 0, p2, p3); break;
        case 5: v = lorentz_fun(z, p1, 0, p2); break;
        case 6: v = moffat_fun(z, p1, 0, p2, p3); break;
        default: v = sech2_fun(z, p1, 0, p2); break;
        }
        if (trunc == 0) return v;
        return (z >= -trunc * p2 && z <= trunc * p2) ? v : 0.f;
    }
    bad = 1;
    return NAN;
}

enum TraitKind { K_RP, K_RH, K_VP, K_VH, K_DP, K_DH, K_ZP, K_SP, K_WP };

// The per-set trait values of the cloud kernels live in fixed-size arrays that are only indexed by
// constants (the loops over the set's n traits are unrolled to the maximum
// with a guard, stores go through selects), so they stay in registers
// instead of the stack.
typedef float TraitVals[GBK_TRAIT_NUM_MAX];

__device__ __forceinline__ void tv_set(TraitVals& o, int i, float v)
{
#pragma unroll
    for (int j = 0; j < GBK_TRAIT_NUM_MAX; ++j) o[j] = i == j ? v : o[j];
}
// sum of the first n values, in index order
__device__ __forceinline__ float tv_sum(const TraitVals& a, int n)
{
    float s = 0;
#pragma unroll
    for (int i = 0; i < GBK_TRAIT_NUM_MAX; ++i)
        if (i < n) s += a[i];
    return s;
}
// sum of a[i] * b[i] over the first n, in index order (b = null: a[i] * 1)
__device__ __forceinline__ float tv_dot(const TraitVals& a, const TraitVals* b, int n)
{
    float s = 0;
#pragma unroll
    for (int i = 0; i < GBK_TRAIT_NUM_MAX; ++i)
        if (i < n) s += a[i] * (b ? (*b)[i] : 1.f);
    return s;
}
// product of the first n values, in index order
__device__ __forceinline__ float tv_prod(const TraitVals& a, int n)
{
    float s = 1;
#pragma unroll
    for (int i = 0; i < GBK_TRAIT_NUM_MAX; ++i)
        if (i < n) s *= a[i];
    return s;
}

// the value of trait uid of a set of kind KIND (traits.hpp:1887-1919)
template<int KIND>
__device__ __forceinline__ float trait_value(int uid, const float* cv, const float* pv,
                                             const Ring& g, float sin_incl, float cos_incl,
                                             float z, int& bad)
{
    float v;
    if (KIND == K_RP) v = p_profile(uid >= 1000 ? uid - 1000 : uid, cv, pv, g, bad);
    else if (KIND == K_DP) v = p_profile(uid, cv, pv, g, bad);
    else if (KIND == K_VP) v = vp_trait(uid, cv, pv, g, sin_incl, cos_incl, bad);
    else if (KIND == K_RH) v = rh_trait(uid, cv, pv, g, z, bad);
    else if (KIND == K_ZP) {
        if (uid == 101) v = nw(g, pv, 0);
        else if (uid == 102) v = p_nw_harmonic(g, cv, pv);
        else { bad = 1; v = NAN; }
    } else if (KIND == K_SP) {
        if (uid == 1) v = azrange(g.theta, pv[0] * GBK_D2R, pv[1] * GBK_D2R);
        else if (uid == 101) v = azrange(g.theta, nw(g, pv, 0) * GBK_D2R,
                                         nw(g, pv, g.nrnodes) * GBK_D2R);
        else { bad = 1; v = NAN; }
    } else {   // K_VH, K_DH, K_WP: the only implemented kind (uid 1) is 1
        if (uid == 1) v = 1.f;
        else { bad = 1; v = NAN; }
    }
    return v;
}

// the n traits of a set into out[i], advancing the constants/parameters
// pointers by the per-trait counts (the smooth-disk kernels)
template<int KIND>
__device__ __forceinline__ void eval_set(float* out, const TraitSet& ts, const Ring& g,
                                         float sin_incl, float cos_incl, float z, int& bad)
{
    const float* cv = ts.cv;
    const float* pv = ts.pv;
    for (int i = 0; i < ts.n; ++i) {
        out[i] = trait_value<KIND>(ts.uids[i], cv, pv, g, sin_incl, cos_incl, z, bad);
        cv += ts.cc[i];
        pv += ts.pc[i];
    }
}

// the same into register-resident values (the cloud kernels: their trait
// values stay off the stack)
template<int KIND>
__device__ __forceinline__ void eval_set_r(TraitVals& out, const TraitSet& ts, const Ring& g,
                                           float sin_incl, float cos_incl, float z, int& bad)
{
    const float* cv = ts.cv;
    const float* pv = ts.pv;
    for (int i = 0; i < ts.n; ++i) {
        tv_set(out, i, trait_value<KIND>(ts.uids[i], cv, pv, g, sin_incl, cos_incl, z, bad));
        cv += ts.cc[i];
        pv += ts.pc[i];
    }
}

// gmodels.hpp:197-215: the first sub-node index with r < node (linear search
// in the reference; the nodes ascend, so a binary search finds the same one)
__device__ __forceinline__ bool disk_info(int& idx, float r, int n, const float* nodes)
{
    if (r < nodes[0]) return false;
    if (r >= nodes[n - 1]) return false;
    int lo = 1, hi = n - 1;   // invariant: nodes[lo-1] <= r < nodes[hi]
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (r < nodes[mid]) hi = mid;
        else lo = mid + 1;
    }
    idx = lo;
    return true;
}

// gmodels.hpp:167-195
__device__ __forceinline__ float rnode_radius(float x, float y, float z, bool thick,
                                              const DiskArgs& a, int i)
{
    float xp = a.loose ? a.xpos[i] : a.xpos[0], yp = a.loose ? a.ypos[i] : a.ypos[0];
    float pa = a.tilted ? a.posa[i] : a.posa[0], in = a.tilted ? a.incl[i] : a.incl[0];
    pa *= GBK_D2R;
    in *= GBK_D2R;
    x -= xp;
    y -= yp;
    float s, c;
    sincosf(pa, &s, &c);
    rot_lh_z(x, y, s, c);
    if (thick) {
        sincosf(in, &s, &c);
        rot_lh_x(y, z, s, c);
    } else {
        y /= cosf(in);
    }
    return sqrtf(x * x + y * y);
}

// gmodels.hpp:217-323 (linear search and "velfi" radius, as there)
static __device__ bool ring_info(int& index, float& radius, float x, float y, float z, bool thick,
                          const DiskArgs& a)
{
    int n = a.nrnodes;
    const float* nodes = a.rnodes;
    if (rnode_radius(x, y, z, thick, a, 0) < nodes[0]) return false;
    if (rnode_radius(x, y, z, thick, a, n - 1) >= nodes[n - 1]) return false;
    for (index = 1; index < n; ++index)
        if (rnode_radius(x, y, z, thick, a, index) < nodes[index]) break;
    float d1 = nodes[index - 1] - rnode_radius(x, y, z, thick, a, index - 1);
    float d2 = nodes[index] - rnode_radius(x, y, z, thick, a, index);
    radius = (nodes[index] * d1 - nodes[index - 1] * d2) / (d1 - d2);
    return true;
}

// gmodels.hpp:92-116: channel window of a line (v -+ 5 sigma, rint, clamped);
// false for an empty window or a non-finite line (UB in the reference)
__device__ __forceinline__ bool line_window(float v, float d, int nz, float step, float zero,
                                            int& zlo, int& zhi)
{
    if (!isfinite(v) || !isfinite(d)) return false;
    float zmin = v - d * GBK_LINE_WIDTH, zmax = v + d * GBK_LINE_WIDTH;
    float a = rintf((zmin - zero) / step), b = rintf((zmax - zero) / step);
    a = a < 0.f ? 0.f : a;
    b = (float)(nz - 1) < b ? (float)(nz - 1) : b;
    zlo = (int)a;
    zhi = (int)b;
    return zlo <= zhi;
}

}  // namespace gbk
