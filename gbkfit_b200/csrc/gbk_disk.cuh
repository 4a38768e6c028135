// Per-spaxel smooth-disk evaluation shared by the drop-in kernels (gmodel.cu)
// and the batched pipeline (batched.cu).
//
// Restates gbkfit/include/gbkfit/gmodel/gmodels.hpp:645-958 of the reference.
#pragma once

#include "gbk_traits.cuh"

namespace gbk {

struct SpaxelOut {
    float rv, vv, dv, wv, orv;
};

// Precomputed per-call constants (identical fp32 values to the per-spaxel
// evaluation of the reference, hoisted out of the loops).
struct DiskConst {
    float sin_pa, cos_pa, cos_in, sin_in, incli;
};

__device__ __forceinline__ DiskConst disk_const(const DiskArgs& a)
{
    DiskConst k;
    float pa = a.posa[0] * GBK_D2R;
    float in = a.incl[0] * GBK_D2R;
    sincosf(pa, &k.sin_pa, &k.cos_pa);
    sincosf(in, &k.sin_in, &k.cos_in);
    k.incli = in;
    return k;
}

// gmodels.hpp:645-914 for spaxel (x, y, z); false if the spaxel contributes
// nothing.  `bad` is raised for unknown trait uids.
static __device__ bool smdisk_spaxel(const DiskArgs& a, const DiskConst& kc, int x, int y, int z,
                              SpaxelOut& o, int& bad)
{
    const bool thin = a.rht.uids == nullptr;
    const bool lt = a.loose || a.tilted;
    float xn = a.zx + x * a.stx, yn = a.zy + y * a.sty, zn = a.zz + z * a.stz;
    Ring g;
    g.rnodes = a.rnodes;
    g.nrnodes = a.nrnodes;
    g.rnidx = -1;
    g.r = 0;
    if (lt && !ring_info(g.rnidx, g.r, xn, yn, zn, !thin, a)) return false;

    float vsysi, xposi, yposi;
    float sin_pa = kc.sin_pa, cos_pa = kc.cos_pa, sin_in = kc.sin_in, cos_in = kc.cos_in;
    if (a.loose) {
        vsysi = lerp(g.r, g.rnidx, a.rnodes, a.xpos, 0);   // gmodels.hpp:726 reads xpos
        xposi = lerp(g.r, g.rnidx, a.rnodes, a.xpos, 0);
        yposi = lerp(g.r, g.rnidx, a.rnodes, a.ypos, 0);
    } else {
        vsysi = a.vsys ? a.vsys[0] : 0.f;
        xposi = a.xpos[0];
        yposi = a.ypos[0];
    }
    float incli = kc.incli;
    if (a.tilted) {
        float pa = lerp(g.r, g.rnidx, a.rnodes, a.posa, 0) * GBK_D2R;
        incli = lerp(g.r, g.rnidx, a.rnodes, a.incl, 0) * GBK_D2R;
        sincosf(pa, &sin_pa, &cos_pa);
        sincosf(incli, &sin_in, &cos_in);
    }
    // world -> disk (gmodels.hpp:143-157)
    xn -= xposi;
    yn -= yposi;
    rot_lh_z(xn, yn, sin_pa, cos_pa);
    if (thin) yn /= cos_in;
    else rot_lh_x(yn, zn, sin_in, cos_in);
    g.theta = atan2f(yn, xn);
    if (!lt) {
        g.r = sqrtf(xn * xn + yn * yn);
        if (!disk_info(g.rnidx, g.r, a.nrnodes, a.rnodes)) return false;
    }

    float pt[GBK_TRAIT_NUM_MAX] = {0, 0, 0, 0}, ht[GBK_TRAIT_NUM_MAX] = {0, 0, 0, 0};
    float rv = 0, vv = 0, dv = 0, wv = 1;
    if (a.spt.uids) {
        eval_set<K_SP>(pt, a.spt, g, 0, 0, 0, bad);
        float sv = 0;
        for (int i = 0; i < a.spt.n; ++i) sv += pt[i];
        if (!sv) return false;
    }
    if (a.zpt.uids) {
        eval_set<K_ZP>(pt, a.zpt, g, 0, 0, 0, bad);
        float zv = 0;
        for (int i = 0; i < a.zpt.n; ++i) zv += pt[i];
        zn += zv;
    }
    if (a.rpt.uids) eval_set<K_RP>(pt, a.rpt, g, 0, 0, 0, bad);
    if (a.rht.uids) eval_set<K_RH>(ht, a.rht, g, 0, 0, fabsf(zn), bad);
    for (int i = 0; i < a.rpt.n; ++i) rv += pt[i] * (thin ? 1.f : ht[i]);
    if (!rv) return false;
    // cos_in and sin_in are sincosf(incli): the values cosf(incli) and
    // sinf(incli) of gmodels.hpp, computed once per set (per spaxel only
    // when the disk is tilted)
    if (thin) rv /= cos_in;
    else rv *= a.stz;
    if (a.vpt.uids) eval_set<K_VP>(pt, a.vpt, g, sin_in, cos_in, 0, bad);
    if (a.vht.uids) eval_set<K_VH>(ht, a.vht, g, 0, 0, fabsf(zn), bad);
    for (int i = 0; i < a.vpt.n; ++i) vv += pt[i] * (thin ? 1.f : ht[i]);
    vv += vsysi;
    if (a.dpt.uids) eval_set<K_DP>(pt, a.dpt, g, 0, 0, 0, bad);
    if (a.dht.uids) eval_set<K_DH>(ht, a.dht, g, 0, 0, fabsf(zn), bad);
    for (int i = 0; i < a.dpt.n; ++i) dv += pt[i] * (thin ? 1.f : ht[i]);
    dv = fabsf(dv);
    if (a.wpt.uids && a.wdata) {
        eval_set<K_WP>(pt, a.wpt, g, 0, 0, 0, bad);
        for (int i = 0; i < a.wpt.n; ++i) wv *= pt[i];
    }
    float orv = rv;
    if (a.opacity) {
        long long sxy = (long long)a.sx * a.sy;
        for (int oz = z + 1; oz < a.sz; ++oz)
            orv -= orv * a.opacity[x + (long long)a.sx * y + sxy * oz];
    }
    o.rv = rv;
    o.vv = vv;
    o.dv = dv;
    o.wv = wv;
    o.orv = orv;
    return true;
}

// smdisk_spaxel for a flat thin disk whose only traits are one node-wise
// density (rpt uid 101), one node-wise rotation curve (vpt uid 101) and one
// node-wise dispersion (dpt uid 101), without opacity: the same fp32
// operations in the same order as the generic path (gmodels.hpp:645-914,
// traits.hpp:138-141, 999-1007), without the trait dispatch.
__device__ __forceinline__ bool smdisk_spaxel_nw(const DiskArgs& a, const DiskConst& kc, int x,
                                                 int y, SpaxelOut& o)
{
    float xn = a.zx + x * a.stx, yn = a.zy + y * a.sty;
    xn -= a.xpos[0];
    yn -= a.ypos[0];
    rot_lh_z(xn, yn, kc.sin_pa, kc.cos_pa);
    yn /= kc.cos_in;
    const float theta = atan2f(yn, xn);
    const float r = sqrtf(xn * xn + yn * yn);
    int k;
    if (!disk_info(k, r, a.nrnodes, a.rnodes)) return false;
    float rv = 0;
    rv += lerp(r, k, a.rnodes, a.rpt.pv, 0) * 1.f;
    if (!rv) return false;
    rv /= kc.cos_in;                                     // cosf(incli), once per set
    const float mtan = cosf(theta) * kc.sin_in;
    const float vt = r == 0 ? 0.f : lerp(r, k, a.rnodes, a.vpt.pv, 0) * mtan;
    float vv = 0;
    vv += vt * 1.f;
    vv += a.vsys ? a.vsys[0] : 0.f;
    float dv = 0;
    dv += lerp(r, k, a.rnodes, a.dpt.pv, 0) * 1.f;
    o.rv = rv;
    o.vv = vv;
    o.dv = fabsf(dv);
    o.wv = 1;
    o.orv = rv;
    return true;
}

// gmodels.hpp:930-957: the non-spectral outputs of an smdisk spaxel
__device__ __forceinline__ void smdisk_side_outputs(const DiskArgs& a, int x, int y, int z,
                                                    const SpaxelOut& o)
{
    long long idx = idx3(x, y, z, a.sx, a.sy);
    if (a.wdata) a.wdata[idx] += o.wv;
    if (a.wdata_cmp) a.wdata_cmp[idx] = o.wv;
    if (a.rdata) a.rdata[idx] += o.rv;
    if (a.rdata_cmp) a.rdata_cmp[idx] = o.rv;
    if (a.ordata) a.ordata[idx] += o.orv;
    if (a.ordata_cmp) a.ordata_cmp[idx] = o.orv;
    if (a.vdata_cmp) a.vdata_cmp[idx] = o.vv;
    if (a.ddata_cmp) a.ddata_cmp[idx] = o.dv;
}

}  // namespace gbk
