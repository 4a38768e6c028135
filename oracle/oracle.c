/*
 * Oracle entry points (TEST INFRASTRUCTURE ONLY; see oracle_impl.h).
 *
 * The smdisk/mcdisk entry points take the reference's argument lists
 * (gbkfit_host/include/gbkfit/host/gmodels.hpp:26-135) so that tests can feed
 * identical packed arrays to the oracle, to the compiled reference in
 * oracle/_ref and to the CUDA product.
 */
#include <math.h>
#include <tgmath.h>
#include <stddef.h>

#define REAL float
#define SFX _f32
#include "oracle_impl.h"
#undef REAL
#undef SFX
#undef TRUNC_PDF
#undef TRUNC_FUN
#undef PI_R
#undef D2R
#undef R

#define REAL double
#define SFX _f64
#include "oracle_impl.h"
#undef REAL
#undef SFX

/* the reference's per-kind trait argument group: uids, cvalues, ccounts,
 * pvalues, pcounts */
#define TRAIT_ARGS(T, p) const int* p##_uids, const T* p##_cv, const int* p##_cc, \
                         const T* p##_pv, const int* p##_pc
#define TRAIT_SET(a, p) a.p##_uids = p##_uids; a.p##_cv = p##_cv; a.p##_cc = p##_cc; \
                        a.p##_pv = p##_pv; a.p##_pc = p##_pc

#define DISK_PARAMS(T) \
    int loose, int tilted, int nrnodes, const T* rnodes, const T* vsys, \
    const T* xpos, const T* ypos, const T* posa, const T* incl, \
    int nrt, TRAIT_ARGS(T, rpt), TRAIT_ARGS(T, rht), \
    int nvt, TRAIT_ARGS(T, vpt), TRAIT_ARGS(T, vht), \
    int ndt, TRAIT_ARGS(T, dpt), TRAIT_ARGS(T, dht), \
    int nzt, TRAIT_ARGS(T, zpt), \
    int nst, TRAIT_ARGS(T, spt), \
    int nwt, TRAIT_ARGS(T, wpt), \
    const T* opacity, \
    int sx, int sy, int sz, T stx, T sty, T stz, T zx, T zy, T zz, \
    int spec_size, T spec_step, T spec_zero, \
    T* image, T* scube, T* wdata, T* wdata_cmp, T* rdata, T* rdata_cmp, \
    T* ordata, T* ordata_cmp, T* vdata_cmp, T* ddata_cmp

#define FILL_ARGS(a) \
    a.loose = loose; a.tilted = tilted; a.nrnodes = nrnodes; a.rnodes = rnodes; a.vsys = vsys; \
    a.xpos = xpos; a.ypos = ypos; a.posa = posa; a.incl = incl; \
    a.nrt = nrt; TRAIT_SET(a, rpt); TRAIT_SET(a, rht); \
    a.nvt = nvt; TRAIT_SET(a, vpt); TRAIT_SET(a, vht); \
    a.ndt = ndt; TRAIT_SET(a, dpt); TRAIT_SET(a, dht); \
    a.nzt = nzt; TRAIT_SET(a, zpt); a.nst = nst; TRAIT_SET(a, spt); \
    a.nwt = nwt; TRAIT_SET(a, wpt); a.opacity = opacity; \
    a.sx = sx; a.sy = sy; a.sz = sz; a.stx = stx; a.sty = sty; a.stz = stz; \
    a.zx = zx; a.zy = zy; a.zz = zz; a.spec_size = spec_size; a.spec_step = spec_step; \
    a.spec_zero = spec_zero; a.image = image; a.scube = scube; a.wdata = wdata; \
    a.wdata_cmp = wdata_cmp; a.rdata = rdata; a.rdata_cmp = rdata_cmp; a.ordata = ordata; \
    a.ordata_cmp = ordata_cmp; a.vdata_cmp = vdata_cmp; a.ddata_cmp = ddata_cmp

int orc_smdisk_evaluate_f32(DISK_PARAMS(float))
{
    disk_args_f32 a;
    FILL_ARGS(a);
    return smdisk_run_f32(&a);
}

int orc_smdisk_evaluate_f64(DISK_PARAMS(double))
{
    disk_args_f64 a;
    FILL_ARGS(a);
    return smdisk_run_f64(&a);
}

int orc_mcdisk_evaluate_f32(float cflux, int nclouds, const int* csum, int csum_len,
                            const unsigned char* hasordint, unsigned long long seed,
                            DISK_PARAMS(float))
{
    (void)csum_len;
    disk_args_f32 a;
    FILL_ARGS(a);
    return mcdisk_run_f32(&a, cflux, nclouds, csum, hasordint, seed);
}

int orc_mcdisk_evaluate_f64(double cflux, int nclouds, const int* csum, int csum_len,
                            const unsigned char* hasordint, unsigned long long seed,
                            DISK_PARAMS(double))
{
    (void)csum_len;
    disk_args_f64 a;
    FILL_ARGS(a);
    return mcdisk_run_f64(&a, cflux, nclouds, csum, hasordint, seed);
}

/* Philox self-check hook: the first four words of Philox(ctr, key) */
void orc_philox4x32(const unsigned ctr[4], unsigned k0, unsigned k1, unsigned out[4])
{
    orc_philox(ctr, k0, k1, out);
}
