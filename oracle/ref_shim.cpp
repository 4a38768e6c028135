// Shim that compiles the REFERENCE's own arithmetic (header-only templates
// under src/gbkfit/driver/native/gbkfit/include and the host RNG header
// gbkfit_host/include/gbkfit/host/random.hpp) into oracle/_ref/libgbkfit_ref.so.
//
// TEST INFRASTRUCTURE ONLY.  Used by the tests to pin the oracle restatement
// and by `bench.py --impl reference` as the timed CPU baseline.  Nothing in the
// product links it.
//
// The loops restate gbkfit_host/include/gbkfit/host/kernels.hpp (the OpenMP
// drivers of the templates); that header itself is not included because it
// pulls <fftw3.h> (FFTW3 is not installed here).  The templates are
// instantiated for float (the reference's own precision) and double.
#include <cmath>
#include <cstdint>
#include <vector>
#include <omp.h>

#include "gbkfit/common.hpp"
#include "gbkfit/host/random.hpp"
#include "gbkfit/dmodel/dmodels.hpp"
#include "gbkfit/gmodel/gmodels.hpp"
#include "gbkfit/objective/objective.hpp"

namespace {

template<typename T> inline void add_atomic(T* p, T v)
{
    #pragma omp atomic update
    p[0] += v;
}
template<typename T> inline void set_atomic(T* p, T v)
{
    #pragma omp atomic write
    p[0] = v;
}

}  // namespace

#define TRAIT_ARGS(T, p) const int* p##_uids, const T* p##_cv, const int* p##_cc, \
                         const T* p##_pv, const int* p##_pc
#define TRAIT_PASS(p) p##_uids, p##_cv, p##_cc, p##_pv, p##_pc

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

#define DISK_PASS \
    (bool)loose, (bool)tilted, nrnodes, rnodes, vsys, xpos, ypos, posa, incl, \
    nrt, TRAIT_PASS(rpt), TRAIT_PASS(rht), \
    nvt, TRAIT_PASS(vpt), TRAIT_PASS(vht), \
    ndt, TRAIT_PASS(dpt), TRAIT_PASS(dht), \
    nzt, TRAIT_PASS(zpt), nst, TRAIT_PASS(spt), nwt, TRAIT_PASS(wpt), \
    opacity, sx, sy, sz, stx, sty, stz, zx, zy, zz, spec_size, spec_step, spec_zero, \
    image, scube, wdata, wdata_cmp, rdata, rdata_cmp, ordata, ordata_cmp, vdata_cmp, ddata_cmp

// host/kernels.hpp:308-423
template<typename T> static void smdisk(DISK_PARAMS(T))
{
    #pragma omp parallel for collapse(3)
    for (int y = 0; y < sy; ++y)
    for (int x = 0; x < sx; ++x)
    for (int z = 0; z < sz; ++z)
        gbkfit::gmodel_smdisk_evaluate_spaxel<add_atomic<T>>(x, y, z, DISK_PASS);
}

// host/kernels.hpp:183-306 (every thread's generator seeded 42, as there)
template<typename T> static void mcdisk(T cflux, int nclouds, const int* csum, int csum_len,
                                        const bool* hasordint, DISK_PARAMS(T))
{
    std::vector<gbkfit::RNG<T>> rngs;
    for (int i = 0; i < omp_get_num_procs(); ++i)
        rngs.push_back(gbkfit::RNG<T>(0, 1, 42));
    #pragma omp parallel for
    for (int ci = 0; ci < nclouds; ++ci) {
        gbkfit::RNG<T>& rng = rngs[omp_get_thread_num()];
        gbkfit::gmodel_mcdisk_evaluate_cloud<set_atomic<T>, add_atomic<T>>(
            rng, ci, cflux, nclouds, csum, csum_len, hasordint, DISK_PASS);
    }
}

// host/kernels.hpp:105-135 (note the d, w, m -> d, m, w swap, as there)
template<typename T> static void moments(int nx, int ny, int nz, T stx, T sty, T stz, T zx, T zy,
                                         T zz, const T* d, const T* w, T cutoff, int norders,
                                         const int* orders, T* mmaps_d, T* mmaps_m, T* mmaps_w)
{
    #pragma omp parallel for collapse(2)
    for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x)
        gbkfit::dmodel_mmaps_moments(x, y, nx, ny, nz, stx, sty, stz, zx, zy, zz, d, w, cutoff,
                                     norders, orders, mmaps_d, mmaps_w, mmaps_m);
}

extern "C" {

void ref_smdisk_evaluate_f32(DISK_PARAMS(float)) { smdisk<float>(DISK_PASS); }
void ref_smdisk_evaluate_f64(DISK_PARAMS(double)) { smdisk<double>(DISK_PASS); }

void ref_mcdisk_evaluate_f32(float cflux, int nclouds, const int* csum, int csum_len,
                             const unsigned char* hasordint, DISK_PARAMS(float))
{
    mcdisk<float>(cflux, nclouds, csum, csum_len, reinterpret_cast<const bool*>(hasordint),
                  DISK_PASS);
}

// Python-facing argument order of the reference native module
// (gbkfit_host/src/dmodels.cpp:79-100): ..., mmaps_d, mmaps_m, mmaps_w
void ref_mmaps_moments_f32(int nx, int ny, int nz, float stx, float sty, float stz, float zx,
                           float zy, float zz, const float* d, const float* w, float cutoff,
                           int norders, const int* orders, float* mmaps_d, float* mmaps_m,
                           float* mmaps_w)
{
    moments<float>(nx, ny, nz, stx, sty, stz, zx, zy, zz, d, w, cutoff, norders, orders,
                   mmaps_d, mmaps_m, mmaps_w);
}

// host/kernels.hpp:55-80
void ref_dcube_downscale_f32(int scx, int scy, int scz, int ofx, int ofy, int ofz, int srx,
                             int sry, int srz, int dsx, int dsy, int dsz, const float* src,
                             float* dst)
{
    #pragma omp parallel for collapse(3)
    for (int z = 0; z < dsz; ++z)
    for (int y = 0; y < dsy; ++y)
    for (int x = 0; x < dsx; ++x)
        gbkfit::dmodel_dcube_downscale(x, y, z, scx, scy, scz, ofx, ofy, ofz, srx, sry, srz,
                                       dsx, dsy, dsz, src, dst);
}

// host/kernels.hpp:82-103
void ref_dcube_mask_f32(float cutoff, int apply, int nx, int ny, int nz, float* d, float* m,
                        float* w)
{
    #pragma omp parallel for collapse(3)
    for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x)
        gbkfit::dmodel_dcube_mask(x, y, z, cutoff, (bool)apply, nx, ny, nz, d, m, w);
}

// host/kernels.hpp:484-514
void ref_residual_f32(const float* od, const float* oe, const float* om, const float* md,
                      const float* mw, const float* mm, int n, float weight, float* res)
{
    #pragma omp parallel for
    for (int i = 0; i < n; ++i)
        gbkfit::objective_residual(i, od, oe, om, md, mw, mm, n, weight, res);
}

void ref_residual_sum_f32(const float* res, int n, int squared, float* sum)
{
    float s = 0;
    #pragma omp parallel for reduction(+:s)
    for (int i = 0; i < n; ++i) {
        const float r = res[i];
        s += squared ? r * r : std::abs(r);
    }
    sum[0] = s;
}

// host/kernels.hpp:137-158
void ref_convolve_f32(int ax, int ay, int az, int bx, int by, int bz, const float* a,
                      const float* b, float* out)
{
    #pragma omp parallel for collapse(3)
    for (int z = 0; z < az; ++z)
    for (int y = 0; y < ay; ++y)
    for (int x = 0; x < ax; ++x)
        gbkfit::gmodel_convolve(x, y, z, ax, ay, az, bx, by, bz, a, b, out);
}

// host/kernels.hpp:160-181
void ref_wcube_evaluate_f32(int sx, int sy, int sz, int spec_z, const float* spat, float* spec)
{
    #pragma omp parallel for collapse(2)
    for (int y = 0; y < sy; ++y)
    for (int x = 0; x < sx; ++x)
        gbkfit::gmodel_wcube_pixel(x, y, sx, sy, sz, spec_z, spat, spec);
}

int ref_num_threads(void) { return omp_get_max_threads(); }
// threads of the following calls (1: the reference's mcdisk draws every cloud
// from one mt19937 stream seeded 42, host/kernels.hpp:239-242)
void ref_set_num_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"
