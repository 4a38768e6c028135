/*
 * gbkb200.h - C ABI of the B200-native GBKFIT model-evaluation library
 * (libgbkb200.so, sm_100a).
 *
 * The entry points replace the methods of the reference's native modules
 * (pybind11 classes FFTf32, DModelf32, GModelf32, Objectivef32 of
 * src/gbkfit/driver/native/gbkfit_{host,cuda}).  Argument lists and argument
 * meaning follow the reference one to one; each declaration cites the
 * reference declaration it replaces (paths relative to
 * src/gbkfit/driver/native/).  The differences are:
 *
 *   - every call takes a context (the "module object"): it carries the CUDA
 *     stream, the synchronous/asynchronous mode and the FFT caches;
 *   - pointers are typed device pointers instead of std::uintptr_t, and
 *     std::array<int, 3> / std::array<T, 3> arguments are passed as pointers
 *     to three host values;
 *   - every call returns a status (GBKB200_OK or an error code) where the
 *     reference returns void and checks nothing.
 *
 * A null pointer means "absent", as in the reference (_detail/native.py maps
 * None to 0).  Outputs documented as accumulated (+=) must be zeroed by the
 * caller, as in the reference.  All device pointers must be on the context's
 * device.  In synchronous mode (the default, the reference's semantics) a call
 * returns after its work finished; in asynchronous mode it only enqueues work
 * on the context's stream.
 */
#ifndef GBKB200_H
#define GBKB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    GBKB200_OK = 0,
    GBKB200_ERR_INVALID_ARG = 1,   /* null handle, bad size, bad shape */
    GBKB200_ERR_UNSUPPORTED = 2,   /* e.g. an FFT length with a prime factor > 61 */
    GBKB200_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    GBKB200_ERR_BAD_TRAIT = 4,     /* a kernel met an unknown trait uid */
    GBKB200_ERR_OOM = 5,           /* device allocation failed */
    GBKB200_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up */
    GBKB200_ERR_TOO_LARGE = 7      /* a size exceeds a documented maximum */
};

typedef struct gbkb200_ctx gbkb200_ctx;

/* ---- context (no reference counterpart: the reference's module objects
 *      are stateless apart from the FFT caches, fft.hpp:209-210) ---------- */

int gbkb200_ctx_create(gbkb200_ctx** out, int device);
int gbkb200_ctx_destroy(gbkb200_ctx* ctx);
/* stream: a cudaStream_t (0 = the legacy default stream) */
int gbkb200_ctx_set_stream(gbkb200_ctx* ctx, void* stream);
/* sync = 1: return after the work finished (reference semantics, wrapper.cu
 * ends every call with cudaDeviceSynchronize); sync = 0: enqueue only */
int gbkb200_ctx_set_sync(gbkb200_ctx* ctx, int sync);
/* seed of the counter-based cloud generator of mcdisk_evaluate and its
 * accumulation mode.  Mode 0 = fast (the default; fp32 atomics, sums depend
 * on the order clouds land in, in the last bits): the lines are accumulated
 * channel-contiguous in scratch cubes held by the context (1 to 8 copies of
 * 4 bytes per scube element, gbkb200_mcdisk_scratch_bytes; each block adds
 * into one copy) with 16-byte vector atomics, then added to scube; when that
 * scratch cannot be allocated, as mode 3.  Mode 1 = deterministic: the
 * accumulated outputs (scube, image, rdata, ordata and their _cmp forms) are
 * summed in 64-bit fixed point, bit-identical run to run and exact to
 * ~2^-(62 - log2 nclouds) of the largest contribution; it takes an extra
 * bound pass over the clouds and scratch of 8 bytes per accumulated element
 * held by the context.  Mode 2 = mode 0 without the fallback (an allocation
 * failure is returned).  Mode 3 = fast with one fp32 atomic per channel into
 * scube (no scratch).  The assigned maps (wdata, vdata_cmp, ddata_cmp) keep
 * the reference's last-writer-wins race in every mode. */
int gbkb200_ctx_set_mcdisk(gbkb200_ctx* ctx, unsigned long long seed, int mode);
/* grows the context's mcdisk scratch to at least `bytes` now (a later call
 * that needs no more allocates nothing on its stream's path) */
int gbkb200_ctx_reserve_scratch(gbkb200_ctx* ctx, size_t bytes);
/* the scratch bytes the fast mcdisk modes use for a call of nclouds clouds
 * on a spat_size_x x spat_size_y x spec_size spectral cube: copies of the
 * channel-contiguous line cube (1 to 8, more for denser clouds, at most
 * 64 MB of copies) */
size_t gbkb200_mcdisk_scratch_bytes(int nclouds, int spat_size_x, int spat_size_y,
                                    int spec_size);
/* waits for the context's stream, then returns the status raised by kernels
 * since the last call (GBKB200_OK, _BAD_TRAIT or _TIMEOUT) and clears it */
int gbkb200_ctx_synchronize(gbkb200_ctx* ctx);
const char* gbkb200_error_string(int code);
/* the CUDA error string of the last GBKB200_ERR_CUDA of this thread */
const char* gbkb200_last_cuda_error(void);

/* ---- FFTf32: gbkfit_host/include/gbkfit/host/fft.hpp:71-125 ------------ */
/* size = {nx, ny, nz} (the reference receives shape[::-1], _detail/native.py
 * :228-250); real data (nz, ny, nx), complex data (nz, ny, nx/2+1) */

/* fft.hpp:71-77  FFT::fft_r2c(size, data_r, data_c) */
int gbkb200_fft_r2c_f32(gbkb200_ctx* ctx, const int size[3], const float* data_r, void* data_c);
/* fft.hpp:79-85  FFT::fft_c2r(size, data_c, data_r); data_c is preserved
 * (unlike FFTW's c2r, which may overwrite its input) */
int gbkb200_fft_c2r_f32(gbkb200_ctx* ctx, const int size[3], const void* data_c, float* data_r);
/* fft.hpp:87-96  FFT::fft_convolve(size, data1_r, data1_c, data2_c):
 * data1_r <- irfft(rfft(data1_r) * data2_c / N); data1_c is work space whose
 * content afterwards is unspecified (the reference multiplies in it and runs
 * FFTW's multi-dimensional c2r on it, which destroys it).  data1_r and the
 * complex buffers must be 8-byte aligned. */
int gbkb200_fft_convolve_f32(gbkb200_ctx* ctx, const int size[3], float* data1_r, void* data1_c,
                             const void* data2_c);
/* fft.hpp:98-125  FFT::fft_convolve_cached(size, data1_r, data2_r): as above
 * with the spectrum of data2_r computed on first use and cached by
 * (size, data2_r) */
int gbkb200_fft_convolve_cached_f32(gbkb200_ctx* ctx, const int size[3], float* data1_r,
                                    const float* data2_r);
/* fft.hpp:56-69  FFT::clear_cache() */
int gbkb200_fft_clear_cache(gbkb200_ctx* ctx);

/* ---- DModelf32: gbkfit_host/include/gbkfit/host/dmodels.hpp:8-34 ------- */

/* dmodels.hpp:11-17  DModel::dcube_downscale(scale, offset, src_size, dst_size, src, dst) */
int gbkb200_dmodel_dcube_downscale_f32(gbkb200_ctx* ctx, const int scale[3], const int offset[3],
                                       const int src_size[3], const int dst_size[3],
                                       const float* src_dcube, float* dst_dcube);
/* dmodels.hpp:19-23  DModel::dcube_mask(cutoff, apply, size, dcube_d, dcube_m, dcube_w);
 * size = {nx, ny, nz}; every voxel is processed (the reference CUDA driver
 * covers only the first plane, gbkfit_cuda/src/wrapper.cu:42-56) */
int gbkb200_dmodel_dcube_mask_f32(gbkb200_ctx* ctx, float cutoff, int apply, const int size[3],
                                  float* dcube_d, float* dcube_m, float* dcube_w);
/* dmodels.hpp:25-33  DModel::mmaps_moments(size, step, zero, dcube_d, dcube_w,
 * cutoff, norders, orders, mmaps_d, mmaps_m, mmaps_w).  As in the reference
 * native module, the map passed in the mmaps_m position receives the weight
 * map and the one in the mmaps_w position the mask map (the reference kernel
 * swaps them, gbkfit_host/include/gbkfit/host/kernels.hpp:124-131, and its
 * Python wrapper passes (d, w, m), _detail/native.py:280-289).  orders is a
 * device array of norders ascending ints; maps are (norders, ny, nx). */
int gbkb200_dmodel_mmaps_moments_f32(gbkb200_ctx* ctx, const int size[3], const float step[3],
                                     const float zero[3], const float* dcube_d,
                                     const float* dcube_w, float cutoff, int norders,
                                     const int* orders, float* mmaps_d, float* mmaps_m,
                                     float* mmaps_w);

/* ---- GModelf32: gbkfit_host/include/gbkfit/host/gmodels.hpp:8-137 ------ */

/* gmodels.hpp:21-27  GModel::wcube_evaluate(spat_size_x, y, z, spec_size_z, spat, spec) */
int gbkb200_gmodel_wcube_evaluate_f32(gbkb200_ctx* ctx, int spat_size_x, int spat_size_y,
                                      int spat_size_z, int spec_size_z, const float* spat_data,
                                      float* spec_data);

/* The trait-table group of one trait kind, as in the reference:
 * uids, cvalues, ccounts, pvalues, pcounts. */
#define GBKB200_TRAIT_ARGS(p) \
    const int* p##_uids, const float* p##_cvalues, const int* p##_ccounts, \
    const float* p##_pvalues, const int* p##_pcounts

#define GBKB200_DISK_ARGS \
    int loose, int tilted, int nrnodes, const float* rnodes, const float* vsys, \
    const float* xpos, const float* ypos, const float* posa, const float* incl, \
    int nrt, GBKB200_TRAIT_ARGS(rpt), GBKB200_TRAIT_ARGS(rht), \
    int nvt, GBKB200_TRAIT_ARGS(vpt), GBKB200_TRAIT_ARGS(vht), \
    int ndt, GBKB200_TRAIT_ARGS(dpt), GBKB200_TRAIT_ARGS(dht), \
    int nzt, GBKB200_TRAIT_ARGS(zpt), \
    int nst, GBKB200_TRAIT_ARGS(spt), \
    int nwt, GBKB200_TRAIT_ARGS(wpt), \
    const float* opacity, \
    int spat_size_x, int spat_size_y, int spat_size_z, \
    float spat_step_x, float spat_step_y, float spat_step_z, \
    float spat_zero_x, float spat_zero_y, float spat_zero_z, \
    int spec_size, float spec_step, float spec_zero, \
    float* image, float* scube, float* wdata, float* wdata_cmp, \
    float* rdata, float* rdata_cmp, float* ordata, float* ordata_cmp, \
    float* vdata_cmp, float* ddata_cmp

/* gmodels.hpp:82-135  GModel::smdisk_evaluate(loose, tilted, nrnodes, rnodes, ...).
 * image, scube, wdata, rdata, ordata are accumulated into. */
int gbkb200_gmodel_smdisk_evaluate_f32(gbkb200_ctx* ctx, GBKB200_DISK_ARGS);

/* gmodels.hpp:26-79  GModel::mcdisk_evaluate(cflux, nclouds, ncloudscsum,
 * ncloudscsum_len, hasordint, loose, tilted, ...).  hasordint is a device
 * array of one byte per density trait.  Clouds draw from a counter-based
 * Philox-4x32-10 stream keyed by (seed, cloud index), see
 * gbkb200_ctx_set_mcdisk; the reference draws from per-thread mt19937
 * generators that all start from seed 42. */
int gbkb200_gmodel_mcdisk_evaluate_f32(gbkb200_ctx* ctx, float cflux, int nclouds,
                                       const int* ncloudscsum, int ncloudscsum_len,
                                       const unsigned char* hasordint, GBKB200_DISK_ARGS);

/* ---- Objectivef32: gbkfit_host/include/gbkfit/host/objective.hpp:8-21 -- */

/* objective.hpp:15-18  Objective::residual(obs_d, obs_e, obs_m, mdl_d, mdl_w,
 * mdl_m, size, weight, residual) */
int gbkb200_objective_residual_f32(gbkb200_ctx* ctx, const float* obs_d, const float* obs_e,
                                   const float* obs_m, const float* mdl_d, const float* mdl_w,
                                   const float* mdl_m, int size, float weight, float* residual);
/* objective.hpp:20  Objective::residual_sum(residual, size, squared, sum);
 * sum is a device pointer to one float (overwritten).  The reduction is
 * deterministic (fixed tree order, fp32 pairwise + fp64 final), unlike the
 * reference's OpenMP reduction. */
int gbkb200_objective_residual_sum_f32(gbkb200_ctx* ctx, const float* residual, int size,
                                       int squared, float* sum);

/* No counterpart in the reference.  The residual sum of
 * gbkb200_objective_residual_sum_f32 for callers that cannot allocate device
 * memory (a host framework that owns every device byte through its own pool,
 * or a loop that must not allocate after start-up): it needs no context and
 * allocates nothing.  Its block partials live in a fixed 64 KiB device array
 * inside the library, held by every GPU that loads the library until exit.
 * size is limited to 268,435,456 residuals (GBKB200_ERR_TOO_LARGE beyond).
 * The call only enqueues work on `stream` (a cudaStream_t, 0 = legacy
 * default stream) on the current device; sum (one device float) is ready
 * when the stream reaches that point.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  After the device's context is re-created
 * (cudaDeviceReset) the next call looks the address up again, so that
 * call also belongs outside any capture.  All calls share the array: calls
 * that overlap on the GPU race and must be ordered by the caller. */
int gbkb200_objective_residual_sum_noalloc_f32(const float* residual, int size, int squared,
                                               float* sum, void* stream);

/* ---- one serving request in one call (no reference counterpart) --------
 * The chain a serving loop runs per request, enqueued on the context's
 * stream: the packed parameters are copied from pinned host memory
 * (blob_host -> blob_dev, blob_bytes), the model cube (size_hi = padded
 * {px, py, pz}) is zeroed and evaluated by smdisk_evaluate (kind 0) or
 * mcdisk_evaluate (kind 1) with the parameter arrays found at byte offsets
 * into blob_dev (-1 = absent; the trait counts of rht/vht/dht are those of
 * rpt/vpt/dpt, as in GBKB200_DISK_ARGS), convolved with the resident
 * spectrum by fft_convolve (work: complex work space of the padded grid),
 * cropped at edge to size (into crop, when not NULL), compared with the data
 * ((model - obs) / err * msk * weight; err and msk may be NULL) and
 * summed in squares (chi2_dev); chi^2 and the context's kernel status word are
 * then copied to chi2_host and status_host (pinned host memory): the result
 * is there once the stream reaches the end of the call.  A nonzero status
 * stays set in the context until gbkb200_ctx_synchronize clears it. */
typedef struct {
    int kind;
    float cflux;
    int nclouds;
    int loose, tilted;
    void* blob_dev;
    const void* blob_host;
    long long blob_bytes;
    long long off_rnodes;
    int nrnodes;
    long long off_vsys, off_xpos, off_ypos, off_posa, off_incl;
    int ntraits[9];            /* rpt, rht, vpt, vht, dpt, dht, zpt, spt, wpt */
    long long off_uids[9], off_cvalues[9], off_ccounts[9], off_pvalues[9], off_pcounts[9];
    long long off_csum;
    int csum_len;
    long long off_hasordint;
    int spat_size[3];
    float spat_step[3], spat_zero[3];
    int spec_size;
    float spec_step, spec_zero;
    int size_hi[3], edge[3], size[3];
    float* scube;
    void* work;
    const void* spectrum;
    float* crop;
    const float *obs, *err, *msk;
    float weight;
    float* chi2_dev;
    float* chi2_host;
    int* status_host;
} gbkb200_serve_args;

int gbkb200_serve_scube_chi2_f32(gbkb200_ctx* ctx, const gbkb200_serve_args* args);
/* The first half of the chain only: the parameters' copy, the zeroing of
 * the spat_size[0] x spat_size[1] x spec_size cube at scube and its model
 * evaluation (kind 0 smdisk, 1 mcdisk) on the geometry of the arguments;
 * the fields after spec_zero other than scube are not read.  For a model
 * that a batched evaluator convolves (gbkb200_batch_evaluate_cubes). */
int gbkb200_serve_model_f32(gbkb200_ctx* ctx, const gbkb200_serve_args* args);

/* ---- differentiable chi^2 of a thin smooth disk (no reference counterpart:
 *      the reference computes no gradients).  A hand-written adjoint of
 *      smdisk_evaluate + fft_convolve_cached + crop + residual + residual_sum
 *      with a multiplicative scale on the convolved model. ------------------ */

/* One pass over the padded cube conv_p (size_p = {px, py, pz}); its crop
 * [offset, offset + size) is compared with the data (size = {nx, ny, nz}):
 *   r = (scale * conv - d) / e * mask * weight   (objective.hpp:7-31 order)
 * Writes g_p = d(chi^2)/d(conv_p) (0 outside the crop; every voxel is written)
 * and out[0] = chi^2 = sum r^2, out[1] = d(chi^2)/d(scale) (fp64 device
 * values, block partials summed in a fixed order). */
int gbkb200_objective_chi2_adjoint_f32(gbkb200_ctx* ctx, const int size_p[3], const int offset[3],
                                       const int size[3], const float* conv_p, const float* obs_d,
                                       const float* obs_e, const float* obs_m, float weight,
                                       float scale, float* g_p, double* out);

/* A thin disk (neither loose nor tilted) with one node-wise surface
 * brightness (density uid 101), one node-wise rotation curve (velocity uid
 * 101, traits.hpp:999-1007) and one node-wise dispersion (uid 101); the
 * sub-node values are those smdisk_evaluate receives as pvalues. */
typedef struct {
    int spat_size[2];          /* evaluation grid (x, y) */
    float spat_step[2];
    float spat_zero[2];
    int spec_size;
    float spec_step;
    float spec_zero;
    int nsub;
    const float* subrnodes;    /* device (nsub) */
    const float* vsys;         /* device (1), or NULL for 0 */
    const float *xpos, *ypos, *posa, *incl;   /* device (1 each), degrees for angles */
    const float *bsub, *vsub, *dsub;          /* device (nsub each) */
} gbkb200_smdisk_nw_desc;

/* Given g_cube = d(chi^2)/d(scube) on the evaluation grid (spec_size,
 * spat_size[1], spat_size[0]), overwrites grad (device, 3 nsub + 5 doubles)
 * with d(chi^2)/d of: the density sub-node values, the rotation sub-node
 * values, the dispersion sub-node values, vsys, xpos, ypos, posa (per
 * degree), incl (per degree).  Each spaxel recomputes its ring position,
 * interpolation weights and line; the truncation of the line window and the
 * ring boundaries are treated as fixed (derivatives almost everywhere).
 * Fixed-order fp64 sums across blocks; within a block fp64 shared atomics
 * (reproducible to rounding).  nsub <= 2046. */
int gbkb200_gmodel_smdisk_nw_adjoint_f32(gbkb200_ctx* ctx, const gbkb200_smdisk_nw_desc* desc,
                                         const float* g_cube, double* grad);

/* ---- batched evaluation (no reference counterpart as one call) ---------
 *
 * Evaluates many parameter sets of one thin smooth disk against one data
 * cube: per set, what the reference computes with GModel::smdisk_evaluate on
 * the padded DCube grid, FFT::fft_convolve_cached with the PSF x LSF cube,
 * DModel::dcube_downscale (crop), Objective::residual and
 * Objective::residual_sum(squared) (objective/objective.py:187-226).  The
 * model is only evaluated on the window that the crop reads (size +
 * kernel_size - 1 per axis) and the FFT grid is chosen freely (factors 2, 3,
 * 5, 7), which leaves the cropped result unchanged.  Kernel truncation:
 * only the kernel_size box of the PSF x LSF cube is used (the reference's
 * one-sided LSF truncation keeps a negative tail beyond it, below 1e-14 of the
 * peak for a Gaussian LSF). */

typedef struct gbkb200_batch gbkb200_batch;

/* trait-kind order of the arrays below: rpt, rht, vpt, vht, dpt, dht, zpt,
 * spt, wpt (rht must be absent: thin disks) */
typedef struct {
    int size[3];            /* data cube (nx, ny, nz) */
    int kernel_size[3];     /* PSF box (x, y) and LSF box (z), odd */
    int fft_size[3];        /* FFT grid >= size + kernel_size - 1; 0 = automatic */
    float spat_step[2];     /* evaluation grid step (x, y) */
    float spat_zero[2];     /* evaluation grid zero (DCube scratch zero, x, y) */
    float spec_step;
    float spec_zero;        /* DCube scratch zero along the spectral axis */
    int loose, tilted, nrnodes;
    const float* rnodes;    /* device: sub-nodes */
    int ntraits[9];
    const int* uids[9];     /* device */
    const float* cvalues[9];
    const int* ccounts[9];
    const int* pcounts[9];
    int npvalues[9];        /* parameter values per set, per kind */
    const double* psf;      /* host: (kernel_size[1], kernel_size[0]) PSF image, centred */
    const double* lsf;      /* host: kernel_size[2] LSF, centred */
    const float* obs_d;     /* device: data (nz, ny, nx) */
    const float* obs_e;     /* device: errors, or NULL */
    const float* obs_m;     /* device: mask, or NULL */
    float weight;
    int max_sets;           /* largest nsets of an evaluate call */
    int chunk;              /* sets per pipeline wave (0 = 8) */
    int rows_k1;            /* spectral rows per shared-memory group of the model kernel (0 = 16) */
    int rows_k5;            /* rows per block of the residual kernel (0 = 8) */
    int conv_mode;          /* 0 = automatic, 1 = FFT, 2 = direct separable FIR */
    int psf_rank;           /* direct mode: PSF = sum_r u_r(y) v_r(x), rank <= 8 */
    const double* psf_u;    /* host: (psf_rank, kernel_size[1]) */
    const double* psf_v;    /* host: (psf_rank, kernel_size[0]) */
    int psf_band;           /* direct mode: output rows per PSF block (0 = automatic) */
    int psf_variant;        /* direct mode: PSF kernel variant 0-7: resident blocks per SM
                             * (0-2: 4, 3-5: 5) x epilogue (variant % 3: 0 residual pass,
                             * 1 residual in the y-FIR items, 2 as 1 with the data
                             * prefetched); 6 = 0 as a persistent kernel (one resident
                             * wave of blocks over all items, each item's range entries
                             * copied in while the previous item runs); 7 = 0 on
                             * 256-thread blocks with twice the shared memory (2 blocks
                             * per SM); 0 = the first */
    int model_variant;      /* direct mode, the model kernel (0-3 give the same values):
                             * 0 = a warp per 32-column chunk stepping every lane through
                             * the union of the lanes' channel windows; 1 = two chunks per
                             * warp on packed FP32 pairs; 2 = a warp per 4 x 8 spaxel tile
                             * (shorter channel unions); 3 = 2 with the range-table masks
                             * from one bit transpose per 32 planes instead of a ballot
                             * per plane; 4 = 3 with the line's exponent as -t^2, t one
                             * multiply-add per channel (the same values up to fp32
                             * rounding) */
} gbkb200_batch_desc;

int gbkb200_batch_create(gbkb200_ctx* ctx, const gbkb200_batch_desc* desc, gbkb200_batch** out);
/* chi2[s] = sum over voxels of residual^2 for set s (device, nsets floats).
 * Per-set inputs are device arrays of nsets rows: vsys, xpos, ypos, posa,
 * incl (1 or nrnodes values per set) and pvalues[k] (npvalues[k] per set).
 * model: optional device (nsets, nz, ny, nx) output of the cropped model. */
int gbkb200_batch_evaluate(gbkb200_batch* b, int nsets, const float* vsys, const float* xpos,
                           const float* ypos, const float* posa, const float* incl,
                           const float* const pvalues[9], float* chi2, float* model);
/* Direct mode: the evaluation window of the model, as the voxel offset of
 * its first voxel in the padded (high-resolution) grid whose zero the
 * descriptor gives, and its size {Wx, Wy, Wz} = data size + FIR lengths - 1
 * (GBKB200_ERR_UNSUPPORTED in FFT mode). */
int gbkb200_batch_window(const gbkb200_batch* b, int offset[3], int size[3]);
/* Direct mode: chi2[s] of given model cubes instead of the evaluator's disk
 * (any gmodel's output sampled on the window: cubes is device (nsets, Wz,
 * Wy, Wx)), through the same LSF FIR, PSF FIR, residual and sum; model as
 * in gbkb200_batch_evaluate (GBKB200_ERR_UNSUPPORTED in FFT mode). */
int gbkb200_batch_evaluate_cubes(gbkb200_batch* b, int nsets, const float* cubes, float* chi2,
                                 float* model);
/* Asynchronous submission (no reference counterpart; the serving loop's
 * launch): copies in_bytes of packed per-set inputs from pinned host memory
 * (in_host) to in_dev, evaluates nsets sets as gbkb200_batch_evaluate (the
 * per-set input pointers point into in_dev), copies chi2 to chi2_host
 * (pinned, nsets floats) and records the evaluator's completion event, all
 * on the context's stream; gbkb200_batch_submit_cubes does the same for
 * given model cubes (gbkb200_batch_evaluate_cubes).  gbkb200_batch_query
 * sets *done to 1 once the last submission has completed (chi2_host is then
 * valid), else 0; one submission may be in flight per evaluator. */
int gbkb200_batch_submit(gbkb200_batch* b, int nsets, const void* in_host, void* in_dev,
                         size_t in_bytes, const float* vsys, const float* xpos, const float* ypos,
                         const float* posa, const float* incl, const float* const pvalues[9],
                         float* chi2_dev, float* chi2_host);
int gbkb200_batch_submit_cubes(gbkb200_batch* b, int nsets, const float* cubes, float* chi2_dev,
                               float* chi2_host);
int gbkb200_batch_query(const gbkb200_batch* b, int* done);
/* after the last submission completed: GBKB200_OK, or the error of the status
 * word its kernels raised (GBKB200_ERR_BAD_TRAIT: a model of the submission
 * met an unknown trait uid), which is then cleared */
int gbkb200_batch_take_status(gbkb200_batch* b);
/* the chosen FFT grid, chunk, the device bytes the evaluator holds (its
 * work space, tables and partials) and the convolution mode (1 = FFT,
 * 2 = direct) */
int gbkb200_batch_info(const gbkb200_batch* b, int fft_size[3], int* chunk, size_t* work_bytes,
                       int* conv_mode);
int gbkb200_batch_destroy(gbkb200_batch* b);

/* The batched evaluator's input rows from raw node values, on the device
 * (replaces the host packing of the trait parameter arrays,
 * gmodels/_disk.py:42-156, when the node -> sub-node interpolation is
 * linear): for sets b < nsets and columns j < width,
 *   out[base[j] + b stride[j]] = (float)(w0[j] raw[b raw_width + k0[j]]
 *                                        + w1[j] raw[b raw_width + k1[j]])
 * in fp64.  raw, the tables and out are device memory; enqueued on stream
 * (a cudaStream_t), nothing is synchronised or allocated. */
int gbkb200_rows_from_nodes(const double* raw, int raw_width, int nsets, const int* k0,
                            const int* k1, const double* w0, const double* w1,
                            const long long* base, const int* stride, int width, float* out,
                            void* stream);

/* Per-stage device timing (no reference counterpart; a measurement aid).
 * With timing enabled, evaluate records a CUDA event pair around every kernel
 * launch; do not capture evaluate into a graph while it is enabled.  Stages:
 * 0 model + lines (direct: LSF FIR too; FFT: x r2c), 1 y FFT, 2 z FFT
 * convolution, 3 inverse y FFT (FFT mode only), 4 PSF FIR or
 * x c2r + residual, 5 chi^2 sum.
 * enable: 0 off, 1 timing and the work counters below, 2 timing alone (the
 * kernels then run without the counters' atomic adds, as in a graph replay).
 * gbkb200_batch_timing synchronizes the stream, returns the summed
 * milliseconds and launch counts per stage since the last call, and resets. */
#define GBKB200_BATCH_STAGES 6
int gbkb200_batch_set_timing(gbkb200_batch* b, int enable);
int gbkb200_batch_timing(gbkb200_batch* b, double ms[GBKB200_BATCH_STAGES],
                         int launches[GBKB200_BATCH_STAGES]);
/* Executed-work counters of the direct-mode kernels (no reference
 * counterpart; a measurement aid), counted while timing mode 1 is enabled:
 * [0] LSF FIR multiply-adds, [1] line values (one exponential each),
 * [2] PSF x FIR multiply-adds, [3] PSF y FIR multiply-adds, [4] residual
 * voxels computed from the model box, [5] spaxel evaluations (one
 * multiply-add is one lane's fused multiply-add).  Synchronizes the stream,
 * returns the sums since the last call and resets them; all zero in FFT
 * mode. */
#define GBKB200_BATCH_COUNTERS 8
int gbkb200_batch_counters(gbkb200_batch* b, unsigned long long out[GBKB200_BATCH_COUNTERS]);

#ifdef __cplusplus
}
#endif

#endif /* GBKB200_H */
