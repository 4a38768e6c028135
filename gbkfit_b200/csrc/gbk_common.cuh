// Shared definitions of the gbkfit_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/gbkb200.h"

#define GBK_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) {                             \
            gbk_set_last_cuda_error(e_);                     \
            return GBKB200_ERR_CUDA;                         \
        }                                                    \
    } while (0)

void gbk_set_last_cuda_error(cudaError_t e);

// Bits of the per-context device status word that kernels may raise.
enum : int {
    GBK_STATUS_BAD_TRAIT = 1,      // unknown trait uid (reference: NaN + assert)
    GBK_STATUS_TIMEOUT = 2,        // a bounded wait gave up
    GBK_STATUS_BAD_INDEX = 4,      // a self-check found an out-of-range index
};

constexpr float GBK_PI = 3.14159265358979323846f;
constexpr float GBK_D2R = GBK_PI / 180.0f;
constexpr int GBK_TRAIT_NUM_MAX = 4;   // constants.hpp:8
constexpr float GBK_LINE_WIDTH = 5.0f; // constants.hpp:5-6

// One trait kind's tables, as the reference passes them: uids, constants,
// constant counts, parameters, parameter counts (gmodel/gmodels.hpp:336-368).
struct TraitSet {
    int n;
    const int* uids;
    const float* cv;
    const int* cc;
    const float* pv;
    const int* pc;
};

// Everything one smdisk/mcdisk call receives, bundled into one kernel
// parameter (the reference passes ~90 arguments,
// gbkfit_host/include/gbkfit/host/gmodels.hpp:26-135).
struct DiskArgs {
    int loose, tilted, nrnodes;
    const float *rnodes, *vsys, *xpos, *ypos, *posa, *incl;
    TraitSet rpt, rht, vpt, vht, dpt, dht, zpt, spt, wpt;
    const float* opacity;
    int sx, sy, sz;
    float stx, sty, stz, zx, zy, zz;
    int spec_size;
    float spec_step, spec_zero;
    float *image, *scube, *wdata, *wdata_cmp, *rdata, *rdata_cmp;
    float *ordata, *ordata_cmp, *vdata_cmp, *ddata_cmp;
};

struct McArgs {
    float cflux;
    int nclouds;
    const int* csum;
    int csum_len;
    const unsigned char* hasordint;
    unsigned long long seed;
};

// Execution context behind the opaque gbkb200_ctx handle.
struct gbkb200_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sync = 1;
    unsigned long long seed = 42;
    int mc_mode = 0;
    int* d_status = nullptr;      // device status word (GBK_STATUS_* bits)
    int* h_status = nullptr;      // pinned mirror
    void* fft_state = nullptr;    // FFT plan / spectrum caches (fft.cu)
    void* reduce_scratch = nullptr;
    size_t reduce_scratch_bytes = 0;
    void* mc_scratch = nullptr;     // fixed-point accumulators of deterministic mcdisk
    size_t mc_scratch_bytes = 0;
    void* serve_scratch = nullptr;  // block partials + last-block counter (serve.cu)
};

int gbk_finish(gbkb200_ctx* ctx);   // launch check, and sync + status read in sync mode
// Raises kernel fn's dynamic shared-memory limit on the current device to at
// least `bytes`, never lowering it: the limit is one setting per function,
// shared by every evaluator and context of the process, so a smaller later
// request must not cut under a larger earlier one.
int gbk_raise_smem_limit(const void* fn, size_t bytes);
int gbk_fft_state_destroy(gbkb200_ctx* ctx);

// Debug builds (-DGBK_CHECKED) bounds-check the accesses of the batched and
// FFT kernels: the first out-of-range (site, index, limit) is recorded in
// gbk_debug_record and the access is skipped.  Release builds compile the
// checks away.
#ifdef GBK_CHECKED
// one record per translation unit (no relocatable device code)
static __device__ long long gbk_debug_record[4];
__device__ inline bool gbk_in_range(long long i, long long n, int site)
{
    if (i >= 0 && i < n) return true;
    if (atomicCAS(reinterpret_cast<unsigned long long*>(&gbk_debug_record[0]), 0ull,
                  (unsigned long long)site) == 0ull) {
        gbk_debug_record[1] = i;
        gbk_debug_record[2] = n;
        gbk_debug_record[3] = blockIdx.x + 65536ll * blockIdx.y;
    }
    return false;
}
#define GBK_OK_IDX(i, n, site) gbk_in_range((long long)(i), (long long)(n), (site))
#else
#define GBK_OK_IDX(i, n, site) true
#endif

__host__ __device__ inline long long idx3(int x, int y, int z, int nx, int ny)
{
    return (long long)x + (long long)nx * ((long long)y + (long long)ny * z);
}
