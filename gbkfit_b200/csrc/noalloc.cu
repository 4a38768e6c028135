// Residual sum that allocates nothing: a variant of
// gbkb200_objective_residual_sum_f32 for callers that cannot allocate device
// memory.  Such callers include host frameworks that own every device byte
// through their own pool or arena and forbid allocations behind their back,
// and long-running loops that must not allocate after start-up, because
// cudaMalloc can synchronize the device and its failures surface at
// unpredictable times.
//
// The block partials live in a file-scope device array of fixed size
// (NOALLOC_MAX_PARTIALS doubles, 64 KiB), which every GPU that loads the
// library keeps until the process exits.  One partial covers
// NOALLOC_PER_BLOCK residuals, so a call takes at most
// NOALLOC_MAX_PARTIALS * NOALLOC_PER_BLOCK = 268,435,456 residuals; larger
// sizes are rejected with GBKB200_ERR_TOO_LARGE before anything is launched.
//
// Every call on a device shares that device's array and leaves its partials
// in it.  Each call writes every partial it reads before reading it, so
// nothing has to be cleared between calls; but calls that overlap on the
// GPU (for instance on two streams) race on the array and must be ordered
// by the caller.
#include "gbk_common.cuh"

#include <cuda.h>

#include <mutex>

namespace {

constexpr int NOALLOC_THREADS = 512;
constexpr int NOALLOC_ITEMS = 64;                                  // per thread
constexpr int NOALLOC_PER_BLOCK = NOALLOC_THREADS * NOALLOC_ITEMS; // 32768
constexpr int NOALLOC_MAX_PARTIALS = 8192;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_PARTIALS];

// Device address of g_noalloc_partials per device, looked up once per device
// and context (cudaGetSymbolAddress with that device current).  The name of
// the array is only a host-side stand-in in host code; kernels get this
// address.  The context it was looked up in is kept beside it: when the
// device's context is re-created (after cudaDeviceReset) the address is
// looked up again instead of pointing into the old context.
struct PartialsAddr {
    CUcontext ctx;
    double* addr;
};
PartialsAddr g_partials_addr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_setup_mutex;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

// cuCtxGetCurrent through the runtime's driver entry point (no link-time
// dependency on the driver library); null where it cannot be resolved
CtxGetCurrentFn ctx_get_current()
{
    static const CtxGetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<CtxGetCurrentFn>(nullptr);
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    return fn;
}

CUcontext current_context()
{
    CUcontext c = nullptr;
    const CtxGetCurrentFn fn = ctx_get_current();
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block b sums residuals [b * PER_BLOCK, (b + 1) * PER_BLOCK) in fp32 (fixed
// per-thread strides, warp shuffles) and stores the block total as a double.
__global__ void __launch_bounds__(NOALLOC_THREADS)
noalloc_partial(const float* r, int n, int squared, double* part)
{
    __shared__ float ws[NOALLOC_THREADS / 32];
    const long long base = (long long)blockIdx.x * NOALLOC_PER_BLOCK;
    float acc = 0.f;
#pragma unroll 4
    for (int k = 0; k < NOALLOC_ITEMS; ++k) {
        long long i = base + (long long)k * NOALLOC_THREADS + threadIdx.x;
        if (i < n) {
            float v = r[i];
            acc += squared ? v * v : fabsf(v);
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < NOALLOC_THREADS / 32 ? ws[threadIdx.x] : 0.f;
        v = warp_sum(v);
        if (threadIdx.x == 0) part[blockIdx.x] = (double)v;
    }
}

// One block adds the nparts partials in index order (fp64) and writes the sum.
__global__ void noalloc_final(const double* part, int nparts, float* out)
{
    if (threadIdx.x == 0) {
        double s = 0;
        for (int i = 0; i < nparts; ++i) s += part[i];
        out[0] = (float)s;
    }
}

int partials_address(double** out)
{
    int dev = 0;
    GBK_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return GBKB200_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    PartialsAddr& e = g_partials_addr[dev];
    if (!e.addr || current_context() != e.ctx) {
        void* p = nullptr;
        GBK_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_partials));   // makes the context current
        e.ctx = current_context();
        e.addr = static_cast<double*>(p);
    }
    *out = e.addr;
    return GBKB200_OK;
}

}  // namespace

extern "C" int gbkb200_objective_residual_sum_noalloc_f32(const float* residual, int size,
                                                          int squared, float* sum, void* stream)
{
    if (!sum || size < 0 || (size > 0 && !residual)) return GBKB200_ERR_INVALID_ARG;
    const long long nparts = ((long long)size + NOALLOC_PER_BLOCK - 1) / NOALLOC_PER_BLOCK;
    if (nparts > NOALLOC_MAX_PARTIALS) return GBKB200_ERR_TOO_LARGE;
    double* part = nullptr;
    int rc = partials_address(&part);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (nparts > 0)
        noalloc_partial<<<(int)nparts, NOALLOC_THREADS, 0, st>>>(residual, size, squared, part);
    noalloc_final<<<1, 32, 0, st>>>(part, (int)nparts, sum);
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}
