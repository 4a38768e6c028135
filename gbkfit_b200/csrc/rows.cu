// The batched evaluator's per-set input rows from the raw node values, on the
// device: the node -> sub-node interpolation and row assembly that the host
// packing does (gmodels/_disk.py:42-156, the trait parameter arrays of
// Disk.evaluate) when the interpolation is linear.  Each output value is then
// a fixed combination of at most two raw values of its set,
//   out = w0 raw[k0] + w1 raw[k1]   (fp64, rounded once to fp32),
// the two interpolation weights of a node-wise parameter's sub-node (1 and 0
// for a value copied as it is), with a host-built table per output column.
#include "gbk_common.cuh"

#include <algorithm>

namespace {

// one thread per (set, column); sets of the batch in blockIdx.y
__global__ void k_rows_from_nodes(const double* __restrict__ raw, int R, int B,
                                  const int* __restrict__ k0, const int* __restrict__ k1,
                                  const double* __restrict__ w0, const double* __restrict__ w1,
                                  const long long* __restrict__ base,
                                  const int* __restrict__ stride, int W, float* __restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= W) return;
    for (int b = blockIdx.y; b < B; b += gridDim.y) {
        const double* r = raw + (long long)b * R;
        const double v = w0[j] * r[k0[j]] + w1[j] * r[k1[j]];
        out[base[j] + (long long)b * stride[j]] = (float)v;
    }
}

}  // namespace

extern "C" int gbkb200_rows_from_nodes(const double* raw, int raw_width, int nsets,
                                       const int* k0, const int* k1, const double* w0,
                                       const double* w1, const long long* base,
                                       const int* stride, int width, float* out, void* stream)
{
    if (nsets < 0 || raw_width < 1 || width < 0) return GBKB200_ERR_INVALID_ARG;
    if (nsets == 0 || width == 0) return GBKB200_OK;
    if (!raw || !k0 || !k1 || !w0 || !w1 || !base || !stride || !out)
        return GBKB200_ERR_INVALID_ARG;
    const int threads = 128;
    const dim3 grid((width + threads - 1) / threads, (unsigned)std::min(nsets, 65535));
    k_rows_from_nodes<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        raw, raw_width, nsets, k0, k1, w0, w1, base, stride, width, out);
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}
