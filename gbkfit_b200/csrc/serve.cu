// One serving request in one call (no reference counterpart): the chain the
// serving loop runs per request, on the context's stream, composed from the
// library's own entry points: the request's packed parameters are copied
// from pinned host memory, the model cube is zeroed and evaluated (smdisk
// or mcdisk, gmodels.hpp), convolved with the dataset's resident PSF x LSF
// spectrum (fft.hpp:87-96), cropped (dmodels.hpp:7-46), its residual and
// sum of squares taken (objective.hpp:7-31, host/kernels.hpp:502-514), and
// chi^2 and the context's kernel status word are copied to pinned host
// memory, so that the caller sees the result without another CUDA call.
#include "gbk_common.cuh"

extern "C" int gbkb200_serve_scube_chi2_f32(gbkb200_ctx* ctx, const gbkb200_serve_args* a)
{
    if (!ctx || !a || !a->blob_dev || !a->scube || !a->work || !a->spectrum || !a->crop ||
        !a->res || !a->obs || !a->chi2_dev || !a->chi2_host || !a->status_host)
        return GBKB200_ERR_INVALID_ARG;
    if (a->kind != 0 && a->kind != 1) return GBKB200_ERR_INVALID_ARG;
    for (int k = 0; k < 3; ++k)
        if (a->size_hi[k] < 1 || a->size[k] < 1 || a->edge[k] < 0 ||
            a->edge[k] + a->size[k] > a->size_hi[k])
            return GBKB200_ERR_INVALID_ARG;
    char* base = static_cast<char*>(a->blob_dev);
    auto at = [&](long long off) -> char* { return off < 0 ? nullptr : base + off; };
    const cudaStream_t st = ctx->stream;
    if (a->blob_bytes > 0) {
        if (!a->blob_host) return GBKB200_ERR_INVALID_ARG;
        GBK_CUDA_TRY(cudaMemcpyAsync(a->blob_dev, a->blob_host, (size_t)a->blob_bytes,
                                     cudaMemcpyHostToDevice, st));
    }
    const long long vhi = (long long)a->size_hi[0] * a->size_hi[1] * a->size_hi[2];
    GBK_CUDA_TRY(cudaMemsetAsync(a->scube, 0, (size_t)vhi * sizeof(float), st));
#define GBK_T(k)                                                                                 \
    reinterpret_cast<const int*>(at(a->off_uids[k])),                                            \
        reinterpret_cast<const float*>(at(a->off_cvalues[k])),                                   \
        reinterpret_cast<const int*>(at(a->off_ccounts[k])),                                     \
        reinterpret_cast<const float*>(at(a->off_pvalues[k])),                                   \
        reinterpret_cast<const int*>(at(a->off_pcounts[k]))
#define GBK_SERVE_DISK                                                                           \
    a->loose, a->tilted, a->nrnodes, reinterpret_cast<const float*>(at(a->off_rnodes)),          \
        reinterpret_cast<const float*>(at(a->off_vsys)),                                         \
        reinterpret_cast<const float*>(at(a->off_xpos)),                                         \
        reinterpret_cast<const float*>(at(a->off_ypos)),                                         \
        reinterpret_cast<const float*>(at(a->off_posa)),                                         \
        reinterpret_cast<const float*>(at(a->off_incl)), a->ntraits[0], GBK_T(0), GBK_T(1),    \
        a->ntraits[2], GBK_T(2), GBK_T(3), a->ntraits[4], GBK_T(4), GBK_T(5), a->ntraits[6],    \
        GBK_T(6), a->ntraits[7], GBK_T(7), a->ntraits[8], GBK_T(8), nullptr, a->spat_size[0],  \
        a->spat_size[1], a->spat_size[2], a->spat_step[0], a->spat_step[1], a->spat_step[2],    \
        a->spat_zero[0], a->spat_zero[1], a->spat_zero[2], a->spec_size, a->spec_step,          \
        a->spec_zero, nullptr, a->scube, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,  \
        nullptr, nullptr
    int rc;
    if (a->kind == 0)
        rc = gbkb200_gmodel_smdisk_evaluate_f32(ctx, GBK_SERVE_DISK);
    else
        rc = gbkb200_gmodel_mcdisk_evaluate_f32(
            ctx, a->cflux, a->nclouds, reinterpret_cast<const int*>(at(a->off_csum)), a->csum_len,
            reinterpret_cast<const unsigned char*>(at(a->off_hasordint)), GBK_SERVE_DISK);
#undef GBK_SERVE_DISK
#undef GBK_T
    if (rc) return rc;
    if ((rc = gbkb200_fft_convolve_f32(ctx, a->size_hi, a->scube, a->work, a->spectrum))) return rc;
    const int one[3] = {1, 1, 1};
    if ((rc = gbkb200_dmodel_dcube_downscale_f32(ctx, one, a->edge, a->size_hi, a->size, a->scube,
                                                 a->crop)))
        return rc;
    const int n = a->size[0] * a->size[1] * a->size[2];
    if ((rc = gbkb200_objective_residual_f32(ctx, a->obs, a->err, a->msk, a->crop, nullptr,
                                             nullptr, n, a->weight, a->res)))
        return rc;
    if ((rc = gbkb200_objective_residual_sum_f32(ctx, a->res, n, 1, a->chi2_dev))) return rc;
    GBK_CUDA_TRY(cudaMemcpyAsync(a->chi2_host, a->chi2_dev, sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
    GBK_CUDA_TRY(cudaMemcpyAsync(a->status_host, ctx->d_status, sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
    GBK_CUDA_TRY(cudaGetLastError());
    return GBKB200_OK;
}
