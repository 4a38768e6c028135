// Explicit instantiations of the batched PSF kernel sized for 4 resident
// blocks per SM (one translation unit per group, so that the library compiles
// in parallel).
#include "gbk_batched.cuh"

namespace gbk {

void kb_register(KbFn* t)
{
    t[0] = kb_psf_residual<5, 4>;
    t[1] = kb_psf_residual<7, 4>;
    t[2] = kb_psf_residual<9, 4>;
    t[3] = kb_psf_residual<11, 4>;
    t[4] = kb_psf_residual<13, 4>;
    t[5] = kb_psf_residual<15, 4>;
    t[6] = kb_psf_residual<17, 4>;
    t[7] = kb_psf_residual<19, 4>;
    t[8] = kb_psf_residual<21, 4>;
    t[9] = kb_psf_residual<23, 4>;
    t[10] = kb_psf_residual<25, 4>;
    t[11] = kb_psf_residual<27, 4>;
    t[12] = kb_psf_residual<29, 4>;
    t[13] = kb_psf_residual<31, 4>;
    t[14] = kb_psf_residual<33, 4>;
}

}  // namespace gbk
