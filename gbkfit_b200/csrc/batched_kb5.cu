// Explicit instantiations of the batched PSF kernel sized for 5 resident
// blocks per SM (one translation unit per group, so that the library compiles
// in parallel).
#include "gbk_batched.cuh"

namespace gbk {

void kb_register5(KbFn* t)
{
    t[0] = kb_psf_residual<5, 5>;
    t[1] = kb_psf_residual<7, 5>;
    t[2] = kb_psf_residual<9, 5>;
    t[3] = kb_psf_residual<11, 5>;
    t[4] = kb_psf_residual<13, 5>;
    t[5] = kb_psf_residual<15, 5>;
    t[6] = kb_psf_residual<17, 5>;
    t[7] = kb_psf_residual<19, 5>;
    t[8] = kb_psf_residual<21, 5>;
    t[9] = kb_psf_residual<23, 5>;
    t[10] = kb_psf_residual<25, 5>;
    t[11] = kb_psf_residual<27, 5>;
    t[12] = kb_psf_residual<29, 5>;
    t[13] = kb_psf_residual<31, 5>;
    t[14] = kb_psf_residual<33, 5>;
}

}  // namespace gbk
