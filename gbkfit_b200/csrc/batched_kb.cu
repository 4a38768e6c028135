// Explicit instantiations of the batched PSF kernel (one translation unit
// per group, so that the library compiles in parallel).
#include "gbk_batched.cuh"

namespace gbk {

void kb_register(KbFn* t)
{
    t[0] = kb_psf_residual<5>;
    t[1] = kb_psf_residual<7>;
    t[2] = kb_psf_residual<9>;
    t[3] = kb_psf_residual<11>;
    t[4] = kb_psf_residual<13>;
    t[5] = kb_psf_residual<15>;
    t[6] = kb_psf_residual<17>;
    t[7] = kb_psf_residual<19>;
    t[8] = kb_psf_residual<21>;
    t[9] = kb_psf_residual<23>;
    t[10] = kb_psf_residual<25>;
    t[11] = kb_psf_residual<27>;
    t[12] = kb_psf_residual<29>;
    t[13] = kb_psf_residual<31>;
    t[14] = kb_psf_residual<33>;
}

}  // namespace gbk
