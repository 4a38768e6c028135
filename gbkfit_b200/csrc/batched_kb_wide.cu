// Explicit instantiations of the batched PSF kernel on 256-thread blocks with
// twice the shared memory (2 resident blocks per SM: a whole band in one pass,
// fewer halo rows), one per odd PSF length.
#include "gbk_batched.cuh"

namespace gbk {

void kb_register_wide(KbFn (*t)[(KB_KMAX - KB_KMIN) / 2 + 1])
{
    t[0][0] = kb_psf_residual<5, 2, 0, false, 256>;
    t[0][1] = kb_psf_residual<7, 2, 0, false, 256>;
    t[0][2] = kb_psf_residual<9, 2, 0, false, 256>;
    t[0][3] = kb_psf_residual<11, 2, 0, false, 256>;
    t[0][4] = kb_psf_residual<13, 2, 0, false, 256>;
    t[0][5] = kb_psf_residual<15, 2, 0, false, 256>;
    t[0][6] = kb_psf_residual<17, 2, 0, false, 256>;
    t[0][7] = kb_psf_residual<19, 2, 0, false, 256>;
    t[0][8] = kb_psf_residual<21, 2, 0, false, 256>;
    t[0][9] = kb_psf_residual<23, 2, 0, false, 256>;
    t[0][10] = kb_psf_residual<25, 2, 0, false, 256>;
    t[0][11] = kb_psf_residual<27, 2, 0, false, 256>;
    t[0][12] = kb_psf_residual<29, 2, 0, false, 256>;
    t[0][13] = kb_psf_residual<31, 2, 0, false, 256>;
    t[0][14] = kb_psf_residual<33, 2, 0, false, 256>;
}

}  // namespace gbk
