// Explicit instantiations of the persistent form of the batched PSF kernel
// (4 resident blocks per SM, residual pass; range entries prefetched), one
// per odd PSF length.
#include "gbk_batched.cuh"

namespace gbk {

void kb_register_pf(KbFn (*t)[(KB_KMAX - KB_KMIN) / 2 + 1])
{
    t[0][0] = kb_psf_residual<5, 4, 0, true, KB_THREADS>;
    t[0][1] = kb_psf_residual<7, 4, 0, true, KB_THREADS>;
    t[0][2] = kb_psf_residual<9, 4, 0, true, KB_THREADS>;
    t[0][3] = kb_psf_residual<11, 4, 0, true, KB_THREADS>;
    t[0][4] = kb_psf_residual<13, 4, 0, true, KB_THREADS>;
    t[0][5] = kb_psf_residual<15, 4, 0, true, KB_THREADS>;
    t[0][6] = kb_psf_residual<17, 4, 0, true, KB_THREADS>;
    t[0][7] = kb_psf_residual<19, 4, 0, true, KB_THREADS>;
    t[0][8] = kb_psf_residual<21, 4, 0, true, KB_THREADS>;
    t[0][9] = kb_psf_residual<23, 4, 0, true, KB_THREADS>;
    t[0][10] = kb_psf_residual<25, 4, 0, true, KB_THREADS>;
    t[0][11] = kb_psf_residual<27, 4, 0, true, KB_THREADS>;
    t[0][12] = kb_psf_residual<29, 4, 0, true, KB_THREADS>;
    t[0][13] = kb_psf_residual<31, 4, 0, true, KB_THREADS>;
    t[0][14] = kb_psf_residual<33, 4, 0, true, KB_THREADS>;
}

}  // namespace gbk
