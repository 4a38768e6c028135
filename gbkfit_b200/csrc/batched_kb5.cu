// Explicit instantiations of the batched PSF kernel sized for 5 resident
// blocks per SM, every epilogue variant (one translation unit per group, so
// that the library compiles in parallel).
#include "gbk_batched.cuh"

namespace gbk {

void kb_register5(KbFn (*t)[(KB_KMAX - KB_KMIN) / 2 + 1])
{
    t[0][0] = kb_psf_residual<5, 5, 0, false, KB_THREADS>;
    t[0][1] = kb_psf_residual<7, 5, 0, false, KB_THREADS>;
    t[0][2] = kb_psf_residual<9, 5, 0, false, KB_THREADS>;
    t[0][3] = kb_psf_residual<11, 5, 0, false, KB_THREADS>;
    t[0][4] = kb_psf_residual<13, 5, 0, false, KB_THREADS>;
    t[0][5] = kb_psf_residual<15, 5, 0, false, KB_THREADS>;
    t[0][6] = kb_psf_residual<17, 5, 0, false, KB_THREADS>;
    t[0][7] = kb_psf_residual<19, 5, 0, false, KB_THREADS>;
    t[0][8] = kb_psf_residual<21, 5, 0, false, KB_THREADS>;
    t[0][9] = kb_psf_residual<23, 5, 0, false, KB_THREADS>;
    t[0][10] = kb_psf_residual<25, 5, 0, false, KB_THREADS>;
    t[0][11] = kb_psf_residual<27, 5, 0, false, KB_THREADS>;
    t[0][12] = kb_psf_residual<29, 5, 0, false, KB_THREADS>;
    t[0][13] = kb_psf_residual<31, 5, 0, false, KB_THREADS>;
    t[0][14] = kb_psf_residual<33, 5, 0, false, KB_THREADS>;
    t[1][0] = kb_psf_residual<5, 5, 1, false, KB_THREADS>;
    t[1][1] = kb_psf_residual<7, 5, 1, false, KB_THREADS>;
    t[1][2] = kb_psf_residual<9, 5, 1, false, KB_THREADS>;
    t[1][3] = kb_psf_residual<11, 5, 1, false, KB_THREADS>;
    t[1][4] = kb_psf_residual<13, 5, 1, false, KB_THREADS>;
    t[1][5] = kb_psf_residual<15, 5, 1, false, KB_THREADS>;
    t[1][6] = kb_psf_residual<17, 5, 1, false, KB_THREADS>;
    t[1][7] = kb_psf_residual<19, 5, 1, false, KB_THREADS>;
    t[1][8] = kb_psf_residual<21, 5, 1, false, KB_THREADS>;
    t[1][9] = kb_psf_residual<23, 5, 1, false, KB_THREADS>;
    t[1][10] = kb_psf_residual<25, 5, 1, false, KB_THREADS>;
    t[1][11] = kb_psf_residual<27, 5, 1, false, KB_THREADS>;
    t[1][12] = kb_psf_residual<29, 5, 1, false, KB_THREADS>;
    t[1][13] = kb_psf_residual<31, 5, 1, false, KB_THREADS>;
    t[1][14] = kb_psf_residual<33, 5, 1, false, KB_THREADS>;
    t[2][0] = kb_psf_residual<5, 5, 2, false, KB_THREADS>;
    t[2][1] = kb_psf_residual<7, 5, 2, false, KB_THREADS>;
    t[2][2] = kb_psf_residual<9, 5, 2, false, KB_THREADS>;
    t[2][3] = kb_psf_residual<11, 5, 2, false, KB_THREADS>;
    t[2][4] = kb_psf_residual<13, 5, 2, false, KB_THREADS>;
    t[2][5] = kb_psf_residual<15, 5, 2, false, KB_THREADS>;
    t[2][6] = kb_psf_residual<17, 5, 2, false, KB_THREADS>;
    t[2][7] = kb_psf_residual<19, 5, 2, false, KB_THREADS>;
    t[2][8] = kb_psf_residual<21, 5, 2, false, KB_THREADS>;
    t[2][9] = kb_psf_residual<23, 5, 2, false, KB_THREADS>;
    t[2][10] = kb_psf_residual<25, 5, 2, false, KB_THREADS>;
    t[2][11] = kb_psf_residual<27, 5, 2, false, KB_THREADS>;
    t[2][12] = kb_psf_residual<29, 5, 2, false, KB_THREADS>;
    t[2][13] = kb_psf_residual<31, 5, 2, false, KB_THREADS>;
    t[2][14] = kb_psf_residual<33, 5, 2, false, KB_THREADS>;
}

}  // namespace gbk
