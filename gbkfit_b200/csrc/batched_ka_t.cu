// Explicit instantiations of the model kernel on 4 x 8 spaxel tiles
// (ka_lines_lsf_t), one per odd LSF length of the direct path, with the
// range-table masks from per-plane ballots (tm = false) or from one bit
// transpose per 32 planes (tm = true), on blocks of four warps or (one_warp,
// with transposed masks) of one warp.
#include "gbk_batched.cuh"

namespace gbk {

void ka_t_register(KaFn* t, bool tm, bool one_warp)
{
    t[0] = one_warp ? ka_lines_lsf_t<1, true, 1> : tm ? ka_lines_lsf_t<1, true, 4> : ka_lines_lsf_t<1, false, 4>;
    t[1] = one_warp ? ka_lines_lsf_t<3, true, 1> : tm ? ka_lines_lsf_t<3, true, 4> : ka_lines_lsf_t<3, false, 4>;
    t[2] = one_warp ? ka_lines_lsf_t<5, true, 1> : tm ? ka_lines_lsf_t<5, true, 4> : ka_lines_lsf_t<5, false, 4>;
    t[3] = one_warp ? ka_lines_lsf_t<7, true, 1> : tm ? ka_lines_lsf_t<7, true, 4> : ka_lines_lsf_t<7, false, 4>;
    t[4] = one_warp ? ka_lines_lsf_t<9, true, 1> : tm ? ka_lines_lsf_t<9, true, 4> : ka_lines_lsf_t<9, false, 4>;
    t[5] = one_warp ? ka_lines_lsf_t<11, true, 1> : tm ? ka_lines_lsf_t<11, true, 4> : ka_lines_lsf_t<11, false, 4>;
    t[6] = one_warp ? ka_lines_lsf_t<13, true, 1> : tm ? ka_lines_lsf_t<13, true, 4> : ka_lines_lsf_t<13, false, 4>;
    t[7] = one_warp ? ka_lines_lsf_t<15, true, 1> : tm ? ka_lines_lsf_t<15, true, 4> : ka_lines_lsf_t<15, false, 4>;
    t[8] = one_warp ? ka_lines_lsf_t<17, true, 1> : tm ? ka_lines_lsf_t<17, true, 4> : ka_lines_lsf_t<17, false, 4>;
    t[9] = one_warp ? ka_lines_lsf_t<19, true, 1> : tm ? ka_lines_lsf_t<19, true, 4> : ka_lines_lsf_t<19, false, 4>;
    t[10] = one_warp ? ka_lines_lsf_t<21, true, 1> : tm ? ka_lines_lsf_t<21, true, 4> : ka_lines_lsf_t<21, false, 4>;
    t[11] = one_warp ? ka_lines_lsf_t<23, true, 1> : tm ? ka_lines_lsf_t<23, true, 4> : ka_lines_lsf_t<23, false, 4>;
    t[12] = one_warp ? ka_lines_lsf_t<25, true, 1> : tm ? ka_lines_lsf_t<25, true, 4> : ka_lines_lsf_t<25, false, 4>;
    t[13] = one_warp ? ka_lines_lsf_t<27, true, 1> : tm ? ka_lines_lsf_t<27, true, 4> : ka_lines_lsf_t<27, false, 4>;
    t[14] = one_warp ? ka_lines_lsf_t<29, true, 1> : tm ? ka_lines_lsf_t<29, true, 4> : ka_lines_lsf_t<29, false, 4>;
    t[15] = one_warp ? ka_lines_lsf_t<31, true, 1> : tm ? ka_lines_lsf_t<31, true, 4> : ka_lines_lsf_t<31, false, 4>;
    t[16] = one_warp ? ka_lines_lsf_t<33, true, 1> : tm ? ka_lines_lsf_t<33, true, 4> : ka_lines_lsf_t<33, false, 4>;
}

}  // namespace gbk
