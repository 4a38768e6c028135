// Explicit instantiations of the model kernel on 4 x 8 spaxel tiles
// (ka_lines_lsf_t), one per odd LSF length of the direct path, with the
// range-table masks from per-plane ballots (tm = false) or from one bit
// transpose per 32 planes (tm = true), the latter also with the scaled line
// exponent (sl).
#include "gbk_batched.cuh"

namespace gbk {

void ka_t_register(KaFn* t, bool tm, bool sl)
{
    t[0] = sl ? ka_lines_lsf_t<1, true, true> : tm ? ka_lines_lsf_t<1, true> : ka_lines_lsf_t<1, false>;
    t[1] = sl ? ka_lines_lsf_t<3, true, true> : tm ? ka_lines_lsf_t<3, true> : ka_lines_lsf_t<3, false>;
    t[2] = sl ? ka_lines_lsf_t<5, true, true> : tm ? ka_lines_lsf_t<5, true> : ka_lines_lsf_t<5, false>;
    t[3] = sl ? ka_lines_lsf_t<7, true, true> : tm ? ka_lines_lsf_t<7, true> : ka_lines_lsf_t<7, false>;
    t[4] = sl ? ka_lines_lsf_t<9, true, true> : tm ? ka_lines_lsf_t<9, true> : ka_lines_lsf_t<9, false>;
    t[5] = sl ? ka_lines_lsf_t<11, true, true> : tm ? ka_lines_lsf_t<11, true> : ka_lines_lsf_t<11, false>;
    t[6] = sl ? ka_lines_lsf_t<13, true, true> : tm ? ka_lines_lsf_t<13, true> : ka_lines_lsf_t<13, false>;
    t[7] = sl ? ka_lines_lsf_t<15, true, true> : tm ? ka_lines_lsf_t<15, true> : ka_lines_lsf_t<15, false>;
    t[8] = sl ? ka_lines_lsf_t<17, true, true> : tm ? ka_lines_lsf_t<17, true> : ka_lines_lsf_t<17, false>;
    t[9] = sl ? ka_lines_lsf_t<19, true, true> : tm ? ka_lines_lsf_t<19, true> : ka_lines_lsf_t<19, false>;
    t[10] = sl ? ka_lines_lsf_t<21, true, true> : tm ? ka_lines_lsf_t<21, true> : ka_lines_lsf_t<21, false>;
    t[11] = sl ? ka_lines_lsf_t<23, true, true> : tm ? ka_lines_lsf_t<23, true> : ka_lines_lsf_t<23, false>;
    t[12] = sl ? ka_lines_lsf_t<25, true, true> : tm ? ka_lines_lsf_t<25, true> : ka_lines_lsf_t<25, false>;
    t[13] = sl ? ka_lines_lsf_t<27, true, true> : tm ? ka_lines_lsf_t<27, true> : ka_lines_lsf_t<27, false>;
    t[14] = sl ? ka_lines_lsf_t<29, true, true> : tm ? ka_lines_lsf_t<29, true> : ka_lines_lsf_t<29, false>;
    t[15] = sl ? ka_lines_lsf_t<31, true, true> : tm ? ka_lines_lsf_t<31, true> : ka_lines_lsf_t<31, false>;
    t[16] = sl ? ka_lines_lsf_t<33, true, true> : tm ? ka_lines_lsf_t<33, true> : ka_lines_lsf_t<33, false>;
}

}  // namespace gbk
