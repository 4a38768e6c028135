// Explicit instantiations of the model kernel on 4 x 8 spaxel tiles
// (ka_lines_lsf_t), one per odd LSF length of the direct path.
#include "gbk_batched.cuh"

namespace gbk {

void ka_t_register(KaFn* t)
{
    t[0] = ka_lines_lsf_t<1>;
    t[1] = ka_lines_lsf_t<3>;
    t[2] = ka_lines_lsf_t<5>;
    t[3] = ka_lines_lsf_t<7>;
    t[4] = ka_lines_lsf_t<9>;
    t[5] = ka_lines_lsf_t<11>;
    t[6] = ka_lines_lsf_t<13>;
    t[7] = ka_lines_lsf_t<15>;
    t[8] = ka_lines_lsf_t<17>;
    t[9] = ka_lines_lsf_t<19>;
    t[10] = ka_lines_lsf_t<21>;
    t[11] = ka_lines_lsf_t<23>;
    t[12] = ka_lines_lsf_t<25>;
    t[13] = ka_lines_lsf_t<27>;
    t[14] = ka_lines_lsf_t<29>;
    t[15] = ka_lines_lsf_t<31>;
    t[16] = ka_lines_lsf_t<33>;
}

}  // namespace gbk
