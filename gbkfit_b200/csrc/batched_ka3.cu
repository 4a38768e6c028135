// Explicit instantiations of the own-window model kernel (ka_lines_lsf3), one
// per odd LSF length of the direct path.
#include "gbk_batched.cuh"

namespace gbk {

void ka3_register(KaFn* t)
{
    t[0] = ka_lines_lsf3<1>;
    t[1] = ka_lines_lsf3<3>;
    t[2] = ka_lines_lsf3<5>;
    t[3] = ka_lines_lsf3<7>;
    t[4] = ka_lines_lsf3<9>;
    t[5] = ka_lines_lsf3<11>;
    t[6] = ka_lines_lsf3<13>;
    t[7] = ka_lines_lsf3<15>;
    t[8] = ka_lines_lsf3<17>;
    t[9] = ka_lines_lsf3<19>;
    t[10] = ka_lines_lsf3<21>;
    t[11] = ka_lines_lsf3<23>;
    t[12] = ka_lines_lsf3<25>;
    t[13] = ka_lines_lsf3<27>;
    t[14] = ka_lines_lsf3<29>;
    t[15] = ka_lines_lsf3<31>;
    t[16] = ka_lines_lsf3<33>;
}

}  // namespace gbk
