// Explicit instantiations of the two-chunk model kernel (ka_lines_lsf2), one
// per odd LSF length of the direct path.
#include "gbk_batched.cuh"

namespace gbk {

void ka2_register(KaFn* t)
{
    t[0] = ka_lines_lsf2<1>;
    t[1] = ka_lines_lsf2<3>;
    t[2] = ka_lines_lsf2<5>;
    t[3] = ka_lines_lsf2<7>;
    t[4] = ka_lines_lsf2<9>;
    t[5] = ka_lines_lsf2<11>;
    t[6] = ka_lines_lsf2<13>;
    t[7] = ka_lines_lsf2<15>;
    t[8] = ka_lines_lsf2<17>;
    t[9] = ka_lines_lsf2<19>;
    t[10] = ka_lines_lsf2<21>;
    t[11] = ka_lines_lsf2<23>;
    t[12] = ka_lines_lsf2<25>;
    t[13] = ka_lines_lsf2<27>;
    t[14] = ka_lines_lsf2<29>;
    t[15] = ka_lines_lsf2<31>;
    t[16] = ka_lines_lsf2<33>;
}

}  // namespace gbk
