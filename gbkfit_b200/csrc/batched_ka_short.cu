// Explicit instantiations of the batched model kernel (one translation unit
// per group, so that the library compiles in parallel).
#include "gbk_batched.cuh"

namespace gbk {

void ka_register_short(KaFn* t)
{
    t[0] = ka_lines_lsf<1>;
    t[1] = ka_lines_lsf<3>;
    t[2] = ka_lines_lsf<5>;
    t[3] = ka_lines_lsf<7>;
    t[4] = ka_lines_lsf<9>;
    t[5] = ka_lines_lsf<11>;
    t[6] = ka_lines_lsf<13>;
    t[7] = ka_lines_lsf<15>;
}

}  // namespace gbk
