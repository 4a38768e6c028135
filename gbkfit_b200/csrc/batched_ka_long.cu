// Explicit instantiations of the batched model kernel (one translation unit
// per group, so that the library compiles in parallel).
#include "gbk_batched.cuh"

namespace gbk {

void ka_register_long(KaFn* t)
{
    t[8] = ka_lines_lsf<17>;
    t[9] = ka_lines_lsf<19>;
    t[10] = ka_lines_lsf<21>;
    t[11] = ka_lines_lsf<23>;
    t[12] = ka_lines_lsf<25>;
    t[13] = ka_lines_lsf<27>;
    t[14] = ka_lines_lsf<29>;
    t[15] = ka_lines_lsf<31>;
    t[16] = ka_lines_lsf<33>;
}

}  // namespace gbk
