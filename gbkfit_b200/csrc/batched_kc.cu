// Explicit instantiations of the LSF FIR of given model cubes (kc_cube_lsf),
// one per odd LSF length of the direct path.
#include "gbk_batched.cuh"

namespace gbk {

void kc_register(KcFn* t)
{
    t[0] = kc_cube_lsf<1>;
    t[1] = kc_cube_lsf<3>;
    t[2] = kc_cube_lsf<5>;
    t[3] = kc_cube_lsf<7>;
    t[4] = kc_cube_lsf<9>;
    t[5] = kc_cube_lsf<11>;
    t[6] = kc_cube_lsf<13>;
    t[7] = kc_cube_lsf<15>;
    t[8] = kc_cube_lsf<17>;
    t[9] = kc_cube_lsf<19>;
    t[10] = kc_cube_lsf<21>;
    t[11] = kc_cube_lsf<23>;
    t[12] = kc_cube_lsf<25>;
    t[13] = kc_cube_lsf<27>;
    t[14] = kc_cube_lsf<29>;
    t[15] = kc_cube_lsf<31>;
    t[16] = kc_cube_lsf<33>;
}

}  // namespace gbk
