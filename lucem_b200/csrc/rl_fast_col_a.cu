// rl_fast_col_a.cu -- instantiations of the register-resident Richardson-Lucy passes
// (rl_pass.cuh) for column lengths 64, 128 and 256, in a translation unit of their own.
#include "rl_pass.cuh"

namespace lucem {
namespace rlp {

int launch_col_64_256(int n, const ColPass &p, cudaStream_t s) {
    switch (n) {
    case 64: return launch_col_fast<8, 8, 16>(p, s);
    // 16 columns per CTA: the z convolution of the 64x512x512 volume (128
    // points) 101 against 103 us with 8; 32 columns 112.6 us.
    case 128: return launch_col_fast<8, 16, 16>(p, s);
    default: return launch_col_fast<16, 16, 16>(p, s);
    }
}

}  // namespace rlp
}  // namespace lucem
