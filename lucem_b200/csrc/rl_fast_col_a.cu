// rl_fast_col_a.cu -- instantiations of the register-resident Richardson-Lucy passes
// (rl_pass.cuh) for column lengths 64, 128 and 256, in a translation unit of their own.
#include "rl_pass.cuh"

namespace lucem {
namespace rlp {

int launch_col_64_256(int n, const ColPass &p, cudaStream_t s) {
    switch (n) {
    case 64: return launch_col_fast<8, 8, 16>(p, s);
    case 128: return launch_col_fast<8, 16, 8>(p, s);
    default: return launch_col_fast<16, 16, 16>(p, s);
    }
}

}  // namespace rlp
}  // namespace lucem
