// rl_fast_row_a.cu -- instantiations of the register-resident Richardson-Lucy passes
// (rl_pass.cuh) for packed row lengths 64, 128 and 256, in a translation unit of their own.
#include "rl_pass.cuh"

namespace lucem {
namespace rlp {

int launch_row_64_256(int m, const RowPass &p, cudaStream_t s) {
    switch (m) {
    case 64: return launch_row_fast<8, 8, 32>(p, s);
    case 128: return launch_row_fast<8, 16, 32>(p, s);
    default: return launch_row_fast<16, 16, 16>(p, s);
    }
}

}  // namespace rlp
}  // namespace lucem
