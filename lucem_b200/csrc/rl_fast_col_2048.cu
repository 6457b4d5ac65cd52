// rl_fast_col_2048.cu -- instantiations of the register-resident Richardson-Lucy passes
// (rl_pass.cuh) for column length 2048, in a translation unit of their own.
#include "rl_pass.cuh"

namespace lucem {
namespace rlp {

int launch_col_2048(const ColPass &p, cudaStream_t s) { return launch_col_fast<32, 64, 8>(p, s); }

}  // namespace rlp
}  // namespace lucem
