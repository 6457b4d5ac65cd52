// rl_fast_col_512.cu -- instantiations of the register-resident Richardson-Lucy passes
// (rl_pass.cuh) for column length 512, in a translation unit of their own.
#include "rl_pass.cuh"

namespace lucem {
namespace rlp {

int launch_col_512(const ColPass &p, cudaStream_t s) { return launch_col_fast<16, 32, 16>(p, s); }

}  // namespace rlp
}  // namespace lucem
