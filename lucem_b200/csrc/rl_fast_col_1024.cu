// rl_fast_col_1024.cu -- instantiations of the register-resident Richardson-Lucy passes
// (rl_pass.cuh) for column length 1024, in a translation unit of their own.
#include "rl_pass.cuh"

namespace lucem {
namespace rlp {

int launch_col_1024(const ColPass &p, cudaStream_t s) { return launch_col_fast<32, 32, 8>(p, s); }

}  // namespace rlp
}  // namespace lucem
