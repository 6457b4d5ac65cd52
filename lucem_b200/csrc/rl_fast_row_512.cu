// rl_fast_row_512.cu -- instantiations of the register-resident Richardson-Lucy passes
// (rl_pass.cuh) for packed row length 512, in a translation unit of their own.
#include "rl_pass.cuh"

namespace lucem {
namespace rlp {

int launch_row_512(const RowPass &p, cudaStream_t s) { return launch_row_fast<16, 32, 16>(p, s); }

}  // namespace rlp
}  // namespace lucem
