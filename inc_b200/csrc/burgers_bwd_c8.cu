// Explicit instantiation of the Burgers bwd kernels with 8 cells per lane.
#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {

template <int CPT, int TPR>
int launch_bwd(Kind kind, const Args& a, cudaStream_t st, int block) {
    return launch_bwd_impl<CPT, TPR>(kind, a, st, block);
}
#define INC_INST(C, T) template int launch_bwd<C, T>(Kind, const Args&, cudaStream_t, int);
INC_BURGERS_SHAPES_C8(INC_INST)

}  // namespace burgers
}  // namespace inc
