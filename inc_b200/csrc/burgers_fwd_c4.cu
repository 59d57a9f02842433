// Explicit instantiation of the Burgers fwd kernels with 4 cells per lane.
#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {

template <int CPT, int TPR>
int launch_fwd(Kind kind, const Args& a, cudaStream_t st, int block) {
    return launch_fwd_impl<CPT, TPR>(kind, a, st, block);
}
#define INC_INST(C, T) template int launch_fwd<C, T>(Kind, const Args&, cudaStream_t, int);
INC_BURGERS_SHAPES_C4(INC_INST)

template <int CPT, int TPR>
int launch_weno(const float* f, float* out, int rows, int n, int dir, cudaStream_t st, int block) {
    return launch_weno_impl<CPT, TPR>(f, out, rows, n, dir, st, block);
}
#define INC_INST_W(C, T) template int launch_weno<C, T>(const float*, float*, int, int, int, cudaStream_t, int);
INC_BURGERS_SHAPES_C4(INC_INST_W)

}  // namespace burgers
}  // namespace inc
