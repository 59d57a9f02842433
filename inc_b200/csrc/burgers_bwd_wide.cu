// Explicit instantiation of the wide-row Burgers backward kernels (one cell per thread, one row per CTA).
#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {

template <int TPR>
int launch_bwd_wide(Kind kind, const Args& a, cudaStream_t st) {
    return launch_bwd_wide_impl<TPR>(kind, a, st);
}
#define INC_INST(T) template int launch_bwd_wide<T>(Kind, const Args&, cudaStream_t);
INC_BURGERS_BWD_WIDE_SHAPES(INC_INST)

}  // namespace burgers
}  // namespace inc
