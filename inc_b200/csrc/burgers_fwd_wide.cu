// Explicit instantiation of the wide-row Burgers forward kernels (1-2 cells per lane, one row per CTA).
#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {

template <int CPT, int TPR>
int launch_wide(Kind kind, const Args& a, cudaStream_t st) {
    return launch_wide_impl<CPT, TPR>(kind, a, st);
}
#define INC_INST(C, T) template int launch_wide<C, T>(Kind, const Args&, cudaStream_t);
INC_BURGERS_WIDE_SHAPES(INC_INST)

}  // namespace burgers
}  // namespace inc
