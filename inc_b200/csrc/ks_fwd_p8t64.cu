// Explicit instantiation of the KS fwd kernels for P=8 values per lane, T=64 lanes per row pair.
#include "ks_kernels.cuh"

namespace inc {
namespace ks {

template <int P, int T>
int launch_fwd(Kind kind, const Args& a, cudaStream_t st, int block) {
    return launch_fwd_impl<P, T>(kind, a, st, block);
}
template int launch_fwd<8, 64>(Kind, const Args&, cudaStream_t, int);

}  // namespace ks
}  // namespace inc
