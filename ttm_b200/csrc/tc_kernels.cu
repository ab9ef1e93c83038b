// Tensor-core paths (tcgen05 / TMEM) of the B200 TTM library.
#include "tc_kernels.cuh"

namespace tlibttm {

bool tc_supported(const View3&, int) { return false; }

cudaError_t launch_tc(const View3&, int, cudaStream_t, int* kid)
{
    *kid = K_NONE;
    return cudaErrorNotSupported;
}

void tc_release_buffers() {}

}  // namespace tlibttm
