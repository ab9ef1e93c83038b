// Tensor-core (tcgen05 / TMEM) paths of the B200 TTM library.
#pragma once

#include "common.cuh"

namespace tlibttm {

// True iff the tensor-core kernel of `precision` can run this dense view.
bool tc_supported(const View3& v, int precision);

// Launches the tensor-core path of `precision` on stream s; *kid receives the
// identifier of the main kernel launched.
cudaError_t launch_tc(const View3& v, int precision, cudaStream_t s, int* kid);

// Frees device state owned by the tensor-core paths on the current device.
void tc_release_buffers();

// Reads and clears the device status word (non-zero: a kernel gave up on a bounded wait).
int tc_read_status();

}  // namespace tlibttm
