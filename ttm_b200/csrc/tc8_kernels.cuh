// 8-bit tensor-core paths of the B200 TTM library: fp8 (e4m3, float operands) and ozaki (int8
// digit slices of double operands, exact int32 products, FP64 recombination).
#pragma once

#include "common.cuh"

namespace tlibttm {

// True iff the 8-bit path of `precision` (TLIBTTM_PREC_FP8 or TLIBTTM_PREC_OZAKI) runs this
// dense view of I/O type `dtype`: m > 16; fp8 takes float, ozaki double with n_q <= 16384.
bool tc8_supported(const View3& v, int precision, int dtype);

// Enqueues the path on stream s: *kid receives the main kernel's identifier and *launches the
// number of kernels enqueued.
cudaError_t launch_tc8(const View3& v, int precision, int dtype, cudaStream_t s, int* kid, int* launches);

// Kernels launch_tc8 enqueues for this view (0 when the path cannot run it).
int tc8_launches(const View3& v, int precision);

}  // namespace tlibttm
