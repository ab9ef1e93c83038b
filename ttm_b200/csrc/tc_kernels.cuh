// Tensor-core (tcgen05 / TMEM) paths of the B200 TTM library.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace tlibttm {

// True iff the tensor-core kernel of `precision` can run this dense view.
bool tc_supported(const View3& v, int precision);

// Launches the tensor-core path of `precision` on stream s; *kid receives the
// identifier of the main kernel launched: K_TC_PAIR (one launch) where tc_pair_supported,
// else K_TC_BF16X3 (the operand-split kernel and the single-SM kernel).
cudaError_t launch_tc(const View3& v, int precision, cudaStream_t s, int* kid);

// Output tiles of the single-SM bf16x3 kernel for this view (128 rows x up to 256 columns each).
int64_t tc_single_tiles(const View3& v);

// The single-SM bf16x3 kernel (and its operand split) whatever the shape.
cudaError_t launch_tc_single(const View3& v, cudaStream_t s, int* kid);

// bf16x3 on pairs of SMs with B resident in tensor memory (tc_pair.cu): float, 128 < m <= 256,
// n_q <= 256, A 16-byte aligned, and either contiguous fibres with n_q % 4 == 0 or inner >= 128
// with inner % 4 == 0. Allocates nothing; `status` is the device status word it raises.
bool tc_pair_supported(const View3& v);
cudaError_t launch_tc_pair(const View3& v, int* status, cudaStream_t s);
// The pair kernels' tensor maps: A in boxes of 64 rows x 64 l (rows of i: 3-D box of 64 i x 64 l
// x 1 k; contiguous fibres: boxes of 16 l x 64 rows, 64-byte swizzle), C in 32 x 32 blocks
// (false when C cannot be a tensor map: the epilogue then stores directly).
bool pair_encode_a(const View3& v, CUtensorMap* map);
bool pair_encode_c(const View3& v, CUtensorMap* map);

// fp8 on pairs of SMs (tc_pair8.cu), A read once: the shapes of tc_pair_supported. Every fibre of
// A and row of B is scaled by 2^(8-e), max|x| = f 2^e with f in [0.5, 1), and rounded to e4m3
// (nearest even, saturating), as the fp8 path of tc8_kernels.cu does; the scales of A's fibres
// are found in shared memory from the resident tile, so no exponent or operand pass precedes it.
bool tc_pair8_supported(const View3& v);
cudaError_t launch_tc_pair8(const View3& v, int* status, cudaStream_t s);

// A grouped bf16x3 launch: many float problems (each with tc_supported) whose tiles are
// numbered one after the other and run by one persistent launch per geometry (rows of i, or
// contiguous fibres), after one operand-split launch for all their B. Created once (tensor
// maps, B images and the problem records in device memory); each run reads the same buffers.
struct TcGroup;
cudaError_t tc_group_create(const View3* views, int count, TcGroup** out);
cudaError_t tc_group_run(TcGroup* g, cudaStream_t s);
int tc_group_launches(const TcGroup* g);   // kernel launches per run
void tc_group_destroy(TcGroup* g);

// Creates the per-device state of the tensor-core paths ahead of time (so that a later stream
// capture does not need to allocate it).
cudaError_t tc_prepare_device();

// TMA-fed exact small-m kernel for strided fibres (inner % 4 == 0, m <= 16, B fits shared memory).
bool stream_supported(const View3& v, int dtype);
cudaError_t launch_stream(const View3& v, int dtype, cudaStream_t s);

// A grouped stream launch: many small-m problems (each with stream_group_eligible: the stream
// kernel takes it with B staged whole) whose units are numbered one after the other and run by one
// persistent launch per (row or column mode, MB build, CTAs per SM) class. Created once (tensor
// maps and problem records in device memory); each run reads the same buffers.
struct StreamGroup;
bool stream_group_eligible(const View3& v, int dtype);
cudaError_t stream_group_create(const View3* views, int count, int dtype, StreamGroup** out);
cudaError_t stream_group_run(StreamGroup* g, cudaStream_t s);
int stream_group_launches(const StreamGroup* g);   // kernel launches per run
void stream_group_destroy(StreamGroup* g);

// Frees device state owned by the tensor-core paths on the current device.
void tc_release_buffers();

// Reads and clears the device status word (non-zero: a kernel gave up on a bounded wait).
int tc_read_status();

// The device status word of device `dev` (created on first use), for kernels in other files.
cudaError_t tc_status_word(int dev, int** out);

// Largest pre-split B image the allocation-free bf16x3 variant can hold (bytes):
// cols(m) * ceil(n_q/32)*32 * 4 bytes, cols(m) = ceil(m/16)*16 for m <= 256 and ceil(m/256)*256
// above (whole 256-row blocks of B), e.g. m = 256 with n_q <= 1024.
constexpr size_t kNoAllocImageBytes = size_t(1) << 20;

// Bytes of the pre-split B image a bf16x3 launch of this view needs.
size_t tc_image_bytes(const View3& v);

// The bf16x3 path with its scratch in file-scope device arrays: allocates no memory.
// Returns cudaErrorInvalidValue when the B image exceeds kNoAllocImageBytes.
cudaError_t launch_tc_noalloc(const View3& v, cudaStream_t s, int* kid);

// Status word of the allocation-free variant (non-zero: its last launch gave up on a bounded wait).
int tc_read_noalloc_status();

}  // namespace tlibttm
