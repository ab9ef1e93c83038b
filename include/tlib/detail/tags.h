/*
 * Policy tags of the tlib::ttm API.
 *
 * Same names, types and constexpr instances as the reference
 * (include/tlib/detail/tags.h:22-69) so that existing callers compile
 * unchanged. In the reference they pick an OpenMP/BLAS threading scheme; on
 * the GPU there is one scheduler (the device planner), so every combination
 * is accepted and computes the same product. This also covers the
 * combinations the reference leaves undefined (its fallback prints a message
 * and computes nothing, include/tlib/detail/ttm.h:391-400) and batched_gemm
 * built without MKL (a no-op there, include/tlib/detail/ttm.h:1345-1401).
 */
#pragma once

namespace tlib::ttm::parallel_policy
{
struct sequential_t         {};
struct parallel_blas_t      {};
struct parallel_loop_t      {};
struct parallel_taskloop_t  {};
struct parallel_task_t      {};
struct parallel_loop_blas_t {};
struct batched_gemm_t       {};
struct combined_t           {};

inline constexpr sequential_t         sequential;
inline constexpr parallel_blas_t      parallel_blas;
inline constexpr parallel_loop_t      parallel_loop;
inline constexpr parallel_taskloop_t  parallel_taskloop;
inline constexpr parallel_task_t      parallel_task;
inline constexpr parallel_loop_blas_t parallel_loop_blas;
inline constexpr batched_gemm_t       batched_gemm;
inline constexpr combined_t           combined;
}

namespace tlib::ttm::slicing_policy
{
struct slice_t     {};
struct subtensor_t {};
struct combined_t  {};

inline constexpr combined_t  combined;
inline constexpr slice_t     slice;
inline constexpr subtensor_t subtensor;
}

namespace tlib::ttm::fusion_policy
{
struct none_t  {};
struct outer_t {};
struct all_t   {};

inline constexpr none_t  none;
inline constexpr outer_t outer;
inline constexpr all_t   all;
}
