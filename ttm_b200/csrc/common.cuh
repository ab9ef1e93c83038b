// Shared definitions of the B200 TTM library (device planner view, launch helpers).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tlibttm {

// Dense slice view of one mode-q TTM.
//
// With qhat = pi^{-1}(q) (one-based position of q in A's layout pi), a tensor
// that is dense under pi is exactly the 3-D row-major array
//     A[outer][nq][inner],   inner = prod_{r<qhat} n_{pi_r},  outer = prod_{r>qhat} n_{pi_r}
// and C, which shares A's layout, is C[outer][m][inner]. Then
//     C[k][j][i] = sum_l A[k][l][i] * B(j, l)
// with B(j,l) = b[j + l*m] (column-major, pib[0]==1) or b[j*nq + l].
// This one view covers all eight layout cases of the reference
// (include/tlib/detail/cases.h:25-37): case 6 is inner == 1, case 7 is
// outer == 1, cases 1-5 are p <= 2 instances, case 8 is the general one
// (include/tlib/detail/ttm.h:1135-1194 slices it as `outer` GEMMs).
struct View3 {
    const void* a;
    const void* b;
    void* c;
    int64_t outer, nq, inner, m;
    int b_cm;
};

// General strided problem (strides not dense under pi): evaluated from the
// definition with the caller's strides.
constexpr int kMaxOrder = 32;
struct StridedProblem {
    const void* a;
    const void* b;
    void* c;
    int p;          // order
    int q;          // zero-based contraction mode
    int b_cm;
    int64_t nq, m;
    int64_t total;  // number of C elements
    int order[kMaxOrder];     // zero-based modes in layout order (fastest first)
    int64_t nc[kMaxOrder];    // C extents (mode order)
    int64_t wa[kMaxOrder];    // A strides (mode order)
    int64_t wc[kMaxOrder];    // C strides (mode order)
};

// Kernel identifiers (for diagnostics and launch counting).
enum KernelId : int {
    K_NONE = 0,
    K_SIMT_GEMM,
    K_COLVEC,
    K_ROWDOT,
    K_STRIDED,
    K_TC_BF16X3,
    K_TC_FP8,
    K_TC_OZAKI,
    K_SPLIT_B,
    K_COUNT
};

const char* kernel_name(int id);

// Launchers (simt_kernels.cu). Return cudaSuccess or the launch error.
cudaError_t launch_simt_gemm(const View3& v, int dtype, cudaStream_t s);
cudaError_t launch_colvec(const View3& v, int dtype, cudaStream_t s);
cudaError_t launch_rowdot(const View3& v, int dtype, cudaStream_t s);
cudaError_t launch_strided(const StridedProblem& sp, int dtype, cudaStream_t s);

// Largest m handled by the small-m bandwidth kernels.
constexpr int64_t kSmallM = 16;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace tlibttm
