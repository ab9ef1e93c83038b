// Shared definitions of the B200 TTM library (device planner view, launch helpers).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tlibttm {

#ifdef __CUDACC__
// Packed FP32 pairs (sm_100): d = a * b + d lane by lane, each lane one correctly rounded fused
// multiply-add like fmaf, two per instruction. Pairs live in 64-bit registers, low half first.
static __device__ __forceinline__ void ffma2(unsigned long long& d, unsigned long long a, unsigned long long b)
{
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
}
static __device__ __forceinline__ unsigned long long pair_dup(float x)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(x));
    return r;
}
static __device__ __forceinline__ float pair_lo(unsigned long long r) { return __uint_as_float((unsigned)r); }
static __device__ __forceinline__ float pair_hi(unsigned long long r) { return __uint_as_float((unsigned)(r >> 32)); }
#endif

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

// One problem of a grouped launch (device copy built by the host plan).
struct GroupDesc {
    const void* a;
    const void* b;
    void* c;
    int64_t outer, nq, inner, m;
    int b_cm;
    int kind;          // 0: slice-GEMM tiles, 1: rows of the small-m kernel
    int flags;         // bit 0: fibres contiguous (inner == 1); bit 1: 16-byte vector access
    int pad;
    int64_t tiles_m;   // slice-GEMM: row tiles; small-m: blocks of 256 rows (256 * 16/sizeof(T) when
                       // strided fibres are read with 16-byte loads)
    int64_t tiles_n;   // slice-GEMM: column tiles; small-m: 1
    int64_t first;     // index of the problem's first work item
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
    K_GROUPED,
    K_STREAM_COLS,
    K_STREAM_ROWS,
    K_TC_PAIR,
    K_BVEC,
    K_TC_FP8_PAIR,
    K_COUNT
};

const char* kernel_name(int id);

// Launchers (simt_kernels.cu). Return cudaSuccess or the launch error.
// The slice-GEMM; when its tiles cannot fill the GPU and n_q is long, the K loop is split over
// more blocks and the parts are added by a second kernel (*launches = 2, else 1).
// force_split: split the K loop whenever n_q >= 2048 (a schedule of its own for the tuner).
cudaError_t launch_simt_gemm(const View3& v, int dtype, cudaStream_t s, int* launches = nullptr,
                             bool force_split = false);
int simt_gemm_launch_count(const View3& v, int dtype);
// Few output rows (outer * inner <= 8), 16 < m <= 256, n_q >= 4096: a kernel that streams B with
// the l range split over the GPU, then a fixed-order reduction (*launches = 2).
bool bvec_supported(const View3& v);
// The same split for small m (m <= kSmallM): few rows and n_q >= 4096.
bool bvec_small_supported(const View3& v);
cudaError_t launch_bvec(const View3& v, int dtype, cudaStream_t s, int* launches = nullptr);
cudaError_t launch_colvec(const View3& v, int dtype, cudaStream_t s);
// colvec with an explicit l split over warps (1 or 8).
cudaError_t launch_colvec_ls(const View3& v, int dtype, int ls, cudaStream_t s);
cudaError_t launch_rowdot(const View3& v, int dtype, cudaStream_t s);
cudaError_t launch_strided(const StridedProblem& sp, int dtype, cudaStream_t s);
// Sets n elements at p (float when dtype == 0, else double) to v.
cudaError_t launch_fill(void* p, int64_t n, int dtype, double v, cudaStream_t s);

// Grouped launch: `count` problems, `total` work items pulled from the device counter `queue`
// (which must be zero at launch) by a persistent grid of `grid` blocks.
cudaError_t launch_grouped(const GroupDesc* d_desc, int count, int64_t total, unsigned long long* queue, int dtype,
                           int grid, cudaStream_t s);
// The same for small-m work items only (kind 1), with more blocks per SM.
cudaError_t launch_grouped_small(const GroupDesc* d_desc, int count, int64_t total, unsigned long long* queue,
                                 int dtype, int grid, cudaStream_t s);
int grouped_small_blocks_per_sm(int dtype);
// Row / column tile sizes of the slice-GEMM for an element type, and rows per small-m work item.
constexpr int kGemmTileF32 = 128, kGemmTileF64 = 64, kGemvRows = 256;
// Blocks per SM the grouped kernel is launched with.
int grouped_blocks_per_sm(int dtype);

// Largest m handled by the small-m bandwidth kernels.
constexpr int64_t kSmallM = 16;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Division of 32-bit unsigned n by a divisor d fixed at set-up, by multiplication (Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994): with l = ceil(log2 d)
// and mul = floor(2^32 (2^l - d) / d) + 1, n / d = (mulhi(n, mul) + n) >> l for every n < 2^32,
// the sum taken in 64 bits. Kernels use it where a runtime divisor would otherwise cost an
// integer division sequence per tile and thread.
struct FastDiv {
    uint32_t d, mul, shift;
};

inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d < 1 ? 1 : d;
    uint32_t l = 0;
    while ((uint64_t(1) << l) < f.d) ++l;
    f.shift = l;
    f.mul = (uint32_t)(((uint64_t(1) << 32) * ((uint64_t(1) << l) - f.d)) / f.d + 1);
    return f;
}

__host__ __device__ inline uint32_t fast_div(uint32_t n, const FastDiv& f)
{
#ifdef __CUDA_ARCH__
    const uint32_t hi = __umulhi(n, f.mul);
#else
    const uint32_t hi = (uint32_t)(((uint64_t)n * f.mul) >> 32);
#endif
    return (uint32_t)(((uint64_t)hi + n) >> f.shift);
}

// Every device allocation of the library goes through these two wrappers (cudaMalloc and the
// stream-ordered cudaMallocAsync), so that a test can make the n-th one fail (tlibttm_inject).
cudaError_t dev_malloc(void** p, size_t bytes);
cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t s);

// Bound of the bounded mbarrier waits of the bf16x3 kernel, in ns (4 s unless a test set it).
unsigned long long wait_limit_ns();
// True once after a test asked for it: the next bf16x3 launch never fills its first pipeline
// stage (no copy, no arrive), so that the bounded waits on that stage run out.
bool take_skip_b();

}  // namespace tlibttm
