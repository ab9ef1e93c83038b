/*
 * tlibttm.h — C ABI of the B200 mode-q tensor-times-matrix library
 * (libtlibttm_cuda.so).
 *
 * This is the boundary a foreign caller (C, ctypes/cffi, cgo, JNI, the C++
 * header include/tlib/ttm.h) binds. Signatures use only plain pointers,
 * size_t metadata arrays and an opaque CUDA stream; no C++ or torch types.
 *
 * Semantics follow the reference tlib::ttm (bassoy/ttm):
 *   C(i1..j..ip) = sum_{iq} A(i1..iq..ip) * B(j,iq)     (README.md:13-18)
 * with C overwritten (beta = 0, include/tlib/detail/mtm.h:92), C laid out with
 * A's layout pi, B of shape nb = (m, n_q) column-major when pib[0] == 1 and
 * row-major otherwise (include/tlib/detail/ttm.h:417), all metadata one-based
 * as in the reference, and the reference's argument checks with the same
 * message texts (include/tlib/ttm.h:65-90).
 *
 * Pointers: a, b and c may each be host memory or device memory of the
 * current CUDA device (managed memory counts as device memory). The library
 * detects which with cudaPointerGetAttributes. If any of them is host memory,
 * it is staged through device buffers the library owns and the call blocks
 * until the result is back in host memory. If all three are device memory,
 * the work is enqueued on `stream` (NULL = the legacy default stream) and the
 * call returns without waiting. The metadata arrays (na, wa, ... ) are always
 * host memory and are not retained after the call.
 *
 * Return value: TLIBTTM_OK (0) or one of the error codes below; the text of
 * the last error on the calling thread is returned by tlibttm_last_error().
 */
#ifndef TLIBTTM_H
#define TLIBTTM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum tlibttm_status {
    TLIBTTM_OK = 0,
    TLIBTTM_ERR_ARG = 1,         /* argument check failed (text = reference runtime_error text) */
    TLIBTTM_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    TLIBTTM_ERR_ALLOC = 3,       /* device or pinned-host allocation failed */
    TLIBTTM_ERR_UNSUPPORTED = 4, /* valid arguments that this build cannot run (e.g. dtype/precision pair) */
    TLIBTTM_ERR_DEVICE = 5       /* a kernel reported failure through its device status word */
};

enum tlibttm_dtype {
    TLIBTTM_F32 = 0,
    TLIBTTM_F64 = 1
};

/*
 * Arithmetic used for the contraction.
 *  PLAIN   exact IEEE FMA in the I/O type (FP32 FFMA / FP64 DFMA). Default.
 *  BF16X3  float only: each FP32 operand is split into bf16 hi + lo parts and
 *          hi*hi + hi*lo + lo*hi run on the tcgen05 tensor cores with FP32
 *          accumulation in TMEM.
 *  FP8     float only: e4m3 operands with a power-of-two scale per slice
 *          (per fibre of A and per row of B), FP32 accumulation. Approximate.
 *  OZAKI   double only: FP64 operands split into int8 slices with a shared
 *          power-of-two exponent per fibre, exact int32 tensor-core products,
 *          FP64 recombination.
 *  AUTO    the library picks per problem (tuned choice among the exact and
 *          the FP32-accurate paths; never FP8).
 * Small-m problems (bandwidth-bound) always run the PLAIN bandwidth kernels.
 */
enum tlibttm_precision {
    TLIBTTM_PREC_DEFAULT = 0,
    TLIBTTM_PREC_PLAIN = 1,
    TLIBTTM_PREC_BF16X3 = 2,
    TLIBTTM_PREC_FP8 = 3,
    TLIBTTM_PREC_OZAKI = 4,
    TLIBTTM_PREC_AUTO = 5
};

/*
 * Replaces tlib::ttm::ttm<float>(ep,sp,fp, q,p, a,na,wa,pia, b,nb,pib, c,nc,wc)
 * (reference include/tlib/ttm.h:54-93). The three policy tags select CPU
 * threading in the reference and have no counterpart on the GPU, so they are
 * not part of the ABI. Uses the process-wide default precision
 * (tlibttm_set_precision, initially PLAIN).
 */
int tlibttm_ttm_f32(unsigned q, unsigned p,
                    const float* a, const size_t* na, const size_t* wa, const size_t* pia,
                    const float* b, const size_t* nb, const size_t* pib,
                    float* c, const size_t* nc, const size_t* wc,
                    void* stream);

/* Same as tlibttm_ttm_f32 for double (reference include/tlib/ttm.h:54-93 with value_t = double). */
int tlibttm_ttm_f64(unsigned q, unsigned p,
                    const double* a, const size_t* na, const size_t* wa, const size_t* pia,
                    const double* b, const size_t* nb, const size_t* pib,
                    double* c, const size_t* nc, const size_t* wc,
                    void* stream);

/*
 * Explicit-precision form of the two calls above (an extension: the
 * reference has one arithmetic, its BLAS's). dtype is a tlibttm_dtype,
 * precision a tlibttm_precision.
 */
int tlibttm_ttm_ex(int dtype, int precision, unsigned q, unsigned p,
                   const void* a, const size_t* na, const size_t* wa, const size_t* pia,
                   const void* b, const size_t* nb, const size_t* pib,
                   void* c, const size_t* nc, const size_t* wc,
                   void* stream);

/*
 * No counterpart in the reference: the bf16x3 contraction (as tlibttm_ttm_ex with
 * TLIBTTM_F32 / TLIBTTM_PREC_BF16X3) for callers that cannot let a library
 * allocate device memory — a host application whose allocator already owns the
 * device's memory, a latency-bound loop that must not risk the implicit device
 * synchronisation of cudaMalloc/cudaFree, or a process under a fixed memory
 * budget. It allocates nothing: its scratch (the bf16 hi/lo image of B and a
 * status word) lives in file-scope device arrays that every GPU loading the
 * library holds until exit.
 *
 * Limits: a, b and c must all be device memory of the current device (no host
 * staging); A and C dense under their layout; m > 16 and either inner >= 17
 * or q == pia[0]; and the B image, cols(m) * ceil(n_q/32)*32 * 4 bytes with
 * cols(m) = ceil(m/16)*16 for m <= 256 and ceil(m/256)*256 above, at most
 * 1 MiB (for example m = 256 with n_q <= 1024, or m = 272 with n_q <= 512). Larger or unsupported problems are rejected with
 * TLIBTTM_ERR_ARG / TLIBTTM_ERR_UNSUPPORTED and a message; nothing is launched.
 *
 * The work is enqueued on `stream`; tlibttm_synchronize reports a failed
 * bounded wait of its kernels. The first call on each device performs a
 * one-time set-up there (it looks up the arrays' device addresses); make that
 * first call before any stream capture. All calls share the arrays, so calls
 * whose work overlaps on the GPU (different streams or host threads) race and
 * must be serialised by the caller.
 */
int tlibttm_ttm_f32_bf16x3_noalloc(unsigned q, unsigned p,
                                   const float* a, const size_t* na, const size_t* wa, const size_t* pia,
                                   const float* b, const size_t* nb, const size_t* pib,
                                   float* c, const size_t* nc, const size_t* wc,
                                   void* stream);

/*
 * Schedules: the kernel choices the planner makes, exposed so that a tuner can
 * time them (an extension; the reference's counterpart is its choice of
 * policy tags, include/tlib/detail/ttm.h:1408-1474, the `combined` heuristic).
 * All but TC_BF16X3 compute in the I/O type with exact FMA.
 */
enum tlibttm_schedule {
    TLIBTTM_SCHED_HEURISTIC = 0,   /* the planner's built-in choice (as tlibttm_ttm_ex, PLAIN) */
    TLIBTTM_SCHED_SIMT_GEMM = 1,   /* slice-GEMM on FFMA/DFMA, any m */
    TLIBTTM_SCHED_COLS = 2,        /* small-m kernel for strided fibres, rows spread over warps (m <= 16, inner >= 2) */
    TLIBTTM_SCHED_COLS_SPLIT = 3,  /* small-m kernel for strided fibres, l split over 8 warps (m <= 16, inner >= 2) */
    TLIBTTM_SCHED_ROWS = 4,        /* small-m kernel for contiguous fibres (m <= 16, q == pia[0]) */
    TLIBTTM_SCHED_TC_BF16X3 = 5,   /* tensor-core bf16x3 on single SMs, float only (FP32-accurate, not exact; m > 16) */
    TLIBTTM_SCHED_COLS_TMA = 6,    /* small-m kernel fed by TMA (m <= 16): strided fibres (inner % 4 == 0), or
                                      contiguous fibres of >= 16 floats / 8 doubles on 16-byte boundaries */
    TLIBTTM_SCHED_TC_BF16X3_PAIR = 7, /* tensor-core bf16x3 on pairs of SMs with B in tensor memory, float only
                                      (128 < m <= 256, n_q <= 256; inner >= 128 or q == pia[0]) */
    TLIBTTM_SCHED_SIMT_SPLIT = 8,  /* slice-GEMM on FFMA/DFMA with its l loop split over blocks whatever the tile
                                      count (n_q >= 2048); a fixed-order second kernel adds the parts */
    TLIBTTM_SCHED_BVEC = 9,        /* few output rows (outer * inner <= 8), 16 < m <= 256, n_q >= 4096: B streamed
                                      by the whole GPU, l split over blocks, fixed-order reduction */
    TLIBTTM_SCHED_COUNT = 10
};

/* Runs one TTM with a given schedule (all operands device memory, A and C dense). */
int tlibttm_ttm_sched(int dtype, int schedule, unsigned q, unsigned p,
                      const void* a, const size_t* na, const size_t* wa, const size_t* pia,
                      const void* b, const size_t* nb, const size_t* pib,
                      void* c, const size_t* nc, const size_t* wc,
                      void* stream);

/* 1 if `schedule` can run a dense TTM with these extents, layout, mode and m; else 0. */
int tlibttm_schedule_valid(int dtype, int schedule, unsigned q, unsigned p, const size_t* na, const size_t* pia,
                           size_t m);

/*
 * Kernels of the learned schedule selector (no counterpart in the reference):
 * a multilayer perceptron over float32 device buffers, activations
 * [batch][features] row-major, weights [out][in].
 *   forward   y = act(x w^T + bias), act = ReLU when relu != 0
 *   backward  dz = dy * act'(y) (into the caller's dz buffer), dw = dz^T x,
 *             db = column sums of dz, dx = dz w (skipped when dx is NULL)
 *   mse_grad  dy = 2 (y - t) mask / count (inv_count = 1/count), loss += mean masked error^2
 *   adam      one Adam step (bias-corrected with `step`, counted from 1)
 */
int tlibttm_mlp_forward(const float* x, const float* w, const float* bias, float* y, int batch, int in, int out,
                        int relu, void* stream);
int tlibttm_mlp_backward(const float* x, const float* w, const float* y, const float* dy, float* dz, float* dx,
                         float* dw, float* db, int batch, int in, int out, int relu, void* stream);
int tlibttm_mlp_mse_grad(const float* y, const float* t, const float* mask, float* dy, float* loss, int n,
                         float inv_count, void* stream);
int tlibttm_mlp_adam(float* p, const float* g, float* m, float* v, int n, float lr, float beta1, float beta2, float eps,
                     int step, void* stream);

/*
 * Plans: many TTMs prepared once, run many times (an extension; the
 * reference's closest counterparts are the MKL-only batched_gemm policy,
 * include/tlib/detail/ttm.h:1321-1403, and ttmpy.ttms,
 * ttmpy/src/wrapped_ttm.cpp:81-222). A plan records device pointers and
 * metadata at creation; running it re-reads the current contents of those
 * buffers. All operands of a plan must be device memory of the current device.
 */
typedef struct tlibttm_plan_s tlibttm_plan;

/* One TTM of a batched plan, with the arguments of tlibttm_ttm_f32/_f64. */
typedef struct tlibttm_problem {
    unsigned q, p;
    const void* a; const size_t* na; const size_t* wa; const size_t* pia;
    const void* b; const size_t* nb; const size_t* pib;
    void* c; const size_t* nc; const size_t* wc;
} tlibttm_problem;

/*
 * Batched plan: `count` independent TTMs of one dtype, in grouped persistent launches:
 * every float problem bf16x3 takes (precision bf16x3, or auto with m > 16) in one
 * tensor-core launch per geometry; small-m problems the TMA-fed kernel takes in one
 * launch per kernel build; the other small-m problems as row-block work items of one
 * launch, except those of at least 2^22 elements of A and those with few rows and a long
 * l range, which get their own launch; the other slice-GEMM problems as tiles of one
 * launch. Problems with non-dense strides get their own launch. Single launches run
 * largest first on worker streams the plan owns, forked from `stream` and joined back
 * into it. Errors name the offending problem ("problem 7: ...").
 * (Reference counterpart: none; the reference runs one TTM per call, ttm.h:100-138.)
 */
int tlibttm_plan_batched(int dtype, int precision, size_t count, const tlibttm_problem* problems,
                         tlibttm_plan** plan);

/* tlibttm_plan_batched with options. TLIBTTM_PLAN_FEW_LAUNCHES: small-m problems of any
 * size become work items of the grouped small-m launch (fewer launches per run, for callers
 * that launch eagerly rather than replay a graph; measured 4-5 % slower on the 512-problem
 * benchmark set under graph replay). */
#define TLIBTTM_PLAN_FEW_LAUNCHES 1u
int tlibttm_plan_batched_ex(int dtype, int precision, size_t count, const tlibttm_problem* problems,
                            unsigned flags, tlibttm_plan** plan);

/*
 * Chain plan (Tucker projection, ttmpy.ttms): C = A x_{modes[0]} B_0 x_{modes[1]} B_1 ... in
 * the given order. A has order p, extents na and layout pia (dense); B_s has shape
 * (ms[s], n) with n the current extent of mode modes[s] and layout pibs[2s..2s+1];
 * every intermediate and C are dense with layout pia. Intermediates live in
 * device buffers the plan owns.
 */
int tlibttm_plan_chain(int dtype, int precision, unsigned p, const void* a, const size_t* na, const size_t* pia,
                       unsigned count, const unsigned* modes, const void* const* bs, const size_t* ms,
                       const size_t* pibs, void* c, tlibttm_plan** plan);

/* Enqueues the plan's launches on `stream`. */
int tlibttm_plan_run(tlibttm_plan* plan, void* stream);

/*
 * Runs the plan as a CUDA graph: the first call captures the plan's launches
 * into a graph and instantiates it, later calls replay it (one launch of the
 * whole plan). With stream == NULL a blocking stream owned by the plan is used
 * (ordered after the work queued on the legacy default stream before the call,
 * as the default stream itself would be) and the call waits for completion.
 */
int tlibttm_plan_run_graph(tlibttm_plan* plan, void* stream);

/* Number of kernel launches one run of the plan performs (grouped + individual). */
int tlibttm_plan_launches(const tlibttm_plan* plan);

/* Frees the plan, its device buffers and its graph. */
int tlibttm_plan_destroy(tlibttm_plan* plan);

/*
 * Host-side fault injection for failure-detection tests (no counterpart in the reference; no
 * GPU fault is ever raised). Each call sets one injection; TLIBTTM_INJECT_NONE clears them all.
 *  FAIL_ALLOC       arg = n > 0: the n-th next device allocation of the library fails with
 *                   cudaErrorMemoryAllocation, and the call that made it returns TLIBTTM_ERR_ALLOC
 *                   (0 disarms).
 *  WAIT_NS          arg = bound in ns of the mbarrier waits of later bf16x3 launches (0: the
 *                   default of 4 s). On expiry the kernel's blocks stop, drain their own copies,
 *                   free tensor memory and raise the status word that tlibttm_synchronize (and
 *                   every blocking call) reports as TLIBTTM_ERR_DEVICE.
 *  SKIP_B_STAGE     arg != 0: the next bf16x3 launch never fills its first pipeline stage (the
 *                   single-SM kernel's first B stage, the pair kernel's first A stage in its
 *                   even CTA), so that the waits on it run out (use with a short WAIT_NS).
 */
enum tlibttm_injection {
    TLIBTTM_INJECT_NONE = 0,
    TLIBTTM_INJECT_FAIL_ALLOC = 1,
    TLIBTTM_INJECT_WAIT_NS = 2,
    TLIBTTM_INJECT_SKIP_B_STAGE = 3
};
int tlibttm_inject(int what, long long arg);

/* Text of the last error reported on the calling thread ("" if none). */
const char* tlibttm_last_error(void);

/* Process-wide default precision used by tlibttm_ttm_f32/_f64. Returns the previous value. */
int tlibttm_set_precision(int precision);
int tlibttm_get_precision(void);

/* Name of the kernel the last successful call on this thread launched (diagnostics, tests). */
const char* tlibttm_last_kernel(void);

/* Number of kernels this library launched on the calling thread since the last reset. */
unsigned long long tlibttm_launch_count(int reset);

/* Waits for all work the library enqueued on `stream`. */
int tlibttm_synchronize(void* stream);

/* Releases the library's staging buffers on the current device. */
int tlibttm_release_buffers(void);

/*
 * Device memory for callers built without the CUDA headers; the device-resident
 * tlib::ttm::device_tensor (include/tlib/detail/device_tensor.h) is written on these.
 *   tlibttm_device_alloc  bytes of memory on the current device (*ptr = NULL when bytes == 0);
 *                         goes through the library's allocator, so FAIL_ALLOC applies
 *                         (TLIBTTM_ERR_ALLOC)
 *   tlibttm_device_free   frees what tlibttm_device_alloc returned (NULL is a no-op)
 *   tlibttm_copy          synchronous copy of `bytes` between any mix of host and device memory
 *   tlibttm_fill          sets `count` elements of type `dtype` (tlibttm_dtype) at device pointer
 *                         `ptr` to `value`, enqueued on `stream`
 */
int tlibttm_device_alloc(void** ptr, size_t bytes);
int tlibttm_device_free(void* ptr);
int tlibttm_copy(void* dst, const void* src, size_t bytes);
int tlibttm_fill(int dtype, void* ptr, size_t count, double value, void* stream);

/*
 * Layout / stride helpers with the reference's semantics, for callers that
 * build metadata without the C++ header:
 *   tlibttm_k_order_layout  reference include/tlib/detail/layout.h:57-76
 *   tlibttm_inverse_mode    reference include/tlib/detail/layout.h:120-144 (0 on error)
 *   tlibttm_strides         reference include/tlib/detail/strides.h:31-57 (incl. the
 *                           all-ones strides of vector/scalar shapes)
 */
int tlibttm_k_order_layout(size_t* layout, size_t p, size_t k);
size_t tlibttm_inverse_mode(const size_t* layout, size_t p, size_t mode);
int tlibttm_strides(const size_t* shape, size_t p, const size_t* layout, size_t* strides);

#ifdef __cplusplus
}
#endif

#endif /* TLIBTTM_H */
