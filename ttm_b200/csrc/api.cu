// C ABI of the B200 TTM library: argument checks, device planner, staging of
// host operands, kernel dispatch. Declarations and contract: include/tlibttm.h.
#include <algorithm>
#include <atomic>
#include <memory>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "tlibttm.h"
#include "tlib/detail/layout.h"
#include "tlib/detail/shape.h"
#include "tlib/detail/strides.h"

#include "common.cuh"
#include "tc8_kernels.cuh"
#include "tc_kernels.cuh"

namespace tlibttm {

const char* kernel_name(int id)
{
    switch (id) {
    case K_SIMT_GEMM: return "simt_gemm";
    case K_COLVEC: return "colvec";
    case K_ROWDOT: return "rowdot";
    case K_STRIDED: return "strided";
    case K_TC_BF16X3: return "tc_bf16x3";
    case K_TC_FP8: return "tc_fp8";
    case K_TC_FP8_PAIR: return "tc_fp8_pair";
    case K_TC_OZAKI: return "tc_ozaki";
    case K_SPLIT_B: return "split_b";
    case K_GROUPED: return "grouped";
    case K_STREAM_COLS: return "stream_cols";
    case K_STREAM_ROWS: return "stream_rows";
    case K_TC_PAIR: return "tc_bf16x3_pair";
    case K_BVEC: return "bvec";
    default: return "";
    }
}

namespace {
bool injected_alloc_failure();
}

cudaError_t dev_malloc(void** p, size_t bytes)
{
    if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
    return cudaMalloc(p, bytes);
}

cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t s)
{
    if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
    return cudaMallocAsync(p, bytes, s);
}

namespace {

thread_local std::string g_err;
thread_local const char* g_last_kernel = "";
thread_local unsigned long long g_launches = 0;

int initial_precision()
{
    const char* e = std::getenv("TLIBTTM_PRECISION");
    if (!e) return TLIBTTM_PREC_PLAIN;
    if (!std::strcmp(e, "plain")) return TLIBTTM_PREC_PLAIN;
    if (!std::strcmp(e, "bf16x3")) return TLIBTTM_PREC_BF16X3;
    if (!std::strcmp(e, "fp8")) return TLIBTTM_PREC_FP8;
    if (!std::strcmp(e, "ozaki")) return TLIBTTM_PREC_OZAKI;
    if (!std::strcmp(e, "auto")) return TLIBTTM_PREC_AUTO;
    return TLIBTTM_PREC_PLAIN;
}

std::atomic<int> g_precision{initial_precision()};

int fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
    g_err = std::string("tlibttm: CUDA error in ") + where + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? TLIBTTM_ERR_ALLOC : TLIBTTM_ERR_CUDA;
}

// Host-side fault injection (tlibttm_inject): the allocation that fails next, the wait bound of
// the bf16x3 kernel and the one-shot skipped B stage.
std::atomic<long long> g_fail_alloc_in{0};
std::atomic<unsigned long long> g_wait_ns{0};
std::atomic<int> g_skip_b{0};

bool injected_alloc_failure()
{
    long long n = g_fail_alloc_in.load();
    while (n > 0) {
        if (g_fail_alloc_in.compare_exchange_weak(n, n - 1)) return n == 1;
    }
    return false;
}

struct Args {
    int dtype;
    unsigned q, p;
    const void* a;
    const size_t *na, *wa, *pia;
    const void* b;
    const size_t *nb, *pib;
    void* c;
    const size_t *nc, *wc;
};

// Reference include/tlib/ttm.h:65-90: same checks, same order, same texts.
// Two additions the reference leaves to asserts or crashes: a null pib, and
// C extents that differ from A's outside mode q (include/tlib/detail/mtm.h:166-167).
int validate(const Args& x)
{
    static const std::string E = "Error in tlib::tensor_times_matrix: ";
    if (x.p == 0) return fail(TLIBTTM_ERR_ARG, E + "input tensor order should be greater zero.");
    if (x.q == 0 || x.q > x.p) return fail(TLIBTTM_ERR_ARG, E + "contraction mode should be greater zero or less than or equal to p.");
    if (!x.a) return fail(TLIBTTM_ERR_ARG, E + "pointer to input tensor A should not be zero.");
    if (!x.b) return fail(TLIBTTM_ERR_ARG, E + "pointer to input vector B should not be zero.");
    if (!x.c) return fail(TLIBTTM_ERR_ARG, E + "pointer to output tensor C should not be zero.");
    if (!x.na) return fail(TLIBTTM_ERR_ARG, E + "pointer to input tensor shape vector na should not be zero.");
    if (!x.nb) return fail(TLIBTTM_ERR_ARG, E + "pointer to input vector shape vector nb should not be zero.");
    if (!x.nc) return fail(TLIBTTM_ERR_ARG, E + "pointer to output tensor shape vector nc should not be zero.");
    if (!x.wa) return fail(TLIBTTM_ERR_ARG, E + "pointer to input tensor stride vector wa should not be zero.");
    if (!x.wc) return fail(TLIBTTM_ERR_ARG, E + "pointer to output tensor stride vector wc should not be zero.");
    if (!x.pia) return fail(TLIBTTM_ERR_ARG, E + "pointer to input tensor permutation vector pia should not be zero.");
    if (x.na[x.q - 1] != x.nb[1]) return fail(TLIBTTM_ERR_ARG, E + "contraction dimension of A and B are not equal.");
    if (x.nc[x.q - 1] != x.nb[0]) return fail(TLIBTTM_ERR_ARG, E + "free dimension of C and B are not equal.");
    if (!tlib::ttm::detail::is_valid_shape(x.na, x.na + x.p)) return fail(TLIBTTM_ERR_ARG, E + "shape vector of A is not valid.");
    if (!tlib::ttm::detail::is_valid_shape(x.nc, x.nc + x.p)) return fail(TLIBTTM_ERR_ARG, E + "shape vector of C is not valid.");
    if (!tlib::ttm::detail::is_valid_layout(x.pia, x.pia + x.p)) return fail(TLIBTTM_ERR_ARG, E + "layout vector of A is not valid.");
    if (!tlib::ttm::detail::is_valid_strides(x.pia, x.pia + x.p, x.wa)) return fail(TLIBTTM_ERR_ARG, E + "stride vector of A is not valid.");
    if (!tlib::ttm::detail::is_valid_strides(x.pia, x.pia + x.p, x.wc)) return fail(TLIBTTM_ERR_ARG, E + "stride vector of C is not valid.");
    if (!x.pib) return fail(TLIBTTM_ERR_ARG, E + "pointer to input matrix layout vector pib should not be zero.");
    for (unsigned r = 0; r < x.p; ++r)
        if (r != x.q - 1 && x.nc[r] != x.na[r])
            return fail(TLIBTTM_ERR_ARG, E + "shape vector of C does not match A outside the contraction mode.");
    return TLIBTTM_OK;
}

// True iff strides w are the dense strides of extents n under layout pi,
// ignoring modes of extent 1 (whose stride never enters an address).
bool dense_under(const size_t* n, const size_t* w, const size_t* pi, unsigned p)
{
    size_t expect = 1;
    for (unsigned r = 0; r < p; ++r) {
        const size_t mode = pi[r] - 1;
        if (n[mode] == 1) continue;
        if (w[mode] != expect) return false;
        expect *= n[mode];
    }
    return true;
}

size_t span_of(const size_t* n, const size_t* w, unsigned p)
{
    size_t s = 1;
    for (unsigned r = 0; r < p; ++r) s += (n[r] - 1) * w[r];
    return s;
}

struct Plan {
    bool dense = true;
    View3 v{};
    StridedProblem sp{};
    size_t a_elems = 0, b_elems = 0, c_elems = 0;   // element spans to stage
};

int make_plan(const Args& x, Plan& pl)
{
    const unsigned p = x.p, q = x.q;
    const size_t* pia = x.pia;
    unsigned qh = 0;
    while (pia[qh] != q) ++qh;   // zero-based position of q in the layout
    int64_t inner = 1, outer = 1;
    for (unsigned r = 0; r < qh; ++r) inner *= (int64_t)x.na[pia[r] - 1];
    for (unsigned r = qh + 1; r < p; ++r) outer *= (int64_t)x.na[pia[r] - 1];
    const int64_t nq = (int64_t)x.na[q - 1], m = (int64_t)x.nb[0];

    pl.dense = dense_under(x.na, x.wa, pia, p) && dense_under(x.nc, x.wc, pia, p);
    pl.b_elems = (size_t)(m * nq);
    if (pl.dense) {
        pl.a_elems = (size_t)(outer * nq * inner);
        pl.c_elems = (size_t)(outer * m * inner);
        pl.v.outer = outer;
        pl.v.nq = nq;
        pl.v.inner = inner;
        pl.v.m = m;
        pl.v.b_cm = x.pib[0] == 1;
    } else {
        if (p > (unsigned)kMaxOrder)
            return fail(TLIBTTM_ERR_UNSUPPORTED, "tlibttm: non-dense strides are supported up to order 32.");
        pl.a_elems = span_of(x.na, x.wa, p);
        pl.c_elems = span_of(x.nc, x.wc, p);
        StridedProblem& sp = pl.sp;
        sp.p = (int)p;
        sp.q = (int)q - 1;
        sp.b_cm = x.pib[0] == 1;
        sp.nq = nq;
        sp.m = m;
        sp.total = 1;
        for (unsigned r = 0; r < p; ++r) {
            sp.order[r] = (int)pia[r] - 1;
            sp.nc[r] = (int64_t)x.nc[r];
            sp.wa[r] = (int64_t)x.wa[r];
            sp.wc[r] = (int64_t)x.wc[r];
            sp.total *= (int64_t)x.nc[r];
        }
    }
    return TLIBTTM_OK;
}

int note_launch(cudaError_t e, int kid)
{
    if (e != cudaSuccess) return cuda_fail(e, kernel_name(kid));
    g_last_kernel = kernel_name(kid);
    ++g_launches;
    return TLIBTTM_OK;
}

constexpr int64_t kStreamMinBytes = int64_t(64) << 20;
constexpr int64_t kPlanStreamMinBytes = int64_t(4) << 20;

// All operands are device memory: enqueue on stream s.
int run_device(const Args& x, Plan& pl, int precision, cudaStream_t s, int64_t stream_min_bytes = kStreamMinBytes)
{
    if (!pl.dense) {
        pl.sp.a = x.a;
        pl.sp.b = x.b;
        pl.sp.c = x.c;
        return note_launch(launch_strided(pl.sp, x.dtype, s), K_STRIDED);
    }
    View3& v = pl.v;
    v.a = x.a;
    v.b = x.b;
    v.c = x.c;
    if (v.m <= kSmallM) {
        // The TMA-fed kernel wins once A streams from HBM; below about half of L2 the plain
        // kernels' shorter start-up wins (both measured on L2-resident repeats). Contiguous
        // fibres of fewer than 16 elements always take the flat-tile row kernel (at 16 the
        // TMA-fed row mode measured 0.87-0.88 of HBM against 0.65-0.72 at m = 8).
        const int64_t a_bytes = v.outer * v.nq * v.inner * (x.dtype == TLIBTTM_F32 ? 4 : 8);
        const bool tma = a_bytes >= stream_min_bytes && stream_supported(v, x.dtype);
        // Few rows (outer * inner <= 8) and a long l range the TMA kernel does not take: the
        // column and row kernels would run a block or two; the l range goes over the GPU instead.
        if (!tma && bvec_small_supported(v)) {
            int n = 1;
            cudaError_t e = launch_bvec(v, x.dtype, s, &n);
            if (e == cudaSuccess && n > 1) g_launches += (unsigned long long)(n - 1);
            return note_launch(e, K_BVEC);
        }
        if (v.inner == 1) {
            if (tma && v.nq >= 16) return note_launch(launch_stream(v, x.dtype, s), K_STREAM_ROWS);
            return note_launch(launch_rowdot(v, x.dtype, s), K_ROWDOT);
        }
        if (tma) return note_launch(launch_stream(v, x.dtype, s), K_STREAM_COLS);
        return note_launch(launch_colvec(v, x.dtype, s), K_COLVEC);
    }
    if (precision == TLIBTTM_PREC_DEFAULT) precision = g_precision.load();
    if (precision == TLIBTTM_PREC_AUTO)
        precision = (x.dtype == TLIBTTM_F32 && tc_supported(v, TLIBTTM_PREC_BF16X3)) ? TLIBTTM_PREC_BF16X3
                                                                                     : TLIBTTM_PREC_PLAIN;
    if (precision == TLIBTTM_PREC_BF16X3 || precision == TLIBTTM_PREC_FP8) {
        if (x.dtype != TLIBTTM_F32)
            return fail(TLIBTTM_ERR_UNSUPPORTED, "tlibttm: the bf16x3 and fp8 precisions take float operands.");
    }
    if (precision == TLIBTTM_PREC_OZAKI && x.dtype != TLIBTTM_F64)
        return fail(TLIBTTM_ERR_UNSUPPORTED, "tlibttm: the ozaki precision takes double operands.");
    if (precision == TLIBTTM_PREC_FP8 || precision == TLIBTTM_PREC_OZAKI) {
        // an explicit 8-bit request never falls back to other arithmetic silently
        if (!tc8_supported(v, precision, x.dtype))
            return fail(TLIBTTM_ERR_UNSUPPORTED, precision == TLIBTTM_PREC_OZAKI
                                                     ? "tlibttm: the ozaki path takes n_q <= 16384 (exact int32 sums)."
                                                     : "tlibttm: the fp8 path cannot run this problem.");
        if (precision == TLIBTTM_PREC_FP8 && tc_pair8_supported(v)) {
            // one launch: the fibre scales and the e4m3 operand are made from the resident tile
            int dev = 0;
            cudaError_t e = cudaGetDevice(&dev);
            int* status = nullptr;
            if (e == cudaSuccess) e = tc_status_word(dev, &status);
            if (e == cudaSuccess) e = launch_tc_pair8(v, status, s);
            return note_launch(e, K_TC_FP8_PAIR);
        }
        int kid = K_NONE, n = 0;
        cudaError_t e = launch_tc8(v, precision, x.dtype, s, &kid, &n);
        if (e == cudaSuccess && n > 1) g_launches += (unsigned long long)(n - 1);   // exponent and slicer kernels
        return note_launch(e, kid);
    }
    // Few output rows and a long l range: stream B over the whole GPU (exact FMA; these shapes are
    // bound by reading B, so a split into bf16 parts would gain nothing).
    if (bvec_supported(v)) {
        int n = 1;
        cudaError_t e = launch_bvec(v, x.dtype, s, &n);
        if (e == cudaSuccess && n > 1) g_launches += (unsigned long long)(n - 1);
        return note_launch(e, K_BVEC);
    }
    if (precision != TLIBTTM_PREC_PLAIN && tc_supported(v, precision)) {
        // The single-SM tensor-core kernel has no K split: when its tiles fill less than half the
        // GPU and the l range is long, the split-K SIMT GEMM (exact) is the faster choice.
        int sms = 0;
        const bool few = !tc_pair_supported(v) && v.nq >= 2048 &&
                         cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0) == cudaSuccess &&
                         tc_single_tiles(v) * 2 < sms;
        if (!few) {
            int kid = K_NONE;
            cudaError_t e = launch_tc(v, precision, s, &kid);
            if (e == cudaSuccess && kid == K_TC_BF16X3) ++g_launches;   // the operand-split kernel that precedes it
            return note_launch(e, kid);
        }
    }
    int n = 1;
    cudaError_t e = launch_simt_gemm(v, x.dtype, s, &n);
    if (e == cudaSuccess && n > 1) g_launches += (unsigned long long)(n - 1);   // the reduction of a split K loop
    return note_launch(e, K_SIMT_GEMM);
}

// ---- staging of host operands ---------------------------------------------------------------
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct Pool {
    std::mutex mu;
    DevBuf a, b, c;
};

std::mutex g_pools_mu;
std::unordered_map<int, Pool*> g_pools;

Pool& pool_for(int dev)
{
    std::lock_guard<std::mutex> lk(g_pools_mu);
    Pool*& p = g_pools[dev];
    if (!p) p = new Pool();
    return *p;
}

cudaError_t ensure(DevBuf& b, size_t bytes)
{
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.ptr) {
        cudaError_t e = cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = dev_malloc(&b.ptr, bytes);
    if (e == cudaSuccess) b.bytes = bytes;
    return e;
}

enum class Where { Host, Device };

int classify(const void* ptr, int dev, Where& w)
{
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        w = Where::Host;
        return TLIBTTM_OK;
    }
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
        if (at.type == cudaMemoryTypeDevice && at.device != dev)
            return fail(TLIBTTM_ERR_ARG, "tlibttm: device operand lives on a device other than the current one.");
        w = Where::Device;
    } else {
        w = Where::Host;
    }
    return TLIBTTM_OK;
}

// ---- pipelined staging of large host operands ----------------------------------------------
// A large TTM with host operands is cut into chunks of whole slices (along `outer`) or, when there
// are few slices, into column blocks of each slice (along `inner`, 2-D copies). Chunk c is copied
// in on the copy-in stream, contracted on the compute stream and copied out on the copy-out
// stream, with a ring of kRing device buffers, so both PCIe directions and the kernels overlap.
constexpr int kRing = 3;
constexpr size_t kChunkBytes = size_t(256) << 20;    // target bytes of A per chunk
constexpr size_t kPipelineMinBytes = size_t(64) << 20;

struct PipeState {
    std::mutex mu;
    bool init = false;
    cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
    cudaEvent_t ev_in[kRing], ev_comp[kRing], ev_out[kRing], ev_b, ev_user, ev_done;
    DevBuf a[kRing], c[kRing], b;
};

std::mutex g_pipe_mu;
std::unordered_map<int, PipeState*> g_pipes;

PipeState* pipe_for(int dev)
{
    std::lock_guard<std::mutex> lk(g_pipe_mu);
    PipeState*& p = g_pipes[dev];
    if (!p) p = new PipeState();
    return p;
}

cudaError_t pipe_init(PipeState& ps)
{
    if (ps.init) return cudaSuccess;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&ps.in, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if ((e = cudaStreamCreateWithFlags(&ps.comp, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if ((e = cudaStreamCreateWithFlags(&ps.out, cudaStreamNonBlocking)) != cudaSuccess) return e;
    for (int i = 0; i < kRing; ++i) {
        if ((e = cudaEventCreateWithFlags(&ps.ev_in[i], cudaEventDisableTiming)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&ps.ev_comp[i], cudaEventDisableTiming)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&ps.ev_out[i], cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    if ((e = cudaEventCreateWithFlags(&ps.ev_b, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&ps.ev_user, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&ps.ev_done, cudaEventDisableTiming)) != cudaSuccess) return e;
    ps.init = true;
    return cudaSuccess;
}

// True when the pipelined path applies: dense, large, A and C both host memory, and chunkable
// either along outer (enough slices) or along inner in multiples of 128.
bool pipeline_applies(const Plan& pl, size_t es, Where wa, Where wc)
{
    if (!pl.dense || wa != Where::Host || wc != Where::Host) return false;
    if (pl.a_elems * es < kPipelineMinBytes) return false;
    return pl.v.outer >= 8 || pl.v.inner % 128 == 0;
}

int run_pipelined(const Args& x, Plan& pl, int precision, cudaStream_t user, Where wb, int dev)
{
    const size_t es = x.dtype == TLIBTTM_F32 ? sizeof(float) : sizeof(double);
    const View3 full = pl.v;
    PipeState& ps = *pipe_for(dev);
    std::lock_guard<std::mutex> lk(ps.mu);
    cudaError_t e = pipe_init(ps);
    if (e != cudaSuccess) return cuda_fail(e, "pipeline set-up");

    // Chunk geometry.
    const size_t slice_bytes = (size_t)(full.nq * full.inner) * es;
    const bool by_outer = full.outer >= 8;
    int64_t kstep = 1, istep = full.inner;
    if (by_outer) {
        kstep = std::max<int64_t>(1, (int64_t)(kChunkBytes / slice_bytes));
        kstep = std::min<int64_t>(kstep, (full.outer + kRing - 1) / kRing);
    } else {
        istep = std::max<int64_t>(128, (int64_t)(kChunkBytes / ((size_t)full.nq * es)) / 128 * 128);
        istep = std::min<int64_t>(istep, full.inner);
    }
    const size_t a_chunk = (size_t)(kstep * full.nq * istep) * es;
    const size_t c_chunk = (size_t)(kstep * full.m * istep) * es;
    for (int i = 0; i < kRing; ++i) {
        if (ensure(ps.a[i], a_chunk) != cudaSuccess || ensure(ps.c[i], c_chunk) != cudaSuccess)
            return fail(TLIBTTM_ERR_ALLOC, "tlibttm: staging allocation failed.");
    }
    // Order after the caller's prior work on its stream.
    if ((e = cudaEventRecord(ps.ev_user, user)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    for (cudaStream_t st : {ps.in, ps.comp, ps.out})
        if ((e = cudaStreamWaitEvent(st, ps.ev_user, 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");

    const void* bdev = x.b;
    if (wb == Where::Host) {
        if (ensure(ps.b, pl.b_elems * es) != cudaSuccess) return fail(TLIBTTM_ERR_ALLOC, "tlibttm: staging allocation for B failed.");
        if ((e = cudaMemcpyAsync(ps.b.ptr, x.b, pl.b_elems * es, cudaMemcpyHostToDevice, ps.in)) != cudaSuccess)
            return cuda_fail(e, "copy of B");
        bdev = ps.b.ptr;
    }
    if ((e = cudaEventRecord(ps.ev_b, ps.in)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if ((e = cudaStreamWaitEvent(ps.comp, ps.ev_b, 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");

    const char* ha = static_cast<const char*>(x.a);
    char* hc = static_cast<char*>(x.c);
    int chunk = 0;
    int rc = TLIBTTM_OK;
    for (int64_t k0 = 0; k0 < full.outer && rc == TLIBTTM_OK; k0 += kstep) {
        const int64_t kn = std::min<int64_t>(kstep, full.outer - k0);
        for (int64_t i0 = 0; i0 < full.inner && rc == TLIBTTM_OK; i0 += istep, ++chunk) {
            const int64_t in = std::min<int64_t>(istep, full.inner - i0);
            const int r = chunk % kRing;
            if (chunk >= kRing) {
                // slot r is free once its previous compute and copy-out are done
                if ((e = cudaStreamWaitEvent(ps.in, ps.ev_comp[r], 0)) != cudaSuccess) return cuda_fail(e, "wait");
                if ((e = cudaStreamWaitEvent(ps.comp, ps.ev_out[r], 0)) != cudaSuccess) return cuda_fail(e, "wait");
            }
            char* da = static_cast<char*>(ps.a[r].ptr);
            char* dc = static_cast<char*>(ps.c[r].ptr);
            if (by_outer) {
                e = cudaMemcpyAsync(da, ha + (size_t)(k0 * full.nq * full.inner) * es, (size_t)(kn * full.nq * full.inner) * es,
                                    cudaMemcpyHostToDevice, ps.in);
            } else {
                e = cudaMemcpy2DAsync(da, (size_t)in * es, ha + (size_t)(k0 * full.nq * full.inner + i0) * es,
                                      (size_t)full.inner * es, (size_t)in * es, (size_t)full.nq, cudaMemcpyHostToDevice, ps.in);
            }
            if (e != cudaSuccess) return cuda_fail(e, "copy of A");
            if ((e = cudaEventRecord(ps.ev_in[r], ps.in)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
            if ((e = cudaStreamWaitEvent(ps.comp, ps.ev_in[r], 0)) != cudaSuccess) return cuda_fail(e, "wait");

            Args d = x;
            d.a = da;
            d.b = bdev;
            d.c = dc;
            Plan sub = pl;
            sub.v.outer = kn;
            sub.v.inner = in;
            rc = run_device(d, sub, precision, ps.comp);
            if (rc) break;
            if ((e = cudaEventRecord(ps.ev_comp[r], ps.comp)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
            if ((e = cudaStreamWaitEvent(ps.out, ps.ev_comp[r], 0)) != cudaSuccess) return cuda_fail(e, "wait");
            if (by_outer) {
                e = cudaMemcpyAsync(hc + (size_t)(k0 * full.m * full.inner) * es, dc, (size_t)(kn * full.m * full.inner) * es,
                                    cudaMemcpyDeviceToHost, ps.out);
            } else {
                e = cudaMemcpy2DAsync(hc + (size_t)(k0 * full.m * full.inner + i0) * es, (size_t)full.inner * es, dc,
                                      (size_t)in * es, (size_t)in * es, (size_t)full.m, cudaMemcpyDeviceToHost, ps.out);
            }
            if (e != cudaSuccess) return cuda_fail(e, "copy of C");
            if ((e = cudaEventRecord(ps.ev_out[r], ps.out)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
        }
    }
    for (cudaStream_t st : {ps.in, ps.comp, ps.out}) {
        cudaError_t e2 = cudaStreamSynchronize(st);
        if (e2 != cudaSuccess && rc == TLIBTTM_OK) rc = cuda_fail(e2, "cudaStreamSynchronize");
    }
    if (rc) return rc;
    if (tc_read_status())
        return fail(TLIBTTM_ERR_DEVICE, "tlibttm: a tensor-core kernel gave up on a bounded wait; its output is invalid.");
    return TLIBTTM_OK;
}

int run(const Args& x, int precision, void* stream)
{
    int rc = validate(x);
    if (rc) return rc;
    Plan pl;
    rc = make_plan(x, pl);
    if (rc) return rc;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    Where wa, wb, wc;
    if ((rc = classify(x.a, dev, wa)) || (rc = classify(x.b, dev, wb)) || (rc = classify(x.c, dev, wc))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    if (wa == Where::Device && wb == Where::Device && wc == Where::Device) return run_device(x, pl, precision, s);

    // At least one host operand: stage through the pool and block until done.
    const size_t es = x.dtype == TLIBTTM_F32 ? sizeof(float) : sizeof(double);
    if (pipeline_applies(pl, es, wa, wc)) return run_pipelined(x, pl, precision, s, wb, dev);
    Pool& pool = pool_for(dev);
    std::lock_guard<std::mutex> lk(pool.mu);
    Args d = x;
    if (wa == Where::Host) {
        if ((e = ensure(pool.a, pl.a_elems * es)) != cudaSuccess) return fail(TLIBTTM_ERR_ALLOC, "tlibttm: staging allocation for A failed.");
        if ((e = cudaMemcpyAsync(pool.a.ptr, x.a, pl.a_elems * es, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(e, "copy of A");
        d.a = pool.a.ptr;
    }
    if (wb == Where::Host) {
        if ((e = ensure(pool.b, pl.b_elems * es)) != cudaSuccess) return fail(TLIBTTM_ERR_ALLOC, "tlibttm: staging allocation for B failed.");
        if ((e = cudaMemcpyAsync(pool.b.ptr, x.b, pl.b_elems * es, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(e, "copy of B");
        d.b = pool.b.ptr;
    }
    if (wc == Where::Host) {
        if ((e = ensure(pool.c, pl.c_elems * es)) != cudaSuccess) return fail(TLIBTTM_ERR_ALLOC, "tlibttm: staging allocation for C failed.");
        // A non-dense C has gaps the kernel does not write: bring them along so they survive.
        if (!pl.dense)
            if ((e = cudaMemcpyAsync(pool.c.ptr, x.c, pl.c_elems * es, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(e, "copy of C");
        d.c = pool.c.ptr;
    }
    rc = run_device(d, pl, precision, s);
    if (rc) {
        cudaStreamSynchronize(s);
        return rc;
    }
    if (wc == Where::Host)
        if ((e = cudaMemcpyAsync(x.c, d.c, pl.c_elems * es, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_fail(e, "copy of C");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    if (tc_read_status())
        return fail(TLIBTTM_ERR_DEVICE, "tlibttm: a tensor-core kernel gave up on a bounded wait; its output is invalid.");
    return TLIBTTM_OK;
}

// ---- plans ----------------------------------------------------------------------------------
// Batched plans: problems with at least this many elements of A take their own launch of the
// kernel the planner picks for them (bf16x3 under auto/bf16x3 for m > 16, the small-m kernels
// for m <= 16); smaller ones share the grouped launch. Measured on the 512-problem workload, the
// specialised kernels beat the grouped launch's generic tiles well below the single-call
// threshold above.
constexpr int64_t kPlanSingleMinElems = int64_t(1) << 18;
// Small-m problems the TMA-fed kernel does not take run on their own from this size
constexpr int64_t kPlanSmallSingleMinElems = int64_t(1) << 22;
constexpr int kPlanStreams = 4;     // worker streams the singles of a batched plan spread over

struct Single {            // one problem launched on its own inside a plan
    int dtype;
    const void* a;
    const void* b;
    void* c;
    Plan pl;
};

int run_single(Single& sg, int precision, cudaStream_t s)
{
    Args x{};
    x.dtype = sg.dtype;
    x.a = sg.a;
    x.b = sg.b;
    x.c = sg.c;
    // a plan streams many problems through HBM: the TMA-fed small-m kernel pays off from 4 MB
    return run_device(x, sg.pl, precision, s, kPlanStreamMinBytes);
}

// Kernels run_device launches for a plan entry (tensor-core paths launch two).
int launches_of(const Single& sg, int dtype, int precision)
{
    if (!sg.pl.dense) return 1;
    if (sg.pl.v.m <= kSmallM) {
        const View3& v = sg.pl.v;
        const int64_t a_bytes = v.outer * v.nq * v.inner * (dtype == TLIBTTM_F32 ? 4 : 8);
        const bool tma = a_bytes >= kPlanStreamMinBytes && stream_supported(v, dtype);
        return (!tma && bvec_small_supported(v)) ? 2 : 1;
    }
    int pr = precision == TLIBTTM_PREC_DEFAULT ? g_precision.load() : precision;
    if (pr == TLIBTTM_PREC_AUTO)
        pr = (dtype == TLIBTTM_F32 && tc_supported(sg.pl.v, TLIBTTM_PREC_BF16X3)) ? TLIBTTM_PREC_BF16X3 : TLIBTTM_PREC_PLAIN;
    if (pr == TLIBTTM_PREC_FP8 && tc_pair8_supported(sg.pl.v)) return 1;
    if (pr == TLIBTTM_PREC_FP8 || pr == TLIBTTM_PREC_OZAKI) return tc8_launches(sg.pl.v, pr);
    if (bvec_supported(sg.pl.v)) return 2;
    if (pr != TLIBTTM_PREC_PLAIN && tc_supported(sg.pl.v, pr)) {
        int sms = 0;
        const bool few = !tc_pair_supported(sg.pl.v) && sg.pl.v.nq >= 2048 &&
                         cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0) == cudaSuccess &&
                         tc_single_tiles(sg.pl.v) * 2 < sms;
        if (!few) return tc_pair_supported(sg.pl.v) ? 1 : 2;
    }
    return simt_gemm_launch_count(sg.pl.v, dtype);
}

}  // namespace

unsigned long long wait_limit_ns()
{
    const unsigned long long v = g_wait_ns.load();
    return v ? v : 4000000000ull;
}

bool take_skip_b() { return g_skip_b.exchange(0) != 0; }

}  // namespace tlibttm

struct tlibttm_plan_s {
    int type = 0;          // 0 batched, 1 chain
    int dtype = 0, precision = 0, dev = 0;
    // batched
    std::vector<tlibttm::GroupDesc> descs;
    tlibttm::GroupDesc* d_desc = nullptr;   // slice-GEMM problems, then small-m problems
    unsigned long long* d_queue = nullptr;   // [2]: work counters of the two grouped launches
    int64_t total = 0;                       // slice-GEMM work items
    int grid = 0;
    int n_small = 0;                         // small-m problems (the last descriptors)
    int64_t stotal = 0;                      // their work items
    int sgrid = 0;
    std::vector<tlibttm::Single> singles;   // individual launches (batched extras, or chain steps)
    tlibttm::TcGroup* tcg = nullptr;         // batched: the grouped bf16x3 launch
    tlibttm::StreamGroup* sg = nullptr;      // batched: the grouped small-m launch
    // chain
    void* bufs[2] = {nullptr, nullptr};
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t own = nullptr;
    // fork/join of batched singles: worker streams and their events (created on first run)
    cudaStream_t workers[tlibttm::kPlanStreams] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t joins[tlibttm::kPlanStreams] = {};
};

namespace tlibttm {
namespace {

int plan_run_impl(tlibttm_plan* P, cudaStream_t s)
{
    int rc;
    cudaError_t e;
    // Batched plans with several singles fork them over worker streams (largest first, round
    // robin) and join them back into s; chain plans run their steps in order on s.
    // The grouped bf16x3 launch takes worker stream 0 and the singles the others, so that they
    // run side by side.
    const bool fan = P->type == 0 && (P->singles.size() > 1 || (P->tcg && !P->singles.empty()));
    const int w0 = (fan && P->tcg) ? 1 : 0;   // first worker stream of the singles
    if (fan) {
        if (!P->fork) {
            if ((e = cudaEventCreateWithFlags(&P->fork, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
            for (int w = 0; w < kPlanStreams; ++w)
                if ((e = cudaStreamCreateWithFlags(&P->workers[w], cudaStreamNonBlocking)) != cudaSuccess ||
                    (e = cudaEventCreateWithFlags(&P->joins[w], cudaEventDisableTiming)) != cudaSuccess)
                    return cuda_fail(e, "cudaStreamCreate");
        }
        if ((e = cudaEventRecord(P->fork, s)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
        for (int w = 0; w < kPlanStreams; ++w)
            if ((e = cudaStreamWaitEvent(P->workers[w], P->fork, 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
    }
    if (P->tcg) {
        if ((rc = note_launch(tc_group_run(P->tcg, fan ? P->workers[0] : s), K_TC_BF16X3))) return rc;
        g_launches += (unsigned long long)(tc_group_launches(P->tcg) - 1);
    }
    if (P->sg && stream_group_launches(P->sg) > 0) {
        if ((rc = note_launch(stream_group_run(P->sg, s), K_STREAM_COLS))) return rc;
        g_launches += (unsigned long long)(stream_group_launches(P->sg) - 1);
    }
    if (P->type == 0 && !P->descs.empty()) {
        e = cudaMemsetAsync(P->d_queue, 0, 2 * sizeof(unsigned long long), s);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
        const int n_gemm = (int)P->descs.size() - P->n_small;
        if (P->total > 0 &&
            (rc = note_launch(launch_grouped(P->d_desc, n_gemm, P->total, P->d_queue, P->dtype, P->grid, s), K_GROUPED)))
            return rc;
        if (P->stotal > 0 &&
            (rc = note_launch(launch_grouped_small(P->d_desc + n_gemm, P->n_small, P->stotal, P->d_queue + 1, P->dtype,
                                                   P->sgrid, s),
                              K_GROUPED)))
            return rc;
    }
    for (size_t i = 0; i < P->singles.size(); ++i)
        if ((rc = run_single(P->singles[i], P->precision,
                             fan ? P->workers[w0 + (int)(i % (size_t)(kPlanStreams - w0))] : s)))
            return rc;
    if (fan) {
        for (int w = 0; w < kPlanStreams; ++w) {
            if ((e = cudaEventRecord(P->joins[w], P->workers[w])) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
            if ((e = cudaStreamWaitEvent(s, P->joins[w], 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
        }
    }
    return TLIBTTM_OK;
}

void plan_free(tlibttm_plan* P)
{
    if (!P) return;
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    if (P->d_desc) cudaFree(P->d_desc);
    if (P->d_queue) cudaFree(P->d_queue);
    tc_group_destroy(P->tcg);
    stream_group_destroy(P->sg);
    for (void* b : P->bufs)
        if (b) cudaFree(b);
    if (P->own) cudaStreamDestroy(P->own);
    for (int w = 0; w < kPlanStreams; ++w) {
        if (P->workers[w]) cudaStreamDestroy(P->workers[w]);
        if (P->joins[w]) cudaEventDestroy(P->joins[w]);
    }
    if (P->fork) cudaEventDestroy(P->fork);
    delete P;
}

std::string problem_prefix(size_t i) { return "problem " + std::to_string(i) + ": "; }



}  // namespace
}  // namespace tlibttm

using namespace tlibttm;

extern "C" {

int tlibttm_ttm_f32(unsigned q, unsigned p, const float* a, const size_t* na, const size_t* wa,
                    const size_t* pia, const float* b, const size_t* nb, const size_t* pib, float* c,
                    const size_t* nc, const size_t* wc, void* stream)
{
    Args x{TLIBTTM_F32, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc};
    return run(x, TLIBTTM_PREC_DEFAULT, stream);
}

int tlibttm_ttm_f64(unsigned q, unsigned p, const double* a, const size_t* na, const size_t* wa,
                    const size_t* pia, const double* b, const size_t* nb, const size_t* pib, double* c,
                    const size_t* nc, const size_t* wc, void* stream)
{
    Args x{TLIBTTM_F64, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc};
    return run(x, TLIBTTM_PREC_DEFAULT, stream);
}

int tlibttm_ttm_ex(int dtype, int precision, unsigned q, unsigned p, const void* a, const size_t* na,
                   const size_t* wa, const size_t* pia, const void* b, const size_t* nb, const size_t* pib,
                   void* c, const size_t* nc, const size_t* wc, void* stream)
{
    if (dtype != TLIBTTM_F32 && dtype != TLIBTTM_F64) return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown dtype.");
    if (precision < TLIBTTM_PREC_DEFAULT || precision > TLIBTTM_PREC_AUTO)
        return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown precision.");
    Args x{dtype, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc};
    return run(x, precision, stream);
}

static bool sched_valid_view(int dtype, int schedule, const View3& v)
{
    switch (schedule) {
    case TLIBTTM_SCHED_HEURISTIC:
    case TLIBTTM_SCHED_SIMT_GEMM: return true;
    case TLIBTTM_SCHED_COLS:
    case TLIBTTM_SCHED_COLS_SPLIT: return v.m <= kSmallM && v.inner >= 2;
    case TLIBTTM_SCHED_ROWS: return v.m <= kSmallM && v.inner == 1;
    case TLIBTTM_SCHED_TC_BF16X3: return dtype == TLIBTTM_F32 && tc_supported(v, TLIBTTM_PREC_BF16X3);
    case TLIBTTM_SCHED_COLS_TMA: return stream_supported(v, dtype);
    case TLIBTTM_SCHED_TC_BF16X3_PAIR: return dtype == TLIBTTM_F32 && tc_pair_supported(v);
    case TLIBTTM_SCHED_SIMT_SPLIT: return v.nq >= 2048;
    case TLIBTTM_SCHED_BVEC: return bvec_supported(v);
    default: return false;
    }
}

int tlibttm_ttm_sched(int dtype, int schedule, unsigned q, unsigned p, const void* a, const size_t* na,
                      const size_t* wa, const size_t* pia, const void* b, const size_t* nb, const size_t* pib,
                      void* c, const size_t* nc, const size_t* wc, void* stream)
{
    if (dtype != TLIBTTM_F32 && dtype != TLIBTTM_F64) return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown dtype.");
    if (schedule < 0 || schedule >= TLIBTTM_SCHED_COUNT) return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown schedule.");
    Args x{dtype, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc};
    int rc = validate(x);
    if (rc) return rc;
    Plan pl;
    if ((rc = make_plan(x, pl))) return rc;
    if (!pl.dense) return fail(TLIBTTM_ERR_UNSUPPORTED, "tlibttm_ttm_sched: A and C must be dense under their layout.");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    Where w1, w2, w3;
    if ((rc = classify(a, dev, w1)) || (rc = classify(b, dev, w2)) || (rc = classify(c, dev, w3))) return rc;
    if (w1 != Where::Device || w2 != Where::Device || w3 != Where::Device)
        return fail(TLIBTTM_ERR_ARG, "tlibttm_ttm_sched: a, b and c must be device memory.");
    View3 v = pl.v;
    v.a = a;
    v.b = b;
    v.c = c;
    if (!sched_valid_view(dtype, schedule, v))
        return fail(TLIBTTM_ERR_UNSUPPORTED, "tlibttm_ttm_sched: the schedule cannot run this problem.");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (schedule) {
    case TLIBTTM_SCHED_HEURISTIC: return run_device(x, pl, TLIBTTM_PREC_PLAIN, s);
    case TLIBTTM_SCHED_SIMT_GEMM: {
        int n = 1;
        e = launch_simt_gemm(v, dtype, s, &n);
        if (e == cudaSuccess && n > 1) g_launches += (unsigned long long)(n - 1);
        return note_launch(e, K_SIMT_GEMM);
    }
    case TLIBTTM_SCHED_COLS: return note_launch(launch_colvec_ls(v, dtype, 1, s), K_COLVEC);
    case TLIBTTM_SCHED_COLS_SPLIT: return note_launch(launch_colvec_ls(v, dtype, 8, s), K_COLVEC);
    case TLIBTTM_SCHED_ROWS: return note_launch(launch_rowdot(v, dtype, s), K_ROWDOT);
    case TLIBTTM_SCHED_COLS_TMA:
        return note_launch(launch_stream(v, dtype, s), v.inner == 1 ? K_STREAM_ROWS : K_STREAM_COLS);
    case TLIBTTM_SCHED_SIMT_SPLIT:
    case TLIBTTM_SCHED_BVEC: {
        int n = 1;
        e = schedule == TLIBTTM_SCHED_BVEC ? launch_bvec(v, dtype, s, &n) : launch_simt_gemm(v, dtype, s, &n, true);
        if (e == cudaSuccess && n > 1) g_launches += (unsigned long long)(n - 1);
        return note_launch(e, schedule == TLIBTTM_SCHED_BVEC ? K_BVEC : K_SIMT_GEMM);
    }
    case TLIBTTM_SCHED_TC_BF16X3_PAIR: {
        int* status = nullptr;
        if ((e = tc_status_word(dev, &status)) != cudaSuccess) return cuda_fail(e, "tensor-core state");
        return note_launch(launch_tc_pair(v, status, s), K_TC_PAIR);
    }
    default: {
        int kid = K_NONE;
        e = launch_tc_single(v, s, &kid);
        if (e == cudaSuccess) ++g_launches;
        return note_launch(e, kid);
    }
    }
}

int tlibttm_schedule_valid(int dtype, int schedule, unsigned q, unsigned p, const size_t* na, const size_t* pia,
                           size_t m)
{
    if (!na || !pia || p == 0 || q == 0 || q > p) return 0;
    if (!tlib::ttm::detail::is_valid_shape(na, na + p) || !tlib::ttm::detail::is_valid_layout(pia, pia + p) || m == 0)
        return 0;
    unsigned qh = 0;
    while (pia[qh] != q) ++qh;
    View3 v{};
    v.inner = 1;
    v.outer = 1;
    for (unsigned r = 0; r < qh; ++r) v.inner *= (int64_t)na[pia[r] - 1];
    for (unsigned r = qh + 1; r < p; ++r) v.outer *= (int64_t)na[pia[r] - 1];
    v.nq = (int64_t)na[q - 1];
    v.m = (int64_t)m;
    alignas(16) static const float aligned_probe[4] = {0, 0, 0, 0};
    v.a = aligned_probe;   // alignment of the real operands is checked again when the schedule runs
    return sched_valid_view(dtype, schedule, v) ? 1 : 0;
}

// No counterpart in the reference: the bf16x3 contraction without any device
// allocation (declaration and contract in include/tlibttm.h).
int tlibttm_ttm_f32_bf16x3_noalloc(unsigned q, unsigned p, const float* a, const size_t* na, const size_t* wa,
                                   const size_t* pia, const float* b, const size_t* nb, const size_t* pib, float* c,
                                   const size_t* nc, const size_t* wc, void* stream)
{
    Args x{TLIBTTM_F32, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc};
    int rc = validate(x);
    if (rc) return rc;
    Plan pl;
    if ((rc = make_plan(x, pl))) return rc;
    if (!pl.dense)
        return fail(TLIBTTM_ERR_UNSUPPORTED, "tlibttm_ttm_f32_bf16x3_noalloc: A and C must be dense under their layout.");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    Where wa_, wb_, wc_;
    if ((rc = classify(x.a, dev, wa_)) || (rc = classify(x.b, dev, wb_)) || (rc = classify(x.c, dev, wc_))) return rc;
    if (wa_ != Where::Device || wb_ != Where::Device || wc_ != Where::Device)
        return fail(TLIBTTM_ERR_ARG, "tlibttm_ttm_f32_bf16x3_noalloc: a, b and c must be device memory "
                                     "(host operands would need staging buffers).");
    View3 v = pl.v;
    v.a = x.a;
    v.b = x.b;
    v.c = x.c;
    if (!tc_supported(v, TLIBTTM_PREC_BF16X3))
        return fail(TLIBTTM_ERR_UNSUPPORTED, "tlibttm_ttm_f32_bf16x3_noalloc: shape not handled by the tensor-core "
                                             "kernel (needs m > 16, and inner >= 17 or q = pi_1).");
    if (tc_image_bytes(v) > kNoAllocImageBytes)
        return fail(TLIBTTM_ERR_ARG, "tlibttm_ttm_f32_bf16x3_noalloc: B needs a " + std::to_string(tc_image_bytes(v)) +
                                         "-byte split image; this entry point holds at most " +
                                         std::to_string(kNoAllocImageBytes) +
                                         " bytes (cols(m) * ceil(n_q/32)*32 * 4 bytes, cols(m) = ceil(m/16)*16 for m <= 256, "
                                         "else ceil(m/256)*256; e.g. m = 256 with n_q <= 1024).");
    int kid = K_NONE;
    e = launch_tc_noalloc(v, static_cast<cudaStream_t>(stream), &kid);
    if (e == cudaSuccess && kid == K_TC_BF16X3) ++g_launches;   // split_b_kernel; note_launch counts the main kernel
    return note_launch(e, kid);
}

int tlibttm_plan_batched(int dtype, int precision, size_t count, const tlibttm_problem* problems,
                         tlibttm_plan** plan)
{
    return tlibttm_plan_batched_ex(dtype, precision, count, problems, 0u, plan);
}

int tlibttm_plan_batched_ex(int dtype, int precision, size_t count, const tlibttm_problem* problems,
                            unsigned flags, tlibttm_plan** plan)
{
    if (!plan) return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_batched: plan pointer is null.");
    *plan = nullptr;
    if (flags & ~TLIBTTM_PLAN_FEW_LAUNCHES) return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_batched_ex: unknown flags.");
    // small-m problems of at least this many elements of A get launches of their own
    const int64_t small_single_min = (flags & TLIBTTM_PLAN_FEW_LAUNCHES) ? INT64_MAX : kPlanSmallSingleMinElems;
    if (dtype != TLIBTTM_F32 && dtype != TLIBTTM_F64) return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown dtype.");
    if (precision < TLIBTTM_PREC_DEFAULT || precision > TLIBTTM_PREC_AUTO)
        return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown precision.");
    if (count && !problems) return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_batched: problems pointer is null.");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    int prec = precision == TLIBTTM_PREC_DEFAULT ? g_precision.load() : precision;
    std::unique_ptr<tlibttm_plan, void (*)(tlibttm_plan*)> P(new tlibttm_plan_s(), plan_free);
    P->type = 0;
    P->dtype = dtype;
    P->precision = precision;
    P->dev = dev;
    const size_t es = dtype == TLIBTTM_F32 ? sizeof(float) : sizeof(double);
    const int64_t tile = dtype == TLIBTTM_F32 ? kGemmTileF32 : kGemmTileF64;
    struct Item { GroupDesc d; double cost; };
    std::vector<Item> items;
    std::vector<View3> tcviews;   // problems of the grouped bf16x3 launch
    std::vector<View3> sgviews;   // problems of the grouped small-m (TMA-fed) launch
    for (size_t i = 0; i < count; ++i) {
        const tlibttm_problem& pr = problems[i];
        Args x{dtype, pr.q, pr.p, pr.a, pr.na, pr.wa, pr.pia, pr.b, pr.nb, pr.pib, pr.c, pr.nc, pr.wc};
        int rc = validate(x);
        if (!rc) {
            Plan pl;
            rc = make_plan(x, pl);
            if (!rc) {
                Where wa, wb, wc;
                if ((rc = classify(x.a, dev, wa)) || (rc = classify(x.b, dev, wb)) || (rc = classify(x.c, dev, wc))) {
                } else if (wa != Where::Device || wb != Where::Device || wc != Where::Device) {
                    rc = fail(TLIBTTM_ERR_ARG, "plans take device operands only.");
                } else {
                    View3 v = pl.v;
                    v.a = x.a;
                    v.b = x.b;
                    v.c = x.c;
                    bool single = false;
                    const int64_t elems = v.outer * v.inner * v.nq;
                    if (pl.dense && v.m > kSmallM && (prec == TLIBTTM_PREC_FP8 || prec == TLIBTTM_PREC_OZAKI)) {
                        // the 8-bit paths run as their own launches; a problem they cannot run is an error
                        if (!tc8_supported(v, prec, dtype)) {
                            rc = fail(TLIBTTM_ERR_UNSUPPORTED, prec == TLIBTTM_PREC_FP8
                                                                   ? "the fp8 precision takes float operands."
                                                                   : "the ozaki precision takes double operands with n_q <= 16384.");
                            return fail(rc, problem_prefix(i) + g_err);
                        }
                        single = true;
                    }
                    if (pl.dense && v.m > kSmallM && dtype == TLIBTTM_F32 &&
                        (prec == TLIBTTM_PREC_BF16X3 || prec == TLIBTTM_PREC_AUTO) && tc_supported(v, TLIBTTM_PREC_BF16X3)) {
                        // bf16x3 (asked for, or chosen by auto as a single call would): every such
                        // problem joins the grouped tensor-core launch
                        tcviews.push_back(v);
                        continue;
                    }
                    // small m: the grouped TMA-fed launch where it takes the problem; else the column and
                    // row kernels, large problems in launches of their own, the others as work items of
                    // the grouped small-m launch
                    if (pl.dense && v.m <= kSmallM && stream_group_eligible(v, dtype)) {
                        sgviews.push_back(v);
                        continue;
                    }
                    if (pl.dense && v.m <= kSmallM && elems >= small_single_min) single = true;
                    // few rows and a long l range: the l-split launch (a work item would be one block)
                    if (pl.dense && bvec_small_supported(v)) single = true;
                    if (!pl.dense || single) {
                        P->singles.push_back(Single{dtype, x.a, x.b, x.c, pl});
                    } else {
                        GroupDesc d{};
                        d.a = x.a;
                        d.b = x.b;
                        d.c = x.c;
                        d.outer = v.outer;
                        d.nq = v.nq;
                        d.inner = v.inner;
                        d.m = v.m;
                        d.b_cm = v.b_cm;
                        const int64_t M = v.outer * v.inner;
                        const int64_t rv = 16 / (int64_t)es;
                        if (v.m <= kSmallM) {
                            d.kind = 1;
                            // work items: 256 rows (contiguous fibres) or 256 rows of one per lane
                            // (strided fibres) -- the tile sizes of rowdot / colvec_async
                            if (v.inner == 1) {
                                d.flags = 1 | ((reinterpret_cast<uintptr_t>(v.a) % 16 == 0 && v.nq % rv == 0) ? 2 : 0);
                                d.tiles_m = ceil_div(M, kGemvRows);
                            } else {
                                // column items: one row per lane (the asynchronous-copy tile takes
                                // any alignment; a 16-byte build would cost the launch registers)
                                d.flags = 0;
                                d.tiles_m = ceil_div(M, 8 * 32);
                            }
                            d.tiles_n = 1;
                        } else {
                            d.kind = 0;
                            d.tiles_m = ceil_div(M, tile);
                            d.tiles_n = ceil_div(v.m, tile);
                            const bool ak = v.inner == 1;
                            bool vec = (reinterpret_cast<uintptr_t>(v.a) % 16 == 0) && (reinterpret_cast<uintptr_t>(v.c) % 16 == 0);
                            vec = vec && (ak ? (v.nq % rv == 0 && v.m % rv == 0) : (v.inner % rv == 0));
                            d.flags = (ak ? 1 : 0) | (vec ? 2 : 0);
                        }
                        // cost ~ work-item count x work per item, for a largest-first order
                        const double per_item = d.kind == 0 ? (double)v.nq * tile * tile
                                                            : (double)v.nq * (d.flags & 1 ? kGemvRows : 8 * 32 * (d.flags & 2 ? rv : 1)) * 16;
                        items.push_back(Item{d, (double)(d.tiles_m * d.tiles_n) * per_item});
                    }
                }
            }
        }
        if (rc) return fail(rc, problem_prefix(i) + g_err);
    }
    std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.cost > y.cost; });
    // singles largest first, so that the round robin over the worker streams balances them
    auto work = [](const Single& sg) {
        const View3& v = sg.pl.v;
        return (double)v.outer * v.inner * v.nq * (1.0 + (double)v.m / 16.0);
    };
    std::stable_sort(P->singles.begin(), P->singles.end(),
                     [&](const Single& x, const Single& y) { return work(x) > work(y); });
    // slice-GEMM items first (one launch), then the small-m ones (the other launch); each list
    // numbers its items from 0, largest problems first
    for (int kind = 0; kind < 2; ++kind) {
        int64_t first = 0;
        for (Item& it : items) {
            if (it.d.kind != kind) continue;
            it.d.first = first;
            first += it.d.tiles_m * it.d.tiles_n;
            P->descs.push_back(it.d);
            if (kind == 1) ++P->n_small;
        }
        (kind == 0 ? P->total : P->stotal) = first;
    }
    if (!P->descs.empty()) {
        if ((e = dev_malloc(reinterpret_cast<void**>(&P->d_desc), P->descs.size() * sizeof(GroupDesc))) != cudaSuccess ||
            (e = dev_malloc(reinterpret_cast<void**>(&P->d_queue), 2 * sizeof(unsigned long long))) != cudaSuccess)
            return fail(TLIBTTM_ERR_ALLOC, "tlibttm_plan_batched: device allocation failed.");
        if ((e = cudaMemcpy(P->d_desc, P->descs.data(), P->descs.size() * sizeof(GroupDesc), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(e, "plan upload");
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        P->grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * grouped_blocks_per_sm(dtype), P->total));
        P->sgrid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * grouped_small_blocks_per_sm(dtype), P->stotal));
    }
    if (!tcviews.empty() && (e = tc_group_create(tcviews.data(), (int)tcviews.size(), &P->tcg)) != cudaSuccess)
        return e == cudaErrorMemoryAllocation ? fail(TLIBTTM_ERR_ALLOC, "tlibttm_plan_batched: device allocation failed.")
                                              : cuda_fail(e, "grouped bf16x3 set-up");
    if (!sgviews.empty() && (e = stream_group_create(sgviews.data(), (int)sgviews.size(), dtype, &P->sg)) != cudaSuccess)
        return e == cudaErrorMemoryAllocation ? fail(TLIBTTM_ERR_ALLOC, "tlibttm_plan_batched: device allocation failed.")
                                              : cuda_fail(e, "grouped small-m set-up");
    if (!P->singles.empty() && (e = tc_prepare_device()) != cudaSuccess) return cuda_fail(e, "tensor-core state");
    *plan = P.release();
    return TLIBTTM_OK;
}

int tlibttm_plan_chain(int dtype, int precision, unsigned p, const void* a, const size_t* na, const size_t* pia,
                       unsigned count, const unsigned* modes, const void* const* bs, const size_t* ms,
                       const size_t* pibs, void* c, tlibttm_plan** plan)
{
    if (!plan) return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_chain: plan pointer is null.");
    *plan = nullptr;
    if (dtype != TLIBTTM_F32 && dtype != TLIBTTM_F64) return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown dtype.");
    if (precision < TLIBTTM_PREC_DEFAULT || precision > TLIBTTM_PREC_AUTO)
        return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown precision.");
    if (count == 0) return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_chain: the chain is empty.");
    if (!na || !pia || !modes || !bs || !ms || !pibs)
        return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_chain: a metadata pointer is null.");
    if (p == 0) return fail(TLIBTTM_ERR_ARG, "Error in tlib::tensor_times_matrix: input tensor order should be greater zero.");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    std::unique_ptr<tlibttm_plan, void (*)(tlibttm_plan*)> P(new tlibttm_plan_s(), plan_free);
    P->type = 1;
    P->dtype = dtype;
    P->precision = precision;
    P->dev = dev;
    const size_t es = dtype == TLIBTTM_F32 ? sizeof(float) : sizeof(double);
    std::vector<size_t> cur(na, na + p), layout(pia, pia + p);
    // sizes of the intermediates (steps 0..count-2)
    size_t max_mid = 0;
    {
        std::vector<size_t> n = cur;
        for (unsigned s = 0; s + 1 < count; ++s) {
            if (modes[s] == 0 || modes[s] > p) break;
            n[modes[s] - 1] = ms[s];
            size_t tot = 1;
            for (size_t x : n) tot *= x;
            max_mid = std::max(max_mid, tot);
        }
    }
    if (count > 1) {
        for (int i = 0; i < 2; ++i)
            if ((e = dev_malloc(&P->bufs[i], std::max<size_t>(max_mid, 1) * es)) != cudaSuccess)
                return fail(TLIBTTM_ERR_ALLOC, "tlibttm_plan_chain: device allocation failed.");
    }
    const void* in = a;
    for (unsigned s = 0; s < count; ++s) {
        std::vector<size_t> nc = cur;
        const unsigned q = modes[s];
        if (q >= 1 && q <= p) nc[q - 1] = ms[s];
        std::vector<size_t> wa(p), wc(p), nb(2);
        tlib::ttm::detail::compute_strides(cur.begin(), cur.end(), layout.begin(), wa.begin());
        tlib::ttm::detail::compute_strides(nc.begin(), nc.end(), layout.begin(), wc.begin());
        nb[0] = ms[s];
        nb[1] = (q >= 1 && q <= p) ? cur[q - 1] : 0;
        void* out = (s + 1 == count) ? c : P->bufs[s & 1];
        // B_s's own column count is checked against the current extent through nb[1]: the caller
        // states B_s's rows only, so its columns are the current extent by construction.
        Args x{dtype, q, p, in, cur.data(), wa.data(), layout.data(), bs[s], nb.data(), pibs + 2 * s, out, nc.data(),
               wc.data()};
        int rc = validate(x);
        if (!rc) {
            Plan pl;
            rc = make_plan(x, pl);
            if (!rc) {
                Where w1, w2, w3;
                if ((rc = classify(in, dev, w1)) || (rc = classify(bs[s], dev, w2)) || (rc = classify(out, dev, w3))) {
                } else if (w1 != Where::Device || w2 != Where::Device || w3 != Where::Device) {
                    rc = fail(TLIBTTM_ERR_ARG, "plans take device operands only.");
                } else {
                    P->singles.push_back(Single{dtype, in, bs[s], out, pl});
                }
            }
        }
        if (rc) return fail(rc, "step " + std::to_string(s) + ": " + g_err);
        in = out;
        cur = nc;
    }
    if ((e = tc_prepare_device()) != cudaSuccess) return cuda_fail(e, "tensor-core state");
    *plan = P.release();
    return TLIBTTM_OK;
}

int tlibttm_plan_run(tlibttm_plan* plan, void* stream)
{
    if (!plan) return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_run: plan is null.");
    return plan_run_impl(plan, static_cast<cudaStream_t>(stream));
}

int tlibttm_plan_run_graph(tlibttm_plan* plan, void* stream)
{
    if (!plan) return fail(TLIBTTM_ERR_ARG, "tlibttm_plan_run_graph: plan is null.");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (!s) {
        // A graph cannot be captured on the legacy default stream; the plan's own stream is a
        // blocking one, so that like the default stream it runs after the work already queued
        // there (the inputs' producers) and before the work queued after it.
        if (!plan->own && (e = cudaStreamCreateWithFlags(&plan->own, cudaStreamDefault)) != cudaSuccess)
            return cuda_fail(e, "cudaStreamCreate");
        s = plan->own;
    }
    if (!plan->exec) {
        if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_fail(e, "cudaStreamBeginCapture");
        const unsigned long long before = g_launches;
        int rc = plan_run_impl(plan, s);
        g_launches = before;   // capture enqueues nothing; the replay below is what runs
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(s, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        plan->graph = g;
        if ((e = cudaGraphInstantiate(&plan->exec, g, 0)) != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    }
    if ((e = cudaGraphLaunch(plan->exec, s)) != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    g_launches += (unsigned long long)tlibttm_plan_launches(plan);
    if (!stream) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
        if (tc_read_status())
            return fail(TLIBTTM_ERR_DEVICE, "tlibttm: a tensor-core kernel gave up on a bounded wait; its output is invalid.");
    }
    return TLIBTTM_OK;
}

int tlibttm_plan_launches(const tlibttm_plan* plan)
{
    if (!plan) return 0;
    int n = (plan->type == 0 && plan->total > 0) ? 1 : 0;
    n += (plan->type == 0 && plan->stotal > 0) ? 1 : 0;
    n += tc_group_launches(plan->tcg) + stream_group_launches(plan->sg);
    for (const Single& sg : plan->singles) n += launches_of(sg, plan->dtype, plan->precision);
    return n;
}

int tlibttm_plan_destroy(tlibttm_plan* plan)
{
    plan_free(plan);
    return TLIBTTM_OK;
}

int tlibttm_inject(int what, long long arg)
{
    switch (what) {
    case TLIBTTM_INJECT_NONE:
        g_fail_alloc_in = 0;
        g_wait_ns = 0;
        g_skip_b = 0;
        return TLIBTTM_OK;
    case TLIBTTM_INJECT_FAIL_ALLOC:
        if (arg < 0) return fail(TLIBTTM_ERR_ARG, "tlibttm_inject: the allocation count must be >= 0.");
        g_fail_alloc_in = arg;
        return TLIBTTM_OK;
    case TLIBTTM_INJECT_WAIT_NS:
        if (arg < 0) return fail(TLIBTTM_ERR_ARG, "tlibttm_inject: the wait bound must be >= 0.");
        g_wait_ns = (unsigned long long)arg;
        return TLIBTTM_OK;
    case TLIBTTM_INJECT_SKIP_B_STAGE:
        g_skip_b = arg ? 1 : 0;
        return TLIBTTM_OK;
    default:
        return fail(TLIBTTM_ERR_ARG, "tlibttm_inject: unknown injection.");
    }
}

const char* tlibttm_last_error(void) { return g_err.c_str(); }

int tlibttm_set_precision(int precision)
{
    if (precision < TLIBTTM_PREC_PLAIN || precision > TLIBTTM_PREC_AUTO) return -1;
    return g_precision.exchange(precision);
}

int tlibttm_get_precision(void) { return g_precision.load(); }

const char* tlibttm_last_kernel(void) { return g_last_kernel; }

unsigned long long tlibttm_launch_count(int reset)
{
    unsigned long long n = g_launches;
    if (reset) g_launches = 0;
    return n;
}

int tlibttm_synchronize(void* stream)
{
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    if (tc_read_status())
        return fail(TLIBTTM_ERR_DEVICE, "tlibttm: a tensor-core kernel gave up on a bounded wait; its output is invalid.");
    if (tc_read_noalloc_status())
        return fail(TLIBTTM_ERR_DEVICE, "tlibttm: the last allocation-free bf16x3 launch gave up on a bounded wait.");
    return TLIBTTM_OK;
}

int tlibttm_release_buffers(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return TLIBTTM_ERR_CUDA;
    Pool& pool = pool_for(dev);
    std::lock_guard<std::mutex> lk(pool.mu);
    for (DevBuf* b : {&pool.a, &pool.b, &pool.c}) {
        if (b->ptr) cudaFree(b->ptr);
        b->ptr = nullptr;
        b->bytes = 0;
    }
    tc_release_buffers();
    return TLIBTTM_OK;
}

int tlibttm_device_alloc(void** ptr, size_t bytes)
{
    if (!ptr) return fail(TLIBTTM_ERR_ARG, "tlibttm_device_alloc: ptr is null.");
    *ptr = nullptr;
    if (bytes == 0) return TLIBTTM_OK;
    cudaError_t e = dev_malloc(ptr, bytes);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return cuda_fail(e, "tlibttm_device_alloc");
    }
    return TLIBTTM_OK;
}

int tlibttm_device_free(void* ptr)
{
    if (!ptr) return TLIBTTM_OK;
    cudaError_t e = cudaFree(ptr);
    return e == cudaSuccess ? TLIBTTM_OK : cuda_fail(e, "tlibttm_device_free");
}

int tlibttm_copy(void* dst, const void* src, size_t bytes)
{
    if (bytes == 0) return TLIBTTM_OK;
    if (!dst || !src) return fail(TLIBTTM_ERR_ARG, "tlibttm_copy: null pointer.");
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDefault);
    return e == cudaSuccess ? TLIBTTM_OK : cuda_fail(e, "tlibttm_copy");
}

int tlibttm_fill(int dtype, void* ptr, size_t count, double value, void* stream)
{
    if (dtype != TLIBTTM_F32 && dtype != TLIBTTM_F64) return fail(TLIBTTM_ERR_ARG, "tlibttm: unknown dtype.");
    if (count == 0) return TLIBTTM_OK;
    if (!ptr) return fail(TLIBTTM_ERR_ARG, "tlibttm_fill: null pointer.");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    Where w;
    int rc = classify(ptr, dev, w);
    if (rc) return rc;
    if (w != Where::Device) return fail(TLIBTTM_ERR_ARG, "tlibttm_fill: ptr must be device memory of the current device.");
    e = launch_fill(ptr, (int64_t)count, dtype, value, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? TLIBTTM_OK : cuda_fail(e, "fill");
}

int tlibttm_k_order_layout(size_t* layout, size_t p, size_t k)
{
    if (!layout || p == 0) return fail(TLIBTTM_ERR_ARG, "Error in tlib::ttm::detail::compute_k_order: range provided by begin and end not correct!");
    tlib::ttm::detail::compute_k_order_layout(layout, layout + p, k);
    return TLIBTTM_OK;
}

size_t tlibttm_inverse_mode(const size_t* layout, size_t p, size_t mode)
{
    try {
        return tlib::ttm::detail::inverse_mode(layout, layout + p, mode);
    } catch (std::exception const& ex) {
        g_err = ex.what();
        return 0;
    }
}

int tlibttm_strides(const size_t* shape, size_t p, const size_t* layout, size_t* strides)
{
    try {
        tlib::ttm::detail::compute_strides(shape, shape + p, layout, strides);
    } catch (std::exception const& ex) {
        return fail(TLIBTTM_ERR_ARG, ex.what());
    }
    return TLIBTTM_OK;
}

}  // extern "C"
