// 8-bit tensor-core paths (tcgen05 / TMEM) of the B200 TTM library.
//
// fp8   (float operands): every fibre of A (one row of the slice GEMM: fixed k, i, all l) and
//       every row of B gets a power-of-two scale that puts its largest magnitude in
//       [128, 256); the scaled values are rounded to e4m3 (round to nearest, saturating) and
//       multiplied on the tensor cores (kind::f8f6f4) with FP32 accumulation in TMEM. The
//       epilogue applies the two scales. Approximate: about 2^-4 relative per product.
//
// ozaki (double operands): the Ozaki scheme with integer slices (Ozaki, Ogita, Oishi & Rump,
//       2012; int8 tensor-core form as in Ootomo, Ozaki & Yokota, 2024). Every fibre of A and
//       row of B is scaled by a power of two 2^-e so that |x| < 1, then cut into S signed
//       7-bit digits: x = 2^e * sum_s d_s 2^-7(s+1), |d_s| <= 127, exactly (S = 7 keeps 49
//       bits). The products d^A_s d^B_t with s + t < S are computed exactly on the int8 tensor
//       cores (kind::i8, int32 accumulation in TMEM, one accumulator per diagonal s + t) and
//       recombined in FP64 in the epilogue: C = 2^(eA+eB) sum_d acc_d 2^-7(d+2). The dropped
//       diagonals and the digit truncation are below 2^-49 relative to the fibre maxima.
//       FP64 arithmetic on the GPU is limited to the exponent extraction, the digit
//       extraction and this recombination.
//
// Both run in three steps per chunk of rows of the slice GEMM: an exponent kernel, a slicer
// that writes the 8-bit operand image in the K-major 32-byte-swizzled layout the MMA reads
// (128 rows x 32 l per 4 KB block, S blocks per (row tile, l chunk)), and the MMA kernel.
// Rows enumerate (k, i) with i fastest, R = k * inner + i, so one code path serves every
// layout; B's rows are j. The operand images are scratch from the stream-ordered pool, at
// most about 1 GB per chunk of rows.
//
// MMA kernel warp roles (320 threads, one CTA per SM, persistent over tiles):
//   warp 0     bulk-copy producer: the A and B image blocks of one l chunk per stage
//   warp 1     TMEM allocator and MMA issuer (one lane)
//   warps 2-9  epilogue: TMEM -> registers -> scaled C, direct stores; two warps per TMEM lane
//              quarter, taking alternate 32-column chunks
// Every mbarrier wait is bounded; on expiry the CTA aborts as the bf16x3 kernel does.
#include <cuda.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <atomic>
#include <cstring>

#include "tc8_kernels.cuh"
#include "tc_kernels.cuh"
#include "tc_ptx.cuh"
#include "tlibttm.h"

namespace tlibttm {
namespace {

constexpr int kRows = 128;             // MMA M
constexpr int kLChunk = 32;            // l per stage (one 8-bit MMA K step)
constexpr int kBlock = kRows * 32;     // bytes of one 128-row image block
constexpr int kOzakiSlices = 7;       // the epilogue's exact two-part combination assumes 7
constexpr int kThreads8 = 10 * 32;           // producer, MMA, 8 epilogue warps
constexpr int kMaxStages8 = 8;
constexpr int kMaxNq8 = 16384;         // int32 accumulators stay exact: 7 * nq * 127^2 < 2^31
enum { MODE_FP8 = 0, MODE_I8 = 1 };

// Rows of an operand: element (R, l) sits at base + (R / d) * s1 + (R % d) * s0 + l * ls.
struct RowView {
    const void* base;
    int64_t rows, d, s1, s0, ls, nq;
};

__device__ __forceinline__ int64_t row_off(const RowView& v, int64_t R)
{
    const int64_t hi = R / v.d;
    return hi * v.s1 + (R - hi * v.d) * v.s0;
}

// exponent e of the largest |x| of each row: max|x| = f 2^e, f in [0.5, 1) (0 for zero rows).
template <typename T>
__global__ void row_exponent_kernel(RowView v, int64_t r0, int64_t nrows, int* __restrict__ ex)
{
    const T* a = static_cast<const T*>(v.base);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nrows; u += stride) {
        const T* p = a + row_off(v, r0 + u);
        T mx = T(0);
        for (int64_t l = 0; l < v.nq; ++l) mx = fmax(mx, fabs(p[l * v.ls]));
        int e = 0;
        if (mx > T(0)) frexp((double)mx, &e);
        ex[u] = e;
    }
}

// Rows whose l run is contiguous (ls == 1, long rows): one warp per row.
template <typename T>
__global__ void row_exponent_warp_kernel(RowView v, int64_t r0, int64_t nrows, int* __restrict__ ex)
{
    const T* a = static_cast<const T*>(v.base);
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < nrows; u += warps) {
        const T* p = a + row_off(v, r0 + u);
        T mx = T(0);
        for (int64_t l = lane; l < v.nq; l += 32) mx = fmax(mx, fabs(p[l]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) {
            int e = 0;
            if (mx > T(0)) frexp((double)mx, &e);
            ex[u] = e;
        }
    }
}

// 2^e as float / double, by construction where e is a normal exponent.
__device__ __forceinline__ float pow2f(int e)
{
    return (e >= -126 && e <= 127) ? __int_as_float((e + 127) << 23) : ldexpf(1.0f, e);
}
__device__ __forceinline__ double pow2d(int e)
{
    return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

// Slicer: rows [r0, r0 + nrows) -> image blocks [tile][kc][S][tile_rows x 32 B], tile_rows rows
// per tile (zero beyond the operand's rows and l extent). One thread per (row, l chunk, half):
// 16 consecutive l -> one 16-byte chunk per slice; the two halves of a row are neighbouring
// lanes, so that a warp writes whole 32-byte rows.
template <typename T, int MODE>
__global__ void slice_kernel(RowView v, int64_t r0, int64_t nrows, const int* __restrict__ ex, int S,
                             int tile_rows, int kchunks, uint8_t* __restrict__ img)
{
    const T* a = static_cast<const T*>(v.base);
    const int64_t tiles = (nrows + tile_rows - 1) / tile_rows;
    const int64_t total = tiles * kchunks * tile_rows * 2;
    const uint32_t block = (uint32_t)tile_rows * 32u;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += stride) {
        const int c = (int)(u & 1);
        const int row = (int)((u >> 1) % tile_rows);
        const int64_t tk = (u >> 1) / tile_rows;
        const int kc = (int)(tk % kchunks);
        const int64_t tile = tk / kchunks;
        const int64_t rr = tile * tile_rows + row;
        const bool rv = rr < nrows;
        const T* p = rv ? a + row_off(v, r0 + rr) : a;
        const int e = rv ? ex[rr] : 0;
        uint8_t* base = img + (size_t)((tile * kchunks + kc) * S) * block;
        {
            const int64_t l0 = (int64_t)kc * kLChunk + c * 16;
            uint8_t* dst = base + kmaj_sw32_off((uint32_t)row, (uint32_t)c);
            if (MODE == MODE_FP8) {
                // x * 2^(8-e) is exact (a power-of-two scaling; below e4m3's range it rounds to 0)
                const int sh = 8 - e;
                const bool fast = sh >= -126 && sh <= 127;
                const float sc = fast ? pow2f(sh) : 1.0f;
                uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    const int64_t l = l0 + t;
                    const float x = (rv && l < v.nq) ? (float)p[l * v.ls] : 0.0f;
                    const __nv_fp8_storage_t b =
                        __nv_cvt_float_to_fp8(fast ? x * sc : ldexpf(x, sh), __NV_SATFINITE, __NV_E4M3);
                    w[t >> 2] |= (uint32_t)b << ((t & 3) * 8);
                }
                *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
            } else {
                // |x| 2^(-e) < 1: its first 7 S bits, truncated, as one integer (exact scaling and
                // truncation toward zero), then cut into base-128 digits carrying x's sign
                const int sh = 7 * S - e;
                const bool fast = sh >= -1022 && sh <= 1023;
                const double sc = fast ? pow2d(sh) : 1.0;
                long long mag[16];
                bool neg[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    const int64_t l = l0 + t;
                    const double x = (rv && l < v.nq) ? (double)p[l * v.ls] : 0.0;
                    const long long X = __double2ll_rz(fast ? x * sc : ldexp(x, sh));
                    neg[t] = X < 0;
                    mag[t] = X < 0 ? -X : X;
                }
                for (int s = 0; s < S; ++s) {
                    const int shift = 7 * (S - 1 - s);
                    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
                    for (int t = 0; t < 16; ++t) {
                        const int d = (int)((mag[t] >> shift) & 127);
                        w[t >> 2] |= (uint32_t)(uint8_t)(int8_t)(neg[t] ? -d : d) << ((t & 3) * 8);
                    }
                    *reinterpret_cast<uint4*>(dst + (size_t)s * block) = make_uint4(w[0], w[1], w[2], w[3]);
                }
            }
        }
    }
}

struct Tc8Params {
    void* c;                  // FP32 (fp8) or FP64 (ozaki) output
    const uint8_t* aimg;      // [mt][kc][S][128 x 32 B] of this chunk of rows
    const uint8_t* bimg;      // [jb][kc][S][NT x 32 B]
    const int* aexp;          // per row of this chunk
    const int* bexp;          // per j
    int* status;
    int64_t r0, nrows;        // rows of this chunk
    int64_t inner, m;         // C(R, j) at (R / inner) * m * inner + j * inner + R % inner
    int64_t tiles;            // tiles_m * jblocks
    int jblocks, kchunks, nt, S, stages, nbuf;
};

// Instruction descriptors (M = 128, A and B K-major): kind::f8f6f4 with e4m3 x e4m3 -> f32, and
// kind::i8 with s8 x s8 -> s32.
__host__ __device__ constexpr uint32_t idesc_8bit(int mode, int n)
{
    return (mode == MODE_FP8 ? (1u << 4) : ((2u << 4) | (1u << 7) | (1u << 10))) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(kRows >> 4) << 24);
}

template <int MODE>
__device__ __forceinline__ void mma_8bit(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    if (MODE == MODE_FP8)
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n}\n"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
            : "memory");
    else
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
            : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(kThreads8, 1) tc8_kernel(Tc8Params P)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = P.S, NT = P.nt, ST = P.stages;
    const uint32_t a_bytes = (uint32_t)S * kBlock, b_block = (uint32_t)NT * 32u, b_bytes = (uint32_t)S * b_block;
    const uint32_t stage_bytes = a_bytes + b_bytes;
    uint8_t* ring = smem;
    uint8_t* ctrl = ring + (size_t)ST * stage_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(ctrl);
    uint64_t* empty = full + kMaxStages8;
    uint64_t* acc_full = empty + kMaxStages8;   // [2]
    uint64_t* acc_empty = acc_full + 2;         // [2]
    uint64_t* drain = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int D = MODE == MODE_FP8 ? 1 : S;     // accumulators per tile

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 8);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int kchunks = P.kchunks;

    if (warp == 0) {
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            int issued[kMaxStages8];
            for (int i = 0; i < kMaxStages8; ++i) issued[i] = -1;
            for (int64_t t = blockIdx.x; t < P.tiles && ok; t += gridDim.x) {
                const int64_t mt = t / P.jblocks, jb = t - mt * P.jblocks;
                for (int kc = 0; kc < kchunks; ++kc) {
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                    issued[s] = (int)ph;
                    mbar_expect_tx(&full[s], stage_bytes);
                    uint8_t* st = ring + (size_t)s * stage_bytes;
                    bulk_load(st, P.aimg + (size_t)(mt * kchunks + kc) * a_bytes, a_bytes, &full[s]);
                    bulk_load(st + a_bytes, P.bimg + (size_t)(jb * kchunks + kc) * b_bytes, b_bytes, &full[s]);
                    if (++s == ST) { s = 0; ph ^= 1; }
                }
            }
            for (int i = 0; i < ST; ++i) {
                if (issued[i] < 0) continue;
                const unsigned long long t0 = gtimer();
                while (!mbar_try(&full[i], (uint32_t)issued[i]) && gtimer() - t0 < kTimeoutNs) {}
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_8bit(MODE, NT);
            int s = 0;
            uint32_t ph = 0;
            int ab = 0;
            uint32_t cph = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; t < P.tiles && ok; t += gridDim.x) {
                if (!mbar_wait(&acc_empty[ab], cph ^ 1, abort_flag)) break;
                tc_fence_after();
                const uint32_t dcol = tmem_base + (uint32_t)(ab * D * NT);
                for (int kc = 0; kc < kchunks; ++kc) {
                    if (!mbar_wait(&full[s], ph, abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t sa = su32(ring + (size_t)s * stage_bytes), sb = sa + a_bytes;
                    // digit pairs (x, y) with x + y < S, accumulated on diagonal x + y; x = 0
                    // opens every diagonal at the first l chunk
                    for (int x = 0; x < S; ++x) {
                        const uint64_t ad = smem_desc(sa + (uint32_t)x * kBlock, 16u, 256u, kLayoutSW32);
                        for (int y = 0; x + y < S; ++y) {
                            const uint64_t bd = smem_desc(sb + (uint32_t)y * b_block, 16u, 256u, kLayoutSW32);
                            const int d = MODE == MODE_FP8 ? 0 : x + y;
                            mma_8bit<MODE>(dcol + (uint32_t)(d * NT), ad, bd, idesc, (kc == 0 && x == 0) ? 0u : 1u);
                        }
                    }
                    mma_commit(&empty[s]);
                    if (++s == ST) { s = 0; ph ^= 1; }
                }
                if (!ok) break;
                mma_commit(&acc_full[ab]);
                if (++ab == P.nbuf) { ab = 0; cph ^= 1; }
            }
            mma_commit(drain);
            const unsigned long long t0 = gtimer();
            while (!mbar_try(drain, 0) && gtimer() - t0 < kTimeoutNs) {}
        }
    } else {
        // ---------------------------------------------------------------- epilogue
        const int q4 = warp & 3;                 // TMEM lane quarter
        const int half = (warp - 2) >> 2;        // 32-column chunks of this parity
        int ab = 0;
        uint32_t aph = 0;
        for (int64_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
            if (!mbar_wait(&acc_full[ab], aph, abort_flag)) break;
            tc_fence_after();
            const int64_t mt = t / P.jblocks, jb = t - mt * P.jblocks;
            const int64_t rl = mt * kRows + q4 * 32 + lane;           // row within the chunk
            const bool rv = rl < P.nrows;
            const int64_t R = P.r0 + rl;
            const int64_t kk = R / P.inner;
            const int64_t cbase = kk * P.m * P.inner + (R - kk * P.inner);
            const int ea = rv ? P.aexp[rl] : 0;
            const uint32_t tb = tmem_base + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(ab * D * NT);
            for (int cc = half * 32; cc < NT; cc += 64) {
                const int64_t j0 = jb * NT + cc;
                const int eb_l = (j0 + lane < P.m) ? P.bexp[j0 + lane] : 0;
                if (MODE == MODE_FP8) {
                    // C = acc 2^(ea-8) 2^(eb-8): two exact power-of-two products
                    uint32_t v[32];
                    tmem_ld32(tb + (uint32_t)cc, v);
                    const float sa = pow2f(ea - 8), sb_l = pow2f(eb_l - 8);
                    float* C = static_cast<float*>(P.c);
                    float y[32];
#pragma unroll
                    for (int c = 0; c < 32; ++c) y[c] = __uint_as_float(v[c]) * sa * __shfl_sync(0xffffffffu, sb_l, c);
                    if (P.inner == 1 && j0 + 32 <= P.m && (((cbase + j0) & 3) == 0)) {
                        // this row's 32 columns are contiguous: 128-bit stores
                        if (rv) {
                            float4* cp = reinterpret_cast<float4*>(C + cbase + j0);
#pragma unroll
                            for (int c = 0; c < 8; ++c) cp[c] = make_float4(y[4 * c], y[4 * c + 1], y[4 * c + 2], y[4 * c + 3]);
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            if (rv && j0 + c < P.m) C[cbase + (j0 + c) * P.inner] = y[c];
                    }
                } else {
                    // sum_d acc_d 2^-7(d+2) = H 2^-28 + L 2^-56 with the exact integers
                    // H = sum_{d<3} acc_d 2^7(2-d) (< 2^43) and L = sum_{d>=3} acc_d 2^7(6-d) (< 2^52)
                    const double sa = pow2d(ea), sb_l = pow2d(eb_l - 28);   // row / this lane's column
                    double* C = static_cast<double*>(P.c);
#pragma unroll
                    for (int h16 = 0; h16 < 32; h16 += 16) {
                        long long H[16], Lo[16];
#pragma unroll
                        for (int c = 0; c < 16; ++c) H[c] = Lo[c] = 0;
#pragma unroll
                        for (int d = 0; d < kOzakiSlices; ++d) {
                            uint32_t v[16];
                            tmem_ld16(tb + (uint32_t)(d * NT + cc + h16), v);
#pragma unroll
                            for (int c = 0; c < 16; ++c) {
                                const long long x = (long long)(int)v[c];
                                if (d < 3) H[c] += x * (1LL << (7 * (2 - d)));
                                else Lo[c] += x * (1LL << (7 * (6 - d)));
                            }
                        }
                        double y[16];
#pragma unroll
                        for (int c = 0; c < 16; ++c)
                            y[c] = fma((double)Lo[c], 0x1p-28, (double)H[c]) * sa * __shfl_sync(0xffffffffu, sb_l, h16 + c);
                        const int64_t jc = j0 + h16;
                        if (P.inner == 1 && jc + 16 <= P.m && (((cbase + jc) & 1) == 0)) {
                            if (rv) {
                                double2* cp = reinterpret_cast<double2*>(C + cbase + jc);
#pragma unroll
                                for (int c = 0; c < 8; ++c) cp[c] = make_double2(y[2 * c], y[2 * c + 1]);
                            }
                        } else {
#pragma unroll
                            for (int c = 0; c < 16; ++c)
                                if (rv && jc + c < P.m) C[cbase + (jc + c) * P.inner] = y[c];
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[ab]);
            if (++ab == P.nbuf) { ab = 0; aph ^= 1; }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicExch(P.status, 1);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(512u));
    }
}

// ------------------------------------------------------------------ host side
int g_sms8 = 0;
std::atomic<uint64_t> g_smem_set8[2];

template <typename T>
cudaError_t launch_exponents(const RowView& v, int64_t r0, int64_t nrows, int* ex, cudaStream_t s)
{
    if (v.ls == 1 && v.nq >= 64) {
        const int64_t blocks = std::min<int64_t>((nrows * 32 + 255) / 256, 65535);
        row_exponent_warp_kernel<T><<<(int)blocks, 256, 0, s>>>(v, r0, nrows, ex);
    } else {
        const int64_t blocks = std::min<int64_t>((nrows + 255) / 256, 65535);
        row_exponent_kernel<T><<<(int)blocks, 256, 0, s>>>(v, r0, nrows, ex);
    }
    return cudaGetLastError();
}

template <typename T, int MODE>
cudaError_t launch_slices(const RowView& v, int64_t r0, int64_t nrows, const int* ex, int S, int tile_rows,
                          int kchunks, uint8_t* img, cudaStream_t s)
{
    const int64_t total = ((nrows + tile_rows - 1) / tile_rows) * kchunks * tile_rows * 2;
    const int64_t blocks = std::min<int64_t>((total + 255) / 256, (int64_t)g_sms8 * 16);
    slice_kernel<T, MODE><<<(int)std::max<int64_t>(blocks, 1), 256, 0, s>>>(v, r0, nrows, ex, S, tile_rows, kchunks,
                                                                            img);
    return cudaGetLastError();
}

struct Plan8 {
    int mode, S, nt, jblocks, kchunks, stages, nbuf;
    size_t smem;
    int64_t chunk_rows;
};

bool plan8(const View3& v, int precision, Plan8& p)
{
    p.mode = precision == TLIBTTM_PREC_FP8 ? MODE_FP8 : MODE_I8;
    p.S = p.mode == MODE_FP8 ? 1 : kOzakiSlices;
    const int D = p.mode == MODE_FP8 ? 1 : p.S;
    // N tile: the accumulators (D per buffer) fit the 512 TMEM columns, two buffers when they can
    const int64_t m16 = ((v.m + 15) / 16) * 16;
    int nt = (int)std::min<int64_t>(256, m16);
    while (nt > 16 && D * nt > 512) nt -= 16;
    if (D * nt > 512) return false;
    p.nt = nt;
    p.nbuf = 2 * D * nt <= 512 ? 2 : 1;
    p.jblocks = (int)((v.m + nt - 1) / nt);
    p.kchunks = (int)((v.nq + kLChunk - 1) / kLChunk);
    const size_t stage = (size_t)p.S * (kBlock + (size_t)nt * 32);
    const size_t avail = 227 * 1024 - 1024 - 256;
    p.stages = (int)std::min<size_t>(kMaxStages8, avail / stage);
    if (p.stages < 2) return false;
    p.smem = 1024 + (size_t)p.stages * stage + 256;
    // rows per chunk: a multiple of 128 with an A image of about 1 GB at most
    const size_t row_bytes = (size_t)p.kchunks * 32 * p.S;
    p.chunk_rows = std::max<int64_t>(kRows, (int64_t)((size_t(1) << 30) / row_bytes) / kRows * kRows);
    return true;
}

}  // namespace

bool tc8_supported(const View3& v, int precision, int dtype)
{
    if (v.m <= kSmallM) return false;
    if (precision == TLIBTTM_PREC_FP8) {
        if (dtype != TLIBTTM_F32) return false;
    } else if (precision == TLIBTTM_PREC_OZAKI) {
        if (dtype != TLIBTTM_F64 || v.nq > kMaxNq8) return false;
    } else {
        return false;
    }
    Plan8 p;
    return plan8(v, precision, p);
}

int tc8_launches(const View3& v, int precision)
{
    Plan8 p;
    if (!plan8(v, precision, p)) return 0;
    const int64_t rows = v.outer * v.inner;
    const int64_t chunk = std::min<int64_t>(p.chunk_rows, ((rows + kRows - 1) / kRows) * kRows);
    return (int)(2 + 3 * ((rows + chunk - 1) / chunk));   // B exponents + slicer, then per chunk three
}

cudaError_t launch_tc8(const View3& v, int precision, int dtype, cudaStream_t s, int* kid, int* launches)
{
    *launches = 0;
    *kid = precision == TLIBTTM_PREC_FP8 ? K_TC_FP8 : K_TC_OZAKI;
    if (!tc8_supported(v, precision, dtype)) return cudaErrorNotSupported;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!g_sms8) {
        e = cudaDeviceGetAttribute(&g_sms8, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    int* status = nullptr;
    if ((e = tc_status_word(dev, &status)) != cudaSuccess) return e;
    Plan8 p;
    plan8(v, precision, p);
    const bool fp8 = p.mode == MODE_FP8;
    const uint64_t bit = dev < 64 ? uint64_t(1) << dev : 0;
    if (!bit || !(g_smem_set8[p.mode].load() & bit)) {
        e = fp8 ? cudaFuncSetAttribute(tc8_kernel<MODE_FP8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)
                : cudaFuncSetAttribute(tc8_kernel<MODE_I8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return e;
        if (bit) g_smem_set8[p.mode].fetch_or(bit);
    }
    const int64_t rows = v.outer * v.inner;
    const int64_t chunk = std::min<int64_t>(p.chunk_rows, ((rows + kRows - 1) / kRows) * kRows);
    // scratch: B exponents + B image, A exponents + A image of one chunk
    const int64_t brows = (int64_t)p.jblocks * p.nt;
    const size_t bimg_bytes = (size_t)brows * p.kchunks * 32 * p.S;
    const size_t aimg_bytes = (size_t)chunk * p.kchunks * 32 * p.S;
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t total = up(brows * sizeof(int)) + up(bimg_bytes) + up(chunk * sizeof(int)) + up(aimg_bytes);
    uint8_t* scratch = nullptr;
    if ((e = dev_malloc_async(reinterpret_cast<void**>(&scratch), total, s)) != cudaSuccess) return e;
    int* bexp = reinterpret_cast<int*>(scratch);
    uint8_t* bimg = scratch + up(brows * sizeof(int));
    int* aexp = reinterpret_cast<int*>(bimg + up(bimg_bytes));
    uint8_t* aimg = reinterpret_cast<uint8_t*>(aexp) + up(chunk * sizeof(int));

    RowView bv{v.b, v.m, v.m, 0, v.b_cm ? 1 : v.nq, v.b_cm ? v.m : 1, v.nq};
    RowView av{v.a, rows, v.inner, v.nq * v.inner, 1, v.inner, v.nq};
    int n = 0;
    if (fp8) {
        e = launch_exponents<float>(bv, 0, v.m, bexp, s);
        if (e == cudaSuccess) e = launch_slices<float, MODE_FP8>(bv, 0, v.m, bexp, p.S, p.nt, p.kchunks, bimg, s);
    } else {
        e = launch_exponents<double>(bv, 0, v.m, bexp, s);
        if (e == cudaSuccess) e = launch_slices<double, MODE_I8>(bv, 0, v.m, bexp, p.S, p.nt, p.kchunks, bimg, s);
    }
    n += 2;
    for (int64_t r0 = 0; r0 < rows && e == cudaSuccess; r0 += chunk) {
        const int64_t nr = std::min<int64_t>(chunk, rows - r0);
        if (fp8) {
            e = launch_exponents<float>(av, r0, nr, aexp, s);
            if (e == cudaSuccess) e = launch_slices<float, MODE_FP8>(av, r0, nr, aexp, p.S, kRows, p.kchunks, aimg, s);
        } else {
            e = launch_exponents<double>(av, r0, nr, aexp, s);
            if (e == cudaSuccess) e = launch_slices<double, MODE_I8>(av, r0, nr, aexp, p.S, kRows, p.kchunks, aimg, s);
        }
        if (e != cudaSuccess) break;
        Tc8Params P{};
        P.c = v.c;
        P.aimg = aimg;
        P.bimg = bimg;
        P.aexp = aexp;
        P.bexp = bexp;
        P.status = status;
        P.r0 = r0;
        P.nrows = nr;
        P.inner = v.inner;
        P.m = v.m;
        P.jblocks = p.jblocks;
        P.kchunks = p.kchunks;
        P.nt = p.nt;
        P.S = p.S;
        P.stages = p.stages;
        P.nbuf = p.nbuf;
        P.tiles = ((nr + kRows - 1) / kRows) * p.jblocks;
        const int grid = (int)std::min<int64_t>(P.tiles, g_sms8);
        if (fp8) tc8_kernel<MODE_FP8><<<grid, kThreads8, p.smem, s>>>(P);
        else tc8_kernel<MODE_I8><<<grid, kThreads8, p.smem, s>>>(P);
        e = cudaGetLastError();
        n += 3;
    }
    cudaFreeAsync(scratch, s);
    *launches = n;
    return e;
}

}  // namespace tlibttm
