// fp8 on pairs of SMs: tcgen05.mma.cta_group::2.kind::f8f6f4 with B held in tensor memory and A
// read from HBM once.
//
// Arithmetic (the fp8 path of tc8_kernels.cu): every fibre of A (one tensor row: fixed k and i, all
// l) and every row j of B is scaled by 2^(8-e), max|x| = f 2^e with f in [0.5, 1) (e = 0 for an
// all-zero fibre), rounded to e4m3 (nearest even, saturating at +-448), multiplied exactly on the
// tensor cores with FP32 accumulation in tensor memory, and the epilogue multiplies by
// 2^(eA-8) 2^(eB-8). The separate path needs an exponent pass and an operand pass over A before
// its MMA kernel; here the converter warps find each fibre's exponent from the tile resident in
// shared memory (n_q <= 256, so a tile's fibres are whole) and convert it in place.
//
// MMA M = 256 rows j of B (CTA c of the cluster holds j in [128c, 128c + 128) as e4m3 in its
// tensor memory, 32 l per 8 columns), N = 64 tensor rows of a tile (32 per CTA, the MMA's B
// operand in shared memory, K-major with 32-byte rows and the 32-byte swizzle), K = 32 l per
// instruction: two instructions per 64-l stage. A tile's fibres must all be resident before any
// is converted, so tiles are kept small (8 KB per 64 l per CTA): up to eight tiles in flight.
//
// Warp roles (448 threads, one CTA per SM, clusters of two, persistent over tiles):
//   warp 0       TMA producer of this CTA's FP32 rows (32 rows x 64 l = 8 KB per stage);
//   warp 1       tensor-memory allocation (both CTAs) and, in the even CTA, the MMA issuer;
//   warps 2-9    converters, one warp per group (one lane per row of the CTA's half tile); group g
//                takes the tiles n = g (mod G) whole: it waits for all of the tile's stages, takes
//                each fibre's maximum, writes the fibre's factor 2^(eA-8) into both CTAs' shared
//                memory, then converts stage after stage in place (the e4m3 rows go to the stage's
//                last 2 KB, whose FP32 values every lane has read before);
//   warps 10-13  B -> e4m3 in tensor memory at the start; then the epilogue: tensor memory ->
//                scaled FP32 -> a 32 x 32 block staged in shared memory -> one TMA store
//                (direct stores when C is not a tensor map).
// Every mbarrier wait is bounded; on expiry the CTA raises its abort flag, drains its own copies
// and MMAs, frees tensor memory and raises the device status word. No TMA load uses multicast.
#include <cuda.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "tc_cluster.cuh"
#include "tc_kernels.cuh"
#include "tc_ptx.cuh"
#include "tlibttm.h"

namespace tlibttm {
namespace {

constexpr int kRows8 = 32;                    // tensor rows per CTA per tile (N / 2)
constexpr int kN8 = 64;                       // MMA N
constexpr int kM8 = 256;                      // MMA M
constexpr int kK8 = 32;                       // l per MMA (32 bytes of e4m3)
constexpr int kStageL8 = 64;                  // l per pipeline stage
constexpr uint32_t kStage8 = kRows8 * kStageL8 * 4;       // 8 KB FP32 stage
constexpr uint32_t kBox8 = kRows8 * 16 * 4;               // contiguous fibres: one 16-l box, 2 KB
constexpr uint32_t kOut8 = kStage8 - 2048;                // the e4m3 rows: the stage's last 2 KB
constexpr uint32_t kKStep8 = kRows8 * kK8;                // 1 KB of e4m3 per K step
constexpr int kConvWarps8 = 8, kGroupWarps8 = 1;          // one converter warp per group
constexpr int kMaxGroups8 = kConvWarps8 / kGroupWarps8;   // 8
constexpr int kEpiWarp08 = 2 + kConvWarps8;
constexpr int kEpiWarps8 = 4;
constexpr int kThreads8P = (kEpiWarp08 + kEpiWarps8) * 32;   // 448
constexpr uint32_t kEpiBuf8 = 32 * 32 * 4;
constexpr uint32_t kEpiBytes8 = kEpiWarps8 * 2 * kEpiBuf8;    // 32 KB
constexpr int kScaleSlots8 = 16;              // tiles whose fibre exponents are held at once
constexpr uint32_t kScaleBytes8 = kScaleSlots8 * kN8 * 4;     // 4 KB
constexpr int kMaxStages8P = 23;
constexpr uint32_t kAccCol8 = 256;            // accumulators at tensor-memory columns 256..511
constexpr size_t kCtrl8 = 1024;

enum { P8_MN = 0, P8_K = 1 };

struct Pair8Params {
    float* c;
    const float* b;
    int* status;
    int64_t outer, nq, inner, m;
    int64_t tiles;          // tiles of 128 tensor rows
    int64_t mper;           // rows mode: tiles per slice
    int kstages;            // 64-l stages per tile
    int nsub;               // 32-l MMA steps holding l < n_q
    int b_cm;
    int stages;             // A ring depth: groups * kstages
    int groups;             // converter groups in use (each owns one tile's slots)
    int tma_c;
    unsigned long long wait_ns;
};

// Instruction descriptor, kind::f8f6f4: D f32, A and B e4m3, both K-major, N = 64, M = 256.
constexpr uint32_t kIdesc8 = (1u << 4) | ((uint32_t)(kN8 >> 3) << 17) | ((uint32_t)(kM8 >> 4) << 24);

__device__ __forceinline__ void mma_pair8(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p, e;\n setp.ne.b32 p, %3, 0;\n elect.sync _|e, 0xffffffff;\n"
        " @e tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], [%1], %2, %4, p;\n}\n"
        ::"r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(acc), "r"(kIdesc8)
        : "memory");
}

__device__ __forceinline__ float pow2f8(int e)
{
    return (e >= -126 && e <= 127) ? __int_as_float((e + 127) << 23) : ldexpf(1.0f, e);
}

// e with max|x| = f 2^e, f in [0.5, 1); 0 for 0.
__device__ __forceinline__ int fibre_exponent(float mx)
{
    int e = 0;
    if (mx > 0.0f) frexpf(mx, &e);
    return e;
}

// x 2^(8-e) rounded to e4m3 (nearest even, saturating); the scaling is exact where 2^(8-e) is a
// normal float (FAST), else done by ldexpf, as the operand pass of the separate fp8 path does.
// Separate builds for the two cases, so that the common one carries no ldexpf.
template <bool FAST>
__device__ __forceinline__ uint32_t to_e4m3(float x, float sc, int sh)
{
    return (uint32_t)__nv_cvt_float_to_fp8(FAST ? x * sc : ldexpf(x, sh), __NV_SATFINITE, __NV_E4M3);
}

// Four values (lowest l in the lowest byte) to e4m3, two conversions at a time.
template <bool FAST>
__device__ __forceinline__ uint32_t pack4_e4m3(const float (&x)[4], float sc, int sh)
{
    float y[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) y[e] = FAST ? x[e] * sc : ldexpf(x[e], sh);
    const uint32_t lo = __nv_cvt_float2_to_fp8x2(make_float2(y[0], y[1]), __NV_SATFINITE, __NV_E4M3);
    const uint32_t hi = __nv_cvt_float2_to_fp8x2(make_float2(y[2], y[3]), __NV_SATFINITE, __NV_E4M3);
    return (lo & 0xffffu) | (hi << 16);
}

// Element (row, l) of an FP32 stage: rows of i are [64 l][32 i]; contiguous fibres are four
// [32 k][16 l] boxes with the 64-byte swizzle.
template <int GEOM>
__device__ __forceinline__ float stage_elem(const uint8_t* st, int row, int l)
{
    if (GEOM == 0) return *reinterpret_cast<const float*>(st + l * (kRows8 * 4) + row * 4);
    const int sb = l >> 4, lc = (l & 15) >> 2;
    return *reinterpret_cast<const float*>(st + sb * kBox8 + row * 64 + ((lc ^ ((row >> 1) & 3)) << 4) + (l & 3) * 4);
}

// One converter lane's row of a stage to e4m3 in the stage's last 2 KB (K-major, 32-byte rows,
// 32-byte swizzle); `hold` carries l 48..63, which live in those bytes and were read before.
template <int GEOM, bool FAST>
__device__ __forceinline__ void convert_row(uint8_t* sp, int row, const float (&hold)[16], float sc, int sh)
{
#pragma unroll
    for (int c = 0; c < 4; ++c) {   // 16-l chunks: K step c / 2, 16-byte half c % 2
        uint32_t w[4];
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            float x[4];
#pragma unroll
            for (int b4 = 0; b4 < 4; ++b4)
                x[b4] = c == 3 ? hold[q4 * 4 + b4] : stage_elem<GEOM>(sp, row, c * 16 + q4 * 4 + b4);
            w[q4] = pack4_e4m3<FAST>(x, sc, sh);
        }
        *reinterpret_cast<uint4*>(sp + kOut8 + (c >> 1) * kKStep8 + kmaj_sw32_off((uint32_t)row, (uint32_t)(c & 1))) =
            make_uint4(w[0], w[1], w[2], w[3]);
    }
}

template <int GEOM>
__global__ void __launch_bounds__(kThreads8P, 1)
    tc_pair8_kernel(const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap cmap, Pair8Params P)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int AS = P.stages, G = P.groups;
    uint8_t* ring = smem;
    uint8_t* epi = smem + (size_t)AS * kStage8;
    float* scales = reinterpret_cast<float*>(epi + kEpiBytes8);   // [kScaleSlots8][128] 2^(eA-8) per fibre
    uint64_t* a_full = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(scales) + kScaleBytes8);
    uint64_t* a_empty = a_full + kMaxStages8P;
    uint64_t* a_conv = a_empty + kMaxStages8P;      // even CTA: both CTAs' converters are done
    uint64_t* acc_full = a_conv + kMaxStages8P;     // [2]
    uint64_t* acc_empty = acc_full + 2;             // [2] even CTA
    uint64_t* drain = acc_empty + 2;                // [1]
    uint64_t* sc_full = drain + 1;                  // [kScaleSlots8] both CTAs' exponents written
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sc_full + kScaleSlots8);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const int64_t cid = cluster_index(), ncl = cluster_count();
    const int64_t tiles = P.tiles;
    const int kst = P.kstages;

    if (threadIdx.x == 0) {
        for (int s = 0; s < AS; ++s) {
            mbar_init(&a_full[s], 1);
            mbar_init(&a_empty[s], 1);
            mbar_init(&a_conv[s], 2 * kGroupWarps8);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2 * kEpiWarps8);
        }
        mbar_init(drain, 1);
        for (int q = 0; q < kScaleSlots8; ++q) mbar_init(&sc_full[q], 2 * kGroupWarps8);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    int eb = 0;   // epilogue lanes: the exponent of their row j of B
    if (warp >= kEpiWarp08) {
        // B -> e4m3 in tensor memory: lane q4 * 32 + lane holds row j = 128 rank + q4 * 32 + lane;
        // 32 l per 8 columns (4 per 32-bit column, lowest l in the lowest byte), zero outside B
        const int q4 = warp & 3;
        const int64_t j = (int64_t)rank * 128 + q4 * 32 + lane;
        const uint32_t trow = tmem_base + ((uint32_t)(q4 * 32) << 16);
        auto bval = [&](int64_t l) -> float {
            return (j < P.m && l < P.nq) ? __ldg(P.b_cm ? P.b + j + l * P.m : P.b + j * P.nq + l) : 0.0f;
        };
        float mx = 0.0f;
        for (int64_t l = 0; l < P.nq; ++l) mx = fmaxf(mx, fabsf(bval(l)));
        eb = fibre_exponent(mx);
        const int sh = 8 - eb;
        const bool fast = sh >= -126 && sh <= 127;
        const float sc = fast ? pow2f8(sh) : 1.0f;
        for (int g = 0; g < P.nsub; ++g) {
            uint32_t w[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                uint32_t x = 0;
#pragma unroll
                for (int b4 = 0; b4 < 4; ++b4) {
                    const float y = bval((int64_t)g * kK8 + c * 4 + b4);
                    x |= (fast ? to_e4m3<true>(y, sc, sh) : to_e4m3<false>(y, sc, sh)) << (8 * b4);
                }
                w[c] = x;
            }
            tmem_st8(trow + (uint32_t)(g * 8), w);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    cluster_sync_all();   // barriers initialised and B resident in both CTAs
    tc_fence_after();

    if (warp == 0) {
        // ------------------------------------------------------------- TMA producer (own rows)
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            int issued[kMaxStages8P];
            for (int i = 0; i < kMaxStages8P; ++i) issued[i] = -1;
            for (int64_t t = cid; t < tiles && ok; t += ncl) {
                int64_t k = 0, r0;
                if (GEOM == P8_MN) {
                    k = t / P.mper;
                    r0 = (t - k * P.mper) * kN8 + (int64_t)rank * kRows8;
                } else {
                    r0 = t * kN8 + (int64_t)rank * kRows8;
                }
                for (int st = 0; st < kst; ++st) {
                    if (!mbar_wait(&a_empty[s], ph ^ 1, abort_flag, P.wait_ns)) { ok = false; break; }
                    issued[s] = (int)ph;
                    mbar_expect_tx(&a_full[s], kStage8);
                    uint8_t* dst = ring + (size_t)s * kStage8;
                    const int l0 = st * kStageL8;
                    if (GEOM == P8_MN) {
                        tma_load_3d(dst, &amap, &a_full[s], (int)r0, l0, (int)k);   // [64 l][32 i]
                    } else {
#pragma unroll
                        for (int sb = 0; sb < 4; ++sb)   // [32 k][16 l] each, 64-byte swizzle
                            tma_load_2d(dst + sb * kBox8, &amap, &a_full[s], l0 + sb * 16, (int)r0);
                    }
                    if (++s == AS) { s = 0; ph ^= 1; }
                }
            }
            for (int i = 0; i < AS; ++i) {
                if (issued[i] < 0) continue;
                const unsigned long long t0 = gtimer();
                while (!mbar_try(&a_full[i], (uint32_t)issued[i]) && gtimer() - t0 < kTimeoutNs) {}
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- MMA issuer (even CTA)
        if (rank == 0) {
            // K-major, 32-byte rows with the 32-byte swizzle: 8-row atoms of 256 bytes
            const uint64_t db0 = smem_desc(su32(ring + kOut8), 16u, 256u, kLayoutSW32);
            int s = 0, ab = 0;
            uint32_t ph = 0, cph = 0;
            bool ok = true;
            for (int64_t t = cid; t < tiles && ok; t += ncl) {
                if (!__all_sync(0xffffffffu, mbar_wait(&acc_empty[ab], cph ^ 1, abort_flag, P.wait_ns))) break;
                tc_fence_after();
                const uint32_t dcol = tmem_base + kAccCol8 + (uint32_t)(ab * kN8);
                for (int st = 0; st < kst; ++st) {
                    if (!__all_sync(0xffffffffu, mbar_wait(&a_conv[s], ph, abort_flag, P.wait_ns))) { ok = false; break; }
                    tc_fence_after();
                    const uint64_t ds = db0 + ((uint64_t)((size_t)s * kStage8) >> 4);
#pragma unroll
                    for (int sub = 0; sub < 2; ++sub) {
                        const int g = st * 2 + sub;
                        if (g >= P.nsub) continue;   // l past n_q in the last stage
                        mma_pair8(dcol, tmem_base + (uint32_t)(g * 8), ds + (uint64_t)((sub * kKStep8) >> 4),
                                  g == 0 ? 0u : 1u);
                    }
                    commit_pair(&a_empty[s], 0x3);   // both CTAs' stage s is free once these are done
                    if (++s == AS) { s = 0; ph ^= 1; }
                }
                if (!ok) break;
                commit_pair(&acc_full[ab], 0x3);
                if (++ab == 2) { ab = 0; cph ^= 1; }
            }
            commit_pair(drain, 0x1);
            const unsigned long long t0 = gtimer();
            while (!mbar_try(drain, 0) && gtimer() - t0 < kTimeoutNs) {}
            __syncwarp();
        }
    } else if (warp < kEpiWarp08) {
        // ------------------------------------------------------------- converters
        const int g = (warp - 2) / kGroupWarps8;
        const int row = lane;                                       // this lane's fibre
        const uint32_t conv0 = peer_addr(su32(&a_conv[0]), 0);      // the even CTA's a_conv[0]
        const uint32_t scf0[2] = {peer_addr(su32(&sc_full[0]), 0), peer_addr(su32(&sc_full[0]), 1)};
        const uint32_t scl0[2] = {peer_addr(su32(scales), 0), peer_addr(su32(scales), 1)};
        bool ok = true;
        int64_t ts = 0;   // tile sequence number of this cluster
        for (int64_t t = cid; t < tiles; t += ncl, ++ts) {
            if (g >= G || (int)(ts % G) != g) continue;
            // Every stage of the tile has landed (the group's slots, stage after stage).
            bool have = ok;
            for (int st = 0; st < kst; ++st) {
                const int64_t n = ts * kst + st;
                const int s = (int)(n % AS);
                const bool got = have && mbar_wait(&a_full[s], (uint32_t)((n / AS) & 1), abort_flag, P.wait_ns);
                have = __all_sync(0xffffffffu, got);
            }
            if (!have) ok = false;
            // The fibre's exponent over all of its l (entries past n_q are the copy's zero fill).
            float mx = 0.0f;
            if (have) {
                float m4[4] = {0.0f, 0.0f, 0.0f, 0.0f};   // four chains, so the loads overlap
                for (int st = 0; st < kst; ++st) {
                    const uint8_t* sp = ring + (size_t)((ts * kst + st) % AS) * kStage8;
#pragma unroll 16
                    for (int l = 0; l < kStageL8; ++l) m4[l & 3] = fmaxf(m4[l & 3], fabsf(stage_elem<GEOM>(sp, row, l)));
                }
                mx = fmaxf(fmaxf(m4[0], m4[1]), fmaxf(m4[2], m4[3]));
            }
            const int ea = fibre_exponent(mx);
            // the fibre's factor 2^(eA-8) goes to both CTAs: the two epilogues scale all 128 columns
            const int q = (int)(ts % kScaleSlots8);
            const uint32_t soff = (uint32_t)((q * kN8 + (int)rank * kRows8 + row) * 4);
            const uint32_t fa = __float_as_uint(pow2f8(ea - 8));
            st_cluster_u32(scl0[0] + soff, fa);
            st_cluster_u32(scl0[1] + soff, fa);
            const int sh = 8 - ea;
            const bool fast = sh >= -126 && sh <= 127;
            const float sc = fast ? pow2f8(sh) : 1.0f;
            for (int st = 0; st < kst; ++st) {
                const int s = (int)((ts * kst + st) % AS);
                uint8_t* sp = ring + (size_t)s * kStage8;
                // l 48..63 occupy the bytes the e4m3 rows go to: read them before anyone writes
                float hold[16];
                if (have) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) hold[e] = stage_elem<GEOM>(sp, row, 48 + e);
                }
                __syncwarp();   // the group is one warp
                if (have) {
                    if (fast) convert_row<GEOM, true>(sp, row, hold, sc, sh);
                    else convert_row<GEOM, false>(sp, row, hold, sc, sh);
                    fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_remote(conv0 + (uint32_t)s * 8u);
                }
            }
            // the factors stored above are published now, after the conversions, so that the
            // cluster-scope fence does not hold up the MMAs (the epilogues need them only once
            // the tile's MMAs are done)
            fence_acq_rel_cluster();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_remote_release_cluster(scf0[0] + (uint32_t)q * 8u);
                mbar_arrive_remote_release_cluster(scf0[1] + (uint32_t)q * 8u);
            }
        }
    } else {
        // ------------------------------------------------------------- epilogue
        const int q4 = warp & 3;
        uint8_t* stage0 = epi + (size_t)(warp - kEpiWarp08) * 2 * kEpiBuf8;
        const int64_t j0 = (int64_t)rank * 128 + q4 * 32;           // first row of C this warp holds
        const int64_t j = j0 + lane;                                 // this lane's row
        const uint32_t empty0 = peer_addr(su32(&acc_empty[0]), 0);
        const int64_t rlim = GEOM == P8_MN ? P.inner : P.outer;     // tensor rows of one slice
        const float sb_l = pow2f8(eb - 8);
        int sb = 0, ab = 0;
        uint32_t aph = 0;
        int64_t ts = 0;
        for (int64_t t = cid; t < tiles; t += ncl, ++ts) {
            if (!mbar_wait(&acc_full[ab], aph, abort_flag, P.wait_ns)) break;
            const int q = (int)(ts % kScaleSlots8);
            if (!mbar_wait_cluster(&sc_full[q], (uint32_t)((ts / kScaleSlots8) & 1), abort_flag, P.wait_ns)) break;
            tc_fence_after();
            int64_t k = 0, r0;
            if (GEOM == P8_MN) {
                k = t / P.mper;
                r0 = (t - k * P.mper) * kN8;
            } else {
                r0 = t * kN8;
            }
            const float* sq = scales + q * kN8;
            const uint32_t tb = tmem_base + ((uint32_t)(q4 * 32) << 16) + kAccCol8 + (uint32_t)(ab * kN8);
            for (int cc = 0; cc < kN8; cc += 32) {
                uint32_t v[32];
                tmem_ld32(tb + (uint32_t)cc, v);
                const int64_t r = r0 + cc;                           // first tensor row of these columns
                if (j0 >= P.m || r >= rlim) continue;                // the block lies outside C
                // C = acc 2^(eA-8) 2^(eB-8): two exact power-of-two products
#pragma unroll
                for (int c = 0; c < 32; ++c) v[c] = __float_as_uint(__uint_as_float(v[c]) * sq[cc + c] * sb_l);
                if (P.tma_c) {
                    uint8_t* buf = stage0 + sb * kEpiBuf8;
                    if (lane == 0) bulk_wait_read1();   // the store that last read `buf` has read it
                    __syncwarp();
                    if (GEOM == P8_MN) {
                        // [32 j][32 i] with the 128-byte swizzle: this lane owns row j
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            *reinterpret_cast<uint4*>(buf + lane * 128 + ((c ^ (lane & 7)) << 4)) =
                                make_uint4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                    } else {
                        // [32 k][32 j]: this lane owns column j
                        float* b32 = reinterpret_cast<float*>(buf);
#pragma unroll
                        for (int c = 0; c < 32; ++c) b32[c * 32 + lane] = __uint_as_float(v[c]);
                    }
                    fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) {
                        if (GEOM == P8_MN) tma_store_3d(&cmap, buf, (int)r, (int)j0, (int)k);
                        else tma_store_2d(&cmap, buf, (int)j0, (int)r);
                        bulk_commit();
                    }
                    sb ^= 1;
                } else if (j < P.m) {
                    // direct stores (C not 16-byte aligned for a tensor map)
                    if (GEOM == P8_MN) {
                        float* p = P.c + (k * P.m + j) * P.inner + r;
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            if (r + c < P.inner) p[c] = __uint_as_float(v[c]);
                    } else {
                        float* p = P.c + r * P.m + j;
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            if (r + c < P.outer) p[(int64_t)c * P.m] = __uint_as_float(v[c]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_remote(empty0 + (uint32_t)ab * 8u);
            if (++ab == 2) { ab = 0; aph ^= 1; }
        }
        if (lane == 0) bulk_wait_all();   // every TMA store of this warp has completed
    }

    tc_fence_before();
    __syncthreads();
    cluster_sync_all();   // the even CTA's MMAs have completed; no arrivals are in flight
    if (threadIdx.x == 0 && *abort_flag) atomicExch(P.status, 1);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(512u));
    }
}

typedef CUresult (*EncodeTiledFn8)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn8 encode_fn8()
{
    static EncodeTiledFn8 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn8>(p);
    });
    return fn;
}

// A in boxes of 32 rows x 64 l: rows of i a 3-D box (32 i, 64 l, 1 k); contiguous fibres 2-D boxes
// of 16 l x 32 rows with the 64-byte swizzle (four per stage).
bool encode_pair8_map(const View3& v, int geom, CUtensorMap* map)
{
    EncodeTiledFn8 enc = encode_fn8();
    if (!enc) return false;
    CUresult r;
    if (geom == P8_MN) {
        cuuint64_t dims[3] = {(cuuint64_t)v.inner, (cuuint64_t)v.nq, (cuuint64_t)v.outer};
        cuuint64_t strides[2] = {(cuuint64_t)v.inner * 4, (cuuint64_t)v.inner * v.nq * 4};
        cuuint32_t box[3] = {kRows8, kStageL8, 1};
        cuuint32_t es[3] = {1, 1, 1};
        r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(v.a), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        cuuint64_t dims[2] = {(cuuint64_t)v.nq, (cuuint64_t)v.outer};
        cuuint64_t strides[1] = {(cuuint64_t)v.nq * 4};
        cuuint32_t box[2] = {16, kRows8};
        cuuint32_t es[2] = {1, 1};
        r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(v.a), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

std::mutex g_pair8_mu;
int g_pair8_clusters[64][2] = {};

template <int GEOM>
cudaError_t launch_pair8_geom(const CUtensorMap& amap, const CUtensorMap& cmap, const Pair8Params& P, size_t smem,
                              int dev, cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(tc_pair8_kernel<GEOM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kThreads8P, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    {
        std::lock_guard<std::mutex> lk(g_pair8_mu);
        clusters = (dev >= 0 && dev < 64) ? g_pair8_clusters[dev][GEOM] : 0;
    }
    if (!clusters) {
        int sms = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        cfg.gridDim = dim3((unsigned)(sms & ~1), 1, 1);
        if ((e = cudaOccupancyMaxActiveClusters(&clusters, tc_pair8_kernel<GEOM>, &cfg)) != cudaSuccess) return e;
        if (clusters < 1) return cudaErrorNotSupported;
        std::lock_guard<std::mutex> lk(g_pair8_mu);
        if (dev >= 0 && dev < 64) g_pair8_clusters[dev][GEOM] = clusters;
    }
    const int64_t ncl = std::min<int64_t>(P.tiles, clusters);
    cfg.gridDim = dim3((unsigned)(2 * ncl), 1, 1);
    e = cudaLaunchKernelEx(&cfg, tc_pair8_kernel<GEOM>, amap, cmap, P);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

}  // namespace

bool tc_pair8_supported(const View3& v) { return tc_pair_supported(v); }

cudaError_t launch_tc_pair8(const View3& v, int* status, cudaStream_t s)
{
    if (!tc_pair8_supported(v)) return cudaErrorNotSupported;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int geom = v.inner == 1 ? P8_K : P8_MN;
    CUtensorMap amap, cmap;
    if (!encode_pair8_map(v, geom, &amap)) return cudaErrorInvalidValue;
    Pair8Params P{};
    P.c = static_cast<float*>(v.c);
    P.b = static_cast<const float*>(v.b);
    P.status = status;
    P.outer = v.outer;
    P.nq = v.nq;
    P.inner = v.inner;
    P.m = v.m;
    P.nsub = (int)((v.nq + kK8 - 1) / kK8);
    P.kstages = (int)((v.nq + kStageL8 - 1) / kStageL8);
    P.b_cm = v.b_cm;
    if (geom == P8_MN) {
        P.mper = (v.inner + kN8 - 1) / kN8;
        P.tiles = v.outer * P.mper;
    } else {
        P.mper = 1;
        P.tiles = (v.outer + kN8 - 1) / kN8;
    }
    P.wait_ns = wait_limit_ns();
    P.tma_c = pair_encode_c(v, &cmap) ? 1 : 0;
    if (!P.tma_c) std::memset(&cmap, 0, sizeof(cmap));
    // Each converter group owns the slots of one tile (stages n of tile n / kstages, group
    // (n / kstages) mod G): the ring is G whole tiles, with G the most groups (at most eight) whose
    // tiles fit beside the epilogue staging, the fibre factors and the barriers. A group then
    // waits on each phase of its own slots in turn, so its phase-parity waits are unambiguous.
    const size_t avail = 227 * 1024 - 1024 - kEpiBytes8 - kScaleBytes8 - kCtrl8;
    const int max_stages = (int)std::min<size_t>(kMaxStages8P, avail / kStage8);
    P.groups = std::min(kMaxGroups8, max_stages / P.kstages);
    if (P.groups < 1) return cudaErrorNotSupported;
    P.stages = P.groups * P.kstages;
    const size_t smem = 1024 + (size_t)P.stages * kStage8 + kEpiBytes8 + kScaleBytes8 + kCtrl8;
    return geom == P8_MN ? launch_pair8_geom<P8_MN>(amap, cmap, P, smem, dev, s)
                         : launch_pair8_geom<P8_K>(amap, cmap, P, smem, dev, s);
}

}  // namespace tlibttm
