// bf16x3 on pairs of SMs: tcgen05.mma.cta_group::2 with B held in tensor memory.
//
// Same arithmetic as tc_bf16x3 (tc_kernels.cu): every FP32 operand x is split into
// x_hi = bf16(x) and x_lo = bf16(x - x_hi), and C = B_hi A_hi + B_lo A_hi + B_hi A_lo is
// accumulated in FP32 in tensor memory. The roles of the operands are swapped so that B, which
// every tile shares, never moves again once loaded:
//
//   MMA M = 256  rows j of B (and of C): CTA rank c of the cluster holds j in [128c, 128c + 128),
//                 its hi and lo parts resident in that CTA's tensor memory for the whole launch
//                 (the MMA's A operand, K-major, 16 l per 8 columns);
//   MMA N = 128  tensor rows r of one tile (128 consecutive i of one slice k, or 128 consecutive
//                 fibres k when the fibres are contiguous): each CTA loads, splits and holds 64 of
//                 them in shared memory (the MMA's B operand);
//   MMA K = 16   l per instruction; three instructions per 16 l (hi*hi, lo*hi, hi*lo).
//
// One issued instruction thus does 256 x 128 x 16 multiply-adds over two SMs, and each SM reads
// 2 KB of shared memory per instruction (its 64 rows), against 12 KB per 128 x 256 x 16 in the
// single-SM kernel; B is read from HBM once per CTA. Limits: 128 < m <= 256 and n_q <= 256 (B's
// hi and lo parts take n_q of the 512 tensor-memory columns, the double-buffered accumulator
// the other 256).
//
// Warp roles (448 threads, one CTA per SM, clusters of two, persistent over tiles):
//   warp 0       TMA producer of this CTA's FP32 rows (64 rows x 64 l per stage);
//   warp 1       tensor-memory allocation (both CTAs) and, in the even CTA, the MMA issuer;
//   warps 2-9    converters in four groups of two warps: FP32 stage -> bf16 hi | lo in place,
//                in the canonical MMA layout, then an arrive on the even CTA's barrier;
//   warps 10-13  B -> tensor memory at the start; then the epilogue: tensor memory -> a 32 x 32
//                block staged in shared memory -> one TMA store (direct stores when C's rows
//                are not 16-byte aligned for a tensor map).
// Every mbarrier wait is bounded; on expiry the CTA raises its abort flag, drains its own copies
// and MMAs, frees tensor memory and raises the device status word. No TMA load uses multicast:
// each CTA loads its own rows into its own shared memory.
#include <cuda.h>
#include <cuda_bf16.h>

#include <atomic>
#include <cstring>
#include <mutex>

#include "tc_cluster.cuh"
#include "tc_kernels.cuh"
#include "tc_ptx.cuh"
#include "tlibttm.h"

namespace tlibttm {
namespace {

constexpr int kRowsCta = 64;                  // tensor rows per CTA per tile (N / 2)
constexpr int kPN = 128;                      // MMA N
constexpr int kPM = 256;                      // MMA M
constexpr int kPK = 16;                       // l per sub-block (one MMA K step)
constexpr int kPSub = 4;                      // sub-blocks per pipeline stage (12 MMAs per barrier round)
constexpr uint32_t kSubBytes = kRowsCta * kPK * 4;        // 4 KB FP32 sub-block
constexpr uint32_t kStageBytes = kPSub * kSubBytes;       // 16 KB
constexpr uint32_t kPartBytes = kRowsCta * kPK * 2;       // 2 KB bf16 part (hi or lo) of a sub-block
constexpr int kConvWarpsP = 8, kConvGroupsP = 4, kGroupWarpsP = kConvWarpsP / kConvGroupsP;
constexpr int kEpiWarp0 = 2 + kConvWarpsP;                // first epilogue warp
constexpr int kEpiWarpsP = 4;                             // one per tensor-memory lane quarter
constexpr int kThreadsP = (kEpiWarp0 + kEpiWarpsP) * 32;  // 448
constexpr uint32_t kEpiBufP = 32 * 32 * 4;                // one 32 x 32 FP32 staging block
constexpr uint32_t kEpiBytesP = kEpiWarpsP * 2 * kEpiBufP;  // double-buffered per epilogue warp
constexpr int kMaxStagesP = 24;
constexpr int kMaxNqP = 256;
constexpr uint32_t kAccCol = 256;                         // accumulators at columns 256..511
constexpr size_t kCtrlBytesP = 1024;

enum { PGEOM_MN = 0, PGEOM_K = 1 };

struct PairParams {
    float* c;
    const float* b;
    int* status;
    int64_t outer, nq, inner, m;
    int64_t tiles;          // tiles of 128 tensor rows
    int64_t mper;           // rows mode: tiles per slice, ceil(inner / 128)
    int kstages;            // pipeline stages per tile, ceil(nsub / 2)
    int nsub;               // 16-l sub-blocks holding l < n_q
    int b_cm;
    int stages;             // A ring depth
    int skip_first;         // test of the bounded waits: the even CTA never fills its first stage
    int tma_c;              // the epilogue stores C through the C tensor map
    unsigned long long wait_ns;
};

// D[tmem] (+)= A[tmem] * B[smem desc], both CTAs of the pair. Called by a whole converged warp
// with warp-uniform operands; one elected lane issues the instruction.
__device__ __forceinline__ void mma_pair(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p, e;\n setp.ne.b32 p, %4, 0;\n elect.sync _|e, 0xffffffff;\n"
        " @e tcgen05.mma.cta_group::2.kind::f16 [%0], [%1], %2, %3, p;\n}\n"
        ::"r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void split_pair(float x0, float x1, uint32_t& hi, uint32_t& lo) { split_bf16x2(x0, x1, hi, lo); }
// Byte offset of the 16-byte chunk of 8 consecutive rows (`rchunk`) at l (0..15) in an MN-major
// 128-byte-swizzled bf16 part of 64 rows x 16 l: [l / 8][l % 8][64 rows, chunk ^ (l % 8)].
__device__ __forceinline__ uint32_t mn64_off(uint32_t l, uint32_t rchunk)
{
    return (l >> 3) * 1024u + (l & 7u) * 128u + ((rchunk ^ (l & 7u)) << 4);
}

template <int GEOM>
__global__ void __launch_bounds__(kThreadsP, 1)
    tc_pair_kernel(const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap cmap, PairParams P)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int AS = P.stages;
    uint8_t* ring = smem;
    uint8_t* epi = smem + (size_t)AS * kStageBytes;
    uint64_t* a_full = reinterpret_cast<uint64_t*>(epi + kEpiBytesP);   // [AS] this CTA's TMA landed
    uint64_t* a_empty = a_full + kMaxStagesP;     // [AS] the pair's MMAs are done with the stage
    uint64_t* a_conv = a_empty + kMaxStagesP;     // [AS] even CTA: both CTAs' converters are done
    uint64_t* acc_full = a_conv + kMaxStagesP;    // [2]  accumulator ready
    uint64_t* acc_empty = acc_full + 2;           // [2]  even CTA: both CTAs' epilogues have read it
    uint64_t* drain = acc_empty + 2;              // [1]  even CTA: its MMAs have completed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
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
            mbar_init(&a_conv[s], 2 * kGroupWarpsP);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2 * kEpiWarpsP);
        }
        mbar_init(drain, 1);
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

    if (warp >= kEpiWarp0) {
        // B -> tensor memory: lane q4 * 32 + lane holds row j = 128 rank + q4 * 32 + lane; 16 l of
        // hi at columns 16 sb .. 16 sb + 7 and of lo at 16 sb + 8 .., zero outside B
        const int q4 = warp & 3;
        const int64_t j = (int64_t)rank * 128 + q4 * 32 + lane;
        const uint32_t trow = tmem_base + ((uint32_t)(q4 * 32) << 16);
        for (int sb = 0; sb < kst * kPSub; ++sb) {
            float x[kPK];
#pragma unroll
            for (int e = 0; e < kPK; ++e) {
                const int64_t l = (int64_t)sb * kPK + e;
                x[e] = (j < P.m && l < P.nq) ? __ldg(P.b_cm ? P.b + j + l * P.m : P.b + j * P.nq + l) : 0.0f;
            }
            uint32_t hi[8], lo[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) split_pair(x[2 * e], x[2 * e + 1], hi[e], lo[e]);
            tmem_st8(trow + (uint32_t)(sb * 16), hi);
            tmem_st8(trow + (uint32_t)(sb * 16 + 8), lo);
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
            int issued[kMaxStagesP];
            for (int i = 0; i < kMaxStagesP; ++i) issued[i] = -1;
            for (int64_t t = cid; t < tiles && ok; t += ncl) {
                int64_t k = 0, r0;
                if (GEOM == PGEOM_MN) {
                    k = t / P.mper;
                    r0 = (t - k * P.mper) * kPN + (int64_t)rank * kRowsCta;
                } else {
                    r0 = t * kPN + (int64_t)rank * kRowsCta;
                }
                for (int st = 0; st < kst; ++st) {
                    if (!mbar_wait(&a_empty[s], ph ^ 1, abort_flag, P.wait_ns)) { ok = false; break; }
                    if (P.skip_first && rank == 0 && t == cid && st == 0) {
                        // test of the bounded waits: this stage is never filled (no copy, no arrive)
                        if (++s == AS) { s = 0; ph ^= 1; }
                        continue;
                    }
                    issued[s] = (int)ph;
                    mbar_expect_tx(&a_full[s], kStageBytes);
                    uint8_t* dst = ring + (size_t)s * kStageBytes;
                    const int l0 = st * kPSub * kPK;
                    if (GEOM == PGEOM_MN) {
                        tma_load_3d(dst, &amap, &a_full[s], (int)r0, l0, (int)k);   // box 64 i x (16 kPSub) l x 1 k
                    } else {
#pragma unroll
                        for (int sb = 0; sb < kPSub; ++sb)   // boxes of 16 l x 64 k
                            tma_load_2d(dst + sb * kSubBytes, &amap, &a_full[s], l0 + sb * kPK, (int)r0);
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
        // The whole warp runs the loop, so that the descriptors and tensor-memory addresses are
        // warp-uniform values; one elected lane issues each MMA and commit. Wait results are
        // made warp-uniform before they steer the loop.
        if (rank == 0) {
            // kind::f16, D f32, A and B bf16, A K-major (tensor memory), B MN-major for rows of
            // consecutive i and K-major for contiguous fibres, N = 128, M = 256
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((GEOM == PGEOM_MN ? 1u : 0u) << 16) |
                                   ((uint32_t)(kPN >> 3) << 17) | ((uint32_t)(kPM >> 4) << 24);
            const uint64_t db0 = GEOM == PGEOM_MN ? smem_desc(su32(ring), 2048u, 1024u, kLayoutSW128)
                                                  : smem_desc(su32(ring), 16u, 256u, kLayoutSW32);
            int s = 0, ab = 0;
            uint32_t ph = 0, cph = 0;
            bool ok = true;
            for (int64_t t = cid; t < tiles && ok; t += ncl) {
                if (!__all_sync(0xffffffffu, mbar_wait(&acc_empty[ab], cph ^ 1, abort_flag, P.wait_ns))) break;
                tc_fence_after();
                const uint32_t dcol = tmem_base + kAccCol + (uint32_t)(ab * kPN);
                for (int st = 0; st < kst; ++st) {
                    if (!__all_sync(0xffffffffu, mbar_wait(&a_conv[s], ph, abort_flag, P.wait_ns))) { ok = false; break; }
                    tc_fence_after();
                    const uint64_t ds = db0 + ((uint64_t)((size_t)s * kStageBytes) >> 4);
#pragma unroll
                    for (int sb = 0; sb < kPSub; ++sb) {
                        const int g = st * kPSub + sb;
                        if (g >= P.nsub) continue;   // all-zero padding of the last stage
                        const uint64_t dhi = ds + (uint64_t)((sb * kSubBytes) >> 4);
                        const uint64_t dlo = dhi + (uint64_t)(kPartBytes >> 4);
                        const uint32_t bhi = tmem_base + (uint32_t)(g * 16), blo = bhi + 8;
                        mma_pair(dcol, bhi, dhi, idesc, g == 0 ? 0u : 1u);
                        mma_pair(dcol, blo, dhi, idesc, 1u);
                        mma_pair(dcol, bhi, dlo, idesc, 1u);
                    }
                    commit_pair(&a_empty[s], 0x3);   // both CTAs' stage s is free once these are done
                    if (++s == AS) { s = 0; ph ^= 1; }
                }
                if (!ok) break;
                commit_pair(&acc_full[ab], 0x3);
                if (++ab == 2) { ab = 0; cph ^= 1; }
            }
            // No MMA of the pair may still be reading or writing when the pair tears down.
            commit_pair(drain, 0x1);
            const unsigned long long t0 = gtimer();
            while (!mbar_try(drain, 0) && gtimer() - t0 < kTimeoutNs) {}
            __syncwarp();
        }
    } else if (warp < kEpiWarp0) {
        // ------------------------------------------------------------- converters (in place)
        const int g = (warp - 2) / kGroupWarpsP;
        const int gt = threadIdx.x - 64 - g * kGroupWarpsP * 32;   // 0 .. 63
        const bool odd = lane & 1;
        const uint32_t conv0 = peer_addr(su32(&a_conv[0]), 0);      // the even CTA's a_conv[0]
        constexpr int kIt = (int)(kStageBytes / 16) / (kGroupWarpsP * 32);   // float4 per thread per stage
        bool ok = true;
        // Stages are numbered n = 0, 1, ... across this cluster's tiles; this group takes those with
        // n % kConvGroupsP == g, in ring slot n % AS with phase (n / AS) & 1. AS being a multiple
        // of kConvGroupsP, the group's slot steps by kConvGroupsP and wraps with a phase flip.
        int rot = 0, s = g;
        uint32_t ph = 0;
        for (int64_t t = cid; t < tiles; t += ncl) {
            for (int st = 0; st < kst; ++st) {
                const bool mine = rot == g;
                if (++rot == kConvGroupsP) rot = 0;
                if (!mine) continue;
                const bool got = ok && mbar_wait(&a_full[s], ph, abort_flag, P.wait_ns);
                const bool have = __all_sync(0xffffffffu, got);
                if (!have) ok = false;
                uint8_t* buf = ring + (size_t)s * kStageBytes;
                float4 x[kIt];
                uint32_t off[kIt];
#pragma unroll
                for (int it = 0; it < kIt; ++it) {
                    const int v = gt + kGroupWarpsP * 32 * it;   // float4 index within the stage
                    if (GEOM == PGEOM_MN) {
                        const int l = v >> 4, w = v & 15;          // [16 kPSub l][64 i], 256-byte rows
                        if (have) x[it] = *reinterpret_cast<const float4*>(buf + l * 256 + w * 16);
                        off[it] = (uint32_t)(l >> 4) * kSubBytes + mn64_off((uint32_t)(l & 15), (uint32_t)(w >> 1));
                    } else {
                        const int sb = v >> 8, vv = v & 255;
                        const int k = vv >> 2, lc = vv & 3;         // [64 k][16 l], TMA 64-byte swizzle
                        if (have)
                            x[it] = *reinterpret_cast<const float4*>(buf + sb * kSubBytes + k * 64 +
                                                                     ((lc ^ ((k >> 1) & 3)) << 4));
                        off[it] = (uint32_t)sb * kSubBytes + kmaj_sw32_off((uint32_t)k, (uint32_t)(lc >> 1));
                    }
                }
                // the whole FP32 stage is in registers before any of it is overwritten
                asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "n"(kGroupWarpsP * 32) : "memory");
                if (have) {
#pragma unroll
                    for (int it = 0; it < kIt; ++it) {
                        uint32_t h0, l0, h1, l1;
                        split_pair(x[it].x, x[it].y, h0, l0);
                        split_pair(x[it].z, x[it].w, h1, l1);
                        // lane pairs hold 8 consecutive elements, one 16-byte chunk of each part:
                        // each lane writes its half of the hi and of the lo chunk
                        const uint32_t half = odd ? 8u : 0u;
                        *reinterpret_cast<uint2*>(buf + off[it] + half) = make_uint2(h0, h1);
                        *reinterpret_cast<uint2*>(buf + kPartBytes + off[it] + half) = make_uint2(l0, l1);
                    }
                    fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_remote(conv0 + (uint32_t)s * 8u);
                }
                s += kConvGroupsP;
                if (s >= AS) { s -= AS; ph ^= 1; }
            }
        }
    } else {
        // ------------------------------------------------------------- epilogue
        const int q4 = warp & 3;
        uint8_t* stage0 = epi + (size_t)(warp - kEpiWarp0) * 2 * kEpiBufP;
        const int64_t j0 = (int64_t)rank * 128 + q4 * 32;           // first row of C this warp holds
        const int64_t j = j0 + lane;                                 // this lane's row
        const uint32_t empty0 = peer_addr(su32(&acc_empty[0]), 0);
        const int64_t rlim = GEOM == PGEOM_MN ? P.inner : P.outer;   // tensor rows of one slice
        int sb = 0, ab = 0;
        uint32_t aph = 0;
        for (int64_t t = cid; t < tiles; t += ncl) {
            if (!mbar_wait(&acc_full[ab], aph, abort_flag, P.wait_ns)) break;
            tc_fence_after();
            int64_t k = 0, r0;
            if (GEOM == PGEOM_MN) {
                k = t / P.mper;
                r0 = (t - k * P.mper) * kPN;
            } else {
                r0 = t * kPN;
            }
            const uint32_t tb = tmem_base + ((uint32_t)(q4 * 32) << 16) + kAccCol + (uint32_t)(ab * kPN);
            for (int cc = 0; cc < kPN; cc += 32) {
                uint32_t v[32];
                tmem_ld32(tb + (uint32_t)cc, v);
                const int64_t r = r0 + cc;                           // first tensor row of these columns
                if (j0 >= P.m || r >= rlim) continue;                // the block lies outside C
                if (P.tma_c) {
                    uint8_t* buf = stage0 + sb * kEpiBufP;
                    if (lane == 0) bulk_wait_read1();   // the store that last read `buf` has read it
                    __syncwarp();
                    if (GEOM == PGEOM_MN) {
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
                        if (GEOM == PGEOM_MN) tma_store_3d(&cmap, buf, (int)r, (int)j0, (int)k);
                        else tma_store_2d(&cmap, buf, (int)j0, (int)r);
                        bulk_commit();
                    }
                    sb ^= 1;
                } else if (j < P.m) {
                    // direct stores (C not 16-byte aligned for a tensor map)
                    if (GEOM == PGEOM_MN) {
                        float* p = P.c + (k * P.m + j) * P.inner + r;
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            if (r + c < P.inner) p[c] = __uint_as_float(v[c]);
                    } else {
                        float* p = P.c + r * P.m + j;   // C[k][j], consecutive lanes consecutive j
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

typedef CUresult (*EncodeTiledFnP)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFnP encode_fn_p()
{
    static EncodeTiledFnP fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFnP>(p);
    });
    return fn;
}

bool encode_pair_map(const View3& v, int geom, CUtensorMap* map)
{
    EncodeTiledFnP enc = encode_fn_p();
    if (!enc) return false;
    CUresult r;
    if (geom == PGEOM_MN) {
        cuuint64_t dims[3] = {(cuuint64_t)v.inner, (cuuint64_t)v.nq, (cuuint64_t)v.outer};
        cuuint64_t strides[2] = {(cuuint64_t)v.inner * 4, (cuuint64_t)v.inner * v.nq * 4};
        cuuint32_t box[3] = {kRowsCta, kPSub * kPK, 1};
        cuuint32_t es[3] = {1, 1, 1};
        r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(v.a), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        cuuint64_t dims[2] = {(cuuint64_t)v.nq, (cuuint64_t)v.outer};
        cuuint64_t strides[1] = {(cuuint64_t)v.nq * 4};
        cuuint32_t box[2] = {kPK, kRowsCta};
        cuuint32_t es[2] = {1, 1};
        r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(v.a), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

// C as a tensor map for the TMA-store epilogue (32 x 32 boxes); false when C's rows or base are
// not 16-byte aligned (the epilogue then stores directly).
bool encode_pair_cmap(const View3& v, int geom, CUtensorMap* map)
{
    EncodeTiledFnP enc = encode_fn_p();
    if (!enc || (reinterpret_cast<uintptr_t>(v.c) & 15u) != 0) return false;
    CUresult r;
    if (geom == PGEOM_MN) {
        cuuint64_t dims[3] = {(cuuint64_t)v.inner, (cuuint64_t)v.m, (cuuint64_t)v.outer};
        cuuint64_t strides[2] = {(cuuint64_t)v.inner * 4, (cuuint64_t)v.inner * v.m * 4};
        cuuint32_t box[3] = {32, 32, 1};
        cuuint32_t es[3] = {1, 1, 1};
        r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, v.c, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        if (v.m % 4 != 0) return false;
        cuuint64_t dims[2] = {(cuuint64_t)v.m, (cuuint64_t)v.outer};
        cuuint64_t strides[1] = {(cuuint64_t)v.m * 4};
        cuuint32_t box[2] = {32, 32};
        cuuint32_t es[2] = {1, 1};
        r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, v.c, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

// Clusters of two that can be resident at once, per device and geometry (queried once).
std::mutex g_pair_mu;
int g_pair_clusters[64][2] = {};

template <int GEOM>
cudaError_t launch_pair_geom(const CUtensorMap& amap, const CUtensorMap& cmap, const PairParams& P, size_t smem, int dev,
                             cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(tc_pair_kernel<GEOM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kThreadsP, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    {
        std::lock_guard<std::mutex> lk(g_pair_mu);
        clusters = (dev >= 0 && dev < 64) ? g_pair_clusters[dev][GEOM] : 0;
    }
    if (!clusters) {
        int sms = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        cfg.gridDim = dim3((unsigned)(sms & ~1), 1, 1);
        if ((e = cudaOccupancyMaxActiveClusters(&clusters, tc_pair_kernel<GEOM>, &cfg)) != cudaSuccess) return e;
        if (clusters < 1) return cudaErrorNotSupported;
        std::lock_guard<std::mutex> lk(g_pair_mu);
        if (dev >= 0 && dev < 64) g_pair_clusters[dev][GEOM] = clusters;
    }
    const int64_t ncl = std::min<int64_t>(P.tiles, clusters);
    cfg.gridDim = dim3((unsigned)(2 * ncl), 1, 1);
    e = cudaLaunchKernelEx(&cfg, tc_pair_kernel<GEOM>, amap, cmap, P);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

}  // namespace

bool pair_encode_a(const View3& v, CUtensorMap* map) { return encode_pair_map(v, v.inner == 1 ? PGEOM_K : PGEOM_MN, map); }
bool pair_encode_c(const View3& v, CUtensorMap* map) { return encode_pair_cmap(v, v.inner == 1 ? PGEOM_K : PGEOM_MN, map); }

bool tc_pair_supported(const View3& v)
{
    if (v.m <= 128 || v.m > kPM || v.nq > kMaxNqP || v.nq < 1) return false;
    if ((reinterpret_cast<uintptr_t>(v.a) & 15u) != 0) return false;
    if (v.outer >= (int64_t(1) << 31) || v.inner >= (int64_t(1) << 31)) return false;
    if (v.inner == 1) return v.nq % 4 == 0;           // fibre rows on 16-byte boundaries for TMA
    return v.inner >= kPN && v.inner % 4 == 0;         // rows of 128 i, 16-byte l stride
}

cudaError_t launch_tc_pair(const View3& v, int* status, cudaStream_t s)
{
    if (!tc_pair_supported(v)) return cudaErrorNotSupported;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int geom = v.inner == 1 ? PGEOM_K : PGEOM_MN;
    CUtensorMap amap;
    if (!encode_pair_map(v, geom, &amap)) return cudaErrorInvalidValue;
    PairParams P{};
    P.c = static_cast<float*>(v.c);
    P.b = static_cast<const float*>(v.b);
    P.status = status;
    P.outer = v.outer;
    P.nq = v.nq;
    P.inner = v.inner;
    P.m = v.m;
    P.nsub = (int)((v.nq + kPK - 1) / kPK);
    P.kstages = (P.nsub + kPSub - 1) / kPSub;
    P.b_cm = v.b_cm;
    if (geom == PGEOM_MN) {
        P.mper = (v.inner + kPN - 1) / kPN;
        P.tiles = v.outer * P.mper;
    } else {
        P.mper = 1;
        P.tiles = (v.outer + kPN - 1) / kPN;
    }
    P.wait_ns = wait_limit_ns();
    P.skip_first = take_skip_b() ? 1 : 0;
    CUtensorMap cmap;
    P.tma_c = encode_pair_cmap(v, geom, &cmap) ? 1 : 0;
    if (!P.tma_c) std::memset(&cmap, 0, sizeof(cmap));
    // A ring: as many stages as fit beside the epilogue staging and the barriers, a multiple of
    // the converter groups. Group g converts the stages n = g (mod groups) in order, waiting on
    // the stage's barrier by phase parity; with the ring a multiple of the groups every slot
    // belongs to one group, which sees each phase of it in turn. Otherwise a group could wait on
    // a slot whose previous load (another group's) has not landed yet, and the parity of that
    // pending phase would read as the completed one before it.
    const size_t avail = 227 * 1024 - 1024 - kEpiBytesP - kCtrlBytesP;
    P.stages = (int)std::min<size_t>(kMaxStagesP, avail / kStageBytes);
    P.stages -= P.stages % kConvGroupsP;
    const size_t smem = 1024 + (size_t)P.stages * kStageBytes + kEpiBytesP + kCtrlBytesP;
    return geom == PGEOM_MN ? launch_pair_geom<PGEOM_MN>(amap, cmap, P, smem, dev, s)
                            : launch_pair_geom<PGEOM_K>(amap, cmap, P, smem, dev, s);
}

}  // namespace tlibttm
