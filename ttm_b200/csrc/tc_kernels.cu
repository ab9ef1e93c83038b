// Tensor-core paths (tcgen05 / TMEM) of the B200 TTM library.
//
// tc_bf16x3: FP32-accurate contraction on the BF16 tensor cores.
//   Each FP32 operand x is split into x_hi = bf16(x) and x_lo = bf16(x - x_hi);
//   C = A_hi*B_hi + A_hi*B_lo + A_lo*B_hi is accumulated in FP32 in TMEM
//   (the "bf16x3" scheme of Henry, Tang & Heinecke, 2019). The dropped term
//   A_lo*B_lo and the split residuals are O(2^-16) relative per product.
//
// Slice view (common.cuh): C[k][j][i] = sum_l A[k][l][i] B(j,l). Two geometries:
//   GEOM_MN (inner % 4 == 0): MMA rows are 128 consecutive i of one slice k;
//            A's tile is MN-major (i contiguous); TMA box (128 i, 32 l, 1 k).
//   GEOM_K  (inner == 1, the contraction mode is the fastest): MMA rows are
//            128 consecutive k; A's tile is K-major; TMA box (32 l, 128 k).
// MMA shape M = 128, N = NT (<= 256, the rows of B in this tile), K = 16 per
// instruction, 32 l (two sub-blocks of 16, six MMAs) per pipeline stage.
//
// Warp roles (736 threads, one CTA per SM, persistent over tiles):
//   warp 0     TMA producer of the FP32 A tile (tensor map).
//   warp 1     TMEM allocator and MMA issuer (one elected lane).
//   warp 2     bulk copies of the pre-split B_hi/B_lo image of this stage.
//   warps 3-18 converters: FP32 tile -> bf16 hi/lo in the swizzled UMMA layout.
//   warps 19-22 epilogue: TMEM -> registers -> global C (double-buffered accumulator).
// Every mbarrier wait is bounded (4 s of %globaltimer); on expiry the CTA raises
// an abort flag, records an error in the device status word, drains its own
// bulk copies, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "tc_kernels.cuh"
#include "tc_ptx.cuh"
#include "tlibttm.h"

namespace tlibttm {
namespace {

constexpr int kConvWarps = 16;                  // converter warps
constexpr int kConvGroups = 4;                  // groups converting different stages at the same time
constexpr int kGroupWarps = kConvWarps / kConvGroups;
constexpr int kThreads = (3 + kConvWarps + 4) * 32;  // A producer, MMA, B producer, converters, 4 epilogue warps
constexpr int kBM = 128;       // MMA M
constexpr int kBK = 16;        // l per sub-block (one MMA K step)
constexpr int kSub = 2;        // sub-blocks per pipeline stage: 3 * kSub MMAs per barrier round
constexpr int kMaxNT = 256;    // MMA N max

enum { GEOM_MN = 0, GEOM_K = 1 };

// Instruction descriptor, kind::f16: D f32, A/B bf16, B K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool a_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(kBM >> 4) << 24);
}

// Called by a whole converged warp with warp-uniform operands (so that they stay in uniform
// registers); one elected lane issues the instruction.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p, e;\n setp.ne.b32 p, %4, 0;\n elect.sync _|e, 0xffffffff;\n"
        " @e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// x -> (hi, lo) bf16 pair, packed two at a time.
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) { split_bf16x2(x0, x1, hi, lo); }

// Byte offset of a 16-byte chunk (8 consecutive MN elements) in an MN-major SW128 bf16 tile of
// 128 MN x 16 K laid out as [K group of 8][MN block of 64][8 K rows][64 MN].
__device__ __forceinline__ uint32_t mnmaj_sw128_off(uint32_t l, uint32_t ichunk)
{
    const uint32_t atom = (l >> 3) * 2u + (ichunk >> 3);
    const uint32_t row = l & 7u, c = ichunk & 7u;
    return atom * 1024u + row * 128u + ((c ^ row) << 4);
}

// One problem of a bf16x3 launch: its tensor maps, pointers and tiling. A single launch passes it
// as a kernel parameter; a grouped launch reads an array of them from device memory (64-byte
// aligned, as TMA requires of a tensor map), ordered by `first`.
struct alignas(64) TcProb {
    CUtensorMap amap;        // A tiles (unused when ldg_a)
    CUtensorMap cmap;        // 32 x 32 blocks of C for the TMA-store epilogue (unused when !tma_c)
    float* c;
    const float* a;          // A itself, for the converters' own loads (ldg_a)
    const float* b;          // B itself, read by the operand split
    const uint8_t* bimg;     // pre-split B: [jb][kc][hi|lo][NT rows x 32 B]
    int64_t outer, nq, inner, m;
    int64_t tiles_m;         // M tiles per j block
    int64_t tiles;           // tiles of this problem
    int64_t first;           // grouped launch: index of its first tile among all problems' tiles
    int nt;                  // MMA N (multiple of 16, <= 256)
    int jblocks;
    int kchunks;             // 16-l sub-blocks of n_q
    int kstages;             // pipeline stages per tile: ceil(kchunks / kSub)
    int ldg_a;               // A rows not 16-byte aligned for TMA: the converters load A
    int tma_c;               // epilogue stores C through the C tensor map
    int fold_kb;             // GEOM_MN with inner <= 64: slices per 128-row tile (1: unfolded)
    int fold_ib_shift;       // log2 of the rows each slice takes in a folded tile (32 or 64)
    int b_cm;
};

// Launch-wide parameters.
struct TcParams {
    int* status;             // device status word (0 = ok)
    const TcProb* group;     // grouped launch: `count` problems in device memory (else unused)
    int count;
    int64_t total;           // tiles over all problems of the launch
    int fstages;             // A ring depth (FP32 tile, converted in place)
    int ostages;             // B ring depth
    uint32_t bslot;          // bytes of one B ring slot (the largest B stage of the launch)
    int acc_stride;          // tensor-memory columns between the two accumulators
    int skip_b;              // test of the bounded waits: the B producer skips its first stage
    unsigned long long wait_ns;   // bound of the pipeline's mbarrier waits
};

// Shared memory: [A ring][B ring][epilogue staging][barriers]. An A stage holds kSub FP32
// sub-blocks of 128 rows x 16 l, each converted in place to [bf16 hi | bf16 lo]; a B stage holds
// [hi | lo] of each sub-block's 16 l of B.
struct SmemLayout {
    uint32_t a_bytes, asub_bytes, abf_bytes, b_bytes, bstage_bytes;
};

__host__ __device__ inline SmemLayout smem_layout(int nt)
{
    SmemLayout L;
    L.asub_bytes = kBM * kBK * 4;           // 8 KB FP32 sub-block (its bf16 hi and lo halves after conversion)
    L.a_bytes = kSub * L.asub_bytes;
    L.abf_bytes = kBM * kBK * 2;            // 4 KB per bf16 part
    L.b_bytes = (uint32_t)nt * kBK * 2;     // per part and sub-block, multiple of 512
    L.bstage_bytes = kSub * 2 * L.b_bytes;
    return L;
}

constexpr int kMaxA = 12, kMaxB = 3;
constexpr uint32_t kEpiBuf = 32 * 32 * 4;        // one 32 x 32 fp32 staging tile
constexpr uint32_t kEpiBytes = 4 * 2 * kEpiBuf;  // 4 epilogue warps, double-buffered
constexpr size_t kCtrlBytes = 1024;
constexpr size_t kSmemBudget = 227 * 1024;

// Ring depths for a given N tile; false if the minimum does not fit.
__host__ inline bool choose_stages(int nt, int& as, int& bs, size_t& smem)
{
    const SmemLayout L = smem_layout(nt);
    const size_t avail = kSmemBudget - 1024 - kCtrlBytes - kEpiBytes;
    // A stages: a multiple of kConvGroups. Group g converts the stages n = g (mod kConvGroups) in
    // order, waiting on each stage's barrier by phase parity; with the ring a multiple of the
    // groups every slot belongs to one group, which sees each phase of it in turn. Otherwise a
    // group could wait on a slot whose previous load (another group's) has not landed yet -- loads
    // may land out of order -- and the parity of that pending phase would read as the completed
    // one before it.
    // B stages (from L2) give way first, down to two, so that A keeps two stages per group
    // (measured at N = 256: 8 A + 2 B stages beat 4 + 3 by 10 %)
    bs = kMaxB;
    while (bs > 2 && (size_t)bs * L.bstage_bytes + 2 * kConvGroups * L.a_bytes > avail) --bs;
    while (bs > 2 && (size_t)bs * L.bstage_bytes + kConvGroups * L.a_bytes > avail) --bs;
    if ((size_t)bs * L.bstage_bytes + kConvGroups * L.a_bytes > avail) return false;
    as = (int)((avail - (size_t)bs * L.bstage_bytes) / L.a_bytes);
    if (as > kMaxA) as = kMaxA;
    as -= as % kConvGroups;
    smem = 1024 + (size_t)as * L.a_bytes + (size_t)bs * L.bstage_bytes + kEpiBytes + kCtrlBytes;
    return true;
}


// Named barrier of one converter group (ids 1..kConvGroups; id 0 is __syncthreads).
__device__ __forceinline__ void conv_barrier(int g)
{
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "n"(kGroupWarps * 32) : "memory");
}

// The problem owning tile t of the launch, and the tile's index within that problem. A role
// visits its tiles in increasing order, so the search goes on from the problem of its previous
// tile (`cur`, 0 at the start).
template <bool GROUP>
__device__ __forceinline__ const TcProb& tile_problem(const TcProb& one, const TcParams& P, int64_t t, int& cur,
                                                      int64_t& lt)
{
    if constexpr (!GROUP) {
        lt = t;
        return one;
    } else {
        while (cur + 1 < P.count && P.group[cur + 1].first <= t) ++cur;
        lt = t - P.group[cur].first;
        return P.group[cur];
    }
}

// A tensor map in device memory is read through the tensor-map proxy: order that read after the
// generic-proxy writes that made the map (the plan's upload) before the first copy using it.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// GROUP = false: one problem, `one`. GROUP = true: the P.count problems of P.group, whose tiles
// are numbered one after the other; every role walks the same tile sequence, so the pipeline
// runs across problem boundaries without draining.
template <int GEOM, bool GROUP>
__global__ void __launch_bounds__(kThreads, 1)
    tc_bf16x3_kernel(const __grid_constant__ TcProb one, TcParams P)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const SmemLayout LA = smem_layout(kMaxNT);   // its A sizes do not depend on N
    const int AS = P.fstages, BS = P.ostages;
    uint8_t* aring = smem;
    uint8_t* bring = smem + (size_t)AS * LA.a_bytes;
    uint8_t* epi = bring + (size_t)BS * P.bslot;
    uint8_t* ctrl = epi + kEpiBytes;
    uint64_t* a_full = reinterpret_cast<uint64_t*>(ctrl);   // [AS]  TMA of the FP32 tile landed
    uint64_t* a_conv = a_full + kMaxA;                        // [AS]  bf16 hi/lo written in place
    uint64_t* a_empty = a_conv + kMaxA;                       // [AS]  MMAs done reading
    uint64_t* b_full = a_empty + kMaxA;                       // [BS]  B image landed
    uint64_t* b_empty = b_full + kMaxB;                       // [BS]  MMAs done reading
    uint64_t* acc_full = b_empty + kMaxB;                     // [2]
    uint64_t* acc_empty = acc_full + 2;                       // [2]
    uint64_t* drain = acc_empty + 2;                          // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto a_at = [&](int s) { return aring + (size_t)s * LA.a_bytes; };
    auto bhi_at = [&](int s) { return bring + (size_t)s * P.bslot; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < AS; ++s) {
            mbar_init(&a_full[s], 1);
            mbar_init(&a_conv[s], kGroupWarps);
            mbar_init(&a_empty[s], 1);
        }
        for (int s = 0; s < BS; ++s) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 4);
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

    const int64_t tiles = P.total;

    if (warp == 0) {
        // ------------------------------------------------------------- A producer (TMA)
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            int issued[kMaxA];
            for (int i = 0; i < kMaxA; ++i) issued[i] = -1;
            const TcProb* last = nullptr;
            int cur = 0;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                int64_t lt;
                const TcProb& pr = tile_problem<GROUP>(one, P, t, cur, lt);
                if (GROUP && &pr != last && !pr.ldg_a) tensormap_acquire(&pr.amap);
                last = &pr;
                const int64_t mt = lt % pr.tiles_m, mper = (pr.inner + kBM - 1) / kBM;
                for (int st = 0; st < pr.kstages; ++st) {
                    if (!mbar_wait(&a_empty[s], ph ^ 1, abort_flag, P.wait_ns)) { ok = false; break; }
                    if (pr.ldg_a) {
                        // no copy: the stage is free for the converters, which load A themselves.
                        // No copy is in flight into it either (its last one landed before the
                        // stage was freed), so the final drain must not wait on it: a phase
                        // recorded by an earlier copy would by then be ambiguous by parity.
                        issued[s] = -1;
                        mbar_arrive(&a_full[s]);
                        if (++s == AS) { s = 0; ph ^= 1; }
                        continue;
                    }
                    issued[s] = (int)ph;
                    // the sub-blocks within n_q (the last box's rows past n_q are zero-filled)
                    const int nsub = min(kSub, pr.kchunks - st * kSub);
                    mbar_expect_tx(&a_full[s], (uint32_t)nsub * LA.asub_bytes);
#pragma unroll
                    for (int sub = 0; sub < kSub; ++sub) {
                        if (sub >= nsub) break;
                        uint8_t* dst = a_at(s) + sub * LA.asub_bytes;
                        const int l0 = (st * kSub + sub) * kBK;
                        if (GEOM == GEOM_MN && pr.fold_kb > 1) {
                            // folded tile: slices mt*KB .. +KB-1, the map ordered (i, k, l)
                            tma_load_3d(dst, &pr.amap, &a_full[s], 0, (int)(mt * pr.fold_kb), l0);
                        } else if (GEOM == GEOM_MN) {
                            const int64_t k = mt / mper, ib = mt - k * mper;
                            tma_load_3d(dst, &pr.amap, &a_full[s], (int)(ib * kBM), l0, (int)k);
                        } else {
                            tma_load_2d(dst, &pr.amap, &a_full[s], l0, (int)(mt * kBM));
                        }
                    }
                    if (++s == AS) { s = 0; ph ^= 1; }
                }
            }
            // None of this CTA's bulk copies may still be in flight when it exits.
            for (int i = 0; i < AS; ++i) {
                if (issued[i] < 0) continue;
                const unsigned long long t0 = gtimer();
                while (!mbar_try(&a_full[i], (uint32_t)issued[i]) && gtimer() - t0 < kTimeoutNs) {}
            }
        }
    } else if (warp == 2) {
        // ------------------------------------------------------------- B producer (bulk copies)
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            int issued[kMaxB];
            for (int i = 0; i < kMaxB; ++i) issued[i] = -1;
            int cur = 0;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                int64_t lt;
                const TcProb& pr = tile_problem<GROUP>(one, P, t, cur, lt);
                const SmemLayout Lp = smem_layout(pr.nt);
                const int64_t jb = lt / pr.tiles_m;
                for (int st = 0; st < pr.kstages; ++st) {
                    if (!mbar_wait(&b_empty[s], ph ^ 1, abort_flag, P.wait_ns)) { ok = false; break; }
                    if (P.skip_b && t == blockIdx.x && st == 0) {
                        // test of the bounded waits: this stage is never filled (no copy, no arrive)
                        if (++s == BS) { s = 0; ph ^= 1; }
                        continue;
                    }
                    issued[s] = (int)ph;
                    mbar_expect_tx(&b_full[s], Lp.bstage_bytes);
                    // the image holds kstages * kSub sub-blocks per j block: one copy per stage
                    const uint8_t* img = pr.bimg + ((size_t)(jb * pr.kstages + st) * Lp.bstage_bytes);
                    bulk_load(bhi_at(s), img, Lp.bstage_bytes, &b_full[s]);
                    if (++s == BS) { s = 0; ph ^= 1; }
                }
            }
            for (int i = 0; i < BS; ++i) {
                if (issued[i] < 0) continue;
                const unsigned long long t0 = gtimer();
                while (!mbar_try(&b_full[i], (uint32_t)issued[i]) && gtimer() - t0 < kTimeoutNs) {}
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- MMA issuer
        // The whole warp runs the loop (warp-uniform descriptors); one elected lane issues each
        // MMA and commit; wait results are made warp-uniform before they steer the loop.
        {
            // descriptors of stage 0's first sub-block; a descriptor's start-address field is
            // address / 16 in its low bits, so other stages and parts are plain additions
            const uint64_t da0 = GEOM == GEOM_MN ? smem_desc(su32(aring), 1024u, 2048u, kLayoutSW128)
                                                 : smem_desc(su32(aring), 16u, 256u, kLayoutSW32);
            const uint64_t db0 = smem_desc(su32(bring), 16u, 256u, kLayoutSW32);
            int as = 0, bs = 0;
            uint32_t aph = 0, bph = 0;
            int ab = 0;
            uint32_t cph = 0;
            bool ok = true;
            int cur = 0;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                int64_t lt;
                const TcProb& pr = tile_problem<GROUP>(one, P, t, cur, lt);
                const int kst = pr.kstages;
                const uint32_t idesc = idesc_bf16(pr.nt, GEOM == GEOM_MN);
                const uint32_t b_bytes = (uint32_t)pr.nt * kBK * 2;   // one part of one sub-block of B
                if (!__all_sync(0xffffffffu, mbar_wait(&acc_empty[ab], cph ^ 1, abort_flag, P.wait_ns))) break;
                tc_fence_after();
                const uint32_t dcol = tmem_base + (uint32_t)(ab * P.acc_stride);
                for (int st = 0; st < kst; ++st) {
                    const bool got = mbar_wait(&b_full[bs], bph, abort_flag, P.wait_ns) &&
                                     mbar_wait(&a_conv[as], aph, abort_flag, P.wait_ns);
                    if (!__all_sync(0xffffffffu, got)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t da = da0 + ((uint64_t)(as * LA.a_bytes) >> 4);
                    const uint64_t db = db0 + ((uint64_t)(bs * P.bslot) >> 4);
#pragma unroll
                    for (int sub = 0; sub < kSub; ++sub) {
                        if (sub > 0 && st * kSub + sub >= pr.kchunks) break;   // zeros past n_q
                        const uint64_t dahi = da + (uint64_t)((sub * LA.asub_bytes) >> 4);
                        const uint64_t dalo = dahi + (uint64_t)(LA.abf_bytes >> 4);
                        const uint64_t dbhi = db + (uint64_t)((sub * 2 * b_bytes) >> 4);
                        const uint64_t dblo = dbhi + (uint64_t)(b_bytes >> 4);
                        mma_bf16(dcol, dahi, dbhi, idesc, (st == 0 && sub == 0) ? 0u : 1u);
                        mma_bf16(dcol, dahi, dblo, idesc, 1u);
                        mma_bf16(dcol, dalo, dbhi, idesc, 1u);
                    }
                    mma_commit_warp(&a_empty[as]);   // stages free once these MMAs have read them
                    mma_commit_warp(&b_empty[bs]);
                    if (++as == AS) { as = 0; aph ^= 1; }
                    if (++bs == BS) { bs = 0; bph ^= 1; }
                }
                if (!ok) break;
                mma_commit_warp(&acc_full[ab]);     // accumulator ready for the epilogue
                if (++ab == 2) { ab = 0; cph ^= 1; }
            }
            // No MMA of this CTA may still be writing TMEM when it is freed.
            mma_commit_warp(drain);
            const unsigned long long t0 = gtimer();
            while (!mbar_try(drain, 0) && gtimer() - t0 < kTimeoutNs) {}
            __syncwarp();
        }
    } else if (warp < 3 + kConvWarps) {
        // ------------------------------------------------------------- converters (in place)
        // kConvGroups groups of kGroupWarps warps; group g converts the stages with sequence number
        // n, n % kConvGroups == g (their kSub sub-blocks one after the other), so that several
        // stages are converted at once.
        const int g = (warp - 3) / kGroupWarps;
        const int gt = threadIdx.x - 96 - g * kGroupWarps * 32;   // 0 .. kGroupWarps*32-1
        const bool odd = lane & 1;
        constexpr int kIters = (kBM * kBK / 4) / (kGroupWarps * 32);
        // this thread's float4 positions in a sub-block: where it reads the FP32 tile and where
        // its 16-byte chunks of the bf16 parts go (the same for every sub-block)
        uint32_t rdo[kIters], wro[kIters];
#pragma unroll
        for (int it = 0; it < kIters; ++it) {
            const int v = gt + kGroupWarps * 32 * it;
            if (GEOM == GEOM_MN) {
                const int l = v >> 5, w = v & 31;
                rdo[it] = (uint32_t)(l * 512 + w * 16);
                wro[it] = mnmaj_sw128_off((uint32_t)l, (uint32_t)(w >> 1));
            } else {
                const int k = v >> 2, lc = v & 3;
                rdo[it] = (uint32_t)(k * 64 + ((lc ^ ((k >> 1) & 3)) << 4));
                wro[it] = kmaj_sw32_off((uint32_t)k, (uint32_t)(lc >> 1));
            }
        }
        bool ok = true;
        // The CTA's stages are numbered n = 0, 1, ... across its tiles; this group takes those with
        // n % kConvGroups == g, which sit in ring slot n % AS with phase (n / AS) & 1. AS being a
        // multiple of kConvGroups, the group's slot steps by kConvGroups and wraps with a phase flip.
        int rot = 0;                 // n % kConvGroups
        int s = g;                   // slot of the group's next stage
        uint32_t ph = 0;
        // Every thread of a group runs every iteration of its residue and reaches the group barrier
        // the same number of times; once the CTA aborts, the waits are skipped and no work is done.
        int cur = 0;
        for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
            int64_t lt;
            const TcProb& pr = tile_problem<GROUP>(one, P, t, cur, lt);
            // the record's fields in registers (stores through generic pointers could alias a
            // grouped launch's records in global memory and force reloads); those of the
            // converters' own loads only where they load A
            const int kst = pr.kstages, kch = pr.kchunks;
            const bool ldg = pr.ldg_a != 0;
            const float* ga = nullptr;
            int64_t gnq = 0, ginner = 0, gouter = 0;
            int fkb = 1, fsh = 0;
            // tile origin for the converters' own loads of A (ldg_a): slice k / first row
            int64_t mt = 0, tk = 0, r0 = 0;
            if (ldg) {
                ga = pr.a;
                gnq = pr.nq;
                ginner = pr.inner;
                gouter = pr.outer;
                fkb = pr.fold_kb;
                fsh = pr.fold_ib_shift;
                const int64_t mper = (ginner + kBM - 1) / kBM;
                mt = lt % pr.tiles_m;
                tk = GEOM == GEOM_MN ? mt / mper : 0;
                r0 = GEOM == GEOM_MN ? (mt - tk * mper) * kBM : mt * kBM;
            }
            for (int st = 0; st < kst; ++st) {
                const bool mine = rot == g;
                if (++rot == kConvGroups) rot = 0;
                if (!mine) continue;
                const bool got = ok && mbar_wait(&a_full[s], ph, abort_flag, P.wait_ns);
                const bool have = __all_sync(0xffffffffu, got);
                if (!have) ok = false;
                // sub-blocks past n_q are zeros that the MMA issuer skips: not converted
                const int nsub = min(kSub, kch - st * kSub);
#pragma unroll 1
                for (int sub = 0; sub < nsub; ++sub) {
                    const int kc = st * kSub + sub;
                    uint8_t* buf = a_at(s) + sub * LA.asub_bytes;
                    float4 x[kIters];
                    uint32_t off[kIters];
#pragma unroll
                    for (int it = 0; it < kIters; ++it) {
                        const int v = gt + kGroupWarps * 32 * it;   // float4 index within the 8 KB tile
                        if (GEOM == GEOM_MN) {
                            const int l = v >> 5, w = v & 31;               // [16 l][128 i], 512-byte rows
                            if (have && ldg) {
                                // elements (l, i .. i+3) of slice tk (of slice tk * KB + row / IB when
                                // folded), zero outside A
                                const int64_t gl = (int64_t)kc * kBK + l;
                                const int64_t sk = fkb > 1 ? mt * fkb + ((w * 4) >> fsh) : tk;
                                const int64_t i = fkb > 1 ? ((w * 4) & ((1 << fsh) - 1)) : r0 + w * 4;
                                const float* src = ga + (sk * gnq + gl) * ginner + i;
                                const bool lv = gl < gnq && sk < gouter;
                                x[it].x = (lv && i < ginner) ? __ldg(src) : 0.0f;
                                x[it].y = (lv && i + 1 < ginner) ? __ldg(src + 1) : 0.0f;
                                x[it].z = (lv && i + 2 < ginner) ? __ldg(src + 2) : 0.0f;
                                x[it].w = (lv && i + 3 < ginner) ? __ldg(src + 3) : 0.0f;
                            } else if (have) {
                                x[it] = *reinterpret_cast<const float4*>(buf + rdo[it]);
                            }
                            off[it] = wro[it];
                        } else {
                            const int k = v >> 2, lc = v & 3;               // [128 k][16 l], TMA 64B swizzle
                            if (have && ldg) {
                                // elements (row, l .. l+3) of the contiguous fibre row, zero outside A
                                const int64_t row = r0 + k, gl = (int64_t)kc * kBK + lc * 4;
                                const float* src = ga + row * gnq + gl;
                                const bool rv = row < gouter;
                                x[it].x = (rv && gl < gnq) ? __ldg(src) : 0.0f;
                                x[it].y = (rv && gl + 1 < gnq) ? __ldg(src + 1) : 0.0f;
                                x[it].z = (rv && gl + 2 < gnq) ? __ldg(src + 2) : 0.0f;
                                x[it].w = (rv && gl + 3 < gnq) ? __ldg(src + 3) : 0.0f;
                            } else if (have) {
                                x[it] = *reinterpret_cast<const float4*>(buf + rdo[it]);
                            }
                            off[it] = wro[it];
                        }
                    }
                    conv_barrier(g);   // the whole FP32 tile is in registers before it is overwritten
                    if (have) {
#pragma unroll
                        for (int it = 0; it < kIters; ++it) {
                            uint32_t h0, l0, h1, l1;
                            split2(x[it].x, x[it].y, h0, l0);
                            split2(x[it].z, x[it].w, h1, l1);
                            // Lane pairs hold 8 consecutive elements, one 16-byte chunk of each part:
                            // each lane writes its half of the hi and of the lo chunk.
                            const uint32_t half = odd ? 8u : 0u;
                            *reinterpret_cast<uint2*>(buf + off[it] + half) = make_uint2(h0, h1);
                            *reinterpret_cast<uint2*>(buf + LA.abf_bytes + off[it] + half) = make_uint2(l0, l1);
                        }
                    }
                }
                if (have) {
                    fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&a_conv[s]);
                }
                s += kConvGroups;
                if (s >= AS) { s -= AS; ph ^= 1; }
            }
        }
    } else {
        // ------------------------------------------------------------- epilogue
        const int q4 = warp & 3;                 // TMEM lane quarter this warp may access
        const int ew = warp - (3 + kConvWarps);  // 0..3
        uint8_t* stage0 = epi + (size_t)ew * 2 * kEpiBuf;
        int sb = 0;
        int ab = 0;
        uint32_t aph = 0;
        const TcProb* last = nullptr;
        int cur = 0;
        for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
            int64_t lt;
            const TcProb& pr = tile_problem<GROUP>(one, P, t, cur, lt);
            if (GROUP && &pr != last && pr.tma_c) tensormap_acquire(&pr.cmap);
            last = &pr;
            const int64_t mper = (pr.inner + kBM - 1) / kBM;
            if (!mbar_wait(&acc_full[ab], aph, abort_flag, P.wait_ns)) break;
            tc_fence_after();
            const int64_t jb = lt / pr.tiles_m, mt = lt - jb * pr.tiles_m;
            int64_t k, r0;            // slice and first row (i for GEOM_MN, k for GEOM_K) of this warp
            if (GEOM == GEOM_MN && pr.fold_kb > 1) {
                // this warp's 32 rows lie in one slice of the folded tile
                k = mt * pr.fold_kb + ((q4 * 32) >> pr.fold_ib_shift);
                r0 = (q4 * 32) & ((1 << pr.fold_ib_shift) - 1);
            } else if (GEOM == GEOM_MN) {
                k = mt / mper;
                r0 = (mt - k * mper) * kBM + q4 * 32;
            } else {
                k = 0;
                r0 = mt * kBM + q4 * 32;
            }
            const int nt = pr.nt;
            // the record's fields the stores use, in registers: a grouped launch's records sit in
            // global memory, where every store to C could alias them and force a reload
            const int64_t e_inner = pr.inner, e_outer = pr.outer, e_m = pr.m;
            float* const e_c = pr.c;
            const bool e_tma = pr.tma_c != 0;
            const int64_t jrem = e_m - (int64_t)jb * nt;
            const int jleft = jrem < nt ? (int)jrem : nt;
            const uint32_t tbase = tmem_base + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(ab * P.acc_stride);
            for (int cc = 0; cc < nt; cc += 32) {
                uint32_t v[32];
                tmem_ld32(tbase + (uint32_t)cc, v);
                if (cc >= jleft) continue;
                const int j0 = jb * nt + cc;
                if (e_tma && GEOM == GEOM_MN && k >= e_outer) {
                    // folded last tile: this warp's slice lies past the end of C, nothing to store
                } else if (e_tma) {
                    // Stage a 32 x 32 block in shared memory and store it with one TMA copy.
                    uint8_t* buf = stage0 + sb * kEpiBuf;
                    if (lane == 0) bulk_wait_read1();      // the copy that last read `buf` has finished reading it
                    __syncwarp();
                    if (GEOM == GEOM_MN) {
                        // smem [32 j][32 i]: this lane owns column i = lane
                        float* b32 = reinterpret_cast<float*>(buf);
#pragma unroll
                        for (int c = 0; c < 32; ++c) b32[c * 32 + lane] = __uint_as_float(v[c]);
                    } else {
                        // smem [32 k][32 j] with the 128-byte swizzle: this lane owns row k = lane
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            *reinterpret_cast<uint4*>(buf + lane * 128 + ((c ^ (lane & 7)) << 4)) =
                                make_uint4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                    }
                    fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) {
                        if (GEOM == GEOM_MN) tma_store_3d(&pr.cmap, buf, (int)r0, j0, (int)k);
                        else tma_store_2d(&pr.cmap, buf, j0, (int)r0);
                        bulk_commit();
                    }
                    sb ^= 1;
                } else if (GEOM == GEOM_MN) {
                    // Direct stores (C rows not 16-byte aligned for a tensor map): lane = i, so each
                    // store instruction writes 32 consecutive elements of one row j of C.
                    const int64_t r = r0 + lane;
                    if (r < e_inner && k < e_outer) {
                        float* p = e_c + (k * e_m + j0) * e_inner + r;
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            if (cc + c < jleft) p[(int64_t)c * e_inner] = __uint_as_float(v[c]);
                    }
                } else {
                    // C rows (m elements each) not 16-byte aligned for a tensor map. A lane holds
                    // one row of the 32 x 32 block, m elements from the next lane's row: the block
                    // goes through shared memory ([row][col ^ row], conflict free both ways) and
                    // out one row segment per store instruction, consecutive lanes on consecutive
                    // elements.
                    float* b32 = reinterpret_cast<float*>(stage0 + sb * kEpiBuf);
                    if (lane == 0) bulk_wait_read0();      // no TMA store is still reading it
                    __syncwarp();
#pragma unroll
                    for (int c = 0; c < 32; ++c) b32[lane * 32 + (c ^ lane)] = __uint_as_float(v[c]);
                    __syncwarp();
                    const int cw = jleft - cc < 32 ? jleft - cc : 32;
                    const int64_t rl = e_outer - r0;
                    const int nrow = rl < 32 ? (int)rl : 32;
                    float* cb = e_c + r0 * e_m + j0 + lane;
                    if (lane < cw)
                        for (int row = 0; row < nrow; ++row) cb[(int64_t)row * e_m] = b32[row * 32 + (lane ^ row)];
                    __syncwarp();
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[ab]);
            if (++ab == 2) { ab = 0; aph ^= 1; }
        }
        if (lane == 0) bulk_wait_all();   // every TMA store of this warp has completed
    }

    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicExch(P.status, 1);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(512u));
    }
}

// B (m x nq, column- or row-major FP32) -> bf16 hi/lo images, one per (j block, K chunk),
// each NT rows x 16 l in the K-major SW32 layout the MMA reads. Zero outside B.
__device__ __forceinline__ void split_b_units(const float* __restrict__ b, int b_cm, int64_t m, int64_t nq, int nt,
                                              int jblocks, int kchunks, uint8_t* __restrict__ img, int64_t u0,
                                              int64_t step)
{
    const int64_t total = (int64_t)jblocks * kchunks * nt * 2;     // 2 chunks of 8 l per row
    const uint32_t part_bytes = (uint32_t)nt * (kBK * 2);
    for (int64_t u = u0; u < total; u += step) {
        const int c = (int)(u & 1);
        const int64_t rrow = u >> 1;
        const int jl = (int)(rrow % nt);
        const int64_t bk = rrow / nt;
        const int kc = (int)(bk % kchunks);
        const int jb = (int)(bk / kchunks);
        const int64_t j = (int64_t)jb * nt + jl;
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int64_t l = (int64_t)kc * kBK + c * 8 + e;
            x[e] = (j < m && l < nq) ? (b_cm ? b[j + l * m] : b[j * nq + l]) : 0.0f;
        }
        uint4 h, lo;
        split2(x[0], x[1], h.x, lo.x);
        split2(x[2], x[3], h.y, lo.y);
        split2(x[4], x[5], h.z, lo.z);
        split2(x[6], x[7], h.w, lo.w);
        uint8_t* base = img + (size_t)((int64_t)jb * kchunks + kc) * 2 * part_bytes;
        const uint32_t off = kmaj_sw32_off((uint32_t)jl, (uint32_t)c);
        *reinterpret_cast<uint4*>(base + off) = h;
        *reinterpret_cast<uint4*>(base + part_bytes + off) = lo;
    }
}

__global__ void split_b_kernel(const float* __restrict__ b, int b_cm, int64_t m, int64_t nq, int nt, int jblocks,
                               int kchunks, uint8_t* __restrict__ img)
{
    split_b_units(b, b_cm, m, nq, nt, jblocks, kchunks, img, (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                  (int64_t)gridDim.x * blockDim.x);
}

// The operand split of every problem of a grouped launch: blockIdx.y + y0 is the problem.
__global__ void split_b_group_kernel(const TcProb* __restrict__ group, int y0)
{
    const TcProb& pr = group[blockIdx.y + y0];
    split_b_units(pr.b, pr.b_cm, pr.m, pr.nq, pr.nt, pr.jblocks, pr.kstages * kSub, const_cast<uint8_t*>(pr.bimg),
                  (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// ------------------------------------------------------------------ TMA-fed small-m kernel
// Exact (FMA in the I/O type) small-m contraction for strided fibres. A producer warp streams
// 16 KB boxes of A into a ring with TMA; 8 consumer warps multiply them with B staged in shared
// memory. A box holds P = 256 * W fibre positions x LB l (n_q l when n_q < LB), where
// W = 16 bytes / element size is the number of consecutive positions one consumer thread owns
// (one 128-bit shared-memory read per l, reused across all m rows of B). The positions are KB consecutive slices k of H * IB
// consecutive i: with H = 1 the tensor map is (i, k, l) and IB a power of two covering inner
// with little waste, so small inner extents still fill whole boxes; with H > 1 (few slices of
// a large inner that IB divides) it is the 4D (i mod IB, i / IB, k, l). The dimensions are
// deliberately not in stride order: either way a box lands in shared memory as
// [l][P positions], position = (k * H + h) * IB + i mod IB.
// Work unit = (tile, l range). When there are too few tiles to fill the GPU, or B is too large
// to stage whole, the l range is split S ways: each unit stages only its rows of B, writes a
// partial tile to a workspace, and the last unit of a tile to finish (atomic counter) adds the
// S partials in a fixed order and stores C, so results do not depend on scheduling.
constexpr int kStreamMaxStages = 8;
constexpr int kStreamThreads = 9 * 32;          // 8 consumer warps + 1 producer warp
constexpr uint32_t kStreamBox = 16384;          // bytes per box

struct StreamParams {
    const void* b;
    void* c;
    void* ws;               // S > 1: partial tiles [tiles][S][MB][P]
    unsigned* cnt;          // S > 1: per-tile arrival counters, zero at launch
    int64_t outer, nq, inner, m;
    int64_t tiles;          // ceil(outer / KB) * mper
    int64_t mper;           // ceil(inner / IB)
    int64_t units;          // tiles * S
    int kchunks;            // ceil(nq / lb)
    int lb;                 // l per box: LB, or n_q when n_q < LB
    int kper;               // l chunks per unit
    int S;                  // l ranges per tile
    int b_cm;
    int ib_shift;           // log2(IB)
    int h_shift;            // log2(H); H > 1 uses the 4D map
    int kb;                 // KB = P / (IB * H)
    FastDiv fd_s, fd_mper;  // division by S and by mper (unit -> tile -> slice block)
};

// One problem of a stream launch: its tensor map and parameters. A single launch passes it as a
// kernel parameter; a grouped launch reads an array of them from device memory (64-byte aligned).
struct alignas(64) StreamProb {
    CUtensorMap amap;
    StreamParams P;
    int64_t first;          // grouped launch: index of the problem's first unit among all units
};

static_assert(sizeof(TcProb) % 64 == 0, "problem records keep their tensor maps 64-byte aligned");
static_assert(sizeof(StreamProb) % 64 == 0, "problem records keep their tensor maps 64-byte aligned");

// Launch-wide parameters of a stream launch.
struct StreamLaunch {
    int* status;
    const StreamProb* group;   // grouped launch: `count` problems in device memory (else unused)
    int count;
    int64_t total;             // units over all problems
    int stages;                // ring depth, <= kStreamMaxStages
    int brows;                 // l rows of B the staging area holds (kper * lb of every problem)
};

// The problem owning unit u of the launch and the unit's index within it; `cur` carries the
// search on from the previous unit (units are visited in increasing order).
template <bool GROUP>
__device__ __forceinline__ const StreamProb& unit_problem(const StreamProb& one, const StreamLaunch& L, int64_t u,
                                                          int& cur, int64_t& lu)
{
    if constexpr (!GROUP) {
        lu = u;
        return one;
    } else {
        while (cur + 1 < L.count && L.group[cur + 1].first <= u) ++cur;
        lu = u - L.group[cur].first;
        return L.group[cur];
    }
}

template <typename T> struct V16Tc;
template <> struct V16Tc<float> { using type = float4; };
template <> struct V16Tc<double> { using type = double2; };

// Column mode: W consecutive positions per thread, a 16 KB stage = one box of P positions x LB
// l, [l][P]. Row mode (contiguous fibres, inner = 1): two fibres (rows) per thread, t and
// t + 256; a 32 KB stage = two boxes of 256 rows x 64 bytes of l (LB = 16 float / 8 double),
// each [row][64 bytes] with the 64-byte swizzle. Two rows per thread halve the shared-memory
// reads of B per FMA; 64-byte rows keep the DRAM accesses long.
template <typename T, bool ROWS = false>
struct StreamGeom {
    static constexpr int W = ROWS ? 2 : 16 / (int)sizeof(T);           // positions per thread
    static constexpr int P = 256 * W;                                  // positions per stage
    static constexpr uint32_t SB = ROWS ? 2 * kStreamBox : kStreamBox; // bytes per stage
    static constexpr int LB = (int)(SB / (P * sizeof(T)));             // l per stage
};

// The kernel comes in two builds by resident CTAs per SM (CPS). A warp's registers come from
// its sub-partition's quarter of the register file (16384), and the nine warps of CPS CTAs spread
// over the four sub-partitions, so the per-thread cap is 16384 / ceil(9 CPS / 4) / 32 rounded
// down to 8: 96 for two CTAs (no spills for m <= 8), 168 for one (any m <= 16).
constexpr int stream_nreg(int cps) { return cps == 2 ? 96 : 168; }

// GROUP = false: one problem, `one`. GROUP = true: the L.count problems of L.group (each with
// S == 1 and B staged whole), their units numbered one after the other; producer and consumers
// walk the same unit sequence, so the ring streams across problem boundaries.
template <typename T, int MB, bool ROWS, int CPS, bool GROUP>
__global__ void __maxnreg__(stream_nreg(CPS))
    stream_cols_kernel(const __grid_constant__ StreamProb one, StreamLaunch L)
{
    using G = StreamGeom<T, ROWS>;
    constexpr int W = G::W, NP = G::P, LB = G::LB;
    using V = typename std::conditional<ROWS, T, typename V16Tc<T>::type>::type;   // W consecutive T
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int stages = L.stages;
    uint8_t* ring = smem;
    constexpr uint32_t SB = G::SB;
    T* bs = reinterpret_cast<T*>(smem + stages * SB);                          // [kper * lb][MB]
    uint64_t* full = reinterpret_cast<uint64_t*>(bs + (size_t)L.brows * MB);
    full = reinterpret_cast<uint64_t*>((reinterpret_cast<uintptr_t>(full) + 15) & ~uintptr_t(15));
    uint64_t* empty = full + kStreamMaxStages;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + kStreamMaxStages);
    volatile int* last_flag = abort_flag + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 8);
        }
        *abort_flag = 0;
        *last_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == 8) {
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            int issued[kStreamMaxStages];
            for (int i = 0; i < kStreamMaxStages; ++i) issued[i] = -1;
            int cur = 0;
            const StreamProb* last = nullptr;
            for (int64_t u = blockIdx.x; u < L.total && ok; u += gridDim.x) {
                int64_t lu;
                const StreamProb& pq = unit_problem<GROUP>(one, L, u, cur, lu);
                if (GROUP && &pq != last) tensormap_acquire(&pq.amap);
                last = &pq;
                const StreamParams& Q = pq.P;
                const int S = Q.S;
                const int IB = 1 << Q.ib_shift;
                const int64_t t = S == 1 ? lu : (int64_t)fast_div((uint32_t)lu, Q.fd_s);
                const int r = (int)(lu - t * S);
                const int64_t kb = fast_div((uint32_t)t, Q.fd_mper), ib = t - kb * Q.mper;
                const int kc0 = r * Q.kper, kc1 = min(kc0 + Q.kper, Q.kchunks);
                for (int kc = kc0; kc < kc1; ++kc) {
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                    issued[s] = (int)ph;
                    mbar_expect_tx(&full[s], (uint32_t)(NP * Q.lb * sizeof(T)));
                    if (ROWS) {
                        tma_load_2d(ring + s * SB, &pq.amap, &full[s], kc * Q.lb, (int)(kb * Q.kb));
                        tma_load_2d(ring + s * SB + SB / 2, &pq.amap, &full[s], kc * Q.lb,
                                    (int)(kb * Q.kb + 256));
                    }
                    else if (Q.h_shift == 0)
                        tma_load_3d(ring + s * SB, &pq.amap, &full[s], (int)(ib * IB), (int)(kb * Q.kb), kc * Q.lb);
                    else
                        tma_load_4d(ring + s * SB, &pq.amap, &full[s], 0, (int)(ib << Q.h_shift), (int)(kb * Q.kb),
                                    kc * Q.lb);
                    if (++s == stages) { s = 0; ph ^= 1; }
                }
            }
            for (int i = 0; i < stages; ++i) {
                if (issued[i] < 0) continue;
                const unsigned long long t0 = gtimer();
                while (!mbar_try(&full[i], (uint32_t)issued[i]) && gtimer() - t0 < kTimeoutNs) {}
            }
        }
    } else {
        const int tid = threadIdx.x;                       // 0..255
        const int pos = tid * W;                           // first owned position
        int s = 0;
        uint32_t ph = 0;
        bool ok = true;
        int staged = -1, staged_p = -1;                    // l range (r) and problem held in bs
        int cur = 0;
        // Every consumer runs every iteration and meets the consumer barriers the same number of
        // times; after an abort the waits are skipped and no work is done.
        for (int64_t u = blockIdx.x; u < L.total; u += gridDim.x) {
            int64_t lu;
            const StreamProb& pq = unit_problem<GROUP>(one, L, u, cur, lu);
            // a grouped launch's record by value: its fields in global memory could otherwise be
            // aliased by the stores to C and to B's staging area and reloaded after each (a single
            // launch's record is a constant kernel parameter)
            const StreamParams Qv = pq.P;
            const StreamParams& Q = GROUP ? Qv : pq.P;
            const int S = Q.S;
            const int IB = 1 << Q.ib_shift;
            const int kk = pos >> (Q.ib_shift + Q.h_shift);
            const int hh = (pos >> Q.ib_shift) & ((1 << Q.h_shift) - 1), ii = pos & (IB - 1);
            const T* Bg = static_cast<const T*>(Q.b);
            T* C = static_cast<T*>(Q.c);
            const int64_t t = S == 1 ? lu : (int64_t)fast_div((uint32_t)lu, Q.fd_s);
            const int r = (int)(lu - t * S);
            const int64_t kb = fast_div((uint32_t)t, Q.fd_mper), ib = t - kb * Q.mper;
            const int kc0 = r * Q.kper, kc1 = min(kc0 + Q.kper, Q.kchunks);
            if (r != staged || cur != staged_p) {
                // stage rows [kc0 * lb, kc1 * lb) of B: bs[l][j] = B(j, l), zero outside B. The
                // loads go out four at a time ahead of their stores: bs is a generic pointer, so
                // the compiler would otherwise wait for each load before the next store.
                asm volatile("bar.sync 1, 256;" ::: "memory");
                const int total = (kc1 - kc0) * Q.lb * MB;
                for (int e0 = tid; e0 < total; e0 += 256 * 4) {
                    T v[4];
#pragma unroll
                    for (int x = 0; x < 4; ++x) {
                        const int e = e0 + x * 256;
                        const int lr = e / MB, j = e - lr * MB;
                        const int64_t l = (int64_t)kc0 * Q.lb + lr;
                        v[x] = (e < total && j < Q.m && l < Q.nq)
                                   ? __ldg(Q.b_cm ? Bg + j + l * Q.m : Bg + j * Q.nq + l) : T(0);
                    }
#pragma unroll
                    for (int x = 0; x < 4; ++x)
                        if (e0 + x * 256 < total) bs[e0 + x * 256] = v[x];
                }
                asm volatile("bar.sync 1, 256;" ::: "memory");
                staged = r;
                staged_p = cur;
            }
            T acc[W][MB];
#pragma unroll
            for (int w = 0; w < W; ++w)
#pragma unroll
                for (int j = 0; j < MB; ++j) acc[w][j] = T(0);
            for (int kc = kc0; kc < kc1; ++kc) {
                const bool got = ok && mbar_wait(&full[s], ph, abort_flag);
                const bool have = __all_sync(0xffffffffu, got);
                if (!have) ok = false;
                if (have && ROWS) {
                    // rows tid and tid + 256: 64 bytes each, in four 16-byte chunks, chunk c stored
                    // at c ^ ((row >> 1) & 3) (the 64-byte swizzle), which also keeps a warp's
                    // reads free of bank conflicts; B is a broadcast read, used for both rows
                    using V16 = typename V16Tc<T>::type;
                    constexpr int EPC = 16 / (int)sizeof(T);
                    const uint8_t* r0p = ring + s * SB + tid * 64;
                    const uint8_t* r1p = r0p + SB / 2;
                    const int sw = (tid >> 1) & 3;
                    const T* brow = bs + (size_t)(kc - kc0) * LB * MB;
                    V16 ch[2][4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        ch[0][c] = *reinterpret_cast<const V16*>(r0p + ((c ^ sw) << 4));
                        ch[1][c] = *reinterpret_cast<const V16*>(r1p + ((c ^ sw) << 4));
                    }
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const T* a0 = reinterpret_cast<const T*>(&ch[0][c]);
                        const T* a1 = reinterpret_cast<const T*>(&ch[1][c]);
#pragma unroll
                        for (int e = 0; e < EPC; ++e) {
                            const T* bl = brow + (c * EPC + e) * MB;
                            if constexpr (MB * sizeof(T) % 16 == 0) {
#pragma unroll
                                for (int q = 0; q < MB * (int)sizeof(T) / 16; ++q) {
                                    const V16 bv = *reinterpret_cast<const V16*>(bl + q * EPC);
                                    const T* b = reinterpret_cast<const T*>(&bv);
#pragma unroll
                                    for (int f = 0; f < EPC; ++f) {
                                        acc[0][q * EPC + f] = fma(a0[e], b[f], acc[0][q * EPC + f]);
                                        acc[1][q * EPC + f] = fma(a1[e], b[f], acc[1][q * EPC + f]);
                                    }
                                }
                            } else {
#pragma unroll
                                for (int j = 0; j < MB; ++j) {
                                    acc[0][j] = fma(a0[e], bl[j], acc[0][j]);
                                    acc[1][j] = fma(a1[e], bl[j], acc[1][j]);
                                }
                            }
                        }
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[s]);
                } else if (have) {
                    const V* box = reinterpret_cast<const V*>(ring + s * SB) + tid;
                    const T* brow = bs + (size_t)(kc - kc0) * Q.lb * MB;
                    const int lb = Q.lb;
                    // all LB reads up front (the builds for m = 16 run one CTA per SM and have
                    // the registers)
                    V av[LB];
#pragma unroll
                    for (int l = 0; l < LB; ++l) av[l] = box[l * (NP / W)];   // in the stage even past lb
#pragma unroll
                    for (int l = 0; l < LB; ++l) {
                        if (l >= lb) break;
                        const V a1 = av[l];
                        const T* a = reinterpret_cast<const T*>(&a1);
                        const T* bl = brow + l * MB;
                        if constexpr (MB % W == 0) {
#pragma unroll
                            for (int c = 0; c < MB / W; ++c) {
                                const V bv = *reinterpret_cast<const V*>(bl + c * W);
                                const T* b = reinterpret_cast<const T*>(&bv);
#pragma unroll
                                for (int e = 0; e < W; ++e)
#pragma unroll
                                    for (int w = 0; w < W; ++w) acc[w][c * W + e] = fma(a[w], b[e], acc[w][c * W + e]);
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < MB; ++j) {
                                const T b = bl[j];
#pragma unroll
                                for (int w = 0; w < W; ++w) acc[w][j] = fma(a[w], b, acc[w][j]);
                            }
                        }
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[s]);
                }
                if (++s == stages) { s = 0; ph ^= 1; }
            }
            if constexpr (ROWS) {
                // rows k0 = tile * 512 + tid and k0 + 256; C[k][j] contiguous in j
                const int64_t kr[2] = {kb * Q.kb + tid, kb * Q.kb + 256 + tid};
                if (S == 1) {
                    if (ok) {
#pragma unroll
                        for (int w = 0; w < 2; ++w)
                            if (kr[w] < Q.outer) {
                                T* cp = C + kr[w] * Q.m;
                                if constexpr (MB * sizeof(T) % 16 == 0) {
                                    // whole rows of MB outputs on 16-byte boundaries: vector stores
                                    if (Q.m == MB && (reinterpret_cast<uintptr_t>(C) & 15u) == 0) {
                                        using V16 = typename V16Tc<T>::type;
                                        constexpr int EPC = 16 / (int)sizeof(T);
#pragma unroll
                                        for (int q = 0; q < MB / EPC; ++q) {
                                            V16 v;
                                            T* vv = reinterpret_cast<T*>(&v);
#pragma unroll
                                            for (int f = 0; f < EPC; ++f) vv[f] = acc[w][q * EPC + f];
                                            *reinterpret_cast<V16*>(cp + q * EPC) = v;
                                        }
                                        continue;
                                    }
                                }
#pragma unroll
                                for (int j = 0; j < MB; ++j)
                                    if (j < Q.m) cp[j] = acc[w][j];
                            }
                    }
                } else {
                    T* wsp = static_cast<T*>(Q.ws) + ((size_t)lu * MB) * NP;
#pragma unroll
                    for (int j = 0; j < MB; ++j) {
                        wsp[(size_t)j * NP + tid] = acc[0][j];
                        wsp[(size_t)j * NP + 256 + tid] = acc[1][j];
                    }
                    __threadfence();
                    asm volatile("bar.sync 1, 256;" ::: "memory");
                    if (tid == 0) *last_flag = (!*abort_flag && atomicAdd(&Q.cnt[t], 1u) == (unsigned)(S - 1)) ? 1 : 0;
                    asm volatile("bar.sync 1, 256;" ::: "memory");
                    if (*last_flag) {
                        __threadfence();
                        const T* w0 = static_cast<const T*>(Q.ws) + ((size_t)t * S * MB) * NP;
#pragma unroll
                        for (int w = 0; w < 2; ++w) {
                            if (kr[w] >= Q.outer) continue;
                            T* cp = C + kr[w] * Q.m;
                            for (int j = 0; j < MB && j < Q.m; ++j) {
                                T sum = T(0);
                                for (int rr = 0; rr < S; ++rr) sum += __ldcg(w0 + ((size_t)rr * MB + j) * NP + w * 256 + tid);
                                cp[j] = sum;
                            }
                        }
                    }
                }
                continue;
            }
            const int64_t k = kb * Q.kb + kk, i = (((ib << Q.h_shift) + hh) << Q.ib_shift) + ii;
            const bool mine = k < Q.outer && i < Q.inner;     // all W positions share k; inner % W == 0
            if (S == 1) {
                if (ok && mine) {
                    T* cp = C + (k * Q.m) * Q.inner + i;
#pragma unroll
                    for (int j = 0; j < MB; ++j) {
                        if (j < Q.m) {
                            V v;
                            T* vv = reinterpret_cast<T*>(&v);
#pragma unroll
                            for (int w = 0; w < W; ++w) vv[w] = acc[w][j];
                            *reinterpret_cast<V*>(cp + (int64_t)j * Q.inner) = v;
                        }
                    }
                }
            } else {
                T* wsp = static_cast<T*>(Q.ws) + ((size_t)lu * MB) * NP + pos;
#pragma unroll
                for (int j = 0; j < MB; ++j) {
                    V v;
                    T* vv = reinterpret_cast<T*>(&v);
#pragma unroll
                    for (int w = 0; w < W; ++w) vv[w] = acc[w][j];
                    *reinterpret_cast<V*>(wsp + (size_t)j * NP) = v;
                }
                __threadfence();
                asm volatile("bar.sync 1, 256;" ::: "memory");
                if (tid == 0) *last_flag = (!*abort_flag && atomicAdd(&Q.cnt[t], 1u) == (unsigned)(S - 1)) ? 1 : 0;
                asm volatile("bar.sync 1, 256;" ::: "memory");
                if (*last_flag) {
                    __threadfence();
                    if (mine) {
                        const T* w0 = static_cast<const T*>(Q.ws) + ((size_t)t * S * MB) * NP + pos;
                        T* cp = C + (k * Q.m) * Q.inner + i;
                        for (int j = 0; j < MB && j < Q.m; ++j) {
                            V sum;
                            T* sv = reinterpret_cast<T*>(&sum);
#pragma unroll
                            for (int w = 0; w < W; ++w) sv[w] = T(0);
                            for (int rr = 0; rr < S; ++rr) {
                                const V v = __ldcg(reinterpret_cast<const V*>(w0 + ((size_t)rr * MB + j) * NP));
                                const T* vv = reinterpret_cast<const T*>(&v);
#pragma unroll
                                for (int w = 0; w < W; ++w) sv[w] += vv[w];
                            }
                            *reinterpret_cast<V*>(cp + (int64_t)j * Q.inner) = sum;
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicExch(L.status, 1);
}

// ------------------------------------------------------------------ host side
// Per-device state: the device status word that kernels raise on a failed bounded wait.
struct DevState {
    int* status = nullptr;
    bool pool_tuned = false;
};
std::mutex g_state_mu;
std::unordered_map<int, DevState> g_state;

cudaError_t state_for(int dev, DevState*& out)
{
    std::lock_guard<std::mutex> lk(g_state_mu);
    DevState& d = g_state[dev];
    if (!d.status) {
        cudaError_t e = dev_malloc(reinterpret_cast<void**>(&d.status), 256);
        if (e != cudaSuccess) return e;
        e = cudaMemset(d.status, 0, 256);
        if (e != cudaSuccess) return e;
    }
    if (!d.pool_tuned) {
        // Scratch comes from the stream-ordered pool (cudaMallocAsync): keep freed blocks cached
        // instead of returning them to the driver at every synchronisation.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        d.pool_tuned = true;
    }
    out = &d;
    return cudaSuccess;
}

int g_sm_count = 0;

// cuTensorMapEncodeTiled through the runtime's driver entry point, so that the
// library itself does not link libcuda (it still loads on machines without a driver).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

bool encode_a_map(const View3& v, int geom, CUtensorMap* map)
{
    EncodeTiledFn cuTensorMapEncodeTiled = encode_fn();
    if (!cuTensorMapEncodeTiled) return false;
    CUresult r;
    if (geom == GEOM_MN) {
        cuuint64_t dims[3] = {(cuuint64_t)v.inner, (cuuint64_t)v.nq, (cuuint64_t)v.outer};
        cuuint64_t strides[2] = {(cuuint64_t)v.inner * 4, (cuuint64_t)v.inner * v.nq * 4};
        cuuint32_t box[3] = {kBM, kBK, 1};
        cuuint32_t es[3] = {1, 1, 1};
        r = cuTensorMapEncodeTiled(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(v.a), dims, strides, box,
                                   es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        cuuint64_t dims[2] = {(cuuint64_t)v.nq, (cuuint64_t)v.outer};
        cuuint64_t strides[1] = {(cuuint64_t)v.nq * 4};
        cuuint32_t box[2] = {kBK, kBM};
        cuuint32_t es[2] = {1, 1};
        r = cuTensorMapEncodeTiled(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(v.a), dims, strides, box,
                                   es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

// A of a folded GEOM_MN tile as the 3-D map (i, k, l) -- dimensions deliberately not in stride
// order -- with boxes of ib i x kb slices x kBK l, which land in shared memory as [l][kb*ib rows]:
// the same layout as an unfolded tile of 128 i.
bool encode_a_map_folded(const View3& v, int ib, int kb, CUtensorMap* map)
{
    EncodeTiledFn cuTensorMapEncodeTiled = encode_fn();
    if (!cuTensorMapEncodeTiled) return false;
    cuuint64_t dims[3] = {(cuuint64_t)v.inner, (cuuint64_t)v.outer, (cuuint64_t)v.nq};
    cuuint64_t strides[2] = {(cuuint64_t)(v.inner * v.nq) * 4, (cuuint64_t)v.inner * 4};
    cuuint32_t box[3] = {(cuuint32_t)ib, (cuuint32_t)kb, (cuuint32_t)kBK};
    cuuint32_t es[3] = {1, 1, 1};
    return cuTensorMapEncodeTiled(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(v.a), dims, strides, box, es,
                                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C as a tensor map for the TMA-store epilogue: 32 x 32 boxes. False when C's rows are not
// 16-byte aligned (the epilogue then stores directly).
bool encode_c_map(const View3& v, int geom, CUtensorMap* map)
{
    EncodeTiledFn cuTensorMapEncodeTiled = encode_fn();
    if (!cuTensorMapEncodeTiled) return false;
    if ((reinterpret_cast<uintptr_t>(v.c) & 15u) != 0) return false;
    CUresult r;
    if (geom == GEOM_MN) {
        cuuint64_t dims[3] = {(cuuint64_t)v.inner, (cuuint64_t)v.m, (cuuint64_t)v.outer};
        cuuint64_t strides[2] = {(cuuint64_t)v.inner * 4, (cuuint64_t)v.inner * v.m * 4};
        cuuint32_t box[3] = {32, 32, 1};
        cuuint32_t es[3] = {1, 1, 1};
        r = cuTensorMapEncodeTiled(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, v.c, dims, strides, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        if (v.m % 4 != 0) return false;
        cuuint64_t dims[2] = {(cuuint64_t)v.m, (cuuint64_t)v.outer};
        cuuint64_t strides[1] = {(cuuint64_t)v.m * 4};
        cuuint32_t box[2] = {32, 32};
        cuuint32_t es[2] = {1, 1};
        r = cuTensorMapEncodeTiled(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, v.c, dims, strides, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

int geometry_of(const View3& v) { return v.inner == 1 ? GEOM_K : GEOM_MN; }

// A's rows (the fibres' 16-l chunks for GEOM_K, the i runs for GEOM_MN) start on 16-byte
// boundaries: TMA can load its tiles. Otherwise the converter warps load A themselves.
bool tma_a_ok(const View3& v, int geom)
{
    if ((reinterpret_cast<uintptr_t>(v.a) & 15u) != 0) return false;
    return geom == GEOM_K ? v.nq % 4 == 0 : v.inner % 4 == 0;
}

// Fills the problem record of the bf16x3 kernel for view v, its pre-split B image at `img`
// (tc_image_bytes(v) bytes); *geom receives its geometry.
void make_tc_prob(const View3& v, uint8_t* img, TcProb& pr, int* geom)
{
    std::memset(&pr, 0, sizeof(pr));
    const int g = geometry_of(v);
    *geom = g;
    pr.nt = (int)std::min<int64_t>(kMaxNT, ((v.m + 15) / 16) * 16);
    pr.jblocks = (int)((v.m + pr.nt - 1) / pr.nt);
    pr.kchunks = (int)((v.nq + kBK - 1) / kBK);
    pr.kstages = (pr.kchunks + kSub - 1) / kSub;
    pr.ldg_a = tma_a_ok(v, g) ? 0 : 1;
    pr.a = static_cast<const float*>(v.a);
    pr.b = static_cast<const float*>(v.b);
    pr.b_cm = v.b_cm ? 1 : 0;
    // inner <= 64: KB = 128 / IB slices share a 128-row tile (IB = 32 or 64 rows each)
    pr.fold_kb = 1;
    pr.fold_ib_shift = 7;
    if (g == GEOM_MN && v.inner <= 64) {
        pr.fold_ib_shift = v.inner <= 32 ? 5 : 6;
        pr.fold_kb = kBM >> pr.fold_ib_shift;
    }
    if (!pr.ldg_a && !(pr.fold_kb > 1 ? encode_a_map_folded(v, 1 << pr.fold_ib_shift, pr.fold_kb, &pr.amap)
                                      : encode_a_map(v, g, &pr.amap)))
        pr.ldg_a = 1;   // the driver declined the map: the converters load A
    if (pr.ldg_a) std::memset(&pr.amap, 0, sizeof(pr.amap));
    pr.tma_c = encode_c_map(v, g, &pr.cmap) ? 1 : 0;
    if (!pr.tma_c) std::memset(&pr.cmap, 0, sizeof(pr.cmap));
    pr.c = static_cast<float*>(v.c);
    pr.bimg = img;
    pr.outer = v.outer;
    pr.nq = v.nq;
    pr.inner = v.inner;
    pr.m = v.m;
    pr.tiles_m = g == GEOM_MN ? (pr.fold_kb > 1 ? (v.outer + pr.fold_kb - 1) / pr.fold_kb
                                                : v.outer * ((v.inner + kBM - 1) / kBM))
                              : (v.outer + kBM - 1) / kBM;
    pr.tiles = pr.tiles_m * pr.jblocks;
    pr.first = 0;
}

// Elements of B's image a problem's operand split writes: kstages * kSub sub-blocks of 16 l per
// j block (zero past n_q), nt rows each, in two 8-l halves.
int64_t split_units(const TcProb& pr) { return (int64_t)pr.jblocks * (pr.kstages * kSub) * pr.nt * 2; }

template <int GEOM, bool GROUP>
cudaError_t launch_tc_kernel(const TcProb& one, const TcParams& P, size_t smem, int grid, cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(tc_bf16x3_kernel<GEOM, GROUP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess) tc_bf16x3_kernel<GEOM, GROUP><<<grid, kThreads, smem, s>>>(one, P);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

// Splits B into `img` (tc_image_bytes(v) bytes) and launches the bf16x3 kernel for v on stream s.
cudaError_t run_bf16x3(const View3& v, uint8_t* img, int* status, int sms, cudaStream_t s)
{
    TcProb pr;
    int geom = GEOM_MN;
    make_tc_prob(v, img, pr, &geom);
    TcParams P{};
    P.status = status;
    P.group = nullptr;
    P.count = 1;
    P.total = pr.tiles;
    P.bslot = smem_layout(pr.nt).bstage_bytes;
    P.acc_stride = pr.nt;
    P.wait_ns = wait_limit_ns();
    P.skip_b = take_skip_b() ? 1 : 0;
    size_t smem = 0;
    if (!choose_stages(pr.nt, P.fstages, P.ostages, smem)) return cudaErrorNotSupported;

    const int64_t total = split_units(pr);
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
    split_b_kernel<<<blocks, 256, 0, s>>>(pr.b, pr.b_cm, pr.m, pr.nq, pr.nt, pr.jblocks, pr.kstages * kSub, img);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int grid = (int)std::min<int64_t>(pr.tiles, sms);
    return geom == GEOM_MN ? launch_tc_kernel<GEOM_MN, false>(pr, P, smem, grid, s)
                           : launch_tc_kernel<GEOM_K, false>(pr, P, smem, grid, s);
}

}  // namespace

// ------------------------------------------------------------------ grouped bf16x3 launch
struct TcGroup {
    TcProb* d_probs = nullptr;    // device records: the GEOM_MN problems, then the GEOM_K ones
    uint8_t* d_img = nullptr;     // all pre-split B images
    int* status = nullptr;
    int count = 0;
    int split_x = 1;              // blocks per problem of the operand split
    TcParams P[2] = {};           // per geometry (count 0: none)
    size_t smem[2] = {0, 0};
    int grid[2] = {0, 0};
};

namespace {
const TcProb g_no_prob{};        // the unused single-problem parameter of grouped launches
}

cudaError_t tc_group_create(const View3* views, int count, TcGroup** out)
{
    *out = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    DevState* st = nullptr;
    if ((e = state_for(dev, st)) != cudaSuccess) return e;
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    std::unique_ptr<TcGroup, void (*)(TcGroup*)> G(new TcGroup(), tc_group_destroy);
    G->status = st->status;
    G->count = count;
    if (count == 0) {
        *out = G.release();
        return cudaSuccess;
    }
    std::vector<size_t> img_off(count);
    size_t img_total = 0;
    for (int i = 0; i < count; ++i) {
        img_off[i] = img_total;
        img_total += (tc_image_bytes(views[i]) + 255) & ~size_t(255);
    }
    if ((e = dev_malloc(reinterpret_cast<void**>(&G->d_img), img_total)) != cudaSuccess) return e;
    std::vector<TcProb> probs(count);
    std::vector<int> geom(count);
    for (int i = 0; i < count; ++i) make_tc_prob(views[i], G->d_img + img_off[i], probs[i], &geom[i]);
    // GEOM_MN first, then GEOM_K; within each, the problems with the heaviest tiles first, so
    // that the round robin of tiles over the persistent CTAs ends on light ones
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    auto tile_cost = [&](int i) { return (int64_t)probs[i].kstages * probs[i].nt; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        if (geom[x] != geom[y]) return geom[x] < geom[y];
        return tile_cost(x) > tile_cost(y);
    });
    std::vector<TcProb> sorted(count);
    int64_t first[2] = {0, 0};
    int ntmax[2] = {16, 16}, n[2] = {0, 0};
    int64_t max_units = 0;
    for (int r = 0; r < count; ++r) {
        const int i = order[r], g = geom[i];
        sorted[r] = probs[i];
        sorted[r].first = first[g];
        first[g] += probs[i].tiles;
        ntmax[g] = std::max(ntmax[g], probs[i].nt);
        ++n[g];
        max_units = std::max(max_units, split_units(probs[i]));
    }
    if ((e = dev_malloc(reinterpret_cast<void**>(&G->d_probs), sizeof(TcProb) * count)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(G->d_probs, sorted.data(), sizeof(TcProb) * count, cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    G->split_x = (int)std::max<int64_t>(1, std::min<int64_t>((max_units + 255) / 256, 64));
    for (int g = 0; g < 2; ++g) {
        TcParams& P = G->P[g];
        P = TcParams{};
        P.count = n[g];
        if (n[g] == 0) continue;
        P.status = G->status;
        P.group = G->d_probs + (g == 0 ? 0 : n[0]);
        P.total = first[g];
        P.bslot = smem_layout(ntmax[g]).bstage_bytes;
        P.acc_stride = ntmax[g];
        if (!choose_stages(ntmax[g], P.fstages, P.ostages, G->smem[g])) return cudaErrorNotSupported;
        G->grid[g] = (int)std::min<int64_t>(P.total, sms);
    }
    *out = G.release();
    return cudaSuccess;
}

cudaError_t tc_group_run(TcGroup* G, cudaStream_t s)
{
    if (!G || G->count == 0) return cudaSuccess;
    for (int y0 = 0; y0 < G->count; y0 += 65535) {
        const int ny = std::min(G->count - y0, 65535);
        split_b_group_kernel<<<dim3((unsigned)G->split_x, (unsigned)ny), 256, 0, s>>>(G->d_probs, y0);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    for (int g = 0; g < 2; ++g) {
        TcParams P = G->P[g];
        if (P.count == 0) continue;
        P.wait_ns = wait_limit_ns();
        P.skip_b = take_skip_b() ? 1 : 0;
        cudaError_t e = g == 0 ? launch_tc_kernel<GEOM_MN, true>(g_no_prob, P, G->smem[g], G->grid[g], s)
                               : launch_tc_kernel<GEOM_K, true>(g_no_prob, P, G->smem[g], G->grid[g], s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int tc_group_launches(const TcGroup* G)
{
    if (!G || G->count == 0) return 0;
    return (G->count + 65534) / 65535 + (G->P[0].count > 0) + (G->P[1].count > 0);
}

void tc_group_destroy(TcGroup* G)
{
    if (!G) return;
    if (G->d_probs) cudaFree(G->d_probs);
    if (G->d_img) cudaFree(G->d_img);
    delete G;
}

namespace {

// A as a tensor map over (i, k, l), or with h > 1 over (i mod ib, i / ib, k, l) (ib must divide
// inner) -- dimensions deliberately not in stride order -- with boxes of ib x [h x] kb x LB.
bool encode_stream_map(const View3& v, int dtype, int ib, int h, int kb, CUtensorMap* map)
{
    EncodeTiledFn cuTensorMapEncodeTiled = encode_fn();
    if (!cuTensorMapEncodeTiled) return false;
    const size_t es = dtype == 0 ? 4 : 8;
    const cuuint32_t LB = dtype == 0 ? (cuuint32_t)StreamGeom<float>::LB : (cuuint32_t)StreamGeom<double>::LB;
    const cuuint32_t lb = (cuuint64_t)v.nq < LB ? (cuuint32_t)v.nq : LB;
    const CUtensorMapDataType ty = dtype == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUresult r;
    if (h <= 1) {
        cuuint64_t dims[3] = {(cuuint64_t)v.inner, (cuuint64_t)v.outer, (cuuint64_t)v.nq};
        cuuint64_t strides[2] = {(cuuint64_t)(v.inner * v.nq) * es, (cuuint64_t)v.inner * es};
        cuuint32_t box[3] = {(cuuint32_t)ib, (cuuint32_t)kb, lb};
        cuuint32_t el[3] = {1, 1, 1};
        r = cuTensorMapEncodeTiled(map, ty, 3, const_cast<void*>(v.a), dims, strides, box, el,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        if (v.inner % ib != 0) return false;
        cuuint64_t dims[4] = {(cuuint64_t)ib, (cuuint64_t)(v.inner / ib), (cuuint64_t)v.outer, (cuuint64_t)v.nq};
        cuuint64_t strides[3] = {(cuuint64_t)ib * es, (cuuint64_t)(v.inner * v.nq) * es, (cuuint64_t)v.inner * es};
        cuuint32_t box[4] = {(cuuint32_t)ib, (cuuint32_t)h, (cuuint32_t)kb, lb};
        cuuint32_t el[4] = {1, 1, 1, 1};
        r = cuTensorMapEncodeTiled(map, ty, 4, const_cast<void*>(v.a), dims, strides, box, el,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

// cudaFuncSetAttribute once per kernel instance and device (devices 0..63): the full dynamic
// shared memory and, when asked, the largest shared-memory carveout (so that two CTAs of
// ~113 KB fit on one SM).
template <typename K>
cudaError_t allow_smem_once(K kernel, int dev, std::atomic<uint64_t>& done, bool max_carveout = false)
{
    const uint64_t bit = dev < 64 ? (uint64_t(1) << dev) : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e == cudaSuccess && max_carveout)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

template <typename T, int MB, bool ROWS, int CPS, bool GROUP>
cudaError_t launch_stream_mb(const StreamProb& one, const StreamLaunch& L, size_t smem, int grid, int dev,
                             cudaStream_t s)
{
    static std::atomic<uint64_t> done{0};
    // the whole unified L1 as shared memory, so that CPS rings fit side by side
    cudaError_t e = allow_smem_once(stream_cols_kernel<T, MB, ROWS, CPS, GROUP>, dev, done, true);
    if (e != cudaSuccess) return e;
    stream_cols_kernel<T, MB, ROWS, CPS, GROUP><<<grid, kStreamThreads, smem, s>>>(one, L);
    return cudaGetLastError();
}

// The build for `cps` CTAs per SM: two for m <= 8, one for any m.
template <typename T, int MB, bool ROWS, bool GROUP>
cudaError_t launch_stream_cps(const StreamProb& one, const StreamLaunch& L, size_t smem, int grid, int dev, int cps,
                              cudaStream_t s)
{
    if constexpr (MB <= 8) {
        if (cps == 2) return launch_stream_mb<T, MB, ROWS, 2, GROUP>(one, L, smem, grid, dev, s);
    }
    return launch_stream_mb<T, MB, ROWS, 1, GROUP>(one, L, smem, grid, dev, s);
}

// `mb`: the MB build (1, 2, 4, 8 or 16) covering every m of the launch.
template <typename T, bool ROWS, bool GROUP>
cudaError_t launch_stream_t(const StreamProb& one, const StreamLaunch& L, int mb, size_t smem, int grid, int dev,
                            int cps, cudaStream_t s)
{
    if (mb <= 1) return launch_stream_cps<T, 1, ROWS, GROUP>(one, L, smem, grid, dev, cps, s);
    if (mb <= 2) return launch_stream_cps<T, 2, ROWS, GROUP>(one, L, smem, grid, dev, cps, s);
    if (mb <= 4) return launch_stream_cps<T, 4, ROWS, GROUP>(one, L, smem, grid, dev, cps, s);
    if (mb <= 8) return launch_stream_cps<T, 8, ROWS, GROUP>(one, L, smem, grid, dev, cps, s);
    return launch_stream_cps<T, 16, ROWS, GROUP>(one, L, smem, grid, dev, cps, s);
}

template <bool GROUP>
cudaError_t launch_stream_any(const StreamProb& one, const StreamLaunch& L, int dtype, bool rows, int mb, size_t smem,
                              int grid, int dev, int cps, cudaStream_t s)
{
    return rows ? (dtype == 0 ? launch_stream_t<float, true, GROUP>(one, L, mb, smem, grid, dev, cps, s)
                              : launch_stream_t<double, true, GROUP>(one, L, mb, smem, grid, dev, cps, s))
                : (dtype == 0 ? launch_stream_t<float, false, GROUP>(one, L, mb, smem, grid, dev, cps, s)
                              : launch_stream_t<double, false, GROUP>(one, L, mb, smem, grid, dev, cps, s));
}

// Row mode: A as the 2-D tensor map (l, row) of its contiguous fibres, boxes of LB l (64 bytes) x
// 256 rows with the 64-byte swizzle.
bool encode_rows_map(const View3& v, int dtype, CUtensorMap* map)
{
    EncodeTiledFn cuTensorMapEncodeTiled = encode_fn();
    if (!cuTensorMapEncodeTiled) return false;
    const size_t es = dtype == 0 ? 4 : 8;
    cuuint64_t dims[2] = {(cuuint64_t)v.nq, (cuuint64_t)v.outer};
    cuuint64_t strides[1] = {(cuuint64_t)v.nq * es};
    cuuint32_t box[2] = {(cuuint32_t)(dtype == 0 ? StreamGeom<float, true>::LB : StreamGeom<double, true>::LB), 256};
    cuuint32_t el[2] = {1, 1};
    CUresult r = cuTensorMapEncodeTiled(map, dtype == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                                        2, const_cast<void*>(v.a), dims, strides, box, el,
                                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Launch geometry of the TMA-fed small-m kernel (one or two CTAs per SM): box shape, ring depth, the
// l split and the dynamic shared memory (ring + staged rows of B + barriers).
struct StreamShape {
    bool rows;
    uint32_t sb;     // bytes per ring stage
    int ib, ib_shift, h_shift, kb, lb, kchunks, kper, S, stages, mb, per_sm;
    int64_t tiles, mper, units;
    size_t smem, ws_bytes;
};

bool stream_tiles(const View3& v, size_t es, int W, int NP, StreamShape& sh);
bool stream_split(const View3& v, size_t es, int NP, int LB, int sms, StreamShape& sh);

bool stream_shape(const View3& v, int dtype, int sms, StreamShape& sh)
{
    const size_t es = dtype == 0 ? 4 : 8;
    sh.rows = v.inner == 1;
    // the kernel's geometry (StreamGeom) for this dtype and mode
    const int W = es == 4 ? (sh.rows ? StreamGeom<float, true>::W : StreamGeom<float, false>::W)
                          : (sh.rows ? StreamGeom<double, true>::W : StreamGeom<double, false>::W);
    const uint32_t SB = sh.rows ? StreamGeom<float, true>::SB : StreamGeom<float, false>::SB;
    sh.sb = SB;
    const int NP = 256 * W, LB = (int)(SB / (NP * es));
    sh.mb = v.m <= 1 ? 1 : v.m <= 2 ? 2 : v.m <= 4 ? 4 : v.m <= 8 ? 8 : 16;
    if (sh.rows) {
        // one tile = 512 consecutive fibres; boxes always hold LB l (fibres of >= LB elements)
        if (v.nq < LB) return false;
        sh.ib_shift = sh.h_shift = 0;
        sh.ib = 1;
        sh.kb = 512;
        sh.mper = 1;
        sh.tiles = (v.outer + 511) / 512;
    } else if (!stream_tiles(v, es, W, NP, sh)) {
        return false;
    }
    return stream_split(v, es, NP, LB, sms, sh);
}

// Column mode: the box shape and tile count.
bool stream_tiles(const View3& v, size_t es, int W, int NP, StreamShape& sh)
{
    // Box shape: among the shapes whose boxes are at most 20% out-of-range fill (positions past
    // inner or outer), the one with the fewest positions, where rows under 32 bytes count
    // double (they use half of each DRAM sector they touch). Candidates: (IB, H = 1) with IB a
    // power of two in [W, 256] (so KB = NP / IB <= 256), and the folded (IB, H > 1) with IB the
    // largest power of two (<= 256, rows >= 128 bytes) dividing inner. None: not supported.
    const int64_t valid = v.inner * v.outer;
    int64_t best_cost = -1;
    auto consider = [&](int ibs, int hs, int64_t tiles, bool narrow) {
        const int64_t pos = tiles * NP;
        if (pos * 4 > valid * 5) return;
        const int64_t cost = narrow ? 2 * pos : pos;
        if (best_cost < 0 || cost < best_cost || (cost == best_cost && hs == 0 && ibs > sh.ib_shift)) {
            best_cost = cost;
            sh.ib_shift = ibs;
            sh.h_shift = hs;
        }
    };
    for (int ibs = 0; (1 << ibs) <= 256; ++ibs) {
        const int64_t ib = int64_t(1) << ibs;
        if (ib < W) continue;
        const int64_t kb = NP / ib;
        consider(ibs, 0, ((v.inner + ib - 1) / ib) * ((v.outer + kb - 1) / kb), ib * (int64_t)es < 32 && ib < v.inner);
    }
    int fb = 0;
    while (fb < 8 && v.inner % (int64_t(1) << (fb + 1)) == 0) ++fb;
    if ((int64_t(1) << fb) * (int64_t)es >= 128) {
        const int64_t ib = int64_t(1) << fb, nhi = v.inner / ib;
        for (int hs = 1; (ib << hs) <= NP; ++hs) {
            const int64_t h = int64_t(1) << hs, kb = NP / (ib * h);
            consider(fb, hs, ((nhi + h - 1) / h) * ((v.outer + kb - 1) / kb), false);
        }
    }
    if (best_cost < 0) return false;
    sh.ib = 1 << sh.ib_shift;
    sh.kb = NP / (sh.ib << sh.h_shift);
    sh.mper = sh.h_shift ? ((v.inner >> sh.ib_shift) + (1 << sh.h_shift) - 1) >> sh.h_shift
                         : (v.inner + sh.ib - 1) / sh.ib;
    sh.tiles = ((v.outer + sh.kb - 1) / sh.kb) * sh.mper;
    return true;
}

// Both modes: ring depth, the l split and the shared memory.
bool stream_split(const View3& v, size_t es, int NP, int LB, int sms, StreamShape& sh)
{
    sh.lb = (int)std::min<int64_t>(LB, v.nq);
    sh.kchunks = (int)((v.nq + sh.lb - 1) / sh.lb);
    // CTAs per SM (one or two share its 228 KB of shared memory, 1 KB each reserved) and the ring
    // of each, measured over the layout/mode sweep: row mode, m > 8 and column mode with fewer
    // tiles than SMs run one CTA (168 registers) with a 128 KB ring; other column-mode shapes two
    // (96 registers) with 48 KB rings. More bytes in flight per SM than that slowed the
    // write-heavy short-n_q cases; three CTAs of 72 registers lost to both.
    sh.per_sm = (sh.rows || sh.mb > 8 || sh.tiles < (int64_t)sms) ? 1 : 2;
    if (sh.per_sm == 2) {
        // one CTA per SM where its last round is much fuller (whole tiles over the slots)
        auto eff = [&](int64_t slots) { return (double)sh.tiles / (double)(slots * ((sh.tiles + slots - 1) / slots)); };
        if (eff(sms) >= eff(2 * (int64_t)sms) + 0.08) sh.per_sm = 1;
    }
    const size_t budget = (sh.per_sm == 2 ? 112 : 227) * 1024 - 1024 - 256;
    const size_t row = (size_t)sh.lb * sh.mb * es;   // staged B bytes per l chunk
    // ring per CTA from hi down to lo while B fits beside it, otherwise fb with B staged a part
    // at a time; at least two stages
    const size_t hi = sh.per_sm == 2 ? 48 * 1024 : 128 * 1024, lo = sh.per_sm == 2 ? 32 * 1024 : 96 * 1024,
                 fb = sh.per_sm == 2 ? 48 * 1024 : 128 * 1024;
    int kper_max = 0;
    sh.stages = 0;
    for (int st = std::max<int>(2, (int)(hi / sh.sb)); st >= std::max<int>(2, (int)(lo / sh.sb)); --st)
        if ((size_t)st * sh.sb + (size_t)sh.kchunks * row <= budget) {
            sh.stages = st;
            kper_max = sh.kchunks;
            break;
        }
    if (!sh.stages) {
        sh.stages = std::max<int>(2, (int)(fb / sh.sb));
        kper_max = (int)((budget - (size_t)sh.stages * sh.sb) / row);
    }
    // l split: the S (at least enough for B to fit) with the shortest estimated makespan, in
    // boxes: rounds of units over the CTA slots x (boxes per unit + 1 for the pipeline ramp
    // + 3 + MB / 2 for writing, fencing and re-reading a partial tile when S > 1); a split must
    // win by 10% (measured: splits cost more than this model says)
    const int64_t slots = (int64_t)sh.per_sm * sms;
    const int64_t s_min = (sh.kchunks + kper_max - 1) / kper_max;
    const int64_t s_max = std::max<int64_t>(s_min, std::min<int64_t>(sh.kchunks, 64));
    double best_t = 0;
    sh.kper = sh.kchunks;
    for (int64_t S = s_min; S <= s_max; ++S) {
        const int64_t kper = (sh.kchunks + S - 1) / S;
        if (kper > kper_max) continue;
        const int64_t s_eff = (sh.kchunks + kper - 1) / kper;
        const int64_t rounds = (sh.tiles * s_eff + slots - 1) / slots;
        const double t = (double)rounds * ((double)kper + 1.0 + (s_eff > 1 ? 3.0 + sh.mb / 2.0 : 0.0));
        if (S == s_min || t < best_t * 0.9) { best_t = t; sh.kper = (int)kper; }
    }
    sh.S = (sh.kchunks + sh.kper - 1) / sh.kper;
    sh.units = sh.tiles * sh.S;
    sh.smem = 1024 + (size_t)sh.stages * sh.sb + (size_t)sh.kper * row + 256;
    sh.ws_bytes = sh.S > 1 ? (size_t)sh.units * sh.mb * NP * es : 0;
    return true;
}

}  // namespace

// Whether the driver accepts tensor maps whose dimensions are not in stride order (checked once,
// on a dummy address: encoding reads no memory).
bool permuted_maps_ok()
{
    static bool ok = false;
    static std::once_flag once;
    std::call_once(once, [] {
        alignas(16) static const double probe[4] = {0, 0, 0, 0};
        View3 v{};
        v.a = probe;
        v.inner = 4;
        v.outer = 3;
        v.nq = 5;
        CUtensorMap map;
        ok = encode_stream_map(v, 0, 4, 1, 256, &map) && encode_stream_map(v, 1, 4, 1, 128, &map);
        v.inner = 256;
        ok = ok && encode_stream_map(v, 0, 32, 4, 8, &map) && encode_stream_map(v, 1, 16, 4, 8, &map);
    });
    return ok;
}

// The per-problem parameters of the stream kernel for view v with shape sh (no workspace).
void fill_stream_params(const View3& v, const StreamShape& sh, StreamParams& P)
{
    P = StreamParams{};
    P.b = v.b;
    P.c = v.c;
    P.outer = v.outer;
    P.nq = v.nq;
    P.inner = v.inner;
    P.m = v.m;
    P.tiles = sh.tiles;
    P.mper = sh.mper;
    P.units = sh.units;
    P.kchunks = sh.kchunks;
    P.lb = sh.lb;
    P.kper = sh.kper;
    P.S = sh.S;
    P.b_cm = v.b_cm;
    P.ib_shift = sh.ib_shift;
    P.h_shift = sh.h_shift;
    P.kb = sh.kb;
    // unit and tile indices fit in 32 bits: a tile holds 256 or more positions
    P.fd_s = make_fastdiv((uint32_t)sh.S);
    P.fd_mper = make_fastdiv((uint32_t)sh.mper);
}

bool stream_supported(const View3& v, int dtype)
{
    const int64_t w = dtype == 0 ? 4 : 2;
    if (v.m > kSmallM) return false;
    if (v.inner == 1) {
        // row mode: fibres start on 16-byte boundaries (the tensor map's row stride)
        if (v.nq % w != 0 || (reinterpret_cast<uintptr_t>(v.a) & 15u) != 0) return false;
    } else {
        if (!permuted_maps_ok()) return false;
        // 16-byte rows and 16-byte vectors of W consecutive positions in A and C
        if (v.inner < w || v.inner % w != 0) return false;
        if (((reinterpret_cast<uintptr_t>(v.a) | reinterpret_cast<uintptr_t>(v.c)) & 15u) != 0) return false;
    }
    if (v.outer >= (int64_t(1) << 31) || v.nq >= (int64_t(1) << 31) || v.inner >= (int64_t(1) << 31)) return false;
    // shapes whose boxes would be mostly out-of-range fill go elsewhere
    StreamShape sh;
    return stream_shape(v, dtype, 148, sh);
}

cudaError_t launch_stream(const View3& v, int dtype, cudaStream_t s)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!g_sm_count) {
        e = cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    DevState* st = nullptr;
    if ((e = state_for(dev, st)) != cudaSuccess) return e;
    StreamShape sh;
    if (!stream_shape(v, dtype, g_sm_count, sh)) return cudaErrorNotSupported;
    StreamProb one;
    std::memset(&one, 0, sizeof(one));
    if (sh.rows ? !encode_rows_map(v, dtype, &one.amap)
                : !encode_stream_map(v, dtype, sh.ib, 1 << sh.h_shift, sh.kb, &one.amap))
        return cudaErrorInvalidValue;
    fill_stream_params(v, sh, one.P);
    StreamLaunch L{};
    L.status = st->status;
    L.count = 1;
    L.total = sh.units;
    L.stages = sh.stages;
    L.brows = sh.kper * sh.lb;
    void* scratch = nullptr;
    if (sh.S > 1) {
        const size_t ws = (sh.ws_bytes + 255) & ~size_t(255);
        if ((e = dev_malloc_async(&scratch, ws + (size_t)sh.tiles * sizeof(unsigned), s)) != cudaSuccess) return e;
        one.P.ws = scratch;
        one.P.cnt = reinterpret_cast<unsigned*>(static_cast<uint8_t*>(scratch) + ws);
        e = cudaMemsetAsync(one.P.cnt, 0, (size_t)sh.tiles * sizeof(unsigned), s);
    }
    const int grid = (int)std::min<int64_t>(sh.units, (int64_t)g_sm_count * sh.per_sm);
    if (e == cudaSuccess)
        e = launch_stream_any<false>(one, L, dtype, sh.rows, sh.mb, sh.smem, grid, dev, sh.per_sm, s);
    if (scratch) cudaFreeAsync(scratch, s);
    return e;
}

// ------------------------------------------------------------------ grouped stream launch
struct StreamGroup {
    struct Cls {
        bool rows;
        int mb, cps, grid;
        size_t smem;
        StreamLaunch L;
    };
    StreamProb* d_probs = nullptr;   // the problems of every class, class after class
    int dtype = 0;
    std::vector<Cls> cls;
};

namespace {
const StreamProb g_no_sprob{};      // the unused single-problem parameter of grouped launches

int group_cps(const StreamShape& sh) { return (sh.rows || sh.mb > 8) ? 1 : 2; }
size_t group_budget(int cps) { return (size_t)(cps == 2 ? 112 : 227) * 1024; }
size_t group_smem(const StreamShape& sh, int stages, int brows, size_t es)
{
    return 1024 + (size_t)stages * sh.sb + (size_t)brows * sh.mb * es + 256;
}
}  // namespace

bool stream_group_eligible(const View3& v, int dtype)
{
    if (!stream_supported(v, dtype)) return false;
    StreamShape sh;
    if (!stream_shape(v, dtype, 148, sh)) return false;
    // B staged whole (no l split) beside a ring of at least two stages
    return group_smem(sh, 2, sh.kchunks * sh.lb, dtype == 0 ? 4 : 8) <= group_budget(group_cps(sh));
}

cudaError_t stream_group_create(const View3* views, int count, int dtype, StreamGroup** out)
{
    *out = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    DevState* st = nullptr;
    if ((e = state_for(dev, st)) != cudaSuccess) return e;
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    std::unique_ptr<StreamGroup, void (*)(StreamGroup*)> G(new StreamGroup(), stream_group_destroy);
    G->dtype = dtype;
    const size_t es = dtype == 0 ? 4 : 8;
    // classes by (row mode, MB build, CTAs per SM): one launch each
    struct Entry { int key; StreamShape sh; int i; };
    std::vector<Entry> ents;
    for (int i = 0; i < count; ++i) {
        StreamShape sh;
        if (!stream_shape(views[i], dtype, sms, sh)) return cudaErrorNotSupported;
        sh.kper = sh.kchunks;   // B staged whole: one unit per tile
        sh.S = 1;
        sh.units = sh.tiles;
        const int cps = group_cps(sh);
        if (group_smem(sh, 2, sh.kchunks * sh.lb, es) > group_budget(cps)) return cudaErrorNotSupported;
        ents.push_back(Entry{(sh.rows ? 100 : 0) + sh.mb * 4 + cps, sh, i});
    }
    std::stable_sort(ents.begin(), ents.end(), [](const Entry& x, const Entry& y) {
        if (x.key != y.key) return x.key < y.key;
        return x.sh.units > y.sh.units;
    });
    std::vector<StreamProb> recs(ents.size());
    for (size_t r = 0; r < ents.size();) {
        size_t r1 = r;
        int brows = 0;
        int64_t first = 0;
        while (r1 < ents.size() && ents[r1].key == ents[r].key) {
            const Entry& en = ents[r1];
            StreamProb& pr = recs[r1];
            std::memset(&pr, 0, sizeof(pr));
            const View3& v = views[en.i];
            if (en.sh.rows ? !encode_rows_map(v, dtype, &pr.amap)
                           : !encode_stream_map(v, dtype, en.sh.ib, 1 << en.sh.h_shift, en.sh.kb, &pr.amap))
                return cudaErrorInvalidValue;
            fill_stream_params(v, en.sh, pr.P);
            pr.first = first;
            first += en.sh.units;
            brows = std::max(brows, en.sh.kchunks * en.sh.lb);
            ++r1;
        }
        const StreamShape& sh = ents[r].sh;
        StreamGroup::Cls c{};
        c.rows = sh.rows;
        c.mb = sh.mb;
        c.cps = group_cps(sh);
        // the ring of the single launches (128 KB, or 48 KB at two CTAs per SM), less while B
        // does not fit beside it
        int stages = std::min<int>(kStreamMaxStages, (int)((c.cps == 2 ? 48 : 128) * 1024 / sh.sb));
        while (stages > 2 && group_smem(sh, stages, brows, es) > group_budget(c.cps)) --stages;
        c.smem = group_smem(sh, stages, brows, es);
        c.L.status = st->status;
        c.L.count = (int)(r1 - r);
        c.L.total = first;
        c.L.stages = stages;
        c.L.brows = brows;
        c.L.group = reinterpret_cast<const StreamProb*>(r);   // index for now; a pointer after the upload
        c.grid = (int)std::min<int64_t>(first, (int64_t)sms * c.cps);
        G->cls.push_back(c);
        r = r1;
    }
    if (!recs.empty()) {
        if ((e = dev_malloc(reinterpret_cast<void**>(&G->d_probs), sizeof(StreamProb) * recs.size())) != cudaSuccess)
            return e;
        if ((e = cudaMemcpy(G->d_probs, recs.data(), sizeof(StreamProb) * recs.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return e;
    }
    for (StreamGroup::Cls& c : G->cls) c.L.group = G->d_probs + reinterpret_cast<uintptr_t>(c.L.group);
    *out = G.release();
    return cudaSuccess;
}

cudaError_t stream_group_run(StreamGroup* G, cudaStream_t s)
{
    if (!G) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    for (const StreamGroup::Cls& c : G->cls)
        if ((e = launch_stream_any<true>(g_no_sprob, c.L, G->dtype, c.rows, c.mb, c.smem, c.grid, dev, c.cps, s)) !=
            cudaSuccess)
            return e;
    return cudaSuccess;
}

int stream_group_launches(const StreamGroup* G) { return G ? (int)G->cls.size() : 0; }

void stream_group_destroy(StreamGroup* G)
{
    if (!G) return;
    if (G->d_probs) cudaFree(G->d_probs);
    delete G;
}

cudaError_t tc_status_word(int dev, int** out)
{
    DevState* st = nullptr;
    cudaError_t e = state_for(dev, st);
    if (e == cudaSuccess) *out = st->status;
    return e;
}

bool tc_supported(const View3& v, int precision)
{
    if (precision != TLIBTTM_PREC_BF16X3) return false;
    if (v.m <= kSmallM) return false;
    const int g = geometry_of(v);
    if ((reinterpret_cast<uintptr_t>(v.a) & 3u) != 0) return false;   // float-aligned A
    if (g == GEOM_MN && v.inner < 17) return false;   // a folded tile gives each slice >= 32 rows
    // TMA coordinates are signed 32-bit.
    if (v.outer >= (int64_t(1) << 31) || v.nq >= (int64_t(1) << 31) || v.inner >= (int64_t(1) << 31)) return false;
    return true;
}

cudaError_t launch_tc(const View3& v, int precision, cudaStream_t s, int* kid)
{
    *kid = K_TC_BF16X3;
    if (precision != TLIBTTM_PREC_BF16X3) return cudaErrorNotSupported;
    if (tc_pair_supported(v)) {
        *kid = K_TC_PAIR;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        DevState* st = nullptr;
        if ((e = state_for(dev, st)) != cudaSuccess) return e;
        return launch_tc_pair(v, st->status, s);
    }
    return launch_tc_single(v, s, kid);
}

int64_t tc_single_tiles(const View3& v)
{
    const int64_t nt = std::min<int64_t>(kMaxNT, ((v.m + 15) / 16) * 16);
    const int64_t jblocks = (v.m + nt - 1) / nt;
    int64_t tiles_m;
    if (geometry_of(v) == GEOM_K) tiles_m = (v.outer + kBM - 1) / kBM;
    else if (v.inner <= 64) tiles_m = (v.outer + (kBM >> (v.inner <= 32 ? 5 : 6)) - 1) / (kBM >> (v.inner <= 32 ? 5 : 6));
    else tiles_m = v.outer * ((v.inner + kBM - 1) / kBM);
    return tiles_m * jblocks;
}

cudaError_t launch_tc_single(const View3& v, cudaStream_t s, int* kid)
{
    *kid = K_TC_BF16X3;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!g_sm_count) {
        e = cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    DevState* st = nullptr;
    if ((e = state_for(dev, st)) != cudaSuccess) return e;
    void* img = nullptr;
    if ((e = dev_malloc_async(&img, tc_image_bytes(v), s)) != cudaSuccess) return e;
    e = run_bf16x3(v, static_cast<uint8_t*>(img), st->status, g_sm_count, s);
    cudaFreeAsync(img, s);
    return e;
}

// ------------------------------------------------------------------ allocation-free variant
// The bf16x3 path above takes its pre-split B image from the stream-ordered pool
// (cudaMallocAsync). Some callers cannot let a library allocate device memory: a
// host application whose own allocator has reserved the device's memory, a
// latency-bound loop that must not risk the implicit device synchronisation of
// cudaMalloc/cudaFree, or a process running under a fixed device-memory budget.
// For them, launch_tc_noalloc runs the same kernels with the B image in this
// file-scope array. Every GPU that loads the library holds the array until exit.
// All calls share it and it keeps the previous call's contents: split_b_kernel
// rewrites every byte a launch reads (zero padding included), and the status
// word is cleared before each launch. Calls whose work overlaps on the GPU (two
// streams, or two host threads) race on the array and must be serialised.
static __device__ __align__(256) uint8_t g_noalloc_image[kNoAllocImageBytes];
static __device__ __align__(256) int g_noalloc_status[64];

struct NoAllocSymbols {
    uint8_t* image = nullptr;
    int* status = nullptr;
};
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocSymbols g_noalloc_syms[kMaxDevices];

// Device addresses of the two arrays on device `dev` (the current device), looked
// up once per device. In host code the array names are host-side stand-ins, not
// device addresses, so kernels only ever receive the looked-up pointers.
cudaError_t noalloc_symbols(int dev, NoAllocSymbols& out)
{
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocSymbols& sy = g_noalloc_syms[dev];
    if (!sy.image) {
        void* img = nullptr;
        void* st = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&img, g_noalloc_image);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress(&st, g_noalloc_status);
        if (e != cudaSuccess) return e;
        sy.image = static_cast<uint8_t*>(img);
        sy.status = static_cast<int*>(st);
    }
    out = sy;
    return cudaSuccess;
}

size_t tc_image_bytes(const View3& v)
{
    const int nt = (int)std::min<int64_t>(kMaxNT, ((v.m + 15) / 16) * 16);
    const int64_t jblocks = (v.m + nt - 1) / nt;
    const int64_t kpad = (v.nq + kSub * kBK - 1) / (kSub * kBK) * kSub;   // sub-blocks, a whole number of stages
    return (size_t)(jblocks * kpad * 2) * smem_layout(nt).b_bytes;
}

cudaError_t launch_tc_noalloc(const View3& v, cudaStream_t s, int* kid)
{
    *kid = K_TC_BF16X3;
    if (!tc_pair_supported(v) && tc_image_bytes(v) > kNoAllocImageBytes) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    NoAllocSymbols sy;
    if ((e = noalloc_symbols(dev, sy)) != cudaSuccess) return e;
    if (tc_pair_supported(v)) {
        // the pair kernel keeps B in tensor memory: no image, only the status word
        *kid = K_TC_PAIR;
        if ((e = cudaMemsetAsync(sy.status, 0, sizeof(int), s)) != cudaSuccess) return e;
        return launch_tc_pair(v, sy.status, s);
    }
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(sy.status, 0, sizeof(int), s)) != cudaSuccess) return e;
    return run_bf16x3(v, sy.image, sy.status, sms, s);
}

cudaError_t tc_prepare_device()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    DevState* st = nullptr;
    return state_for(dev, st);
}

int tc_read_status()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lk(g_state_mu);
    auto it = g_state.find(dev);
    if (it == g_state.end() || !it->second.status) return 0;
    int st = 0;
    if (cudaMemcpy(&st, it->second.status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    if (st) cudaMemset(it->second.status, 0, sizeof(int));
    return st;
}

int tc_read_noalloc_status()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    int* p = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        p = g_noalloc_syms[dev].status;
    }
    if (!p) return 0;
    int st = 0;
    if (cudaMemcpy(&st, p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    if (st) cudaMemset(p, 0, sizeof(int));
    return st;
}

void tc_release_buffers()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lk(g_state_mu);
    auto it = g_state.find(dev);
    if (it == g_state.end()) return;
    cudaDeviceSynchronize();
    if (it->second.status) cudaFree(it->second.status);
    g_state.erase(it);
}

}  // namespace tlibttm
