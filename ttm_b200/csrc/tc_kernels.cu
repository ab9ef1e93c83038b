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
// instruction, 32 l per pipeline stage.
//
// Warp roles (320 threads, one CTA per SM, persistent over tiles):
//   warp 0     TMA producer: FP32 A tile (tensor map) + the pre-split B_hi/B_lo
//              image of this K chunk (bulk copy) into stage s.
//   warp 1     TMEM allocator and MMA issuer (one elected lane).
//   warps 2-5  converters: FP32 tile -> bf16 hi/lo in the swizzled UMMA layout.
//   warps 6-9  epilogue: TMEM -> registers -> global C (double-buffered accumulator).
// Every mbarrier wait is bounded (4 s of %globaltimer); on expiry the CTA raises
// an abort flag, records an error in the device status word, drains its own
// bulk copies, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdio>
#include <mutex>
#include <unordered_map>

#include "tc_kernels.cuh"
#include "tlibttm.h"

namespace tlibttm {
namespace {

constexpr int kThreads = 320;
constexpr int kBM = 128;       // MMA M
constexpr int kBK = 32;        // l per stage
constexpr int kMaxNT = 256;    // MMA N max
constexpr int kMaxStages = 6;
constexpr unsigned long long kTimeoutNs = 4000000000ull;

enum { GEOM_MN = 0, GEOM_K = 1 };

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait: false when the CTA is aborting or this wait expired (which starts the abort).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, volatile int* abort_flag)
{
    if (mbar_try(bar, phase)) return true;
    const unsigned long long t0 = gtimer();
    while (true) {
        if (mbar_try(bar, phase)) return true;
        if (*abort_flag) return false;
        if (gtimer() - t0 > kTimeoutNs) {
            *abort_flag = 1;
            return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(su32(dst)), "l"(map), "r"(su32(bar)), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(su32(dst)), "l"(map), "r"(su32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(su32(dst)), "l"(src), "r"(bytes), "r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor (tcgen05): start, leading/stride byte offsets, version 1, layout type.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)(layout & 7u) << 61;
    return d;
}
constexpr uint32_t kLayoutSW128 = 2, kLayoutSW64 = 4;

// Instruction descriptor, kind::f16: D f32, A/B bf16, B K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool a_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// x -> (hi, lo) bf16 pair, packed two at a time.
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    const float r0 = x0 - __low2float(h);
    const float r1 = x1 - __high2float(h);
    __nv_bfloat162 l = __floats2bfloat162_rn(r0, r1);
    hi = *reinterpret_cast<uint32_t*>(&h);
    lo = *reinterpret_cast<uint32_t*>(&l);
}

// Byte offset of a 16-byte chunk inside a K-major SW64 bf16 tile with 64-byte rows (32 l per row).
__host__ __device__ __forceinline__ uint32_t kmaj_sw64_off(uint32_t row, uint32_t chunk)
{
    return (row >> 3) * 512u + (row & 7u) * 64u + ((chunk ^ ((row >> 1) & 3u)) << 4);
}

// Byte offset of a 16-byte chunk (8 consecutive MN elements) in an MN-major SW128 bf16 tile of
// 128 MN x 32 K laid out as [K group of 8][MN block of 64][8 K rows][64 MN].
__device__ __forceinline__ uint32_t mnmaj_sw128_off(uint32_t l, uint32_t ichunk)
{
    const uint32_t atom = (l >> 3) * 2u + (ichunk >> 3);
    const uint32_t row = l & 7u, c = ichunk & 7u;
    return atom * 1024u + row * 128u + ((c ^ row) << 4);
}

struct TcParams {
    float* c;
    const uint8_t* bimg;     // pre-split B: [jb][kc][hi|lo][NT rows x 64 B]
    int* status;             // device status word (0 = ok)
    int64_t outer, nq, inner, m;
    int64_t tiles_m;         // M tiles per j block
    int64_t tiles;           // total tiles
    int nt;                  // MMA N (multiple of 16, <= 256)
    int jblocks;
    int kchunks;
    int stages;
    int vec_c;               // GEOM_K epilogue may use 16-byte stores
};

struct SmemLayout {
    uint32_t f32_bytes, abf_bytes, b_bytes, stage_bytes;
};

__host__ __device__ inline SmemLayout smem_layout(int nt)
{
    SmemLayout L;
    L.f32_bytes = kBM * kBK * 4;            // 16 KB
    L.abf_bytes = kBM * kBK * 2;            // 8 KB per part
    L.b_bytes = (uint32_t)nt * kBK * 2;     // per part
    L.stage_bytes = L.f32_bytes + 2 * L.abf_bytes + 2 * L.b_bytes;
    return L;
}

template <int GEOM>
__global__ void __launch_bounds__(kThreads, 1) tc_bf16x3_kernel(const __grid_constant__ CUtensorMap amap, TcParams P)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned base (swizzle atoms are address-based).
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const SmemLayout L = smem_layout(P.nt);
    const int S = P.stages;
    uint8_t* ctrl = smem + (size_t)S * L.stage_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(ctrl);           // [S]
    uint64_t* conv = full + S;                                      // [S]
    uint64_t* empty = conv + S;                                     // [S]
    uint64_t* acc_full = empty + S;                                 // [2]
    uint64_t* acc_empty = acc_full + 2;                             // [2]
    uint64_t* drain = acc_empty + 2;                                // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto stage_f32 = [&](int s) { return smem + (size_t)s * L.stage_bytes; };
    auto stage_ahi = [&](int s) { return stage_f32(s) + L.f32_bytes; };
    auto stage_alo = [&](int s) { return stage_ahi(s) + L.abf_bytes; };
    auto stage_bhi = [&](int s) { return stage_alo(s) + L.abf_bytes; };
    auto stage_blo = [&](int s) { return stage_bhi(s) + L.b_bytes; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&conv[s], 4);
            mbar_init(&empty[s], 1);
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

    const int64_t tiles = P.tiles;
    const int kchunks = P.kchunks;
    const uint32_t tx_bytes = L.f32_bytes + 2 * L.b_bytes;

    if (warp == 0) {
        // ------------------------------------------------------------- TMA producer
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            int issued[kMaxStages];
            for (int i = 0; i < kMaxStages; ++i) issued[i] = -1;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                const int64_t jb = t / P.tiles_m, mt = t - jb * P.tiles_m;
                for (int kc = 0; kc < kchunks; ++kc) {
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                    issued[s] = (int)ph;
                    mbar_expect_tx(&full[s], tx_bytes);
                    if (GEOM == GEOM_MN) {
                        const int64_t mper = (P.inner + kBM - 1) / kBM;
                        const int64_t k = mt / mper, ib = mt - k * mper;
                        tma_load_3d(stage_f32(s), &amap, &full[s], (int)(ib * kBM), kc * kBK, (int)k);
                    } else {
                        tma_load_2d(stage_f32(s), &amap, &full[s], kc * kBK, (int)(mt * kBM));
                    }
                    const uint8_t* img = P.bimg + ((size_t)(jb * kchunks + kc) * 2) * L.b_bytes;
                    bulk_load(stage_bhi(s), img, L.b_bytes, &full[s]);
                    bulk_load(stage_blo(s), img + L.b_bytes, L.b_bytes, &full[s]);
                    if (++s == S) { s = 0; ph ^= 1; }
                }
            }
            // Drain: none of this CTA's bulk copies may still be in flight when it exits.
            for (int i = 0; i < S; ++i) {
                if (issued[i] < 0) continue;
                const unsigned long long t0 = gtimer();
                while (!mbar_try(&full[i], (uint32_t)issued[i]) && gtimer() - t0 < kTimeoutNs) {}
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(P.nt, GEOM == GEOM_MN);
            int s = 0;
            uint32_t ph = 0;
            int ab = 0;
            uint32_t aph = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                if (!mbar_wait(&acc_empty[ab], aph ^ 1, abort_flag)) break;
                tc_fence_after();
                const uint32_t dcol = tmem_base + (uint32_t)(ab * P.nt);
                for (int kc = 0; kc < kchunks; ++kc) {
                    if (!mbar_wait(&conv[s], ph, abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t ahi = su32(stage_ahi(s)), alo = su32(stage_alo(s));
                    const uint32_t bhi = su32(stage_bhi(s)), blo = su32(stage_blo(s));
#pragma unroll
                    for (int kk = 0; kk < kBK / 16; ++kk) {
                        uint64_t dahi, dalo;
                        if (GEOM == GEOM_MN) {
                            dahi = smem_desc(ahi + kk * 4096u, 1024u, 2048u, kLayoutSW128);
                            dalo = smem_desc(alo + kk * 4096u, 1024u, 2048u, kLayoutSW128);
                        } else {
                            dahi = smem_desc(ahi + kk * 32u, 16u, 512u, kLayoutSW64);
                            dalo = smem_desc(alo + kk * 32u, 16u, 512u, kLayoutSW64);
                        }
                        const uint64_t dbhi = smem_desc(bhi + kk * 32u, 16u, 512u, kLayoutSW64);
                        const uint64_t dblo = smem_desc(blo + kk * 32u, 16u, 512u, kLayoutSW64);
                        const uint32_t first = (kc == 0 && kk == 0) ? 0u : 1u;
                        mma_bf16(dcol, dahi, dbhi, idesc, first);
                        mma_bf16(dcol, dahi, dblo, idesc, 1u);
                        mma_bf16(dcol, dalo, dbhi, idesc, 1u);
                    }
                    mma_commit(&empty[s]);     // stage free once these MMAs have read it
                    if (++s == S) { s = 0; ph ^= 1; }
                }
                if (!ok) break;
                mma_commit(&acc_full[ab]);     // accumulator ready for the epilogue
                if (++ab == 2) { ab = 0; aph ^= 1; }
            }
            // No MMA of this CTA may still be writing TMEM when it is freed.
            mma_commit(drain);
            const unsigned long long t0 = gtimer();
            while (!mbar_try(drain, 0) && gtimer() - t0 < kTimeoutNs) {}
        }
    } else if (warp < 6) {
        // ------------------------------------------------------------- converters
        const int ct = threadIdx.x - 64;   // 0..127
        int s = 0;
        uint32_t ph = 0;
        bool ok = true;
        for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
            for (int kc = 0; kc < kchunks; ++kc) {
                if (!mbar_wait(&full[s], ph, abort_flag)) { ok = false; break; }
                const float* f = reinterpret_cast<const float*>(stage_f32(s));
                uint8_t* ahi = stage_ahi(s);
                uint8_t* alo = stage_alo(s);
#pragma unroll
                for (int it = 0; it < 4; ++it) {
                    const int u = ct + 128 * it;
                    float4 x0, x1;
                    uint32_t off;
                    if (GEOM == GEOM_MN) {
                        const int l = u >> 4, ic = u & 15;           // fp32 tile [32 l][128 i], rows of 512 B
                        const float4* src = reinterpret_cast<const float4*>(f + l * kBM + ic * 8);
                        x0 = src[0];
                        x1 = src[1];
                        off = mnmaj_sw128_off(l, ic);
                    } else {
                        const int k = u >> 2, c = u & 3;             // fp32 tile [128 k][32 l], TMA SW128
                        const uint32_t base = (uint32_t)k * 128u;
                        const uint32_t c0 = (uint32_t)(2 * c), c1 = (uint32_t)(2 * c + 1);
                        x0 = *reinterpret_cast<const float4*>(reinterpret_cast<const uint8_t*>(f) + base + ((c0 ^ (k & 7)) << 4));
                        x1 = *reinterpret_cast<const float4*>(reinterpret_cast<const uint8_t*>(f) + base + ((c1 ^ (k & 7)) << 4));
                        off = kmaj_sw64_off((uint32_t)k, (uint32_t)c);
                    }
                    uint4 h, lo;
                    split2(x0.x, x0.y, h.x, lo.x);
                    split2(x0.z, x0.w, h.y, lo.y);
                    split2(x1.x, x1.y, h.z, lo.z);
                    split2(x1.z, x1.w, h.w, lo.w);
                    *reinterpret_cast<uint4*>(ahi + off) = h;
                    *reinterpret_cast<uint4*>(alo + off) = lo;
                }
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) mbar_arrive(&conv[s]);
                if (++s == S) { s = 0; ph ^= 1; }
            }
        }
    } else {
        // ------------------------------------------------------------- epilogue
        const int q4 = warp & 3;                 // TMEM lane quarter this warp may access
        const int row = q4 * 32 + lane;          // accumulator row = MMA M index
        int ab = 0;
        uint32_t aph = 0;
        for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
            if (!mbar_wait(&acc_full[ab], aph, abort_flag)) break;
            tc_fence_after();
            const int64_t jb = t / P.tiles_m, mt = t - jb * P.tiles_m;
            int64_t cbase;
            bool rvalid;
            if (GEOM == GEOM_MN) {
                const int64_t mper = (P.inner + kBM - 1) / kBM;
                const int64_t k = mt / mper, i = (mt - k * mper) * kBM + row;
                rvalid = i < P.inner;
                cbase = k * P.m * P.inner + i;
            } else {
                const int64_t k = mt * kBM + row;
                rvalid = k < P.outer;
                cbase = k * P.m;
            }
            const uint32_t tbase = tmem_base + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(ab * P.nt);
            for (int cc = 0; cc < P.nt; cc += 32) {
                uint32_t v[32];
                tmem_ld32(tbase + (uint32_t)cc, v);
                const int64_t j0 = (int64_t)jb * P.nt + cc;
                if (rvalid) {
                    if (GEOM == GEOM_MN) {
#pragma unroll
                        for (int c = 0; c < 32; ++c) {
                            const int64_t j = j0 + c;
                            if (j < P.m) P.c[cbase + j * P.inner] = __uint_as_float(v[c]);
                        }
                    } else if (P.vec_c && j0 + 32 <= P.m) {
                        float4* dst = reinterpret_cast<float4*>(P.c + cbase + j0);
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            dst[c] = make_float4(__uint_as_float(v[4 * c]), __uint_as_float(v[4 * c + 1]),
                                                 __uint_as_float(v[4 * c + 2]), __uint_as_float(v[4 * c + 3]));
                    } else {
#pragma unroll
                        for (int c = 0; c < 32; ++c) {
                            const int64_t j = j0 + c;
                            if (j < P.m) P.c[cbase + j] = __uint_as_float(v[c]);
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[ab]);
            if (++ab == 2) { ab = 0; aph ^= 1; }
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

// B (m x nq, column- or row-major FP32) -> bf16 hi/lo images, one per (j block, K chunk),
// each NT rows x 32 l in the K-major SW64 layout the MMA reads. Zero outside B.
__global__ void split_b_kernel(const float* __restrict__ b, int b_cm, int64_t m, int64_t nq, int nt, int jblocks,
                               int kchunks, uint8_t* __restrict__ img)
{
    const int64_t total = (int64_t)jblocks * kchunks * nt * 4;     // 4 chunks of 8 l per row
    const uint32_t part_bytes = (uint32_t)nt * 64u;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(u & 3);
        const int64_t rrow = u >> 2;
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
        const uint32_t off = kmaj_sw64_off((uint32_t)jl, (uint32_t)c);
        *reinterpret_cast<uint4*>(base + off) = h;
        *reinterpret_cast<uint4*>(base + part_bytes + off) = lo;
    }
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
        cudaError_t e = cudaMalloc(&d.status, 256);
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
                                   es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

int geometry_of(const View3& v)
{
    if (v.inner == 1) return (v.nq % 4 == 0) ? GEOM_K : -1;
    return (v.inner % 4 == 0) ? GEOM_MN : -1;
}

}  // namespace

bool tc_supported(const View3& v, int precision)
{
    if (precision != TLIBTTM_PREC_BF16X3) return false;
    if (v.m <= kSmallM) return false;
    const int g = geometry_of(v);
    if (g < 0) return false;
    if ((reinterpret_cast<uintptr_t>(v.a) & 15u) != 0) return false;
    if (g == GEOM_MN && v.inner < 32) return false;
    // TMA coordinates are signed 32-bit.
    if (v.outer >= (int64_t(1) << 31) || v.nq >= (int64_t(1) << 31) || v.inner >= (int64_t(1) << 31)) return false;
    return true;
}

cudaError_t launch_tc(const View3& v, int precision, cudaStream_t s, int* kid)
{
    *kid = K_TC_BF16X3;
    if (precision != TLIBTTM_PREC_BF16X3) return cudaErrorNotSupported;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!g_sm_count) {
        e = cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    const int geom = geometry_of(v);
    const int nt = (int)std::min<int64_t>(kMaxNT, ((v.m + 15) / 16) * 16);
    const int jblocks = (int)((v.m + nt - 1) / nt);
    const int kchunks = (int)((v.nq + kBK - 1) / kBK);
    const SmemLayout L = smem_layout(nt);
    const size_t img_bytes = (size_t)jblocks * kchunks * 2 * L.b_bytes;

    DevState* st = nullptr;
    if ((e = state_for(dev, st)) != cudaSuccess) return e;
    void* img = nullptr;
    if ((e = cudaMallocAsync(&img, img_bytes, s)) != cudaSuccess) return e;

    CUtensorMap amap;
    if (!encode_a_map(v, geom, &amap)) {
        cudaFreeAsync(img, s);
        return cudaErrorInvalidValue;
    }

    TcParams P{};
    P.c = static_cast<float*>(v.c);
    P.bimg = static_cast<const uint8_t*>(img);
    P.status = st->status;
    P.outer = v.outer;
    P.nq = v.nq;
    P.inner = v.inner;
    P.m = v.m;
    P.tiles_m = geom == GEOM_MN ? v.outer * ((v.inner + kBM - 1) / kBM) : (v.outer + kBM - 1) / kBM;
    P.tiles = P.tiles_m * jblocks;
    P.nt = nt;
    P.jblocks = jblocks;
    P.kchunks = kchunks;
    P.vec_c = (geom == GEOM_K) && (v.m % 4 == 0) && ((reinterpret_cast<uintptr_t>(v.c) & 15u) == 0);
    const size_t ctrl = 1024;
    const size_t budget = 227 * 1024 - 1024 - ctrl;
    int stages = (int)(budget / L.stage_bytes);
    if (stages > kMaxStages) stages = kMaxStages;
    if (stages < 2) {
        cudaFreeAsync(img, s);
        return cudaErrorNotSupported;
    }
    P.stages = stages;
    const size_t smem = 1024 + (size_t)stages * L.stage_bytes + ctrl;

    // split B once per call
    {
        const int64_t total = (int64_t)jblocks * kchunks * nt * 4;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
        split_b_kernel<<<blocks, 256, 0, s>>>(static_cast<const float*>(v.b), v.b_cm, v.m, v.nq, nt, jblocks,
                                              kchunks, static_cast<uint8_t*>(img));
        if ((e = cudaGetLastError()) != cudaSuccess) {
            cudaFreeAsync(img, s);
            return e;
        }
    }
    const int grid = (int)std::min<int64_t>(P.tiles, g_sm_count);
    if (geom == GEOM_MN) {
        e = cudaFuncSetAttribute(tc_bf16x3_kernel<GEOM_MN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) tc_bf16x3_kernel<GEOM_MN><<<grid, kThreads, smem, s>>>(amap, P);
    } else {
        e = cudaFuncSetAttribute(tc_bf16x3_kernel<GEOM_K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) tc_bf16x3_kernel<GEOM_K><<<grid, kThreads, smem, s>>>(amap, P);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
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
    const int64_t kchunks = (v.nq + kBK - 1) / kBK;
    return (size_t)(jblocks * kchunks * 2) * smem_layout(nt).b_bytes;
}

cudaError_t launch_tc_noalloc(const View3& v, cudaStream_t s, int* kid)
{
    *kid = K_TC_BF16X3;
    if (tc_image_bytes(v) > kNoAllocImageBytes) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    NoAllocSymbols sy;
    if ((e = noalloc_symbols(dev, sy)) != cudaSuccess) return e;
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;

    const int geom = geometry_of(v);
    const int nt = (int)std::min<int64_t>(kMaxNT, ((v.m + 15) / 16) * 16);
    const int jblocks = (int)((v.m + nt - 1) / nt);
    const int kchunks = (int)((v.nq + kBK - 1) / kBK);
    const SmemLayout L = smem_layout(nt);

    CUtensorMap amap;
    if (!encode_a_map(v, geom, &amap)) return cudaErrorInvalidValue;
    if ((e = cudaMemsetAsync(sy.status, 0, sizeof(int), s)) != cudaSuccess) return e;

    TcParams P{};
    P.c = static_cast<float*>(v.c);
    P.bimg = sy.image;
    P.status = sy.status;
    P.outer = v.outer;
    P.nq = v.nq;
    P.inner = v.inner;
    P.m = v.m;
    P.tiles_m = geom == GEOM_MN ? v.outer * ((v.inner + kBM - 1) / kBM) : (v.outer + kBM - 1) / kBM;
    P.tiles = P.tiles_m * jblocks;
    P.nt = nt;
    P.jblocks = jblocks;
    P.kchunks = kchunks;
    P.vec_c = (geom == GEOM_K) && (v.m % 4 == 0) && ((reinterpret_cast<uintptr_t>(v.c) & 15u) == 0);
    const size_t ctrl = 1024;
    int stages = (int)((227 * 1024 - 1024 - ctrl) / L.stage_bytes);
    if (stages > kMaxStages) stages = kMaxStages;
    if (stages < 2) return cudaErrorNotSupported;
    P.stages = stages;
    const size_t smem = 1024 + (size_t)stages * L.stage_bytes + ctrl;

    const int64_t total = (int64_t)jblocks * kchunks * nt * 4;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
    split_b_kernel<<<blocks, 256, 0, s>>>(static_cast<const float*>(v.b), v.b_cm, v.m, v.nq, nt, jblocks, kchunks,
                                          sy.image);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int grid = (int)std::min<int64_t>(P.tiles, sms);
    if (geom == GEOM_MN) {
        e = cudaFuncSetAttribute(tc_bf16x3_kernel<GEOM_MN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) tc_bf16x3_kernel<GEOM_MN><<<grid, kThreads, smem, s>>>(amap, P);
    } else {
        e = cudaFuncSetAttribute(tc_bf16x3_kernel<GEOM_K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) tc_bf16x3_kernel<GEOM_K><<<grid, kThreads, smem, s>>>(amap, P);
    }
    return e == cudaSuccess ? cudaGetLastError() : e;
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
