// SIMT kernels of the B200 TTM library: the exact-arithmetic ("plain") paths.
//
//  simt_gemm  slice-GEMM over the dense view C[k][j][i] = sum_l A[k][l][i] B(j,l),
//             FP32 FFMA or FP64 DFMA, 128x128 (f32) / 64x64 (f64) CTA tiles,
//             register-double-buffered shared-memory stages. Rows of the GEMM
//             are the flattened (k, i) pairs, so one kernel covers every
//             layout case without transposing anything.
//  colvec     bandwidth kernel for small m when A's fibres along mode q are
//             strided (inner >= 2): each thread owns W consecutive i of one k
//             and streams 16-byte loads along l; B is staged in shared memory.
//  rowdot     bandwidth kernel for small m when the fibres are contiguous
//             (inner == 1, q = pi_1): a group of G lanes reads one fibre with
//             16-byte loads and reduces the m partial sums by warp shuffles.
//  strided    definition-level kernel for non-dense (but valid) strides.
//
// All index arithmetic is 64-bit (a 256^4 tensor has 2^32 elements).
#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace tlibttm {
namespace {

template <typename T> struct V16;
template <> struct V16<float> { using type = float4; };
template <> struct V16<double> { using type = double2; };

template <typename T, int W>
__device__ __forceinline__ void load_vec(T (&r)[W], const T* p)
{
    if constexpr (W == 1) {
        r[0] = __ldg(p);
    } else if constexpr (W * sizeof(T) == 16) {
        typename V16<T>::type v = __ldg(reinterpret_cast<const typename V16<T>::type*>(p));
        const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int w = 0; w < W; ++w) r[w] = e[w];
    } else {
#pragma unroll
        for (int w = 0; w < W; ++w) r[w] = __ldg(p + w);
    }
}

template <typename T, int W>
__device__ __forceinline__ void store_vec(T* p, const T (&r)[W])
{
    if constexpr (W * sizeof(T) == 16) {
        typename V16<T>::type v;
        T* e = reinterpret_cast<T*>(&v);
#pragma unroll
        for (int w = 0; w < W; ++w) e[w] = r[w];
        *reinterpret_cast<typename V16<T>::type*>(p) = v;
    } else {
#pragma unroll
        for (int w = 0; w < W; ++w) p[w] = r[w];
    }
}

__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }

// ---------------------------------------------------------------------------------------------
// simt_gemm
//   AK   : A is K-major (inner == 1, fibres contiguous); otherwise rows (i) are contiguous.
//   VEC  : 16-byte vector loads of A and vector stores of C (alignment and divisibility checked
//          by the host).
//   BCM  : B column-major.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct GemmSmem {
    static constexpr int RV = 16 / sizeof(T);
    __align__(16) T As[2][8][32 * RV];
    __align__(16) T Bs[2][8][32 * RV];
};

// One BM x BN output tile (rows m0.., columns n0..) of the slice-GEMM, all 256 threads of the block.
template <typename T, bool AK, bool VEC, bool BCM>
__device__ __forceinline__ void gemm_tile(const View3& v, int64_t m0, int64_t n0, GemmSmem<T>& sm,
                                          int64_t l_begin = 0, int64_t l_end = -1)
{
    constexpr int RV = 16 / sizeof(T);   // elements per 16-byte vector
    constexpr int BM = 32 * RV, BN = 32 * RV, BK = 8;
    constexpr int TM = 2 * RV, TN = 2 * RV;
    constexpr int NT = 256;
    constexpr int WA = VEC ? RV : 1;
    // A tile: BM rows x BK columns, loaded as NVA vectors of WA elements.
    constexpr int NVA = BM * BK / WA;
    constexpr int LA = NVA / NT;
    constexpr int ACONT = AK ? BK : BM;          // extent of A's contiguous tile dimension
    // B tile: BK x BN, scalar loads.
    constexpr int LB = BN * BK / NT;

    auto& As = sm.As;
    auto& Bs = sm.Bs;

    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t inner = v.inner, m = v.m;
    // the l range of this tile: all of n_q, or one part of a split K loop (l_begin % BK == 0)
    const int64_t nq = l_end < 0 ? v.nq : l_end;
    const int64_t nq_full = v.nq;
    const int64_t M = v.outer * inner;
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;

    // Per-slot A addressing, fixed for the whole K loop.
    int64_t abase[LA];
    int a_loff[LA], a_roff[LA];
    bool arow_ok[LA];
#pragma unroll
    for (int s = 0; s < LA; ++s) {
        const int vi = tid + s * NT;
        const int c = (vi % (ACONT / WA)) * WA;
        const int o = vi / (ACONT / WA);
        const int roff = AK ? o : c;
        const int loff = AK ? c : o;
        const int64_t row = m0 + roff;
        arow_ok[s] = row < M;
        const int64_t k = arow_ok[s] ? row / inner : 0;
        const int64_t i = arow_ok[s] ? row - k * inner : 0;
        abase[s] = k * inner * nq_full + i;
        a_loff[s] = loff;
        a_roff[s] = roff;
    }

    T ra[LA][WA];
    T rb[LB];

    auto load_tiles = [&](int64_t l0) {
#pragma unroll
        for (int s = 0; s < LA; ++s) {
            const int64_t l = l0 + a_loff[s];
            if (arow_ok[s] && l < nq) {
                load_vec<T, WA>(ra[s], A + abase[s] + l * inner);
            } else {
#pragma unroll
                for (int w = 0; w < WA; ++w) ra[s][w] = T(0);
            }
        }
#pragma unroll
        for (int s = 0; s < LB; ++s) {
            const int vi = tid + s * NT;
            int jo, lo;
            if (BCM) { jo = vi % BN; lo = vi / BN; }
            else     { lo = vi % BK; jo = vi / BK; }
            const int64_t j = n0 + jo, l = l0 + lo;
            T val = T(0);
            if (j < m && l < nq) val = __ldg(BCM ? B + j + l * m : B + j * nq_full + l);
            rb[s] = val;
        }
    };
    auto store_tiles = [&](int buf) {
#pragma unroll
        for (int s = 0; s < LA; ++s) {
#pragma unroll
            for (int w = 0; w < WA; ++w) {
                if (AK) As[buf][a_loff[s] + w][a_roff[s]] = ra[s][w];
                else    As[buf][a_loff[s]][a_roff[s] + w] = ra[s][w];
            }
        }
#pragma unroll
        for (int s = 0; s < LB; ++s) {
            const int vi = tid + s * NT;
            int jo, lo;
            if (BCM) { jo = vi % BN; lo = vi / BN; }
            else     { lo = vi % BK; jo = vi / BK; }
            Bs[buf][lo][jo] = rb[s];
        }
    };

    // FP32 accumulates in packed column pairs (acc2[i][j / 2], column j in the low half when j
    // is even): half the FMA instructions of one per output
    constexpr bool PK = std::is_same<T, float>::value;
    T acc[TM][TN];
    unsigned long long acc2[PK ? TM : 1][PK ? TN / 2 : 1];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
    if constexpr (PK) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN / 2; ++j) acc2[i][j] = 0ull;
    }

    const int64_t nk = ceil_div(nq - l_begin, BK);
    load_tiles(l_begin);
    store_tiles(0);
    __syncthreads();

    for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) load_tiles(l_begin + (kt + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            if constexpr (PK) {
                const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * RV]);
                const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][BM / 2 + ty * RV]);
                const ulonglong2 b0 = *reinterpret_cast<const ulonglong2*>(&Bs[buf][kk][tx * RV]);
                const ulonglong2 b1 = *reinterpret_cast<const ulonglong2*>(&Bs[buf][kk][BN / 2 + tx * RV]);
                const unsigned long long bp[TN / 2] = {b0.x, b0.y, b1.x, b1.y};
                const float af[TM] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
                for (int i = 0; i < TM; ++i) {
                    const unsigned long long ap = pair_dup(af[i]);
#pragma unroll
                    for (int j = 0; j < TN / 2; ++j) ffma2(acc2[i][j], ap, bp[j]);
                }
                continue;
            }
            T af[TM], bf[TN];
            typedef typename V16<T>::type VT;
            VT a0 = *reinterpret_cast<const VT*>(&As[buf][kk][ty * RV]);
            VT a1 = *reinterpret_cast<const VT*>(&As[buf][kk][BM / 2 + ty * RV]);
            VT b0 = *reinterpret_cast<const VT*>(&Bs[buf][kk][tx * RV]);
            VT b1 = *reinterpret_cast<const VT*>(&Bs[buf][kk][BN / 2 + tx * RV]);
#pragma unroll
            for (int r = 0; r < RV; ++r) {
                af[r] = reinterpret_cast<const T*>(&a0)[r];
                af[RV + r] = reinterpret_cast<const T*>(&a1)[r];
                bf[r] = reinterpret_cast<const T*>(&b0)[r];
                bf[RV + r] = reinterpret_cast<const T*>(&b1)[r];
            }
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fma_t(af[i], bf[j], acc[i][j]);
        }
        if (kt + 1 < nk) store_tiles(buf ^ 1);
        __syncthreads();
    }

    if constexpr (PK) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN / 2; ++j) {
                acc[i][2 * j] = pair_lo(acc2[i][j]);
                acc[i][2 * j + 1] = pair_hi(acc2[i][j]);
            }
    }

    // Epilogue: C(row, j) = cbase(row) + j*inner, cbase = (row/inner)*inner*m + row%inner.
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int64_t row0 = m0 + h * (BM / 2) + ty * RV;
        if (!AK && VEC) {
            // RV consecutive rows share one k (inner % RV == 0): one vector per column.
            if (row0 < M) {
                const int64_t k = row0 / inner;
                const int64_t cb = k * inner * m + (row0 - k * inner);
#pragma unroll
                for (int g = 0; g < 2; ++g)
#pragma unroll
                    for (int c = 0; c < RV; ++c) {
                        const int64_t j = n0 + g * (BN / 2) + tx * RV + c;
                        if (j < m) {
                            T r[RV];
#pragma unroll
                            for (int w = 0; w < RV; ++w) r[w] = acc[h * RV + w][g * RV + c];
                            store_vec<T, RV>(Cp + cb + j * inner, r);
                        }
                    }
            }
        } else if (AK && VEC) {
            // inner == 1 and m % RV == 0: RV consecutive columns are contiguous.
#pragma unroll
            for (int w = 0; w < RV; ++w) {
                const int64_t row = row0 + w;
                if (row < M) {
#pragma unroll
                    for (int g = 0; g < 2; ++g) {
                        const int64_t j0 = n0 + g * (BN / 2) + tx * RV;
                        if (j0 < m) {
                            T r[RV];
#pragma unroll
                            for (int c = 0; c < RV; ++c) r[c] = acc[h * RV + w][g * RV + c];
                            store_vec<T, RV>(Cp + row * m + j0, r);
                        }
                    }
                }
            }
        } else {
#pragma unroll
            for (int w = 0; w < RV; ++w) {
                const int64_t row = row0 + w;
                if (row < M) {
                    const int64_t k = row / inner;
                    const int64_t cb = k * inner * m + (row - k * inner);
#pragma unroll
                    for (int g = 0; g < 2; ++g)
#pragma unroll
                        for (int c = 0; c < RV; ++c) {
                            const int64_t j = n0 + g * (BN / 2) + tx * RV + c;
                            if (j < m) Cp[cb + j * inner] = acc[h * RV + w][g * RV + c];
                        }
                }
            }
        }
    }
}

// Two CTAs per SM in float (at most 128 registers a thread: 16 warps of 128 fill each
// sub-partition's quarter of the register file), three in double (at most 80).
template <typename T, bool AK, bool VEC, bool BCM>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? 3 : 2)) simt_gemm_kernel(View3 v)
{
    constexpr int RV = 16 / sizeof(T);
    __shared__ GemmSmem<T> sm;
    gemm_tile<T, AK, VEC, BCM>(v, (int64_t)blockIdx.x * (32 * RV), (int64_t)blockIdx.y * (32 * RV), sm);
}

// The K loop split `gridDim.z` ways: part z covers l in [z * lper, min(n_q, (z + 1) * lper)) and
// writes its partial tile into ws + z * (outer * m * inner), a buffer with C's own layout;
// split_reduce_kernel then adds the parts in a fixed order, so the result does not depend on
// scheduling.
template <typename T, bool AK, bool VEC, bool BCM>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? 3 : 2)) simt_gemm_split_kernel(View3 v, int64_t lper, T* ws)
{
    constexpr int RV = 16 / sizeof(T);
    __shared__ GemmSmem<T> sm;
    const int64_t l0 = (int64_t)blockIdx.z * lper;
    const int64_t l1 = l0 + lper < v.nq ? l0 + lper : v.nq;
    View3 part = v;
    part.c = ws + (size_t)blockIdx.z * (size_t)(v.outer * v.m * v.inner);
    gemm_tile<T, AK, VEC, BCM>(part, (int64_t)blockIdx.x * (32 * RV), (int64_t)blockIdx.y * (32 * RV), sm, l0, l1);
}

// ---------------------------------------------------------------------------------------------
// colvec: small m (<= MB), strided fibres (inner >= 2). Each lane owns W consecutive rows (i of
// one slice; 16-byte loads when W = 16/sizeof(T)). The block's 8 warps are split into 8/LS row
// chunks of LS warps each; the LS warps of a chunk split the l loop (warp w takes l = w, w+LS,
// ...) and reduce through shared memory at the end. LS = 1 gives 8*32*W rows per block and no
// reduction (problems with many rows); LS = 8 gives 32*W rows per block and 8 independent load
// streams per row chunk (problems with few rows). B is staged in shared memory as [l][MB].
// ---------------------------------------------------------------------------------------------
constexpr int kColWarps = 8;
constexpr int kColUnroll1 = 8;   // l steps unrolled with one scalar row per lane

template <typename T, int MB>
struct ColvecSmem {
    static constexpr int MBP = MB < 4 ? 4 : MB;
    static constexpr int LB = (32768 / (MBP * (int)sizeof(T))) < 512 ? 32768 / (MBP * (int)sizeof(T)) : 512;  // l per staged chunk of B
    __align__(16) T bs[LB][MBP];
    __align__(16) T red[kColWarps][32 * (16 / sizeof(T))];
};

template <typename T, int MB, int W, int LS>
__device__ __forceinline__ void colvec_tile(const View3& v, int64_t row0, ColvecSmem<T, MB>& sm)
{
    constexpr int LB = ColvecSmem<T, MB>::LB;
    constexpr int MBP = MB < 4 ? 4 : MB;
    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t inner = v.inner, nq = v.nq, m = v.m;
    const int64_t M = v.outer * inner;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int chunk = warp / LS, part = warp % LS;
    const int64_t row = row0 + ((int64_t)chunk * 32 + lane) * W;
    const bool valid = row < M;
    const int64_t k = valid ? row / inner : 0;
    const int64_t i = valid ? row - k * inner : 0;
    const T* ap = A + k * inner * nq + i;

    T acc[MB][W];
#pragma unroll
    for (int j = 0; j < MB; ++j)
#pragma unroll
        for (int w = 0; w < W; ++w) acc[j][w] = T(0);

    for (int64_t l0 = 0; l0 < nq; l0 += LB) {
        const int lc = (int)((nq - l0) < LB ? (nq - l0) : LB);
        __syncthreads();
        for (int e = threadIdx.x; e < lc * MBP; e += blockDim.x) {
            const int l = e / MBP, j = e % MBP;
            const int64_t gl = l0 + l;
            sm.bs[l][j] = (j < m) ? (v.b_cm ? B[j + gl * m] : B[j * nq + gl]) : T(0);
        }
        __syncthreads();
        if (valid) {
            // scalar rows (W = 1) take more l steps at a time, so that more loads are in flight
#pragma unroll (W == 1 ? kColUnroll1 : 4)
            for (int l = part; l < lc; l += LS) {
                T a[W];
                load_vec<T, W>(a, ap + (l0 + l) * inner);
                T bj[MBP];
                if constexpr (MBP * sizeof(T) % 16 == 0) {
#pragma unroll
                    for (int c = 0; c < MBP * (int)sizeof(T) / 16; ++c) {
                        typename V16<T>::type t = *reinterpret_cast<const typename V16<T>::type*>(&sm.bs[l][c * (16 / sizeof(T))]);
#pragma unroll
                        for (int e = 0; e < (int)(16 / sizeof(T)); ++e) bj[c * (16 / sizeof(T)) + e] = reinterpret_cast<const T*>(&t)[e];
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < MBP; ++j) bj[j] = sm.bs[l][j];
                }
#pragma unroll
                for (int j = 0; j < MB; ++j)
#pragma unroll
                    for (int w = 0; w < W; ++w) acc[j][w] = fma_t(a[w], bj[j], acc[j][w]);
            }
        }
    }
    T* cp = Cp + k * inner * m + i;
    if constexpr (LS == 1) {
        if (valid) {
#pragma unroll
            for (int j = 0; j < MB; ++j)
                if (j < m) store_vec<T, W>(cp + j * inner, acc[j]);
        }
    } else {
        // Reduce the LS warps' partial sums, one output column at a time.
#pragma unroll
        for (int j = 0; j < MB; ++j) {
            if (j >= m) break;
            __syncthreads();
#pragma unroll
            for (int w = 0; w < W; ++w) sm.red[warp][lane * W + w] = acc[j][w];
            __syncthreads();
            if (part == 0 && valid) {
                T r[W];
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    T t = T(0);
#pragma unroll
                    for (int q = 0; q < LS; ++q) t += sm.red[chunk * LS + q][lane * W + w];
                    r[w] = t;
                }
                store_vec<T, W>(cp + j * inner, r);
            }
        }
    }
}

template <typename T, int MB, int W, int LS>
__global__ void __launch_bounds__(256) colvec_kernel(View3 v)
{
    __shared__ ColvecSmem<T, MB> sm;
    colvec_tile<T, MB, W, LS>(v, (int64_t)blockIdx.x * (kColWarps / LS) * 32 * W, sm);
}

// colvec_async: the column kernel for rows without 16-byte alignment (one row per lane). Each
// thread streams its own row's elements A[k][l][i] into a ring of shared memory with 4- or 8-byte
// asynchronous copies (cp.async, any 4-byte alignment), kColAsyncStages - 1 stages of LC l
// (8 float, 4 double) ahead of the one it multiplies, so that many loads are in flight without
// holding them in registers. A thread reads back only what it copied itself: the ring needs no block barrier,
// only the thread's own wait on its copy groups. B is staged per chunk of LB l as in colvec.
constexpr int kColAsyncStages = 4;
constexpr bool kColAsync = true;   // rows without 16-byte alignment take colvec_async

template <typename T, int MB>
struct ColvecAsyncSmem {
    static constexpr int MBP = MB < 4 ? 4 : MB;
    static constexpr int LC = sizeof(T) == 8 ? 4 : 8;                      // l per stage
    static constexpr int LB = sizeof(T) == 8 ? 64 : 128;                   // l of B per chunk
    __align__(16) T a[kColAsyncStages][LC][256];
    __align__(16) T bs[LB][MBP];
    __align__(16) T red[kColWarps][32];
};

__device__ __forceinline__ void cp_async_elem(void* smem_dst, const void* src, int bytes, int src_bytes)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename T, int MB, int LS>
__device__ __forceinline__ void colvec_async_tile(const View3& v, int64_t row0, ColvecAsyncSmem<T, MB>& sm)
{
    using SM = ColvecAsyncSmem<T, MB>;
    constexpr int LB = SM::LB, LC = SM::LC, MBP = SM::MBP, ST = kColAsyncStages;
    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t inner = v.inner, nq = v.nq, m = v.m;
    const int64_t M = v.outer * inner;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int chunk = warp / LS, part = warp % LS;
    const int64_t row = row0 + (int64_t)chunk * 32 + lane;
    const bool valid = row < M;
    const int64_t k = valid ? row / inner : 0;
    const int64_t i = valid ? row - k * inner : 0;
    const T* ap = A + k * inner * nq + i;

    T acc[MB];
#pragma unroll
    for (int j = 0; j < MB; ++j) acc[j] = T(0);

    for (int64_t l0 = 0; l0 < nq; l0 += LB) {
        const int lc = (int)((nq - l0) < LB ? (nq - l0) : LB);
        __syncthreads();
        for (int e = tid; e < lc * MBP; e += blockDim.x) {
            const int l = e / MBP, j = e % MBP;
            const int64_t gl = l0 + l;
            sm.bs[l][j] = (j < m) ? (v.b_cm ? B[j + gl * m] : B[j * nq + gl]) : T(0);
        }
        __syncthreads();
        // this thread's l in the chunk: part, part + LS, ...; n of them, in stages of LC
        const int n = lc > part ? (lc - part + LS - 1) / LS : 0;
        const int nst = (n + LC - 1) / LC;
        const T* base = ap + l0 * inner;
        auto issue = [&](int st) {
            T* dst = &sm.a[st % ST][0][tid];
#pragma unroll
            for (int c = 0; c < LC; ++c) {
                const int idx = st * LC + c;
                const bool ok = valid && idx < n;
                cp_async_elem(dst + c * 256, ok ? base + (int64_t)(part + idx * LS) * inner : A, (int)sizeof(T),
                              ok ? (int)sizeof(T) : 0);
            }
        };
        // one commit group per stage (empty ones too), so that wait_group counts stages
#pragma unroll
        for (int st = 0; st < ST - 1; ++st) {
            if (st < nst) issue(st);
            cp_async_commit();
        }
        for (int st = 0; st < nst; ++st) {
            // refill the slot the previous stage used, then wait for this stage's copies
            if (st + ST - 1 < nst) issue(st + ST - 1);
            cp_async_commit();
            cp_async_wait<ST - 1>();
#pragma unroll
            for (int c = 0; c < LC; ++c) {
                const int idx = st * LC + c;
                if (idx >= n) break;
                const T a = sm.a[st % ST][c][tid];
                const int l = part + idx * LS;
                T bj[MBP];
                if constexpr (MBP * sizeof(T) % 16 == 0) {
#pragma unroll
                    for (int q = 0; q < MBP * (int)sizeof(T) / 16; ++q) {
                        typename V16<T>::type t = *reinterpret_cast<const typename V16<T>::type*>(&sm.bs[l][q * (16 / sizeof(T))]);
#pragma unroll
                        for (int e = 0; e < (int)(16 / sizeof(T)); ++e) bj[q * (16 / sizeof(T)) + e] = reinterpret_cast<const T*>(&t)[e];
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < MBP; ++j) bj[j] = sm.bs[l][j];
                }
#pragma unroll
                for (int j = 0; j < MB; ++j) acc[j] = fma_t(a, bj[j], acc[j]);
            }
        }
        cp_async_wait<0>();   // no copy into the ring is pending when the next chunk restarts it
    }
    T* cp = Cp + k * inner * m + i;
    if constexpr (LS == 1) {
        if (valid) {
#pragma unroll
            for (int j = 0; j < MB; ++j)
                if (j < m) cp[j * inner] = acc[j];
        }
    } else {
        // Reduce the LS warps' partial sums, one output column at a time.
#pragma unroll
        for (int j = 0; j < MB; ++j) {
            if (j >= m) break;
            __syncthreads();
            sm.red[warp][lane] = acc[j];
            __syncthreads();
            if (part == 0 && valid) {
                T t = T(0);
#pragma unroll
                for (int q = 0; q < LS; ++q) t += sm.red[chunk * LS + q][lane];
                cp[j * inner] = t;
            }
        }
    }
}

template <typename T, int MB, int LS>
__global__ void __launch_bounds__(256) colvec_async_kernel(View3 v)
{
    __shared__ ColvecAsyncSmem<T, MB> sm;
    colvec_async_tile<T, MB, LS>(v, (int64_t)blockIdx.x * (kColWarps / LS) * 32, sm);
}

// ---------------------------------------------------------------------------------------------
// rowdot: small m (<= MB), contiguous fibres (inner == 1): C[k][j] = sum_l A[k][l] B(j,l).
// Each warp owns 32 rows; the block walks l in chunks of LC = 128/sizeof(T): every warp copies
// its 32 x LC tile of A into padded shared memory with coalesced 16-byte loads, the block stages
// B[l][MB] for the chunk, then each lane accumulates its own row from shared memory.
// ---------------------------------------------------------------------------------------------
template <typename T, int MB>
struct RowdotSmem {
    static constexpr int LC = 128 / sizeof(T);          // l per chunk (one 128-byte line per row)
    T a[8][32][LC + 1];                                  // per warp, padded rows
    __align__(16) T bs[LC][MB < 4 ? 4 : MB];
};

template <typename T, int MB, bool VEC>
__device__ __forceinline__ void rowdot_tile(const View3& v, int64_t row0, RowdotSmem<T, MB>& sm)
{
    constexpr int LC = RowdotSmem<T, MB>::LC;
    constexpr int MBP = MB < 4 ? 4 : MB;
    constexpr int RV = 16 / sizeof(T);
    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t nq = v.nq, m = v.m, rows = v.outer;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t wrow0 = row0 + warp * 32;
    const int64_t row = wrow0 + lane;
    T acc[MB];
#pragma unroll
    for (int j = 0; j < MB; ++j) acc[j] = T(0);

    for (int64_t l0 = 0; l0 < nq; l0 += LC) {
        const int lc = (int)((nq - l0) < LC ? (nq - l0) : LC);
        __syncthreads();
        // B chunk
        for (int e = threadIdx.x; e < LC * MBP; e += blockDim.x) {
            const int l = e / MBP, j = e % MBP;
            const int64_t gl = l0 + l;
            sm.bs[l][j] = (j < m && l < lc) ? (v.b_cm ? B[j + gl * m] : B[j * nq + gl]) : T(0);
        }
        // this warp's A tile: rows wrow0 .. +31, columns l0 .. l0+LC-1
        if (VEC) {
            // (LC / RV) lanes per row, 32 / (LC / RV) rows per step
            constexpr int LPR = LC / RV, RPS = 32 / LPR;
            const int r_in = lane / LPR, c = (lane % LPR) * RV;
#pragma unroll
            for (int r = r_in; r < 32; r += RPS) {
                const int64_t gr = wrow0 + r;
                T x[RV];
                if (gr < rows && c < lc) load_vec<T, RV>(x, A + gr * nq + l0 + c);
                else {
#pragma unroll
                    for (int e = 0; e < RV; ++e) x[e] = T(0);
                }
#pragma unroll
                for (int e = 0; e < RV; ++e) sm.a[warp][r][c + e] = x[e];
            }
        } else {
            // lane c copies column c of the warp's rows: the loads of RB rows go out before their
            // stores, so that many are in flight
            constexpr int RB = 16;
            const int c = lane;
#pragma unroll 1
            for (int rb = 0; rb < 32; rb += RB) {
                T x[RB];
#pragma unroll
                for (int r = 0; r < RB; ++r) {
                    const int64_t gr = wrow0 + rb + r;
                    x[r] = (c < LC && c < lc && gr < rows) ? __ldg(A + gr * nq + l0 + c) : T(0);
                }
                if (c < LC) {
#pragma unroll
                    for (int r = 0; r < RB; ++r) sm.a[warp][rb + r][c] = x[r];
                }
            }
        }
        __syncthreads();
#pragma unroll 8
        for (int l = 0; l < lc; ++l) {
            const T a = sm.a[warp][lane][l];
            T bj[MBP];
            if constexpr (MBP * sizeof(T) % 16 == 0) {
#pragma unroll
                for (int cc = 0; cc < MBP * (int)sizeof(T) / 16; ++cc) {
                    typename V16<T>::type t = *reinterpret_cast<const typename V16<T>::type*>(&sm.bs[l][cc * RV]);
#pragma unroll
                    for (int e = 0; e < RV; ++e) bj[cc * RV + e] = reinterpret_cast<const T*>(&t)[e];
                }
            } else {
#pragma unroll
                for (int j = 0; j < MBP; ++j) bj[j] = sm.bs[l][j];
            }
#pragma unroll
            for (int j = 0; j < MB; ++j) acc[j] = fma_t(a, bj[j], acc[j]);
        }
    }
    if (row < rows) {
#pragma unroll
        for (int j = 0; j < MB; ++j)
            if (j < m) Cp[row * m + j] = acc[j];
    }
}

template <typename T, int MB, bool VEC>
__global__ void __launch_bounds__(256) rowdot_kernel(View3 v)
{
    __shared__ RowdotSmem<T, MB> sm;
    rowdot_tile<T, MB, VEC>(v, (int64_t)blockIdx.x * 256, sm);
}

// ---------------------------------------------------------------------------------------------
// rowflat: small m, contiguous fibres of at most kFlatMaxNq elements (inner == 1, short rows).
// A warp's wr consecutive rows are wr * nq contiguous elements: the warp copies them with
// coalesced loads into shared memory with rows padded to nq + 1 (conflict-free row reads), then
// each lane computes every 32nd row. B sits in shared memory as bs[l][j]. With STAGE, the m
// outputs of 32 consecutive rows (32 * m contiguous elements of C) are staged in shared memory
// (rows padded to an odd stride) and written with coalesced stores, 32 consecutive elements per
// instruction; without it each lane stores its own row (a stride of m elements between lanes),
// which measured faster where a row's outputs are short or the fibres long.
// ---------------------------------------------------------------------------------------------
constexpr int kFlatMaxNq = 16;

template <typename T, int MB, bool STAGE>
__global__ void __launch_bounds__(256) rowflat_kernel(View3 v, int wr)
{
    constexpr int MBP = MB < 4 ? 4 : MB;
    extern __shared__ __align__(16) unsigned char flat_raw[];
    T* smf = reinterpret_cast<T*>(flat_raw);
    const int nq = (int)v.nq, stride = nq + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T* tile = smf + (size_t)warp * wr * stride;
    T* bs = smf + (size_t)8 * wr * stride;
    const T* __restrict__ B = static_cast<const T*>(v.b);
    for (int e = threadIdx.x; e < nq * MBP; e += blockDim.x) {
        const int l = e / MBP, j = e - l * MBP;
        bs[e] = j < v.m ? (v.b_cm ? B[j + (int64_t)l * v.m] : B[(int64_t)j * nq + l]) : T(0);
    }
    __syncthreads();
    const int64_t wrow0 = ((int64_t)blockIdx.x * 8 + warp) * wr;
    if (wrow0 >= v.outer) return;
    const int nrow = (int)((v.outer - wrow0) < wr ? (v.outer - wrow0) : wr);
    const T* __restrict__ A = static_cast<const T*>(v.a) + wrow0 * nq;
    const int cnt = nrow * nq;
    // e / nq == umulhi(e, ceil(2^32 / nq)) for these e (nq > 1; 2^32 itself does not fit)
    const uint32_t inv = nq > 1 ? (uint32_t)((0x100000000ull + nq - 1) / nq) : 0u;
#pragma unroll 16
    for (int e = lane; e < cnt; e += 32) {
        const int r = nq > 1 ? (int)__umulhi((uint32_t)e, inv) : e;
        tile[r * stride + (e - r * nq)] = __ldg(A + e);
    }
    __syncwarp();
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int m = (int)v.m;
    if constexpr (!STAGE) {
        for (int r = lane; r < nrow; r += 32) {
            T acc[MB];
#pragma unroll
            for (int j = 0; j < MB; ++j) acc[j] = T(0);
            const T* row = tile + r * stride;
            for (int l = 0; l < nq; ++l) {
                const T a = row[l];
#pragma unroll
                for (int j = 0; j < MB; ++j) acc[j] = fma_t(a, bs[l * MBP + j], acc[j]);
            }
            T* cp = Cp + (wrow0 + r) * (int64_t)m;
#pragma unroll
            for (int j = 0; j < MB; ++j)
                if (j < m) cp[j] = acc[j];
        }
        return;
    }
    // staged: this warp's 32 x (m | 1) outputs after B (odd row stride, conflict-free writes)
    const int ms = m | 1;
    T* ostage = bs + (size_t)nq * MBP + (size_t)warp * 32 * ms;
    // e / m == umulhi(e, ceil(2^32 / m)) for e < 32 * m (m > 1)
    const uint32_t minv = m > 1 ? (uint32_t)((0x100000000ull + m - 1) / m) : 0u;
    for (int r0 = 0; r0 < nrow; r0 += 32) {
        const int r = r0 + lane;
        if (r < nrow) {
            T acc[MB];
#pragma unroll
            for (int j = 0; j < MB; ++j) acc[j] = T(0);
            const T* row = tile + r * stride;
            for (int l = 0; l < nq; ++l) {
                const T a = row[l];
#pragma unroll
                for (int j = 0; j < MB; ++j) acc[j] = fma_t(a, bs[l * MBP + j], acc[j]);
            }
#pragma unroll
            for (int j = 0; j < MB; ++j)
                if (j < m) ostage[lane * ms + j] = acc[j];
        }
        __syncwarp();
        // rows r0 .. r0 + nr - 1: nr * m contiguous outputs from C[(wrow0 + r0) * m]
        const int nr = (nrow - r0) < 32 ? (nrow - r0) : 32;
        T* cp = Cp + (wrow0 + r0) * (int64_t)m;
        for (int e = lane; e < nr * m; e += 32) {
            const int rr = m > 1 ? (int)__umulhi((uint32_t)e, minv) : e;
            cp[e] = ostage[rr * ms + (e - rr * m)];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------------
// rowspan: small m, contiguous fibres of NQ in {1, 2, 4, 8, 16} elements (at most a span), A
// 16-byte aligned. Thread t reads the 64-byte span (16 floats / 8 doubles) holding the R = span /
// NQ whole fibres t*R .. t*R + R-1 with 128-bit loads: consecutive threads read consecutive
// spans, so a warp's loads are fully coalesced and nothing is staged. Its R*m outputs are
// contiguous in C. B sits in shared memory (broadcast reads). Used where a thread's outputs take
// at most 64 bytes (measured: more outputs per thread scatter the stores too widely).
// ---------------------------------------------------------------------------------------------
template <typename T, int MB, int NQ>
__global__ void __launch_bounds__(256) rowspan_kernel(View3 v)
{
    constexpr int E = 64 / (int)sizeof(T), R = E / NQ, VW = 16 / (int)sizeof(T), NV = E / VW;
    static_assert(NQ <= E, "a fibre fits a span");
    __shared__ T bs[NQ * MB];
    const T* __restrict__ B = static_cast<const T*>(v.b);
    for (int e = threadIdx.x; e < NQ * MB; e += blockDim.x) {
        const int l = e / MB, j = e - l * MB;
        bs[e] = j < v.m ? (v.b_cm ? B[j + (int64_t)l * v.m] : B[(int64_t)j * NQ + l]) : T(0);
    }
    __syncthreads();
    const T* __restrict__ A = static_cast<const T*>(v.a);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t rows = v.outer, spans = (rows + R - 1) / R;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < spans; t += stride) {
        const int64_t r0 = t * R;
        T a[E];
        if (r0 + R <= rows) {
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                T x[VW];
                load_vec<T, VW>(x, A + r0 * NQ + q * VW);
#pragma unroll
                for (int w = 0; w < VW; ++w) a[q * VW + w] = x[w];
            }
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) a[e] = (r0 + e / NQ < rows) ? __ldg(A + r0 * NQ + e) : T(0);
        }
        T* cp = Cp + r0 * v.m;
        // R*m contiguous outputs: with m == MB, a 16-byte aligned C and R*MB a multiple of VW,
        // written VW at a time (a vector covers MB / VW of a row, or VW / MB rows)
        const bool vec = r0 + R <= rows && v.m == MB && (R * MB) % VW == 0 &&
                         (reinterpret_cast<uintptr_t>(cp) & 15u) == 0;
        if (vec) {
#pragma unroll
            for (int q = 0; q < R * MB / VW; ++q) {
                T x[VW];
#pragma unroll
                for (int w = 0; w < VW; ++w) {
                    const int o = q * VW + w, r = o / MB, j = o - r * MB;
                    T acc = T(0);
#pragma unroll
                    for (int l = 0; l < NQ; ++l) acc = fma_t(a[r * NQ + l], bs[l * MB + j], acc);
                    x[w] = acc;
                }
                store_vec<T, VW>(cp + q * VW, x);
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r0 + r >= rows) break;
#pragma unroll
                for (int j = 0; j < MB; ++j) {
                    if (j >= v.m) break;
                    T acc = T(0);
#pragma unroll
                    for (int l = 0; l < NQ; ++l) acc = fma_t(a[r * NQ + l], bs[l * MB + j], acc);
                    cp[(int64_t)r * v.m + j] = acc;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// strided: one thread per C element, strides taken from the caller.
// ---------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) strided_kernel(StridedProblem sp)
{
    const T* __restrict__ A = static_cast<const T*>(sp.a);
    const T* __restrict__ B = static_cast<const T*>(sp.b);
    T* __restrict__ Cp = static_cast<T*>(sp.c);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < sp.total; e += stride) {
        int64_t rem = e, aoff = 0, coff = 0, j = 0;
        for (int r = 0; r < sp.p; ++r) {
            const int mode = sp.order[r];
            const int64_t ext = sp.nc[mode];
            const int64_t idx = rem % ext;
            rem /= ext;
            coff += idx * sp.wc[mode];
            if (mode == sp.q) j = idx;
            else aoff += idx * sp.wa[mode];
        }
        const int64_t wq = sp.wa[sp.q];
        T acc = T(0);
        for (int64_t l = 0; l < sp.nq; ++l) {
            const T bv = sp.b_cm ? B[j + l * sp.m] : B[j * sp.nq + l];
            acc = fma_t(A[aoff + l * wq], bv, acc);
        }
        Cp[coff] = acc;
    }
}

// ---------------------------------------------------------------------------------------------
// grouped: many independent TTMs in one persistent launch. Blocks pull work items from a device
// counter; an item is one slice-GEMM tile of a problem (m > 16) or a block of 256 rows of a
// small-m problem. Problems are ordered largest first by the host, so the tail is short.
// ---------------------------------------------------------------------------------------------
template <typename T>
union GroupedSmem {
    GemmSmem<T> gemm;
    ColvecSmem<T, 16> col;
    RowdotSmem<T, 16> row;
};

// ASYNC: unaligned column items take colvec_async (its ring must be part of SM).
template <typename T, int MB, bool ASYNC, class SM>
__device__ __forceinline__ void grouped_small(const View3& v, int flags, int64_t local, SM& sm)
{
    constexpr int RV = 16 / sizeof(T);
    auto& col = reinterpret_cast<ColvecSmem<T, MB>&>(sm.col);
    auto& row = reinterpret_cast<RowdotSmem<T, MB>&>(sm.row);
    if (flags & 1) {
        if (flags & 2) rowdot_tile<T, MB, true>(v, local * 256, row);
        else rowdot_tile<T, MB, false>(v, local * 256, row);
    } else {
        if (!ASYNC && (flags & 2)) colvec_tile<T, MB, RV, 1>(v, local * kColWarps * 32 * RV, col);
        else if constexpr (ASYNC) colvec_async_tile<T, MB, 1>(v, local * kColWarps * 32, reinterpret_cast<ColvecAsyncSmem<T, MB>&>(sm.cola));
        else colvec_tile<T, MB, 1, 1>(v, local * kColWarps * 32, col);
    }
}

// Two CTAs per SM (at most 128 registers; a few spill): measured faster on the batched workload
// than one CTA of 255 registers.
template <typename T>
__global__ void __launch_bounds__(256, 2) grouped_kernel(const GroupDesc* __restrict__ desc, int count, int64_t total,
                                                      unsigned long long* queue)
{
    constexpr int RV = 16 / sizeof(T);
    constexpr int BM = 32 * RV, BN = 32 * RV;
    __shared__ GroupedSmem<T> sm;
    __shared__ int64_t item_s;
    for (;;) {
        if (threadIdx.x == 0) item_s = (int64_t)atomicAdd(queue, 1ull);
        __syncthreads();
        const int64_t item = item_s;
        if (item >= total) break;
        int lo = 0, hi = count - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (desc[mid].first <= item) lo = mid;
            else hi = mid - 1;
        }
        const GroupDesc g = desc[lo];
        const int64_t local = item - g.first;
        View3 v;
        v.a = g.a;
        v.b = g.b;
        v.c = g.c;
        v.outer = g.outer;
        v.nq = g.nq;
        v.inner = g.inner;
        v.m = g.m;
        v.b_cm = g.b_cm;
        if (g.kind == 0) {
            const int64_t m0 = (local % g.tiles_m) * BM, n0 = (local / g.tiles_m) * BN;
            const bool ak = g.flags & 1, vec = g.flags & 2;
            if (ak) {
                if (vec) { if (g.b_cm) gemm_tile<T, true, true, true>(v, m0, n0, sm.gemm); else gemm_tile<T, true, true, false>(v, m0, n0, sm.gemm); }
                else     { if (g.b_cm) gemm_tile<T, true, false, true>(v, m0, n0, sm.gemm); else gemm_tile<T, true, false, false>(v, m0, n0, sm.gemm); }
            } else {
                if (vec) { if (g.b_cm) gemm_tile<T, false, true, true>(v, m0, n0, sm.gemm); else gemm_tile<T, false, true, false>(v, m0, n0, sm.gemm); }
                else     { if (g.b_cm) gemm_tile<T, false, false, true>(v, m0, n0, sm.gemm); else gemm_tile<T, false, false, false>(v, m0, n0, sm.gemm); }
            }
        } else {
            if (g.m <= 1) grouped_small<T, 1, false>(v, g.flags, local, sm);
            else if (g.m <= 2) grouped_small<T, 2, false>(v, g.flags, local, sm);
            else if (g.m <= 4) grouped_small<T, 4, false>(v, g.flags, local, sm);
            else if (g.m <= 8) grouped_small<T, 8, false>(v, g.flags, local, sm);
            else grouped_small<T, 16, false>(v, g.flags, local, sm);
        }
        __syncthreads();
    }
}

template <typename T>
union SmallSmem {
    ColvecSmem<T, 16> col;
    ColvecAsyncSmem<T, 16> cola;
    RowdotSmem<T, 16> row;
};

// Grouped launch of small-m problems only: the same work items as grouped_kernel's small-m ones,
// without the slice-GEMM's registers and shared memory, so that more blocks share an SM (their
// loads in flight are what these bandwidth-bound items need). Measured against one launch per
// MB build (each launch leaves a tail) and against the MB = 16 build for every item (small m then
// computes 16 columns): one launch that picks the build per item is the fastest of the three. A
// block's items come from the queue in increasing order, so the problem search goes on from the
// previous item's.
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) grouped_small_kernel(const GroupDesc* __restrict__ desc, int count,
                                                           int64_t total, unsigned long long* queue)
{
    __shared__ SmallSmem<T> sm;
    __shared__ int64_t item_s;
    int cur = 0;
    for (;;) {
        if (threadIdx.x == 0) item_s = (int64_t)atomicAdd(queue, 1ull);
        __syncthreads();
        const int64_t item = item_s;
        if (item >= total) break;
        while (cur + 1 < count && desc[cur + 1].first <= item) ++cur;
        const GroupDesc g = desc[cur];
        const int64_t local = item - g.first;
        View3 v;
        v.a = g.a;
        v.b = g.b;
        v.c = g.c;
        v.outer = g.outer;
        v.nq = g.nq;
        v.inner = g.inner;
        v.m = g.m;
        v.b_cm = g.b_cm;
        if (g.m <= 1) grouped_small<T, 1, kColAsync>(v, g.flags, local, sm);
        else if (g.m <= 2) grouped_small<T, 2, kColAsync>(v, g.flags, local, sm);
        else if (g.m <= 4) grouped_small<T, 4, kColAsync>(v, g.flags, local, sm);
        else if (g.m <= 8) grouped_small<T, 8, kColAsync>(v, g.flags, local, sm);
        else grouped_small<T, 16, kColAsync>(v, g.flags, local, sm);
        __syncthreads();
    }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename T>
cudaError_t simt_gemm_dispatch(const View3& v, cudaStream_t s, int split = 1, int64_t lper = 0, T* ws = nullptr)
{
    constexpr int RV = 16 / sizeof(T);
    constexpr int BM = 32 * RV, BN = 32 * RV;
    const bool ak = v.inner == 1;
    bool vec = aligned16(v.a) && aligned16(split > 1 ? static_cast<const void*>(ws) : v.c);
    if (ak) vec = vec && (v.nq % RV == 0) && (v.m % RV == 0);
    else vec = vec && (v.inner % RV == 0);
    const int64_t M = v.outer * v.inner;
    dim3 grid((unsigned)ceil_div(M, BM), (unsigned)ceil_div(v.m, BN), (unsigned)split);
    dim3 block(256);
#define TLIBTTM_GEMM(AKv, VECv, BCMv)                                                            \
    do {                                                                                        \
        if (split > 1) simt_gemm_split_kernel<T, AKv, VECv, BCMv><<<grid, block, 0, s>>>(v, lper, ws); \
        else simt_gemm_kernel<T, AKv, VECv, BCMv><<<grid, block, 0, s>>>(v);                     \
    } while (0)
    if (ak) {
        if (vec) { if (v.b_cm) TLIBTTM_GEMM(true, true, true); else TLIBTTM_GEMM(true, true, false); }
        else     { if (v.b_cm) TLIBTTM_GEMM(true, false, true); else TLIBTTM_GEMM(true, false, false); }
    } else {
        if (vec) { if (v.b_cm) TLIBTTM_GEMM(false, true, true); else TLIBTTM_GEMM(false, true, false); }
        else     { if (v.b_cm) TLIBTTM_GEMM(false, false, true); else TLIBTTM_GEMM(false, false, false); }
    }
#undef TLIBTTM_GEMM
    return cudaGetLastError();
}

template <typename T, int W, int LS>
cudaError_t colvec_dispatch_ls(const View3& v, cudaStream_t s)
{
    const int64_t M = v.outer * v.inner;
    dim3 grid((unsigned)ceil_div(M, (kColWarps / LS) * 32 * W)), block(256);
#define TLIBTTM_COLVEC(MBv)                                                                \
    do {                                                                                   \
        if (W == 1 && kColAsync) colvec_async_kernel<T, MBv, LS><<<grid, block, 0, s>>>(v); \
        else colvec_kernel<T, MBv, W, LS><<<grid, block, 0, s>>>(v);                       \
    } while (0)
    if (v.m <= 1) TLIBTTM_COLVEC(1);
    else if (v.m <= 2) TLIBTTM_COLVEC(2);
    else if (v.m <= 4) TLIBTTM_COLVEC(4);
    else if (v.m <= 8) TLIBTTM_COLVEC(8);
    else TLIBTTM_COLVEC(16);
#undef TLIBTTM_COLVEC
    return cudaGetLastError();
}

// Few rows (fewer than ~32 warps of rows per SM): split the l loop across warps.
template <typename T, int W>
cudaError_t colvec_dispatch_w(const View3& v, cudaStream_t s)
{
    const int64_t row_warps = ceil_div(v.outer * v.inner, 32 * W);
    return row_warps < 148 * 32 ? colvec_dispatch_ls<T, W, 8>(v, s) : colvec_dispatch_ls<T, W, 1>(v, s);
}

template <typename T>
cudaError_t colvec_dispatch(const View3& v, cudaStream_t s)
{
    constexpr int RV = 16 / sizeof(T);
    const bool vec = aligned16(v.a) && aligned16(v.c) && (v.inner % RV == 0);
    return vec ? colvec_dispatch_w<T, RV>(v, s) : colvec_dispatch_w<T, 1>(v, s);
}

template <typename T, bool VEC>
cudaError_t rowdot_dispatch_v(const View3& v, cudaStream_t s)
{
    dim3 grid((unsigned)ceil_div(v.outer, 256)), block(256);
    if (v.m <= 1) rowdot_kernel<T, 1, VEC><<<grid, block, 0, s>>>(v);
    else if (v.m <= 2) rowdot_kernel<T, 2, VEC><<<grid, block, 0, s>>>(v);
    else if (v.m <= 4) rowdot_kernel<T, 4, VEC><<<grid, block, 0, s>>>(v);
    else if (v.m <= 8) rowdot_kernel<T, 8, VEC><<<grid, block, 0, s>>>(v);
    else rowdot_kernel<T, 16, VEC><<<grid, block, 0, s>>>(v);
    return cudaGetLastError();
}

template <typename T, int MB, bool STAGE>
cudaError_t rowflat_launch_s(const View3& v, cudaStream_t s)
{
    // rows per warp: about 4 KB of A, a multiple of 32, with the block's tiles, B and the output
    // staging (8 warps x 32 rows x (m | 1)) within 44 KB of shared memory where that allows 32 rows
    const int64_t es = (int64_t)sizeof(T), ms = STAGE ? (v.m | 1) : 0;
    const int64_t fixed = 16 * 16 * es + 8 * 32 * ms * es;
    const int64_t want = 4096 / (v.nq * es);
    const int64_t cap = (44 * 1024 - fixed) / (8 * (v.nq + 1) * es);
    const int wr = (int)std::max<int64_t>(32, std::min(want, cap) / 32 * 32);
    const size_t smem = ((size_t)8 * wr * (v.nq + 1) + (size_t)v.nq * (MB < 4 ? 4 : MB) + (size_t)8 * 32 * ms) * sizeof(T);
    const int64_t blocks = ceil_div(v.outer, (int64_t)8 * wr);
    if (smem > 48 * 1024) {
        // staged double outputs of m up to 16 with 32-row tiles: up to 70 KB
        const cudaError_t e = cudaFuncSetAttribute(rowflat_kernel<T, MB, STAGE>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    rowflat_kernel<T, MB, STAGE><<<(unsigned)blocks, 256, smem, s>>>(v, wr);
    return cudaGetLastError();
}

// Staged (coalesced) output stores where a row's outputs take at least 64 bytes, or at least 32
// bytes with fibres of at most 4 elements (measured on A of 2^26 elements, n_q 2..16, m 4..16).
template <typename T, int MB>
cudaError_t rowflat_launch(const View3& v, cudaStream_t s)
{
    const int64_t ob = v.m * (int64_t)sizeof(T);
    const bool stage = ob >= 64 || (ob >= 32 && v.nq <= 4);
    return stage ? rowflat_launch_s<T, MB, true>(v, s) : rowflat_launch_s<T, MB, false>(v, s);
}

template <typename T, int NQ>
cudaError_t rowspan_launch(const View3& v, cudaStream_t s)
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t spans = ceil_div(v.outer, (int64_t)(64 / sizeof(T) / NQ));
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(spans, 256), (int64_t)sms * 16));
    if (v.m <= 1) rowspan_kernel<T, 1, NQ><<<blocks, 256, 0, s>>>(v);
    else if (v.m <= 2) rowspan_kernel<T, 2, NQ><<<blocks, 256, 0, s>>>(v);
    else if (v.m <= 4) rowspan_kernel<T, 4, NQ><<<blocks, 256, 0, s>>>(v);
    else if (v.m <= 8) rowspan_kernel<T, 8, NQ><<<blocks, 256, 0, s>>>(v);
    else rowspan_kernel<T, 16, NQ><<<blocks, 256, 0, s>>>(v);
    return cudaGetLastError();
}

template <typename T>
cudaError_t rowdot_dispatch(const View3& v, cudaStream_t s)
{
    const int64_t span = 64 / (int64_t)sizeof(T);
    const int64_t mb = v.m <= 1 ? 1 : v.m <= 2 ? 2 : v.m <= 4 ? 4 : v.m <= 8 ? 8 : 16;
    if (aligned16(v.a) && v.nq <= span && (span / v.nq) * mb * (int64_t)sizeof(T) <= 64) {
        switch (v.nq) {
        case 1: return rowspan_launch<T, 1>(v, s);
        case 2: return rowspan_launch<T, 2>(v, s);
        case 4: return rowspan_launch<T, 4>(v, s);
        case 8: return rowspan_launch<T, 8>(v, s);
        case 16: if constexpr (sizeof(T) == 4) return rowspan_launch<T, 16>(v, s); break;
        default: break;
        }
    }
    if (v.nq <= kFlatMaxNq) {
        if (v.m <= 1) return rowflat_launch<T, 1>(v, s);
        if (v.m <= 2) return rowflat_launch<T, 2>(v, s);
        if (v.m <= 4) return rowflat_launch<T, 4>(v, s);
        if (v.m <= 8) return rowflat_launch<T, 8>(v, s);
        return rowflat_launch<T, 16>(v, s);
    }
    constexpr int RV = 16 / sizeof(T);
    const bool vec = aligned16(v.a) && (v.nq % RV == 0);
    return vec ? rowdot_dispatch_v<T, true>(v, s) : rowdot_dispatch_v<T, false>(v, s);
}

// Sum of the `parts` partial results of a split K loop, in a fixed order: c[i] = sum_z ws[z][i].
template <typename T>
__global__ void __launch_bounds__(256) split_reduce_kernel(const T* __restrict__ ws, int parts, int64_t n, T* __restrict__ c)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T sum = ws[i];
        for (int z = 1; z < parts; ++z) sum += ws[(size_t)z * n + i];
        c[i] = sum;
    }
}

// ---------------------------------------------------------------------------------------------
// bvec: few output rows (R = outer * inner <= 8) and m <= 256: C[r][j] = sum_l A[r][l] B(j,l),
// bound by reading B (m x n_q), e.g. the order-1 product c = B a. Block b of G streams the
// contiguous l range [b lper, (b + 1) lper) of B; its partial C goes to ws[b][r][j] and
// bvec_reduce_kernel adds the G partials in a fixed order.
//   column-major B (B(j,l) = b[j + l m], the range is one contiguous block of B): thread =
//     (j vector jv of W consecutive j, l lane ls of LS); a warp's loads for one l are
//     consecutive; the LS lane partials are added in lane order at the end;
//   row-major B (B(j,l) = b[j n_q + l]): the range is cut into tiles of kBvecTile l; warp w owns
//     rows j = w, w + 8, ... and reads W consecutive l per lane (A's tile stays in L1 across the
//     rows); warp shuffles reduce, and the warp alone adds into its rows' shared partials.
// W = 16 / sizeof(T) when the vector accesses are aligned (VEC), else 1.
// ---------------------------------------------------------------------------------------------
constexpr int kBvecMaxR = 8, kBvecMaxM = 256, kBvecTile = 1024;
constexpr int64_t kBvecSmallMaxRows = 65536;   // small m: row tiles of 8 up to this many rows

// Offsets in A of (row r0 + r, l = 0) for the R rows of a row tile (r = k inner + i); A's element
// (row, l) is then at offset + l inner.
template <int R>
__device__ __forceinline__ void bvec_rows(const View3& v, int64_t r0, int Rv, int64_t (&off)[R])
{
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t row = r0 + (r < Rv ? r : 0);
        const int64_t k = row / v.inner, i = row - k * v.inner;
        off[r] = k * v.nq * v.inner + i;
    }
}

// A's element (row, l), row = k inner + i
template <typename T>
__device__ __forceinline__ T bvec_a(const T* __restrict__ A, const View3& v, int64_t row, int64_t l)
{
    const int64_t k = row / v.inner, i = row - k * v.inner;
    return __ldg(A + (k * v.nq + l) * v.inner + i);
}

template <typename T, int R, bool VEC>
__global__ void __launch_bounds__(256) bvec_cm_kernel(View3 v, int64_t lper, T* __restrict__ ws)
{
    constexpr int W = VEC ? 16 / (int)sizeof(T) : 1;
    extern __shared__ __align__(16) uint8_t bvec_smem[];
    T* red = reinterpret_cast<T*>(bvec_smem);                 // [LS][R][m]
    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    const int64_t m = v.m;
    const int JV = (int)((m + W - 1) / W), LS = 256 / JV;
    const int tid = threadIdx.x, jv = tid % JV, ls = tid / JV;
    const int64_t l0 = (int64_t)blockIdx.x * lper, l1 = l0 + lper < v.nq ? l0 + lper : v.nq;
    // rows r0 .. r0 + R - 1 of this block's row tile (blockIdx.y), Rv of them in A
    const int64_t r0 = (int64_t)blockIdx.y * R, rrem = v.outer * v.inner - r0;
    const int Rv = (int)(rrem < R ? rrem : R);
    int64_t aoff[R];
    bvec_rows<R>(v, r0, Rv, aoff);
    T acc[W][R];
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
        for (int r = 0; r < R; ++r) acc[w][r] = T(0);
    if (ls < LS) {
#pragma unroll 4
        for (int64_t l = l0 + ls; l < l1; l += LS) {
            T a[R];
#pragma unroll
            for (int r = 0; r < R; ++r) a[r] = r < Rv ? __ldg(A + aoff[r] + l * v.inner) : T(0);
            T b[W];
            const T* bp = B + l * m + (int64_t)jv * W;
            if constexpr (VEC) {
                typedef typename V16<T>::type VT;
                const VT x = __ldg(reinterpret_cast<const VT*>(bp));
#pragma unroll
                for (int w = 0; w < W; ++w) b[w] = reinterpret_cast<const T*>(&x)[w];
            } else {
                b[0] = __ldg(bp);
            }
#pragma unroll
            for (int w = 0; w < W; ++w)
#pragma unroll
                for (int r = 0; r < R; ++r) acc[w][r] = fma_t(a[r], b[w], acc[w][r]);
        }
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const int64_t j = (int64_t)jv * W + w;
            if (j < m) {
#pragma unroll
                for (int r = 0; r < R; ++r) red[((size_t)ls * R + r) * m + j] = acc[w][r];
            }
        }
    }
    __syncthreads();
    // ws[g][row][j] over all row tiles: this block's rows start at r0
    T* wb = ws + ((size_t)blockIdx.x * gridDim.y * R + (size_t)r0) * (size_t)m;
    for (int e = tid; e < R * m; e += 256) {
        T sum = red[e];
        for (int q = 1; q < LS; ++q) sum += red[(size_t)q * R * m + e];
        wb[e] = sum;
    }
}

template <typename T, int R, bool VEC>
__global__ void __launch_bounds__(256) bvec_rm_kernel(View3 v, int64_t lper, T* __restrict__ ws)
{
    constexpr int W = VEC ? 16 / (int)sizeof(T) : 1;
    __shared__ T part[R][kBvecMaxM];
    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    const int64_t m = v.m, nq = v.nq;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t l0 = (int64_t)blockIdx.x * lper, l1 = l0 + lper < nq ? l0 + lper : nq;
    const int64_t r0 = (int64_t)blockIdx.y * R, rrem = v.outer * v.inner - r0;
    const int Rv = (int)(rrem < R ? rrem : R);
    for (int e = tid; e < R * kBvecMaxM; e += 256) part[e / kBvecMaxM][e % kBvecMaxM] = T(0);
    __syncthreads();
    for (int64_t t0 = l0; t0 < l1; t0 += kBvecTile) {
        const int64_t t1 = t0 + kBvecTile < l1 ? t0 + kBvecTile : l1;
        for (int64_t j = warp; j < m; j += 8) {
            const T* bj = B + j * nq;
            T acc[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = T(0);
#pragma unroll 2
            for (int64_t l = t0 + (int64_t)lane * W; l < t1; l += 32 * W) {
                T b[W], a[W][R];
                if constexpr (VEC) {
                    typedef typename V16<T>::type VT;
                    const VT x = __ldg(reinterpret_cast<const VT*>(bj + l));
#pragma unroll
                    for (int w = 0; w < W; ++w) b[w] = reinterpret_cast<const T*>(&x)[w];
                    if constexpr (R == 1) {
                        // one row, inner == 1 (VEC requires it for R == 1): A's W values in one load
                        const VT y = __ldg(reinterpret_cast<const VT*>(A + l));
#pragma unroll
                        for (int w = 0; w < W; ++w) a[w][0] = reinterpret_cast<const T*>(&y)[w];
                    } else {
#pragma unroll
                        for (int w = 0; w < W; ++w)
#pragma unroll
                            for (int r = 0; r < R; ++r) a[w][r] = r < Rv ? bvec_a<T>(A, v, r0 + r, l + w) : T(0);
                    }
                } else {
                    b[0] = __ldg(bj + l);
#pragma unroll
                    for (int r = 0; r < R; ++r) a[0][r] = r < Rv ? bvec_a<T>(A, v, r0 + r, l) : T(0);
                }
#pragma unroll
                for (int w = 0; w < W; ++w)
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] = fma_t(a[w][r], b[w], acc[r]);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int r = 0; r < R; ++r) part[r][j] += acc[r];
            }
        }
    }
    __syncthreads();
    T* wb = ws + ((size_t)blockIdx.x * gridDim.y * R + (size_t)r0) * (size_t)m;
    for (int e = tid; e < R * m; e += 256) wb[e] = part[e / m][e % m];
}

// ws[g][r][j] -> C[k][j][i] (r = k inner + i): sum over the G block partials in block order.
template <typename T>
__global__ void __launch_bounds__(256) bvec_reduce_kernel(const T* __restrict__ ws, int G, View3 v, int R)
{
    T* C = static_cast<T*>(v.c);
    const int64_t n = (int64_t)R * v.m;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / v.m, j = e - r * v.m;
        if (r >= v.outer * v.inner) continue;
        T sum = T(0);
        for (int g = 0; g < G; ++g) sum += ws[(size_t)g * n + e];
        const int64_t k = r / v.inner, i = r - k * v.inner;
        C[(k * v.m + j) * v.inner + i] = sum;
    }
}

template <typename T, int R>
cudaError_t bvec_launch_r(const View3& v, dim3 G, int64_t lper, bool vec, T* ws, cudaStream_t s)
{
    if (v.b_cm) {
        constexpr int WV = 16 / (int)sizeof(T);
        const int W = vec ? WV : 1;
        const int JV = (int)((v.m + W - 1) / W), LS = 256 / JV;
        const size_t smem = (size_t)LS * R * v.m * sizeof(T);
        if (vec) bvec_cm_kernel<T, R, true><<<G, 256, smem, s>>>(v, lper, ws);
        else bvec_cm_kernel<T, R, false><<<G, 256, smem, s>>>(v, lper, ws);
    } else {
        if (vec) bvec_rm_kernel<T, R, true><<<G, 256, 0, s>>>(v, lper, ws);
        else bvec_rm_kernel<T, R, false><<<G, 256, 0, s>>>(v, lper, ws);
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t bvec_dispatch(const View3& v, int sms, cudaStream_t s, int* launches)
{
    constexpr int WV = 16 / (int)sizeof(T);
    const int64_t R = v.outer * v.inner;
    const int Rt = R <= 1 ? 1 : R <= 2 ? 2 : R <= 4 ? 4 : 8;
    // more than 8 rows (small m only): row tiles of 8 along the grid's y dimension
    const int64_t ty = ceil_div(R, Rt);
    // 16-byte accesses: B's j vectors (column-major) or l vectors (row-major; for one row also A's)
    bool vec = aligned16(v.b) && (v.b_cm ? v.m % WV == 0 : v.nq % WV == 0);
    if (!v.b_cm && Rt == 1) vec = vec && v.inner == 1 && aligned16(v.a);
    // contiguous l ranges of at least 4096 l, eight blocks per SM at most; starts on vector boundaries
    // (with row tiles: about eight blocks per SM over all tiles, l ranges of at least 1024 l)
    const int G = ty == 1 ? (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(v.nq, 4096), (int64_t)sms * 8))
                          : (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(v.nq, 1024), ceil_div((int64_t)sms * 8, ty)));
    const int64_t lper = ceil_div(ceil_div(v.nq, G), WV) * WV;
    const int Gr = (int)ceil_div(v.nq, lper);
    T* ws = nullptr;
    cudaError_t e = dev_malloc_async(reinterpret_cast<void**>(&ws), (size_t)Gr * ty * Rt * v.m * sizeof(T), s);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)Gr, (unsigned)ty);
    switch (Rt) {
    case 1: e = bvec_launch_r<T, 1>(v, grid, lper, vec, ws, s); break;
    case 2: e = bvec_launch_r<T, 2>(v, grid, lper, vec, ws, s); break;
    case 4: e = bvec_launch_r<T, 4>(v, grid, lper, vec, ws, s); break;
    default: e = bvec_launch_r<T, 8>(v, grid, lper, vec, ws, s); break;
    }
    if (e == cudaSuccess) {
        const int64_t n = ty * Rt * v.m;
        bvec_reduce_kernel<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), 1024)), 256, 0, s>>>(
            ws, Gr, v, (int)(ty * Rt));
        e = cudaGetLastError();
    }
    cudaFreeAsync(ws, s);
    if (launches) *launches = 2;
    return e;
}

int g_sms_simt = 0;

cudaError_t sms_of_device(int& sms)
{
    if (!g_sms_simt) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_sms_simt, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    sms = g_sms_simt;
    return cudaSuccess;
}

// Parts of the K loop for a slice-GEMM whose tiles cannot fill the GPU (1 when none is needed).
// `force` (a tuner's schedule): split whenever n_q >= 2048, into enough parts for two rounds of
// blocks.
template <typename T>
int gemm_split_parts(const View3& v, int sms, int64_t& lper, bool force = false)
{
    constexpr int RV = 16 / sizeof(T);
    constexpr int64_t BM = 32 * RV, BN = 32 * RV, BK = 8;
    const int64_t tiles = ceil_div(v.outer * v.inner, BM) * ceil_div(v.m, BN);
    const int64_t slots = (int64_t)sms * (sizeof(T) == 8 ? 3 : 2);
    lper = v.nq;
    if (v.nq < 2048 || (!force && tiles * 2 > slots)) return 1;
    int64_t S = std::min<int64_t>(ceil_div(slots, tiles), v.nq / 1024);
    if (force) S = std::max<int64_t>(2, std::min<int64_t>(ceil_div(2 * slots, tiles), v.nq / 1024));
    S = std::min<int64_t>(S, 256);
    // workspace of S partial results at most 1 GiB
    const int64_t nc = v.outer * v.m * v.inner;
    while (S > 1 && S * nc * (int64_t)sizeof(T) > (int64_t(1) << 30)) --S;
    if (S <= 1) return 1;
    lper = ceil_div(ceil_div(v.nq, S), BK) * BK;
    return (int)ceil_div(v.nq, lper);
}

template <typename T>
cudaError_t simt_gemm_launch(const View3& v, cudaStream_t s, int* launches, bool force)
{
    int sms = 0;
    cudaError_t e = sms_of_device(sms);
    if (e != cudaSuccess) return e;
    int64_t lper = 0;
    const int S = gemm_split_parts<T>(v, sms, lper, force);
    if (launches) *launches = S > 1 ? 2 : 1;
    if (S <= 1) return simt_gemm_dispatch<T>(v, s);
    const int64_t nc = v.outer * v.m * v.inner;
    T* ws = nullptr;
    if ((e = dev_malloc_async(reinterpret_cast<void**>(&ws), (size_t)S * nc * sizeof(T), s)) != cudaSuccess) return e;
    e = simt_gemm_dispatch<T>(v, s, S, lper, ws);
    if (e == cudaSuccess) {
        split_reduce_kernel<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(nc, 256), 4096)), 256, 0, s>>>(
            ws, S, nc, static_cast<T*>(v.c));
        e = cudaGetLastError();
    }
    cudaFreeAsync(ws, s);
    return e;
}

}  // namespace

cudaError_t launch_simt_gemm(const View3& v, int dtype, cudaStream_t s, int* launches, bool force_split)
{
    return dtype == 0 ? simt_gemm_launch<float>(v, s, launches, force_split)
                      : simt_gemm_launch<double>(v, s, launches, force_split);
}

int simt_gemm_launch_count(const View3& v, int dtype)
{
    int sms = 0;
    if (sms_of_device(sms) != cudaSuccess) return 1;
    int64_t lper = 0;
    const int S = dtype == 0 ? gemm_split_parts<float>(v, sms, lper) : gemm_split_parts<double>(v, sms, lper);
    return S > 1 ? 2 : 1;
}

bool bvec_supported(const View3& v)
{
    return v.m > kSmallM && v.m <= kBvecMaxM && v.outer * v.inner <= kBvecMaxR && v.nq >= 4096;
}

bool bvec_small_supported(const View3& v)
{
    const int64_t R = v.outer * v.inner;
    if (v.m < 1 || v.m > kSmallM) return false;
    if (R <= kBvecMaxR) return v.nq >= 4096;
    // row tiles: rows too few for the column and row kernels to fill the GPU, l long enough to
    // split (measured at m = 8, 16-4095 rows: against the row kernel from n_q = 1024 on, against
    // the column kernel's l-split form only for long l ranges)
    return R <= kBvecSmallMaxRows && v.nq >= (v.inner == 1 ? 1024 : 16384);
}

cudaError_t launch_bvec(const View3& v, int dtype, cudaStream_t s, int* launches)
{
    int sms = 0;
    cudaError_t e = sms_of_device(sms);
    if (e != cudaSuccess) return e;
    return dtype == 0 ? bvec_dispatch<float>(v, sms, s, launches) : bvec_dispatch<double>(v, sms, s, launches);
}

cudaError_t launch_colvec(const View3& v, int dtype, cudaStream_t s)
{
    return dtype == 0 ? colvec_dispatch<float>(v, s) : colvec_dispatch<double>(v, s);
}

cudaError_t launch_colvec_ls(const View3& v, int dtype, int ls, cudaStream_t s)
{
    constexpr int RF = 4, RD = 2;
    if (dtype == 0) {
        const bool vec = aligned16(v.a) && aligned16(v.c) && (v.inner % RF == 0);
        if (vec) return ls == 8 ? colvec_dispatch_ls<float, RF, 8>(v, s) : colvec_dispatch_ls<float, RF, 1>(v, s);
        return ls == 8 ? colvec_dispatch_ls<float, 1, 8>(v, s) : colvec_dispatch_ls<float, 1, 1>(v, s);
    }
    const bool vec = aligned16(v.a) && aligned16(v.c) && (v.inner % RD == 0);
    if (vec) return ls == 8 ? colvec_dispatch_ls<double, RD, 8>(v, s) : colvec_dispatch_ls<double, RD, 1>(v, s);
    return ls == 8 ? colvec_dispatch_ls<double, 1, 8>(v, s) : colvec_dispatch_ls<double, 1, 1>(v, s);
}

cudaError_t launch_rowdot(const View3& v, int dtype, cudaStream_t s)
{
    return dtype == 0 ? rowdot_dispatch<float>(v, s) : rowdot_dispatch<double>(v, s);
}

int grouped_blocks_per_sm(int dtype)
{
    int n = 0;
    cudaError_t e = dtype == 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, grouped_kernel<float>, 256, 0)
                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, grouped_kernel<double>, 256, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

cudaError_t launch_grouped(const GroupDesc* d_desc, int count, int64_t total, unsigned long long* queue, int dtype,
                           int grid, cudaStream_t s)
{
    if (dtype == 0) grouped_kernel<float><<<grid, 256, 0, s>>>(d_desc, count, total, queue);
    else grouped_kernel<double><<<grid, 256, 0, s>>>(d_desc, count, total, queue);
    return cudaGetLastError();
}

int grouped_small_blocks_per_sm(int dtype)
{
    int n = 0;
    cudaError_t e = dtype == 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, grouped_small_kernel<float>, 256, 0)
                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, grouped_small_kernel<double>, 256, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

cudaError_t launch_grouped_small(const GroupDesc* d_desc, int count, int64_t total, unsigned long long* queue,
                                 int dtype, int grid, cudaStream_t s)
{
    if (dtype == 0) grouped_small_kernel<float><<<grid, 256, 0, s>>>(d_desc, count, total, queue);
    else grouped_small_kernel<double><<<grid, 256, 0, s>>>(d_desc, count, total, queue);
    return cudaGetLastError();
}

cudaError_t launch_strided(const StridedProblem& sp, int dtype, cudaStream_t s)
{
    int64_t blocks = ceil_div(sp.total, 256);
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    if (dtype == 0) strided_kernel<float><<<(unsigned)blocks, 256, 0, s>>>(sp);
    else strided_kernel<double><<<(unsigned)blocks, 256, 0, s>>>(sp);
    return cudaGetLastError();
}

template <class T>
__global__ void __launch_bounds__(256) fill_kernel(T* __restrict__ p, int64_t n, T v)
{
    const int64_t step = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += step) p[i] = v;
}

cudaError_t launch_fill(void* p, int64_t n, int dtype, double v, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    int sms = 148;
    cudaError_t e = sms_of_device(sms);
    if (e != cudaSuccess) return e;
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), int64_t(sms) * 8);
    if (dtype == 0) fill_kernel<float><<<(unsigned)blocks, 256, 0, s>>>(static_cast<float*>(p), n, float(v));
    else fill_kernel<double><<<(unsigned)blocks, 256, 0, s>>>(static_cast<double*>(p), n, v);
    return cudaGetLastError();
}

}  // namespace tlibttm
