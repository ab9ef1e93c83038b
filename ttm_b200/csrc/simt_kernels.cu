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
__device__ __forceinline__ void gemm_tile(const View3& v, int64_t m0, int64_t n0, GemmSmem<T>& sm)
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
    const int64_t inner = v.inner, nq = v.nq, m = v.m;
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
        abase[s] = k * inner * nq + i;
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
            if (j < m && l < nq) val = __ldg(BCM ? B + j + l * m : B + j * nq + l);
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

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

    const int64_t nk = ceil_div(nq, BK);
    load_tiles(0);
    store_tiles(0);
    __syncthreads();

    for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) load_tiles((kt + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
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

template <typename T, bool AK, bool VEC, bool BCM>
__global__ void __launch_bounds__(256) simt_gemm_kernel(View3 v)
{
    constexpr int RV = 16 / sizeof(T);
    __shared__ GemmSmem<T> sm;
    gemm_tile<T, AK, VEC, BCM>(v, (int64_t)blockIdx.x * (32 * RV), (int64_t)blockIdx.y * (32 * RV), sm);
}

// ---------------------------------------------------------------------------------------------
// colvec: small m, W consecutive i per thread (W | inner).
// ---------------------------------------------------------------------------------------------
template <typename T, int MB, int W>
__global__ void __launch_bounds__(256) colvec_kernel(View3 v)
{
    constexpr int LBS = 8192 / MB;   // l values per shared-memory chunk (32 KB f32 / 64 KB f64 max)
    constexpr int LB = (LBS * MB * sizeof(T) > 32768) ? 32768 / (MB * sizeof(T)) : LBS;
    __shared__ __align__(16) T Bs[LB][MB];

    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t inner = v.inner, nq = v.nq, m = v.m;
    const int64_t M = v.outer * inner;
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * W;
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
        for (int e = threadIdx.x; e < lc * MB; e += blockDim.x) {
            const int l = e / MB, j = e % MB;
            const int64_t gl = l0 + l;
            Bs[l][j] = (j < m) ? (v.b_cm ? B[j + gl * m] : B[j * nq + gl]) : T(0);
        }
        __syncthreads();
        if (valid) {
            const T* p = ap + l0 * inner;
#pragma unroll 4
            for (int l = 0; l < lc; ++l) {
                T a[W];
                load_vec<T, W>(a, p + (int64_t)l * inner);
#pragma unroll
                for (int j = 0; j < MB; ++j) {
                    const T bj = Bs[l][j];
#pragma unroll
                    for (int w = 0; w < W; ++w) acc[j][w] = fma_t(a[w], bj, acc[j][w]);
                }
            }
        }
    }
    if (valid) {
        T* cp = Cp + k * inner * m + i;
#pragma unroll
        for (int j = 0; j < MB; ++j)
            if (j < m) store_vec<T, W>(cp + j * inner, acc[j]);
    }
}

// ---------------------------------------------------------------------------------------------
// rowdot: small m, inner == 1. A group of G lanes reads one contiguous fibre A[k][0..nq).
// ---------------------------------------------------------------------------------------------
template <typename T, int MB, int G, int W, bool BSMEM>
__global__ void __launch_bounds__(256) rowdot_kernel(View3 v)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* Bs = reinterpret_cast<T*>(smem_raw);   // [m][nq], row-major in j

    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t nq = v.nq, m = v.m, rows = v.outer;

    if (BSMEM) {
        for (int64_t e = threadIdx.x; e < m * nq; e += blockDim.x) {
            const int64_t j = e / nq, l = e - j * nq;
            Bs[e] = v.b_cm ? B[j + l * m] : B[j * nq + l];
        }
        __syncthreads();
    }
    const int lane = threadIdx.x % G;
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const bool valid = row < rows;

    T acc[MB];
#pragma unroll
    for (int j = 0; j < MB; ++j) acc[j] = T(0);
    if (valid) {
        const T* ap = A + row * nq;
        for (int64_t l = (int64_t)lane * W; l < nq; l += (int64_t)G * W) {
            T a[W];
            load_vec<T, W>(a, ap + l);
#pragma unroll
            for (int j = 0; j < MB; ++j) {
                if (j < m) {
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const T bj = BSMEM ? Bs[j * nq + l + w]
                                           : __ldg(v.b_cm ? B + j + (l + w) * m : B + j * nq + l + w);
                        acc[j] = fma_t(a[w], bj, acc[j]);
                    }
                }
            }
        }
    }
    // All lanes (valid or not) take part in the shuffles: G divides 32.
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
        for (int j = 0; j < MB; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], off);
    if (valid && lane == 0) {
#pragma unroll
        for (int j = 0; j < MB; ++j)
            if (j < m) Cp[row * m + j] = acc[j];
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
__device__ __forceinline__ void gemv_rows(const View3& v, int64_t row0, T* bsm)
{
    constexpr int MB = 16;
    constexpr int LB = (int)(sizeof(GemmSmem<T>) / sizeof(T)) / MB;
    const T* __restrict__ A = static_cast<const T*>(v.a);
    const T* __restrict__ B = static_cast<const T*>(v.b);
    T* __restrict__ Cp = static_cast<T*>(v.c);
    const int64_t inner = v.inner, nq = v.nq, m = v.m;
    const int64_t M = v.outer * inner;
    const int64_t row = row0 + threadIdx.x;
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
        for (int e = threadIdx.x; e < lc * MB; e += blockDim.x) {
            const int l = e / MB, j = e % MB;
            const int64_t gl = l0 + l;
            bsm[e] = (j < m) ? (v.b_cm ? B[j + gl * m] : B[j * nq + gl]) : T(0);
        }
        __syncthreads();
        if (valid) {
            for (int l = 0; l < lc; ++l) {
                const T a = __ldg(ap + (l0 + l) * inner);
#pragma unroll
                for (int j = 0; j < MB; ++j) acc[j] = fma_t(a, bsm[l * MB + j], acc[j]);
            }
        }
    }
    if (valid) {
        T* cp = Cp + k * inner * m + i;
#pragma unroll
        for (int j = 0; j < MB; ++j)
            if (j < m) cp[j * inner] = acc[j];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) grouped_kernel(const GroupDesc* __restrict__ desc, int count, int64_t total,
                                                      unsigned long long* queue)
{
    constexpr int RV = 16 / sizeof(T);
    constexpr int BM = 32 * RV, BN = 32 * RV;
    __shared__ GemmSmem<T> sm;
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
                if (vec) { if (g.b_cm) gemm_tile<T, true, true, true>(v, m0, n0, sm); else gemm_tile<T, true, true, false>(v, m0, n0, sm); }
                else     { if (g.b_cm) gemm_tile<T, true, false, true>(v, m0, n0, sm); else gemm_tile<T, true, false, false>(v, m0, n0, sm); }
            } else {
                if (vec) { if (g.b_cm) gemm_tile<T, false, true, true>(v, m0, n0, sm); else gemm_tile<T, false, true, false>(v, m0, n0, sm); }
                else     { if (g.b_cm) gemm_tile<T, false, false, true>(v, m0, n0, sm); else gemm_tile<T, false, false, false>(v, m0, n0, sm); }
            }
        } else {
            gemv_rows<T>(v, local * kGemvRows, reinterpret_cast<T*>(&sm));
        }
        __syncthreads();
    }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename T>
cudaError_t simt_gemm_dispatch(const View3& v, cudaStream_t s)
{
    constexpr int RV = 16 / sizeof(T);
    constexpr int BM = 32 * RV, BN = 32 * RV;
    const bool ak = v.inner == 1;
    bool vec = aligned16(v.a) && aligned16(v.c);
    if (ak) vec = vec && (v.nq % RV == 0) && (v.m % RV == 0);
    else vec = vec && (v.inner % RV == 0);
    const int64_t M = v.outer * v.inner;
    dim3 grid((unsigned)ceil_div(M, BM), (unsigned)ceil_div(v.m, BN));
    dim3 block(256);
#define TLIBTTM_GEMM(AKv, VECv, BCMv) simt_gemm_kernel<T, AKv, VECv, BCMv><<<grid, block, 0, s>>>(v)
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

template <typename T, int W>
cudaError_t colvec_dispatch_w(const View3& v, cudaStream_t s)
{
    const int64_t M = v.outer * v.inner;
    const int64_t threads = ceil_div(M, W);
    dim3 grid((unsigned)ceil_div(threads, 256)), block(256);
    if (v.m <= 1) colvec_kernel<T, 1, W><<<grid, block, 0, s>>>(v);
    else if (v.m <= 2) colvec_kernel<T, 2, W><<<grid, block, 0, s>>>(v);
    else if (v.m <= 4) colvec_kernel<T, 4, W><<<grid, block, 0, s>>>(v);
    else if (v.m <= 8) colvec_kernel<T, 8, W><<<grid, block, 0, s>>>(v);
    else colvec_kernel<T, 16, W><<<grid, block, 0, s>>>(v);
    return cudaGetLastError();
}

template <typename T>
cudaError_t colvec_dispatch(const View3& v, cudaStream_t s)
{
    constexpr int RV = 16 / sizeof(T);
    const bool vec = aligned16(v.a) && aligned16(v.c) && (v.inner % RV == 0);
    return vec ? colvec_dispatch_w<T, RV>(v, s) : colvec_dispatch_w<T, 1>(v, s);
}

template <typename T, int MB, int G, int W>
cudaError_t rowdot_launch(const View3& v, cudaStream_t s)
{
    const size_t bbytes = (size_t)(v.m * v.nq) * sizeof(T);
    const bool bsm = bbytes <= 48 * 1024;
    const int64_t threads = v.outer * G;
    dim3 grid((unsigned)ceil_div(threads, 256)), block(256);
    if (bsm) rowdot_kernel<T, MB, G, W, true><<<grid, block, bbytes, s>>>(v);
    else rowdot_kernel<T, MB, G, W, false><<<grid, block, 0, s>>>(v);
    return cudaGetLastError();
}

template <typename T, int MB>
cudaError_t rowdot_dispatch_m(const View3& v, cudaStream_t s)
{
    constexpr int RV = 16 / sizeof(T);
    const bool vec = aligned16(v.a) && (v.nq % RV == 0);
    const bool wide = v.nq >= 32 * RV;
    if (vec) return wide ? rowdot_launch<T, MB, 32, RV>(v, s) : rowdot_launch<T, MB, 4, RV>(v, s);
    return wide ? rowdot_launch<T, MB, 32, 1>(v, s) : rowdot_launch<T, MB, 4, 1>(v, s);
}

template <typename T>
cudaError_t rowdot_dispatch(const View3& v, cudaStream_t s)
{
    return v.m <= 4 ? rowdot_dispatch_m<T, 4>(v, s) : rowdot_dispatch_m<T, 16>(v, s);
}

}  // namespace

cudaError_t launch_simt_gemm(const View3& v, int dtype, cudaStream_t s)
{
    return dtype == 0 ? simt_gemm_dispatch<float>(v, s) : simt_gemm_dispatch<double>(v, s);
}

cudaError_t launch_colvec(const View3& v, int dtype, cudaStream_t s)
{
    return dtype == 0 ? colvec_dispatch<float>(v, s) : colvec_dispatch<double>(v, s);
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

cudaError_t launch_strided(const StridedProblem& sp, int dtype, cudaStream_t s)
{
    int64_t blocks = ceil_div(sp.total, 256);
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    if (dtype == 0) strided_kernel<float><<<(unsigned)blocks, 256, 0, s>>>(sp);
    else strided_kernel<double><<<(unsigned)blocks, 256, 0, s>>>(sp);
    return cudaGetLastError();
}

}  // namespace tlibttm
