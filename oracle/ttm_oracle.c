/*
 * CPU oracle for the mode-q tensor-times-matrix product.
 *
 * TEST INFRASTRUCTURE ONLY. This file restates, in plain C, the algorithm of
 * the reference tlib::ttm (bassoy/ttm) so that the CUDA path can be checked
 * against it. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it, and only as the checker. The product library never links,
 * loads or calls it.
 *
 * Pinning: tests/test_oracle.py checks this restatement against (1) the
 * closed-form known answers of the reference's own unit test
 * (test/src/gtest_tlib_ttm.cpp:29-134) and (2) outputs of the reference
 * itself, compiled from its headers with OpenBLAS (oracle/_ref, see
 * oracle/Makefile), committed as fixtures under tests/golden/.
 *
 * Semantics restated (reference file:line):
 *   C(i1..j..ip) = sum_{iq} A(i1..iq..ip) * B(j,iq)           README.md:13-18
 *   argument checks and their messages                         include/tlib/ttm.h:65-90
 *   case classification 1..8                                   include/tlib/detail/cases.h:25-37
 *   qhat = pi^{-1}(q)                                          include/tlib/detail/layout.h:120-144
 *   nnq = n[pi1]*..*n[pi(qhat-1)],  num = n[pi(qhat+1)]*..*n[pip]
 *                                                              include/tlib/detail/ttm.h:1150-1171
 *   outer slice step of A and C = w[pi(qhat+1)] (case 8)        include/tlib/detail/ttm.h:1159-1160
 *   per slice: C_k(nnq x m) = A_k(nnq x nq) * B^T, beta = 0     include/tlib/detail/ttm.h:1174-1190, mtm.h:90-97
 *   cases 1..7: one dense GEMM/GEMV over the whole tensor       include/tlib/detail/mtm.h:186-223
 *   B column-major iff pib[0] == 1                              include/tlib/detail/ttm.h:417
 *
 * Accumulation: the f64 oracle sums in long double (x87 80-bit, 64-bit
 * mantissa) and rounds once; the f32 oracle sums float inputs in double and
 * rounds once. Both are therefore at least as accurate as any BLAS ordering,
 * which is what a "relative error vs FP64 oracle" statement needs.
 */
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#define ORACLE_MSG_LEN 256
static _Thread_local char g_msg[ORACLE_MSG_LEN];

const char* oracle_last_error(void) { return g_msg; }

static int fail(const char* m)
{
    strncpy(g_msg, m, ORACLE_MSG_LEN - 1);
    g_msg[ORACLE_MSG_LEN - 1] = '\0';
    return 1;
}

/* include/tlib/detail/shape.h:31-35 */
static int valid_shape(const size_t* n, unsigned p)
{
    if (p == 0) return 0;
    for (unsigned r = 0; r < p; ++r) if (n[r] == 0) return 0;
    return 1;
}

/* include/tlib/detail/layout.h:29-55 */
static int valid_layout(const size_t* pi, unsigned p)
{
    if (p == 0) return 0;
    for (unsigned r = 0; r < p; ++r) {
        if (pi[r] == 0 || pi[r] > p) return 0;
        for (unsigned s = r + 1; s < p; ++s) if (pi[s] == pi[r]) return 0;
    }
    return 1;
}

/* include/tlib/detail/strides.h:76-101 (monotone along the layout) */
static int valid_strides(const size_t* pi, unsigned p, const size_t* w)
{
    if (p == 1 && w[0] == 1) return 1;
    for (unsigned r = 1; r < p; ++r)
        if (w[pi[r - 1] - 1] > w[pi[r] - 1]) return 0;
    return 1;
}

/* include/tlib/ttm.h:65-90, same order and messages */
static int check_args(unsigned q, unsigned p, const void* a, const size_t* na, const size_t* wa,
                      const size_t* pia, const void* b, const size_t* nb, const size_t* pib,
                      const void* c, const size_t* nc, const size_t* wc)
{
    const char* E = "Error in tlib::tensor_times_matrix: ";
    char buf[ORACLE_MSG_LEN];
#define FAIL(text) do { snprintf(buf, sizeof buf, "%s%s", E, text); return fail(buf); } while (0)
    if (p == 0) FAIL("input tensor order should be greater zero.");
    if (q == 0 || q > p) FAIL("contraction mode should be greater zero or less than or equal to p.");
    if (!a) FAIL("pointer to input tensor A should not be zero.");
    if (!b) FAIL("pointer to input vector B should not be zero.");
    if (!c) FAIL("pointer to output tensor C should not be zero.");
    if (!na) FAIL("pointer to input tensor shape vector na should not be zero.");
    if (!nb) FAIL("pointer to input vector shape vector nb should not be zero.");
    if (!nc) FAIL("pointer to output tensor shape vector nc should not be zero.");
    if (!wa) FAIL("pointer to input tensor stride vector wa should not be zero.");
    if (!wc) FAIL("pointer to output tensor stride vector wc should not be zero.");
    if (!pia) FAIL("pointer to input tensor permutation vector pia should not be zero.");
    if (na[q - 1] != nb[1]) FAIL("contraction dimension of A and B are not equal.");
    if (nc[q - 1] != nb[0]) FAIL("free dimension of C and B are not equal.");
    if (!valid_shape(na, p)) FAIL("shape vector of A is not valid.");
    if (!valid_shape(nc, p)) FAIL("shape vector of C is not valid.");
    if (!valid_layout(pia, p)) FAIL("layout vector of A is not valid.");
    if (!valid_strides(pia, p, wa)) FAIL("stride vector of A is not valid.");
    if (!valid_strides(pia, p, wc)) FAIL("stride vector of C is not valid.");
    (void)pib;
#undef FAIL
    g_msg[0] = '\0';
    return 0;
}

/* include/tlib/detail/cases.h:25-37 */
int oracle_case(unsigned p, size_t q, const size_t* pi)
{
    if (p == 1) return 1;
    if (p == 2) {
        if (q == 1 && pi[0] == 1) return 2;
        if (q == 2 && pi[0] == 1) return 3;
        if (q == 1 && pi[0] == 2) return 4;
        if (q == 2 && pi[0] == 2) return 5;
        return 0;
    }
    if (pi[0] == q) return 6;
    if (pi[p - 1] == q) return 7;
    return 8;
}

/* include/tlib/detail/layout.h:120-144 (one-based result) */
static unsigned inverse_mode(const size_t* pi, unsigned p, size_t q)
{
    for (unsigned r = 0; r < p; ++r) if (pi[r] == q) return r + 1;
    return 0;
}

/* include/tlib/detail/ttm.h:181-191: n[pi[start-1]] * ... * n[pi[finish-2]] */
static size_t product(const size_t* n, const size_t* pi, unsigned start, unsigned finish)
{
    size_t nn = 1;
    for (unsigned r = start - 1; r < finish - 1; ++r) nn *= n[pi[r] - 1];
    return nn;
}

/* The slice geometry every reference path reduces to. */
typedef struct {
    size_t inner;   /* nnq: product of extents before qhat in layout order */
    size_t nq;      /* contraction extent */
    size_t m;       /* rows of B */
    size_t outer;   /* number of subtensor slices */
    size_t astep;   /* pointer step between slices of A */
    size_t cstep;   /* pointer step between slices of C */
    int b_cm;       /* B column-major */
} geom_t;

static void make_geom(unsigned q, unsigned p, const size_t* na, const size_t* wa, const size_t* pia,
                      const size_t* nb, const size_t* pib, const size_t* wc, geom_t* g)
{
    unsigned qh = inverse_mode(pia, p, q);
    g->inner = product(na, pia, 1, qh);
    g->outer = product(na, pia, qh + 1, p + 1);
    g->nq = na[q - 1];
    g->m = nb[0];
    g->b_cm = pib[0] == 1;
    if (oracle_case(p, q, pia) == 8) {
        /* include/tlib/detail/ttm.h:1159-1160: waq = wa[pia[qh]-1] */
        g->astep = wa[pia[qh] - 1];
        g->cstep = wc[pia[qh] - 1];
    } else {
        /* mtm.h:186-223: one dense matrix, slices are contiguous */
        g->astep = g->inner * g->nq;
        g->cstep = g->inner * g->m;
    }
}

#define ORACLE_BODY(T, ACC)                                                              \
    _Pragma("omp parallel for collapse(2) schedule(static)")                             \
    for (size_t k = 0; k < g.outer; ++k)                                                 \
        for (size_t j = 0; j < g.m; ++j) {                                               \
            const T* ak = a + k * g.astep;                                               \
            T* ck = c + k * g.cstep + j * g.inner;                                       \
            for (size_t i = 0; i < g.inner; ++i) {                                       \
                ACC s = 0;                                                               \
                for (size_t l = 0; l < g.nq; ++l) {                                      \
                    T bv = g.b_cm ? b[j + l * g.m] : b[j * g.nq + l];                    \
                    s += (ACC)ak[l * g.inner + i] * (ACC)bv;                             \
                }                                                                        \
                ck[i] = (T)s;                                                            \
            }                                                                            \
        }

int oracle_ttm_f64(unsigned q, unsigned p, const double* a, const size_t* na, const size_t* wa,
                   const size_t* pia, const double* b, const size_t* nb, const size_t* pib,
                   double* c, const size_t* nc, const size_t* wc)
{
    if (check_args(q, p, a, na, wa, pia, b, nb, pib, c, nc, wc)) return 1;
    if (!pib) return fail("Error in tlib::tensor_times_matrix: pointer to input matrix layout vector pib should not be zero.");
    geom_t g;
    make_geom(q, p, na, wa, pia, nb, pib, wc, &g);
    ORACLE_BODY(double, long double)
    return 0;
}

int oracle_ttm_f32(unsigned q, unsigned p, const float* a, const size_t* na, const size_t* wa,
                   const size_t* pia, const float* b, const size_t* nb, const size_t* pib,
                   float* c, const size_t* nc, const size_t* wc)
{
    if (check_args(q, p, a, na, wa, pia, b, nb, pib, c, nc, wc)) return 1;
    if (!pib) return fail("Error in tlib::tensor_times_matrix: pointer to input matrix layout vector pib should not be zero.");
    geom_t g;
    make_geom(q, p, na, wa, pia, nb, pib, wc, &g);
    ORACLE_BODY(float, double)
    return 0;
}

/*
 * Sampled fibres, for checking full-size results whose dense oracle would
 * take too long: for each of nf (k, i) pairs, out[f*m + j] = C_k(j, i) in
 * double, accumulated in long double. A and B are f32 (dtype 0) or f64
 * (dtype 1). The caller guarantees the dense geometry (no checks here).
 */
int oracle_fibres(int dtype, unsigned q, unsigned p, const void* a, const size_t* na,
                  const size_t* wa, const size_t* pia, const void* b, const size_t* nb,
                  const size_t* pib, const size_t* wc, const size_t* fk, const size_t* fi,
                  size_t nf, double* out)
{
    geom_t g;
    make_geom(q, p, na, wa, pia, nb, pib, wc, &g);
    #pragma omp parallel for schedule(static)
    for (size_t f = 0; f < nf; ++f) {
        size_t k = fk[f], i = fi[f];
        for (size_t j = 0; j < g.m; ++j) {
            long double s = 0;
            for (size_t l = 0; l < g.nq; ++l) {
                size_t ai = k * g.astep + l * g.inner + i;
                size_t bi = g.b_cm ? j + l * g.m : j * g.nq + l;
                long double av = dtype ? ((const double*)a)[ai] : ((const float*)a)[ai];
                long double bv = dtype ? ((const double*)b)[bi] : ((const float*)b)[bi];
                s += av * bv;
            }
            out[f * g.m + j] = (double)s;
        }
    }
    return 0;
}
