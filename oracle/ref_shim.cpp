/*
 * C-ABI wrapper around the UNMODIFIED reference tlib::ttm headers.
 *
 * TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles this file with
 * -I<reference>/include and links it against the bundled OpenBLAS, producing
 * oracle/_ref/libtlibttm_ref.so. Tests use it to pin the oracle and to make
 * golden fixtures; bench.py's reference arm times it on the host cores. The
 * product path never loads it.
 *
 * Each entry point calls the reference's own public low-level interface
 * tlib::ttm::ttm(ep,sp,fp, q,p, a,na,wa,pia, b,nb,pib, c,nc,wc)
 * (include/tlib/ttm.h:54-93) with one of the policy-tag combinations the
 * reference defines (include/tlib/detail/ttm.h:405-1474), and turns a thrown
 * std::runtime_error into a non-zero return plus the exception text.
 */
#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <vector>

#include <tlib/ttm.h>

namespace {

using namespace tlib::ttm;

// Policy ids. 0 is what operator* and ttmpy use (include/tlib/ttm.h:133-138).
enum policy_id {
    P_COMBINED = 0,
    P_SEQ_SLICE_NONE,
    P_SEQ_SUBT_NONE,
    P_BLAS_SLICE_NONE,
    P_BLAS_SUBT_NONE,
    P_BLAS_SLICE_ALL,
    P_BLAS_SUBT_ALL,
    P_LOOP_SLICE_OUTER,
    P_LOOP_SLICE_ALL,
    P_LOOP_SUBT_ALL,
    P_LOOPBLAS_SLICE_ALL,
    P_LOOPBLAS_SUBT_ALL,
    P_TASKLOOP_SLICE_NONE,
    P_TASKLOOP_SUBT_NONE,
    P_TASK_SLICE_NONE,
    P_TASK_SUBT_NONE,
    P_COUNT
};

template <class T>
int run(int policy, unsigned q, unsigned p,
        const T* a, const size_t* na, const size_t* wa, const size_t* pia,
        const T* b, const size_t* nb, const size_t* pib,
        T* c, const size_t* nc, const size_t* wc,
        char* err, size_t errlen)
{
    try {
        switch (policy) {
        case P_COMBINED:
            ttm(parallel_policy::combined, slicing_policy::combined, fusion_policy::all,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_SEQ_SLICE_NONE:
            ttm(parallel_policy::sequential, slicing_policy::slice, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_SEQ_SUBT_NONE:
            ttm(parallel_policy::sequential, slicing_policy::subtensor, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_BLAS_SLICE_NONE:
            ttm(parallel_policy::parallel_blas, slicing_policy::slice, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_BLAS_SUBT_NONE:
            ttm(parallel_policy::parallel_blas, slicing_policy::subtensor, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_BLAS_SLICE_ALL:
            ttm(parallel_policy::parallel_blas, slicing_policy::slice, fusion_policy::all,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_BLAS_SUBT_ALL:
            ttm(parallel_policy::parallel_blas, slicing_policy::subtensor, fusion_policy::all,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_LOOP_SLICE_OUTER:
            ttm(parallel_policy::parallel_loop, slicing_policy::slice, fusion_policy::outer,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_LOOP_SLICE_ALL:
            ttm(parallel_policy::parallel_loop, slicing_policy::slice, fusion_policy::all,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_LOOP_SUBT_ALL:
            ttm(parallel_policy::parallel_loop, slicing_policy::subtensor, fusion_policy::all,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_LOOPBLAS_SLICE_ALL:
            ttm(parallel_policy::parallel_loop_blas, slicing_policy::slice, fusion_policy::all,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_LOOPBLAS_SUBT_ALL:
            ttm(parallel_policy::parallel_loop_blas, slicing_policy::subtensor, fusion_policy::all,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_TASKLOOP_SLICE_NONE:
            ttm(parallel_policy::parallel_taskloop, slicing_policy::slice, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_TASKLOOP_SUBT_NONE:
            ttm(parallel_policy::parallel_taskloop, slicing_policy::subtensor, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_TASK_SLICE_NONE:
            ttm(parallel_policy::parallel_task, slicing_policy::slice, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        case P_TASK_SUBT_NONE:
            ttm(parallel_policy::parallel_task, slicing_policy::subtensor, fusion_policy::none,
                q, p, a, na, wa, pia, b, nb, pib, c, nc, wc); break;
        default:
            if (err && errlen) std::snprintf(err, errlen, "unknown policy id %d", policy);
            return 2;
        }
    } catch (std::exception const& e) {
        if (err && errlen) {
            std::strncpy(err, e.what(), errlen - 1);
            err[errlen - 1] = '\0';
        }
        return 1;
    }
    return 0;
}

} // namespace

extern "C" {

int tlibref_policy_count(void) { return P_COUNT; }

unsigned tlibref_cores(void) { return tlib::ttm::detail::cores; }

int tlibref_ttm_f32(int policy, unsigned q, unsigned p,
                    const float* a, const size_t* na, const size_t* wa, const size_t* pia,
                    const float* b, const size_t* nb, const size_t* pib,
                    float* c, const size_t* nc, const size_t* wc,
                    char* err, size_t errlen)
{
    return run<float>(policy, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc, err, errlen);
}

int tlibref_ttm_f64(int policy, unsigned q, unsigned p,
                    const double* a, const size_t* na, const size_t* wa, const size_t* pia,
                    const double* b, const size_t* nb, const size_t* pib,
                    double* c, const size_t* nc, const size_t* wc,
                    char* err, size_t errlen)
{
    return run<double>(policy, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc, err, errlen);
}

/* Layout / shape / stride helpers of the reference (include/tlib/detail/
 * layout.h, shape.h, strides.h), exported so tests can pin this project's
 * own helpers against them. Return 1 on success / true, 0 on false, -1 when
 * the reference throws. */
int tlibref_compute_k_order_layout(size_t* layout, size_t n, size_t k)
{
    try { tlib::ttm::detail::compute_k_order_layout(layout, layout + n, k); }
    catch (std::exception const&) { return -1; }
    return 1;
}

int tlibref_is_valid_layout(const size_t* layout, size_t n)
{
    return tlib::ttm::detail::is_valid_layout(layout, layout + n) ? 1 : 0;
}

int tlibref_inverse_mode(const size_t* layout, size_t n, size_t mode, size_t* out)
{
    try { *out = tlib::ttm::detail::inverse_mode(layout, layout + n, mode); }
    catch (std::exception const&) { return -1; }
    return 1;
}

int tlibref_compute_strides(const size_t* shape, size_t n, const size_t* layout, size_t* strides)
{
    try { tlib::ttm::detail::compute_strides(shape, shape + n, layout, strides); }
    catch (std::exception const&) { return -1; }
    return 1;
}

int tlibref_is_valid_strides(const size_t* layout, size_t n, const size_t* strides)
{
    try { return tlib::ttm::detail::is_valid_strides(layout, layout + n, strides) ? 1 : 0; }
    catch (std::exception const&) { return -1; }
}

int tlibref_shape_kind(const size_t* shape, size_t n)
{
    /* bit 0 valid, bit 1 scalar, bit 2 vector, bit 3 matrix, bit 4 tensor */
    using namespace tlib::ttm::detail;
    int r = 0;
    if (is_valid_shape(shape, shape + n)) r |= 1;
    if (is_scalar(shape, shape + n)) r |= 2;
    if (is_vector(shape, shape + n)) r |= 4;
    if (is_matrix(shape, shape + n)) r |= 8;
    if (is_tensor(shape, shape + n)) r |= 16;
    return r;
}

int tlibref_is_case(unsigned case_nr, unsigned p, size_t q, const size_t* pi)
{
    using namespace tlib::ttm::detail;
    switch (case_nr) {
    case 1: return is_case<1>(p, q, pi);
    case 2: return is_case<2>(p, q, pi);
    case 3: return is_case<3>(p, q, pi);
    case 4: return is_case<4>(p, q, pi);
    case 5: return is_case<5>(p, q, pi);
    case 6: return is_case<6>(p, q, pi);
    case 7: return is_case<7>(p, q, pi);
    case 8: return is_case<8>(p, q, pi);
    default: return -1;
    }
}

} // extern "C"
