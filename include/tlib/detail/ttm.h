/*
 * Dispatch layer of the tlib::ttm C++ API onto the B200 library.
 *
 * The reference implements 21 detail::ttm overloads, one per policy-tag
 * combination, each slicing the tensor into CPU BLAS calls
 * (include/tlib/detail/ttm.h:391-1474). Here every combination forwards to
 * the same device planner behind the C ABI (include/tlibttm.h), which checks
 * the arguments with the reference's texts, picks a kernel and runs it on the
 * current CUDA device. Errors come back as std::runtime_error carrying the
 * library's message, like the reference's checks (include/tlib/ttm.h:65-90).
 *
 * Calls are synchronous: when ttm() returns, C holds the result, whether the
 * pointers are host or device memory.
 */
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../tlibttm.h"
#include "cases.h"
#include "layout.h"
#include "shape.h"
#include "strides.h"
#include "tags.h"

namespace tlib::ttm::detail
{

// Host core count, kept for callers that report per-core rates the way the
// reference's benchmark does (example/measure.cpp:113 reads detail::cores,
// defined at include/tlib/detail/ttm.h:60-96). The device planner does not use it.
inline unsigned get_number_cores()
{
    const unsigned n = std::thread::hardware_concurrency();
    return n == 0 ? 1u : n;
}
inline const unsigned cores = get_number_cores();

// Metadata arrays as std::size_t (copied when the caller's index type differs).
template <class size_type>
class size_t_array
{
public:
    size_t_array(size_type const* v, std::size_t n)
    {
        if constexpr (std::is_same_v<size_type, std::size_t>) {
            ptr_ = v;
        } else if (v) {
            buf_.assign(v, v + n);
            ptr_ = buf_.data();
        }
    }
    std::size_t const* get() const { return ptr_; }

private:
    std::vector<std::size_t> buf_;
    std::size_t const* ptr_ = nullptr;
};

template <class value_t, class size_type>
inline void ttm_device(unsigned const q, unsigned const p,
                       const value_t* a, size_type const* const na, size_type const* const wa, size_type const* const pia,
                       const value_t* b, size_type const* const nb, size_type const* const pib,
                       value_t* c, size_type const* const nc, size_type const* const wc)
{
    static_assert(std::is_same_v<value_t, float> || std::is_same_v<value_t, double>,
                  "tlib::ttm: element type must be float or double.");
    const size_t_array<size_type> na_(na, p), wa_(wa, p), pia_(pia, p), nb_(nb, 2), pib_(pib, 2),
        nc_(nc, p), wc_(wc, p);
    int rc;
    if constexpr (std::is_same_v<value_t, float>)
        rc = tlibttm_ttm_f32(q, p, a, na_.get(), wa_.get(), pia_.get(), b, nb_.get(), pib_.get(), c,
                             nc_.get(), wc_.get(), nullptr);
    else
        rc = tlibttm_ttm_f64(q, p, a, na_.get(), wa_.get(), pia_.get(), b, nb_.get(), pib_.get(), c,
                             nc_.get(), wc_.get(), nullptr);
    if (rc == TLIBTTM_OK) rc = tlibttm_synchronize(nullptr);
    if (rc != TLIBTTM_OK) throw std::runtime_error(tlibttm_last_error());
}

// Any (parallel, slicing, fusion) tag combination.
template <class value_t, class size_type, class parallel_policy, class slicing_policy, class fusion_policy>
inline void ttm(parallel_policy, slicing_policy, fusion_policy,
                unsigned const q, unsigned const p,
                const value_t* a, size_type const* const na, size_type const* const wa, size_type const* const pia,
                const value_t* b, size_type const* const nb, size_type const* const pib,
                value_t* c, size_type const* const nc, size_type const* const wc)
{
    ttm_device(q, p, a, na, wa, pia, b, nb, pib, c, nc, wc);
}

// The reference's overloads with a thread-split `ratio` (include/tlib/detail/ttm.h:843, 1258):
// the ratio has no meaning on the GPU and is ignored.
template <class value_t, class size_type, class slicing_policy>
inline void ttm(parallel_policy::parallel_loop_blas_t, slicing_policy, fusion_policy::all_t,
                unsigned const q, unsigned const p, double /*ratio*/,
                const value_t* a, size_type const* const na, size_type const* const wa, size_type const* const pia,
                const value_t* b, size_type const* const nb, size_type const* const pib,
                value_t* c, size_type const* const nc, size_type const* const wc)
{
    ttm_device(q, p, a, na, wa, pia, b, nb, pib, c, nc, wc);
}

} // namespace tlib::ttm::detail
