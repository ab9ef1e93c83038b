/*
 * Layout (index permutation) helpers of the tlib::ttm API.
 *
 * A layout pi is a one-based permutation of the modes 1..p listing them from
 * the fastest-varying (pi[0]) to the slowest (pi[p-1]). "k-order" layouts are
 * (k, k-1, ..., 1, k+1, ..., p); k = 1 is first-order (column-major), k = p
 * (or 0) last-order (row-major). Names, signatures and results match the
 * reference (include/tlib/detail/layout.h:29-144).
 */
#pragma once

#include <algorithm>
#include <cassert>
#include <iterator>
#include <stdexcept>
#include <type_traits>
#include <vector>

namespace tlib::ttm::detail
{

// True iff [begin,end) is a non-empty permutation of 1..n (reference layout.h:29-55).
template <class InputIt>
inline bool is_valid_layout(InputIt begin, InputIt end)
{
    const auto n = std::distance(begin, end);
    if (n <= 0) return false;
    for (auto it = begin; it != end; ++it) {
        const auto v = *it;
        if (v == 0u || static_cast<std::size_t>(v) > static_cast<std::size_t>(n)) return false;
        if (std::find(std::next(it), end, v) != end) return false;
    }
    return true;
}

// Writes the k-order layout into [begin,end); k == 0 means last-order (reference layout.h:57-76).
template <class OutputIt, class size_t>
inline void compute_k_order_layout(OutputIt begin, OutputIt end, size_t k)
{
    const auto n_signed = std::distance(begin, end);
    if (n_signed <= 0)
        throw std::runtime_error("Error in tlib::ttm::detail::compute_k_order: range provided by begin and end not correct!");
    using value_t = typename std::iterator_traits<OutputIt>::value_type;
    const auto n = static_cast<std::size_t>(n_signed);
    std::size_t kk = static_cast<std::size_t>(k);
    if (kk == 0u) kk = n;
    const std::size_t head = std::min(kk, n);
    std::size_t r = 0;
    for (auto it = begin; it != end; ++it, ++r)
        *it = static_cast<value_t>(r < head ? head - r : r + 1);
}

template <class size_t>
inline auto generate_k_order_layout(size_t p, size_t k)
{
    std::vector<size_t> v(p);
    compute_k_order_layout(v.begin(), v.end(), k);
    return v;
}

template <class InputIt>
inline bool is_first_order(InputIt begin, InputIt end)
{
    using value_type = typename std::iterator_traits<InputIt>::value_type;
    value_type expect = 1;
    for (; begin != end; ++begin, ++expect)
        if (*begin != expect) return false;
    return true;
}

template <class InputIt>
inline bool is_last_order(InputIt begin, InputIt end)
{
    using value_type = typename std::iterator_traits<InputIt>::value_type;
    auto expect = static_cast<value_type>(std::distance(begin, end));
    for (; begin != end; ++begin, --expect)
        if (*begin != expect) return false;
    return true;
}

template <class OutputIt>
inline void compute_first_order_layout(OutputIt begin, OutputIt end)
{
    compute_k_order_layout(begin, end, 1u);
}

template <class OutputIt>
inline void compute_last_order_layout(OutputIt begin, OutputIt end)
{
    compute_k_order_layout(begin, end, 0u);
}

// One-based position of the one-based `mode` in the layout, i.e. pi^{-1}(mode)
// (reference layout.h:120-144, same exception texts).
template <class InputIt, class SizeType>
inline auto inverse_mode(InputIt layout_begin, InputIt layout_end, SizeType mode)
{
    using value_type = typename std::iterator_traits<InputIt>::value_type;
    if (!is_valid_layout(layout_begin, layout_end))
        throw std::runtime_error("Error in tlib::ttm::detail::inverse_mode(): input layout is not valid.");
    const auto p_signed = std::distance(layout_begin, layout_end);
    if (p_signed <= 0)
        throw std::runtime_error("Error in tlib::ttm::detail::inverse_mode(): input layout is invalid.");
    const auto p = static_cast<value_type>(p_signed);
    if (mode == 0u || mode > SizeType(p))
        throw std::runtime_error("Error in tlib::ttm::detail::inverse_mode(): mode should be one-based and equal to or less than layout size.");
    value_type r = 0;
    while (r < p && layout_begin[r] != value_type(mode)) ++r;
    assert(r < p);
    return static_cast<value_type>(r + 1);
}

} // namespace tlib::ttm::detail
