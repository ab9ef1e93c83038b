/*
 * Stride helpers of the tlib::ttm API (reference include/tlib/detail/strides.h:31-101).
 *
 * compute_strides writes the dense strides of shape n under layout pi:
 * w[pi_1] = 1, w[pi_r] = w[pi_{r-1}] * n[pi_{r-1}]. Like the reference it
 * returns all-ones strides for scalar and vector shapes (and leaves ones for
 * shapes that are neither matrix nor tensor); addresses are unaffected
 * because the modes concerned have extent 1.
 *
 * is_valid_strides only checks that strides do not decrease along pi, which
 * is the reference's (weak) contract; the device planner separately decides
 * whether strides are dense enough for the slice kernels.
 */
#pragma once

#include <algorithm>
#include <array>
#include <cstddef>
#include <iterator>
#include <stdexcept>
#include <vector>

#include "layout.h"
#include "shape.h"

namespace tlib::ttm::detail
{

template <class InputIt1, class InputIt2, class OutputIt>
inline void compute_strides(InputIt1 shape_begin, InputIt1 shape_end, InputIt2 layout_begin, OutputIt strides_begin)
{
    if (!is_valid_shape(shape_begin, shape_end))
        throw std::runtime_error("Error in tlib::detail::compute_strides(): input shape is not valid.");
    const auto n = std::distance(shape_begin, shape_end);
    if (!is_valid_layout(layout_begin, layout_begin + n))
        throw std::runtime_error("Error in tlib::detail::compute_strides(): input layout is not valid.");

    std::fill(strides_begin, strides_begin + n, 1u);
    if (is_vector(shape_begin, shape_end) || is_scalar(shape_begin, shape_end)) return;
    if (!is_matrix(shape_begin, shape_end) && !is_tensor(shape_begin, shape_end)) return;

    for (std::ptrdiff_t r = 1; r < n; ++r) {
        const auto cur = layout_begin[r] - 1;
        const auto prev = layout_begin[r - 1] - 1;
        strides_begin[cur] = strides_begin[prev] * shape_begin[prev];
    }
}

template <class size_type>
inline auto generate_strides(std::vector<size_type> const& shape, std::vector<size_type> const& layout)
{
    auto strides = std::vector<size_type>(shape.size());
    compute_strides(shape.begin(), shape.end(), layout.begin(), strides.begin());
    return strides;
}

template <class size_type, std::size_t N>
inline auto generate_strides(std::array<size_type, N> const& shape, std::array<size_type, N> const& layout)
{
    static_assert(N > 0, "Static error in tlib::detail::generate_strides(): N, i.e. length of array should be greater than zero.");
    auto strides = std::array<size_type, N>{};
    compute_strides(shape.begin(), shape.end(), layout.begin(), strides.begin());
    return strides;
}

template <class InputIt1, class InputIt2>
inline bool is_valid_strides(InputIt1 layout_begin, InputIt1 layout_end, InputIt2 stride_begin)
{
    if (!is_valid_layout(layout_begin, layout_end))
        throw std::runtime_error("Error in tlib::detail::is_valid_strides(): input layout is not valid.");
    for (auto it = layout_begin; std::next(it) != layout_end; ++it)
        if (stride_begin[*it - 1] > stride_begin[*std::next(it) - 1]) return false;
    return true;
}

} // namespace tlib::ttm::detail
