/*
 * Shape predicates of the tlib::ttm API (reference include/tlib/detail/shape.h:31-96).
 *
 *  valid   non-empty, no zero extent
 *  scalar  valid and all extents 1
 *  vector  one extent > 1 among the first two, the other 1, all later extents 1
 *          (a single extent > 1 for order 1)
 *  matrix  order >= 2, first two extents > 1, all later extents 1
 *  tensor  order >= 3 and some extent after the second > 1
 */
#pragma once

#include <algorithm>
#include <cstddef>
#include <iterator>
#include <stdexcept>
#include <vector>

namespace tlib::ttm::detail
{

template <class InputIt>
inline bool is_valid_shape(InputIt begin, InputIt end)
{
    if (begin == end) return false;
    for (; begin != end; ++begin)
        if (*begin == 0u) return false;
    return true;
}

template <class InputIt>
inline bool is_scalar(InputIt begin, InputIt end)
{
    if (!is_valid_shape(begin, end)) return false;
    for (; begin != end; ++begin)
        if (*begin != 1u) return false;
    return true;
}

template <class InputIt>
inline bool is_vector(InputIt begin, InputIt end)
{
    if (!is_valid_shape(begin, end)) return false;
    const auto n = std::distance(begin, end);
    if (n == 1) return *begin > 1u;
    const auto e0 = begin[0], e1 = begin[1];
    const bool one_big = (e0 > 1u) != (e1 > 1u);
    for (auto it = begin + 2; it != end; ++it)
        if (*it != 1u) return false;
    return one_big;
}

template <class InputIt>
inline bool is_matrix(InputIt begin, InputIt end)
{
    if (!is_valid_shape(begin, end)) return false;
    if (std::distance(begin, end) < 2) return false;
    if (!(begin[0] > 1u && begin[1] > 1u)) return false;
    for (auto it = begin + 2; it != end; ++it)
        if (*it != 1u) return false;
    return true;
}

template <class InputIt>
inline bool is_tensor(InputIt begin, InputIt end)
{
    if (!is_valid_shape(begin, end)) return false;
    if (std::distance(begin, end) < 3) return false;
    for (auto it = begin + 2; it != end; ++it)
        if (*it > 1u) return true;
    return false;
}

} // namespace tlib::ttm::detail
