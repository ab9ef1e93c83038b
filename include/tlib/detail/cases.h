/*
 * Layout cases of a mode-q TTM (reference include/tlib/detail/cases.h:25-37).
 *
 *  1  p == 1                         (matrix-times-vector)
 *  2..5  p == 2, by q and pi[0]      (a single matrix-times-matrix)
 *  6  p >= 3, q == pi[0]             (contraction mode is the fastest: inner == 1)
 *  7  p >= 3, q == pi[p-1]           (contraction mode is the slowest: outer == 1)
 *  8  p >= 3, otherwise              (strided slices)
 *
 * The device planner does not branch on the case: all eight are instances of
 * the one slice view [outer][n_q][inner]. The classifier is kept because it
 * is part of the reference's public detail API and its tests.
 */
#pragma once

#include <cstddef>

namespace tlib::ttm::detail
{

template <unsigned case_nr>
inline constexpr bool is_case(unsigned p, std::size_t q, std::size_t const* const pi)
{
    static_assert(case_nr > 0u && case_nr < 9u, "tlib::ttm::detail::is_case: only 8 cases from 1 to 8 are covered.");
    if constexpr (case_nr == 1u) return p == 1u;
    else if constexpr (case_nr == 2u) return p == 2u && q == 1u && pi[0] == 1u;
    else if constexpr (case_nr == 3u) return p == 2u && q == 2u && pi[0] == 1u;
    else if constexpr (case_nr == 4u) return p == 2u && q == 1u && pi[0] == 2u;
    else if constexpr (case_nr == 5u) return p == 2u && q == 2u && pi[0] == 2u;
    else if constexpr (case_nr == 6u) return p >= 3u && pi[0] == q;
    else if constexpr (case_nr == 7u) return p >= 3u && pi[p - 1] == q;
    else return p >= 3u && !(pi[0] == q || pi[p - 1] == q);
}

} // namespace tlib::ttm::detail
