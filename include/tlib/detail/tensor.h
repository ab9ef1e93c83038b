/*
 * Host tensor container of the tlib::ttm C++ API (same interface as the
 * reference include/tlib/detail/tensor.h:39-189): a std::vector holding the
 * elements in the order given by a layout pi, its shape, and a view
 * A(q) that carries the contraction mode for `A(q) * B`.
 */
#pragma once

#include <cstddef>
#include <functional>
#include <numeric>
#include <ostream>
#include <stdexcept>
#include <vector>

#include "layout.h"
#include "shape.h"
#include "strides.h"

namespace tlib::ttm
{

template <class value_t>
class tensor;

template <class _value_t>
struct tensor_view
{
public:
    using value_t = _value_t;
    using tensor_t = tensor<value_t>;
    tensor_view() = delete;
    tensor_view(tensor_view const&) = delete;
    tensor_view& operator=(tensor_view const&) = delete;
    inline tensor_t const& get_tensor() const { return _tensor; }
    inline std::size_t contraction_mode() const { return _q; }

private:
    friend class tensor<value_t>;
    tensor_view(tensor_t const& t, std::size_t q) : _tensor(t), _q(q) {}
    tensor_t const& _tensor;
    std::size_t _q;
};

template <class value_t>
class tensor
{
public:
    using shape_t = std::vector<std::size_t>;
    using layout_t = std::vector<std::size_t>;
    using strides_t = std::vector<std::size_t>;
    using vector_t = std::vector<value_t>;
    using tensor_view_t = tensor_view<value_t>;

    tensor() = delete;

    tensor(shape_t const& n, layout_t const& pi)
        : _n(n), _pi(pi), _data(std::accumulate(n.begin(), n.end(), std::size_t{1}, std::multiplies<>()))
    {
        if (n.size() != pi.size())
            throw std::runtime_error("Error in tlib::tensor: shape vector and layout vector must have the same length.");
        if (!detail::is_valid_shape(n.begin(), n.end()))
            throw std::runtime_error("Error in tlib::tensor: shape vector of tensor is not valid.");
        if (!detail::is_valid_layout(pi.begin(), pi.end()))
            throw std::runtime_error("Error in tlib::tensor: layout vector of tensor is not valid.");
    }

    explicit tensor(shape_t const& n) : tensor(n, detail::generate_k_order_layout(n.size(), std::size_t{1})) {}

    tensor& operator=(value_t v)
    {
        std::fill(_data.begin(), _data.end(), v);
        return *this;
    }

    tensor_view_t operator()(std::size_t contraction_mode) const
    {
        if (1ul > contraction_mode || contraction_mode > this->order())
            throw std::runtime_error("Error in tlib::tensor: specified contraction mode should be greater than one and equal to or less than the order.");
        return tensor_view_t(*this, contraction_mode);
    }

    auto begin() const { return _data.begin(); }
    auto end() const { return _data.end(); }
    decltype(auto) begin() { return _data.begin(); }
    decltype(auto) end() { return _data.end(); }

    auto const& data() const { return _data; }
    auto& data() { return _data; }
    auto const& shape() const { return _n; }
    auto const& layout() const { return _pi; }
    auto strides() const { return detail::generate_strides(_n, _pi); }
    auto order() const { return _n.size(); }

    auto const& operator[](std::size_t k) const { return _data[k]; }
    auto& operator[](std::size_t k) { return _data[k]; }

private:
    shape_t _n;
    layout_t _pi;
    vector_t _data;
};

} // namespace tlib::ttm

// MATLAB-style printing. The text is part of the interface (callers' output is compared
// against the reference's), so it follows this format exactly; `v` is an element printed with
// the stream's own formatting, elements taken in memory order of the named modes:
//   order 1:  "[ \n"   then "v, " for each i1   then "];\n"
//   order 2:  "[ ... \n"  then per i2: "v, " for each i1, then "...\n"  then "];\n"
//   order p >= 3: nested blocks. Level r >= 3 opens with "cat(r,...\n", holds one level-(r-1)
//     block per index of mode r, and closes with ");\n" when r == p, else "), ...\n". The
//     innermost level-2 block is "[ ... \n", then per i1 the elements over i2 joined by ", " and
//     ended by "; ...\n", then "],...\n".
namespace tlib::ttm::detail
{
template <class value_type>
void print_level2(std::ostream& out, tlib::ttm::tensor<value_type> const& a, std::size_t base)
{
    const auto w = a.strides();
    const auto& n = a.shape();
    out << "[ ... " << std::endl;
    for (std::size_t r = 0; r < n[0]; ++r) {
        const std::size_t row = base + r * w[0];
        for (std::size_t c = 0; c < n[1]; ++c) out << a[row + c * w[1]] << (c + 1 < n[1] ? ", " : "; ...");
        out << std::endl;
    }
    out << "],..." << std::endl;
}
} // namespace tlib::ttm::detail

template <class value_type>
std::ostream& operator<<(std::ostream& out, tlib::ttm::tensor<value_type> const& a)
{
    const auto w = a.strides();
    const auto& n = a.shape();
    const std::size_t p = a.order();
    if (p == 1u) {
        out << "[ " << std::endl;
        for (std::size_t i = 0; i < n[0]; ++i) out << a[i * w[0]] << ", ";
        out << "];" << std::endl;
        return out;
    }
    if (p == 2u) {
        out << "[ ... " << std::endl;
        for (std::size_t c = 0; c < n[1]; ++c) {
            for (std::size_t r = 0; r < n[0]; ++r) out << a[c * w[1] + r * w[0]] << ", ";
            out << "..." << std::endl;
        }
        out << "];" << std::endl;
        return out;
    }
    // p >= 3: walk modes 3..p as an odometer (mode 3 fastest), opening and closing the
    // cat(...) levels as their indices start and wrap.
    std::vector<std::size_t> idx(p + 1, 0);
    for (std::size_t r = p; r >= 3; --r) out << "cat(" << r << ",..." << std::endl;
    while (true) {
        std::size_t base = 0;
        for (std::size_t r = 3; r <= p; ++r) base += idx[r] * w[r - 1];
        tlib::ttm::detail::print_level2(out, a, base);
        std::size_t r = 3;
        for (; r <= p; ++r) {
            if (++idx[r] < n[r - 1]) break;
            idx[r] = 0;
            out << (r == p ? ");" : "), ...") << std::endl;
        }
        if (r > p) break;
        for (std::size_t s = r - 1; s >= 3; --s) out << "cat(" << s << ",..." << std::endl;
    }
    return out;
}
