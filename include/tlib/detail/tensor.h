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

// MATLAB-style printing, same format as the reference (tensor.h:131-189):
// order 1 as a row, order 2 as rows of mode 1, higher orders as nested cat(r, ...).
template <class value_type>
void stream_out(std::ostream& out, tlib::ttm::tensor<value_type> const& a, std::size_t j, unsigned r)
{
    const auto w = a.strides();
    const auto& n = a.shape();
    const auto p = a.order();
    if (r >= 3) {
        out << "cat(" << r << ",..." << std::endl;
        for (std::size_t ir = 0; ir < n[r - 1]; ++ir, j += w[r - 1]) stream_out(out, a, j, r - 1);
        out << (r == p ? ");" : "), ...") << std::endl;
    } else if (r == 2) {
        out << "[ ... " << std::endl;
        for (std::size_t i1 = 0; i1 < n[0]; ++i1, j += w[0]) {
            std::size_t j2 = 0;
            for (std::size_t i2 = 0; i2 + 1 < n[1]; ++i2, j2 += w[1]) out << a[j + j2] << ", ";
            out << a[j + j2] << "; ..." << std::endl;
        }
        out << "],..." << std::endl;
    }
}

template <class value_type>
std::ostream& operator<<(std::ostream& out, tlib::ttm::tensor<value_type> const& a)
{
    const auto w = a.strides();
    const auto& n = a.shape();
    const auto p = a.order();
    std::size_t j = 0;
    if (p == 1u) {
        out << "[ " << std::endl;
        for (std::size_t i1 = 0; i1 < n[0]; ++i1, j += w[0]) out << a[j] << ", ";
        out << "];" << std::endl;
    } else if (p == 2u) {
        out << "[ ... " << std::endl;
        for (std::size_t i2 = 0; i2 < n[1]; ++i2, j += w[1]) {
            std::size_t j2 = 0;
            for (std::size_t i1 = 0; i1 < n[0]; ++i1, j2 += w[0]) out << a[j + j2] << ", ";
            out << "..." << std::endl;
        }
        out << "];" << std::endl;
    } else {
        stream_out(out, a, j, static_cast<unsigned>(p));
    }
    return out;
}
