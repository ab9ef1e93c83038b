/*
 * Device-resident tensor of the tlib::ttm C++ API.
 *
 * The reference's tensor (include/tlib/detail/tensor.h:59-121) keeps its elements in a host
 * std::vector, so every product on the GPU would copy A and B in and C out. device_tensor has
 * the same interface (shape, layout, strides, order, the A(q) view, assignment of a value) with
 * the elements in memory of the CUDA device that was current when it was made. ttm(q, A, B)
 * and A(q) * B on device tensors (include/tlib/ttm.h) run without host staging and return a
 * device tensor; to_host() and the constructor from a host tensor move data between the two.
 *
 * Memory comes from the library's allocator (tlibttm_device_alloc), so this header needs no
 * CUDA headers. A failed allocation throws std::bad_alloc, as std::vector does for the host
 * tensor; any other library error throws std::runtime_error with the library's message.
 * Copies are deep (device to device); moves transfer ownership.
 */
#pragma once

#include <cstddef>
#include <functional>
#include <new>
#include <numeric>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../tlibttm.h"
#include "layout.h"
#include "shape.h"
#include "strides.h"
#include "tensor.h"

namespace tlib::ttm
{

template <class value_t>
class device_tensor;

/** A(q) on a device tensor: the tensor and its contraction mode, for `A(q) * B`. */
template <class _value_t>
struct device_tensor_view
{
public:
    using value_t = _value_t;
    using tensor_t = device_tensor<value_t>;
    device_tensor_view() = delete;
    device_tensor_view(device_tensor_view const&) = delete;
    device_tensor_view& operator=(device_tensor_view const&) = delete;
    inline tensor_t const& get_tensor() const { return _tensor; }
    inline std::size_t contraction_mode() const { return _q; }

private:
    friend class device_tensor<value_t>;
    device_tensor_view(tensor_t const& t, std::size_t q) : _tensor(t), _q(q) {}
    tensor_t const& _tensor;
    std::size_t _q;
};

namespace detail
{
inline void device_check(int rc)
{
    if (rc == TLIBTTM_OK) return;
    if (rc == TLIBTTM_ERR_ALLOC) throw std::bad_alloc();
    throw std::runtime_error(tlibttm_last_error());
}

template <class value_t>
constexpr int dtype_of()
{
    static_assert(std::is_same_v<value_t, float> || std::is_same_v<value_t, double>,
                  "tlib::ttm::device_tensor: element type must be float or double.");
    return std::is_same_v<value_t, float> ? TLIBTTM_F32 : TLIBTTM_F64;
}
} // namespace detail

template <class value_t>
class device_tensor
{
public:
    using shape_t = std::vector<std::size_t>;
    using layout_t = std::vector<std::size_t>;
    using strides_t = std::vector<std::size_t>;
    using tensor_view_t = device_tensor_view<value_t>;
    using host_tensor_t = tensor<value_t>;

    device_tensor() = delete;

    /** Elements set to zero, like the host tensor's value-initialised vector. */
    device_tensor(shape_t const& n, layout_t const& pi) : device_tensor(n, pi, no_fill{}) { *this = value_t(0); }

    explicit device_tensor(shape_t const& n) : device_tensor(n, detail::generate_k_order_layout(n.size(), std::size_t{1})) {}

    /** Same checks, elements left unset: for outputs that a product overwrites whole. */
    static device_tensor uninitialized(shape_t const& n, layout_t const& pi) { return device_tensor(n, pi, no_fill{}); }

    /** Upload of a host tensor (same shape, layout and element order). */
    explicit device_tensor(host_tensor_t const& h) : _n(h.shape()), _pi(h.layout())
    {
        allocate();
        guarded([&] { detail::device_check(tlibttm_copy(_ptr, h.data().data(), bytes())); });
    }

    device_tensor(device_tensor const& o) : _n(o._n), _pi(o._pi)
    {
        allocate();
        guarded([&] { detail::device_check(tlibttm_copy(_ptr, o._ptr, bytes())); });
    }

    device_tensor(device_tensor&& o) noexcept : _n(std::move(o._n)), _pi(std::move(o._pi)), _ptr(o._ptr), _size(o._size)
    {
        o._ptr = nullptr;
        o._size = 0;
    }

    device_tensor& operator=(device_tensor const& o)
    {
        if (this != &o) {
            device_tensor t(o);
            swap(t);
        }
        return *this;
    }

    device_tensor& operator=(device_tensor&& o) noexcept
    {
        swap(o);
        return *this;
    }

    ~device_tensor() { tlibttm_device_free(_ptr); }

    /** Sets every element to v (enqueued on the default stream, then waited for). */
    device_tensor& operator=(value_t v)
    {
        detail::device_check(tlibttm_fill(detail::dtype_of<value_t>(), _ptr, _size, double(v), nullptr));
        detail::device_check(tlibttm_synchronize(nullptr));
        return *this;
    }

    tensor_view_t operator()(std::size_t contraction_mode) const
    {
        if (1ul > contraction_mode || contraction_mode > this->order())
            throw std::runtime_error("Error in tlib::tensor: specified contraction mode should be greater than one and equal to or less than the order.");
        return tensor_view_t(*this, contraction_mode);
    }

    /** Download into a host tensor with the same shape and layout. */
    host_tensor_t to_host() const
    {
        host_tensor_t h(_n, _pi);
        detail::device_check(tlibttm_copy(h.data().data(), _ptr, bytes()));
        return h;
    }

    value_t* data() { return _ptr; }
    value_t const* data() const { return _ptr; }
    std::size_t size() const { return _size; }
    auto const& shape() const { return _n; }
    auto const& layout() const { return _pi; }
    auto strides() const { return detail::generate_strides(_n, _pi); }
    auto order() const { return _n.size(); }

    void swap(device_tensor& o) noexcept
    {
        std::swap(_n, o._n);
        std::swap(_pi, o._pi);
        std::swap(_ptr, o._ptr);
        std::swap(_size, o._size);
    }

private:
    struct no_fill {};

    device_tensor(shape_t const& n, layout_t const& pi, no_fill) : _n(n), _pi(pi)
    {
        if (n.size() != pi.size())
            throw std::runtime_error("Error in tlib::tensor: shape vector and layout vector must have the same length.");
        if (!detail::is_valid_shape(n.begin(), n.end()))
            throw std::runtime_error("Error in tlib::tensor: shape vector of tensor is not valid.");
        if (!detail::is_valid_layout(pi.begin(), pi.end()))
            throw std::runtime_error("Error in tlib::tensor: layout vector of tensor is not valid.");
        allocate();
    }

    std::size_t bytes() const { return _size * sizeof(value_t); }

    // Runs a constructor's fill or copy; frees the allocation if it throws (no destructor runs then).
    template <class F>
    void guarded(F&& f)
    {
        try {
            f();
        } catch (...) {
            tlibttm_device_free(_ptr);
            _ptr = nullptr;
            throw;
        }
    }

    void allocate()
    {
        (void)detail::dtype_of<value_t>();
        _size = std::accumulate(_n.begin(), _n.end(), std::size_t{1}, std::multiplies<>());
        void* p = nullptr;
        detail::device_check(tlibttm_device_alloc(&p, bytes()));
        _ptr = static_cast<value_t*>(p);
    }

    shape_t _n;
    layout_t _pi;
    value_t* _ptr = nullptr;
    std::size_t _size = 0;
};

} // namespace tlib::ttm
