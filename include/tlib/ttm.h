/*
 * tlib::ttm — mode-q tensor-times-matrix product, B200 implementation.
 *
 *   C(i1..j..ip) = sum_{iq} A(i1..iq..ip) * B(j, iq)
 *
 * Drop-in for the reference header of the same name (bassoy/ttm,
 * include/tlib/ttm.h): the same three interfaces, names, template parameters
 * and exception texts, so callers written against the reference compile
 * unchanged and link against libtlibttm_cuda.so instead of a CPU BLAS.
 *
 *  1. low-level  ttm(ep,sp,fp, q,p, a,na,wa,pia, b,nb,pib, c,nc,wc)   (reference ttm.h:54-93)
 *  2. high-level ttm(q, A, B, ep,sp,fp) -> tensor                     (reference ttm.h:100-125)
 *  3. operator   A(q) * B -> tensor                                    (reference ttm.h:133-138)
 *
 * Interfaces 2 and 3 also take device_tensor (detail/device_tensor.h), whose elements stay in
 * GPU memory: the product then runs with no host copies and returns a device_tensor.
 *
 * The pointers of interface 1 may be host or device memory; the call blocks
 * until C is written. The policy tags are accepted for compatibility and do
 * not change the result (see detail/tags.h).
 */
#pragma once

#include "detail/device_tensor.h"
#include "detail/tags.h"
#include "detail/tensor.h"
#include "detail/ttm.h"

namespace tlib::ttm
{

/**
 * Low-level interface. q is the one-based contraction mode (1 <= q <= p);
 * na/wa/pia are A's extents, strides and one-based layout; nb = (m, n_q) and
 * pib the layout of B (pib[0] == 1: column-major); nc/wc are C's extents and
 * strides, C sharing A's layout. C is overwritten.
 */
template <class value_t, class size_t, class parallel_policy, class slicing_policy, class fusion_policy>
inline void ttm(parallel_policy ep, slicing_policy sp, fusion_policy fp,
                unsigned const q, unsigned const p,
                const value_t* a, size_t const* const na, size_t const* const wa, size_t const* const pia,
                const value_t* b, size_t const* const nb, size_t const* const pib,
                value_t* c, size_t const* const nc, size_t const* const wc)
{
    detail::ttm(ep, sp, fp, q, p, a, na, wa, pia, b, nb, pib, c, nc, wc);
}

/** High-level interface: allocates C with A's layout and nc[q-1] = nb[0], then runs interface 1. */
template <class value_t, class execution_policy, class slicing_policy, class fusion_policy>
inline auto ttm(std::size_t q, ttm::tensor<value_t> const& a, ttm::tensor<value_t> const& b,
                execution_policy ep, slicing_policy sp, fusion_policy fp)
{
    auto const p = a.order();
    if (p == 0) throw std::runtime_error("Error in tlib::tensor_times_matrix: input tensor order should be greater zero.");
    if (q == 0 || q > p) throw std::runtime_error("Error in tlib::tensor_times_matrix: contraction mode should be greater zero or less than or equal to p.");

    auto nc = a.shape();
    auto nb = b.shape();
    nc[q - 1] = nb.at(0);
    auto c = tensor<value_t>(nc, a.layout());

    ttm(ep, sp, fp, static_cast<unsigned>(q), static_cast<unsigned>(p),
        a.data().data(), a.shape().data(), a.strides().data(), a.layout().data(),
        b.data().data(), b.shape().data(), b.layout().data(),
        c.data().data(), c.shape().data(), c.strides().data());
    return c;
}

/** High-level interface on device-resident tensors: the same checks and texts as above; C is
 *  made on the device (A's layout, nc[q-1] = nb[0]) and written by the product, with no host copy. */
template <class value_t, class execution_policy, class slicing_policy, class fusion_policy>
inline auto ttm(std::size_t q, ttm::device_tensor<value_t> const& a, ttm::device_tensor<value_t> const& b,
                execution_policy ep, slicing_policy sp, fusion_policy fp)
{
    auto const p = a.order();
    if (p == 0) throw std::runtime_error("Error in tlib::tensor_times_matrix: input tensor order should be greater zero.");
    if (q == 0 || q > p) throw std::runtime_error("Error in tlib::tensor_times_matrix: contraction mode should be greater zero or less than or equal to p.");

    auto nc = a.shape();
    auto nb = b.shape();
    nc[q - 1] = nb.at(0);
    auto c = device_tensor<value_t>::uninitialized(nc, a.layout());

    ttm(ep, sp, fp, static_cast<unsigned>(q), static_cast<unsigned>(p),
        a.data(), a.shape().data(), a.strides().data(), a.layout().data(),
        b.data(), b.shape().data(), b.layout().data(),
        c.data(), c.shape().data(), c.strides().data());
    return c;
}

} // namespace tlib::ttm

/** Operator interface: C = A(q) * B, with the combined policies (reference ttm.h:133-138). */
template <class value_t>
inline auto operator*(tlib::ttm::tensor_view<value_t> const& a, tlib::ttm::tensor<value_t> const& b)
{
    return tlib::ttm::ttm(a.contraction_mode(), a.get_tensor(), b, tlib::ttm::parallel_policy::combined,
                          tlib::ttm::slicing_policy::combined, tlib::ttm::fusion_policy::all);
}

/** Operator interface on device-resident tensors: C = A(q) * B stays on the device. */
template <class value_t>
inline auto operator*(tlib::ttm::device_tensor_view<value_t> const& a, tlib::ttm::device_tensor<value_t> const& b)
{
    return tlib::ttm::ttm(a.contraction_mode(), a.get_tensor(), b, tlib::ttm::parallel_policy::combined,
                          tlib::ttm::slicing_policy::combined, tlib::ttm::fusion_policy::all);
}
