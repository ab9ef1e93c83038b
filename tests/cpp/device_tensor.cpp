// Exercises tlib::ttm::device_tensor (include/tlib/detail/device_tensor.h) on the GPU library:
// products of device-resident tensors through A(q) * B and ttm(q, A, B, ...) must give exactly
// the bits the host-tensor interfaces give (the same kernels run on the same data) and agree
// with the definition; the result stays in device memory; copies are deep, moves transfer
// ownership; assignment of a value fills; bad arguments throw the host tensor's texts and a
// failed allocation throws std::bad_alloc. Exit code 0 on success; each failure is printed.
#include <tlib/ttm.h>

#include <cuda_runtime.h>

#include "check.h"

#include <cmath>
#include <cstdio>
#include <new>
#include <numeric>
#include <string>
#include <vector>

using namespace tlib::ttm;

static bool on_device(const void* p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice;
}

template <class T>
static void products(const char* tname)
{
    const std::vector<std::vector<std::size_t>> shapes = {{9, 7, 6, 5}, {40, 3, 33}, {300, 257}, {1000}};
    for (const auto& na : shapes) {
        const std::size_t p = na.size();
        for (std::size_t k : {1ul, p}) {    // first-order and last-order layouts
            const auto pia = detail::generate_k_order_layout(p, k);
            for (unsigned q = 1; q <= p; ++q) {
                for (std::size_t m : {3ul, 24ul, 130ul}) {
                    auto A = tensor<T>(na, pia);
                    for (std::size_t i = 0; i < A.data().size(); ++i) A[i] = T(std::sin(0.71 * double(i) + q));
                    auto B = tensor<T>({m, na[q - 1]});
                    for (std::size_t i = 0; i < B.data().size(); ++i) B[i] = T(std::cos(0.13 * double(i)));
                    const std::string tag = std::string(tname) + " p=" + std::to_string(p) + " k=" +
                                            std::to_string(k) + " q=" + std::to_string(q) + " m=" + std::to_string(m);

                    const auto host = A(q) * B;
                    const device_tensor<T> dA(A), dB(B);
                    const auto dC = dA(q) * dB;
                    check(dC.shape() == host.shape() && dC.layout() == pia, "shape/layout " + tag);
                    check(on_device(dC.data()), "result in device memory " + tag);
                    const auto got = dC.to_host();
                    check(got.data() == host.data(), "device == host bits " + tag);
                    std::size_t ncn = 1;
                    for (auto x : host.shape()) ncn *= x;
                    const auto want = naive_double<T>(q, na, A.strides(), A.data().data(), B.data().data(), true,
                                                      m, host.strides(), ncn);
                    const auto abs_sums = naive_double<T>(q, na, A.strides(), A.data().data(), B.data().data(),
                                                          true, m, host.strides(), ncn, true);
                    check(within_dot_bound(got.data(), want, abs_sums, na[q - 1]), "definition " + tag);
                    const auto dC2 = ttm(q, dA, dB, parallel_policy::parallel_loop, slicing_policy::slice,
                                         fusion_policy::outer);
                    check(dC2.to_host().data() == host.data(), "ttm(q,A,B,tags) " + tag);
                }
            }
        }
    }
}

template <class T>
static void ownership(const char* tname)
{
    const std::string t(tname);
    device_tensor<T> a({4, 5, 6}, {2, 1, 3});
    auto h = a.to_host();
    bool zeros = true;
    for (auto x : h) zeros = zeros && x == T(0);
    check(zeros, "zero-initialised " + t);
    a = T(2.5);
    auto b = a;                                        // deep copy
    check(b.data() != a.data() && b.layout() == a.layout(), "copy is a new buffer " + t);
    b = T(-1);
    bool two = true, minus = true;
    for (auto x : a.to_host()) two = two && x == T(2.5);
    for (auto x : b.to_host()) minus = minus && x == T(-1);
    check(two && minus, "copies are independent " + t);
    const T* pa = a.data();
    device_tensor<T> c(std::move(a));
    check(c.data() == pa && a.data() == nullptr && a.size() == 0, "move transfers ownership " + t);
    c = std::move(b);
    check(c.to_host()[0] == T(-1), "move assignment " + t);
    tensor<T> hv({3, 4});
    std::iota(hv.begin(), hv.end(), T(1));
    device_tensor<T> dv(hv);
    check(dv.to_host().data() == hv.data() && dv.strides() == hv.strides(), "upload/download round trip " + t);
}

static void errors()
{
    auto expect = [](auto&& f, const std::string& text) {
        try {
            f();
            check(false, "no exception for: " + text);
        } catch (std::runtime_error const& e) {
            check(std::string(e.what()) == text, std::string("exception text: ") + e.what());
        }
    };
    expect([] { device_tensor<float>({4, 3}, {1, 1}); }, "Error in tlib::tensor: layout vector of tensor is not valid.");
    expect([] { device_tensor<float>({4, 0}); }, "Error in tlib::tensor: shape vector of tensor is not valid.");
    expect([] { device_tensor<float>({4, 3}, {1, 2, 3}); },
           "Error in tlib::tensor: shape vector and layout vector must have the same length.");
    expect([] { device_tensor<float> a({4, 3}); (void)a(3); },
           "Error in tlib::tensor: specified contraction mode should be greater than one and equal to or less than the order.");
    expect([] { device_tensor<double> a({4, 3, 2}), b({5, 4}); (void)(a(2) * b); },
           "Error in tlib::tensor_times_matrix: contraction dimension of A and B are not equal.");
    // The next device allocation of the library fails: the constructor throws std::bad_alloc.
    tlibttm_inject(TLIBTTM_INJECT_FAIL_ALLOC, 1);
    try {
        device_tensor<float> a({64, 64});
        check(false, "no std::bad_alloc under an injected allocation failure");
    } catch (std::bad_alloc const&) {
    }
    tlibttm_inject(TLIBTTM_INJECT_NONE, 0);
    device_tensor<float> ok({64, 64});
    check(ok.data() != nullptr, "allocation after the injection is cleared");
}

int main()
{
    products<float>("float");
    products<double>("double");
    ownership<float>("float");
    ownership<double>("double");
    errors();
    if (g_fail) {
        std::printf("%d failures\n", g_fail);
        return 1;
    }
    std::printf("device_tensor ok\n");
    return 0;
}
