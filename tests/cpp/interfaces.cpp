// Exercises the three tlib::ttm interfaces of include/tlib/ttm.h on the GPU library:
//   1. low-level ttm(ep,sp,fp, q,p, a,na,wa,pia, b,nb,pib, c,nc,wc) with host and with device
//      pointers (reference include/tlib/ttm.h:54-93);
//   2. high-level ttm(q, A, B, ep,sp,fp) under several policy-tag combinations (ttm.h:100-125);
//   3. A(q) * B (ttm.h:133-138);
// and the reference's exception texts for bad arguments. Every result is compared with a plain
// loop over the definition C(i1..j..ip) = sum_iq A(i1..iq..ip) * B(j, iq). Exit code 0 on
// success; each failure is printed.
#include <tlib/ttm.h>

#include <cuda_runtime.h>

#include "check.h"

#include <cmath>
#include <cstdio>
#include <numeric>
#include <string>
#include <vector>

using namespace tlib::ttm;

template <class T>
static void high_level_and_operator(const char* tname)
{
    for (std::size_t k : {1ul, 0ul}) {
        for (unsigned q = 1; q <= 4; ++q) {
            const std::vector<std::size_t> na = {5, 4, 3, 6};
            const auto pia = detail::generate_k_order_layout(na.size(), k);
            auto A = tensor<T>(na, pia);
            std::iota(A.begin(), A.end(), T(1));
            const std::size_t m = 7;
            auto B = tensor<T>({m, na[q - 1]}, detail::generate_k_order_layout(std::size_t{2}, std::size_t{1}));
            for (std::size_t i = 0; i < B.data().size(); ++i) B[i] = T((i % 5) + 1) / T(4);
            auto nc = na;
            nc[q - 1] = m;
            const auto wc = detail::generate_strides(nc, pia);
            std::size_t ncn = 1;
            for (auto x : nc) ncn *= x;
            const auto want = naive<T>(q, na, A.strides(), A.data().data(), B.data().data(), true, m, wc, ncn);
            const std::string tag = std::string(tname) + " k=" + std::to_string(k) + " q=" + std::to_string(q);

            auto C0 = A(q) * B;
            check(C0.shape() == nc && C0.layout() == pia && close(C0.data(), want), "operator* " + tag);
            auto C1 = ttm(q, A, B, parallel_policy::parallel_blas, slicing_policy::slice, fusion_policy::none);
            check(close(C1.data(), want), "ttm parallel_blas/slice/none " + tag);
            auto C2 = ttm(q, A, B, parallel_policy::parallel_loop, slicing_policy::subtensor, fusion_policy::all);
            check(close(C2.data(), want), "ttm parallel_loop/subtensor/all " + tag);
            auto C3 = ttm(q, A, B, parallel_policy::sequential, slicing_policy::slice, fusion_policy::none);
            check(close(C3.data(), want), "ttm sequential/slice/none " + tag);
            auto C4 = ttm(q, A, B, parallel_policy::batched_gemm, slicing_policy::subtensor, fusion_policy::all);
            check(close(C4.data(), want), "ttm batched_gemm/subtensor/all " + tag);
            auto C5 = ttm(q, A, B, parallel_policy::combined, slicing_policy::combined, fusion_policy::all);
            check(close(C5.data(), want), "ttm combined " + tag);
        }
    }
}

template <class T>
static void low_level(const char* tname)
{
    // A of order 3, layout (2,3,1), B row-major (pib = {2,1}); host and device pointers.
    const std::vector<std::size_t> na = {33, 20, 18}, pia = {2, 3, 1};
    for (unsigned q = 1; q <= 3; ++q) {
        const std::size_t m = q == 2 ? 40 : 5;   // m = 40 runs a slice-GEMM kernel, m = 5 a small-m one
        const auto wa = detail::generate_strides(na, pia);
        auto nc = na;
        nc[q - 1] = m;
        const auto wc = detail::generate_strides(nc, pia);
        const std::vector<std::size_t> nb = {m, na[q - 1]}, pib = {2, 1};
        std::size_t nan = 1, ncn = 1;
        for (auto x : na) nan *= x;
        for (auto x : nc) ncn *= x;
        std::vector<T> a(nan), b(m * na[q - 1]), c(ncn, T(-1));
        for (std::size_t i = 0; i < nan; ++i) a[i] = T(std::sin(0.37 * (double)i));
        for (std::size_t i = 0; i < b.size(); ++i) b[i] = T(std::cos(0.11 * (double)i));
        const auto want = naive<T>(q, na, wa, a.data(), b.data(), false, m, wc, ncn);
        const std::string tag = std::string(tname) + " q=" + std::to_string(q);

        ttm(parallel_policy::parallel_loop, slicing_policy::slice, fusion_policy::outer, q, 3u, a.data(), na.data(),
            wa.data(), pia.data(), b.data(), nb.data(), pib.data(), c.data(), nc.data(), wc.data());
        check(close(c, want), "low-level host " + tag);

        T *da = nullptr, *db = nullptr, *dc = nullptr;
        if (cudaMalloc(&da, nan * sizeof(T)) != cudaSuccess || cudaMalloc(&db, b.size() * sizeof(T)) != cudaSuccess ||
            cudaMalloc(&dc, ncn * sizeof(T)) != cudaSuccess) {
            check(false, "cudaMalloc " + tag);
            return;
        }
        cudaMemcpy(da, a.data(), nan * sizeof(T), cudaMemcpyHostToDevice);
        cudaMemcpy(db, b.data(), b.size() * sizeof(T), cudaMemcpyHostToDevice);
        cudaMemset(dc, 0, ncn * sizeof(T));
        ttm(parallel_policy::parallel_taskloop, slicing_policy::subtensor, fusion_policy::none, q, 3u, da, na.data(),
            wa.data(), pia.data(), db, nb.data(), pib.data(), dc, nc.data(), wc.data());
        std::vector<T> got(ncn);
        cudaMemcpy(got.data(), dc, ncn * sizeof(T), cudaMemcpyDeviceToHost);
        check(close(got, want), "low-level device " + tag);
        // the ratio overload of parallel_loop_blas (reference detail/ttm.h:843)
        cudaMemset(dc, 0, ncn * sizeof(T));
        detail::ttm(parallel_policy::parallel_loop_blas, slicing_policy::slice, fusion_policy::all, q, 3u, 0.5, da,
                    na.data(), wa.data(), pia.data(), db, nb.data(), pib.data(), dc, nc.data(), wc.data());
        cudaMemcpy(got.data(), dc, ncn * sizeof(T), cudaMemcpyDeviceToHost);
        check(close(got, want), "detail::ttm parallel_loop_blas ratio " + tag);
        cudaFree(da);
        cudaFree(db);
        cudaFree(dc);
    }
}

static void errors()
{
    const std::vector<std::size_t> na = {4, 3, 2}, pia = {1, 2, 3}, wa = {1, 4, 12}, nb = {5, 4}, pib = {1, 2};
    const std::vector<std::size_t> nc = {5, 3, 2}, wc = {1, 5, 15};
    std::vector<float> a(24, 1.f), b(20, 1.f), c(30, 0.f);
    auto expect = [&](unsigned q, unsigned p, const float* pa, const std::string& text) {
        try {
            ttm(parallel_policy::combined, slicing_policy::combined, fusion_policy::all, q, p, pa, na.data(),
                wa.data(), pia.data(), b.data(), nb.data(), pib.data(), c.data(), nc.data(), wc.data());
            check(false, "no exception for: " + text);
        } catch (std::runtime_error const& e) {
            check(std::string(e.what()) == "Error in tlib::tensor_times_matrix: " + text,
                  std::string("exception text: ") + e.what());
        }
    };
    expect(1, 0, a.data(), "input tensor order should be greater zero.");
    expect(0, 3, a.data(), "contraction mode should be greater zero or less than or equal to p.");
    expect(4, 3, a.data(), "contraction mode should be greater zero or less than or equal to p.");
    expect(1, 3, nullptr, "pointer to input tensor A should not be zero.");
    expect(2, 3, a.data(), "contraction dimension of A and B are not equal.");
    try {
        auto A = tensor<float>({4, 3, 2});
        (void)A(4);
        check(false, "A(4) did not throw");
    } catch (std::runtime_error const&) {
    }
}

int main()
{
    high_level_and_operator<float>("float");
    high_level_and_operator<double>("double");
    low_level<float>("float");
    low_level<double>("double");
    errors();
    if (g_fail) {
        std::printf("%d failures\n", g_fail);
        return 1;
    }
    std::printf("interfaces ok\n");
    return 0;
}
