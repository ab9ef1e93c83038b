// Helpers shared by the C++ test programs: a failure counter, C = A x_q B from its definition
// (a plain loop in double), and a relative Frobenius comparison.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <string>
#include <vector>

inline int g_fail = 0;

inline void check(bool ok, const std::string& what)
{
    if (!ok) {
        std::printf("FAIL %s\n", what.c_str());
        ++g_fail;
    }
}

// C = A x_q B from the definition in double, on strided host arrays (B column-major when b_cm);
// with `absolute`, C of |A| x_q |B| instead.
template <class T>
inline std::vector<double> naive_double(unsigned q, const std::vector<std::size_t>& na,
                                        const std::vector<std::size_t>& wa, const T* a, const T* b, bool b_cm,
                                        std::size_t m, const std::vector<std::size_t>& wc, std::size_t nc_elems,
                                        bool absolute = false)
{
    const unsigned p = (unsigned)na.size();
    std::vector<double> c(nc_elems, 0.0);
    const std::size_t nq = na[q - 1];
    std::size_t total = 1;
    for (unsigned r = 0; r < p; ++r)
        if (r != q - 1) total *= na[r];
    for (std::size_t t = 0; t < total; ++t) {
        std::size_t rem = t, oa = 0, oc = 0;
        for (unsigned r = 0; r < p; ++r) {
            if (r == q - 1) continue;
            const std::size_t i = rem % na[r];
            rem /= na[r];
            oa += i * wa[r];
            oc += i * wc[r];
        }
        for (std::size_t j = 0; j < m; ++j) {
            double s = 0;
            for (std::size_t l = 0; l < nq; ++l) {
                const double x = (double)a[oa + l * wa[q - 1]] * (double)b[b_cm ? j + l * m : j * nq + l];
                s += absolute ? std::fabs(x) : x;
            }
            c[oc + j * wc[q - 1]] = s;
        }
    }
    return c;
}

// The same, rounded to T.
template <class T>
inline std::vector<T> naive(unsigned q, const std::vector<std::size_t>& na, const std::vector<std::size_t>& wa,
                            const T* a, const T* b, bool b_cm, std::size_t m, const std::vector<std::size_t>& wc,
                            std::size_t nc_elems)
{
    const auto d = naive_double(q, na, wa, a, b, b_cm, m, wc, nc_elems);
    return std::vector<T>(d.begin(), d.end());
}

// Relative Frobenius distance within tol (default: 1e-6 float, 1e-13 double, for short sums).
template <class T>
inline bool close(const std::vector<T>& x, const std::vector<T>& y, double tol = sizeof(T) == 4 ? 1e-6 : 1e-13)
{
    if (x.size() != y.size()) return false;
    double num = 0, den = 0;
    for (std::size_t i = 0; i < x.size(); ++i) {
        num += ((double)x[i] - y[i]) * ((double)x[i] - y[i]);
        den += (double)y[i] * y[i];
    }
    return std::sqrt(num) <= tol * std::sqrt(den) + 1e-30;
}

// The dot-product error bound: a sum of n products computed in T, in any order and with or
// without FMA, is within gamma_n * sum |a_l b_l| of the exact sum (gamma_n = n u / (1 - n u),
// u the unit roundoff of T). `abs_sums` is C of |A| x_q |B| in double; the bound is doubled to
// cover the rounding of the stored result and of the double reference.
template <class T>
inline bool within_dot_bound(const std::vector<T>& got, const std::vector<double>& want,
                             const std::vector<double>& abs_sums, std::size_t n)
{
    const double u = sizeof(T) == 4 ? 5.96e-8 : 1.11e-16;
    const double gamma = double(n + 1) * u / (1.0 - double(n + 1) * u);
    if (got.size() != want.size() || got.size() != abs_sums.size()) return false;
    for (std::size_t i = 0; i < got.size(); ++i)
        if (std::fabs((double)got[i] - want[i]) > 2.0 * gamma * abs_sums[i] + 1e-300) return false;
    return true;
}

