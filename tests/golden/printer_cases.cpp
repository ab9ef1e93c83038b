#include <cassert>
// Prints tensors of orders 1..5 (first- and last-order layouts, values 1, 2, ...) with the
// tlib::ttm printer; compiled against the reference headers it writes printer_ref.txt.
#include <tlib/detail/tensor.h>
#include <iostream>
#include <numeric>
using namespace tlib::ttm;
int main() {
  std::vector<std::vector<std::size_t>> shapes = {{3},{2,3},{3,2},{2,3,2},{2,2,3,2},{2,1,2,2,3},{1,1,1},{3,1,2}};
  for (auto& s : shapes) for (std::size_t k : {1ul, 0ul}) {
    auto pi = detail::generate_k_order_layout(s.size(), k);
    tensor<float> A(s, pi);
    std::iota(A.begin(), A.end(), 1.0f);
    std::cout << A << std::endl;
  }
}
