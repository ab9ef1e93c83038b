"""Layout / shape / stride helpers and the C++ drop-in headers, against the
reference's own tables (test/src/gtest_tlib_{layout,strides,shape}.cpp) and,
when present, the reference build itself."""
import itertools
import os
import shutil
import subprocess

import pytest

from ttm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_k_order_layouts_table():
    # gtest_tlib_layout.cpp:40-166: k-order layouts of orders 1..4 for k = 1..4.
    want = {1: [[1], [1, 2], [1, 2, 3], [1, 2, 3, 4]],
            2: [[1], [2, 1], [2, 1, 3], [2, 1, 3, 4]],
            3: [[1], [2, 1], [3, 2, 1], [3, 2, 1, 4]],
            4: [[1], [2, 1], [3, 2, 1], [4, 3, 2, 1]]}
    for k, rows in want.items():
        for p, row in enumerate(rows, start=1):
            assert _lib.k_order_layout(p, k) == row
    assert _lib.k_order_layout(4, 0) == [4, 3, 2, 1]


def test_inverse_mode_all_k_orders():
    # gtest_tlib_layout.cpp:191-211
    for order in range(1, 11):
        for k in range(1, order + 1):
            lay = _lib.k_order_layout(order, k)
            for mode in range(1, order + 1):
                r = _lib.inverse_mode(lay, mode)
                assert 1 <= r <= order and lay[r - 1] == mode
    with pytest.raises(RuntimeError, match="mode should be one-based"):
        _lib.inverse_mode([1, 2], 3)
    with pytest.raises(RuntimeError, match="input layout is not valid"):
        _lib.inverse_mode([1, 1], 1)


def test_strides_tables():
    # gtest_tlib_strides.cpp:34-147
    assert _lib.strides([1], [1]) == [1]
    assert _lib.strides([1, 1], [1, 2]) == [1, 1]
    for ext in ([1, 2], [1, 4], [1, 8], [2, 1], [4, 1], [8, 1]):
        for lay in ([1, 2], [2, 1]):
            assert _lib.strides(ext, lay) == [1, 1]
    for ext in ([2, 2], [2, 4], [4, 2], [4, 4], [2, 8], [8, 2], [4, 8], [8, 4], [8, 8]):
        assert _lib.strides(ext, [1, 2]) == [1, ext[0]]
        assert _lib.strides(ext, [2, 1]) == [ext[1], 1]
    first = ([2, 1, 2], [1, 2, 2]), ([1, 2, 2], [1, 1, 2]), ([2, 2, 2], [1, 2, 4]), ([2, 4, 2], [1, 2, 8]), \
            ([4, 4, 2], [1, 4, 16]), ([2, 4, 4], [1, 2, 8])
    for ext, ref in first:
        assert _lib.strides(ext, [1, 2, 3]) == ref
    last = ([2, 1, 2], [2, 2, 1]), ([1, 2, 2], [4, 2, 1]), ([2, 2, 2], [4, 2, 1]), ([2, 4, 2], [8, 2, 1]), \
           ([2, 4, 4], [16, 4, 1])
    for ext, ref in last:
        assert _lib.strides(ext, [3, 2, 1]) == ref
    second = ([2, 1, 2], [1, 1, 2]), ([1, 2, 2], [2, 1, 2]), ([2, 2, 2], [2, 1, 4]), ([2, 4, 2], [4, 1, 8]), \
             ([2, 2, 4], [2, 1, 4]), ([4, 2, 2], [2, 1, 8])
    for ext, ref in second:
        assert _lib.strides(ext, [2, 1, 3]) == ref


def test_helpers_match_reference_build(reference):
    for p in range(1, 6):
        for k in range(0, p + 1):
            assert _lib.k_order_layout(p, k) == reference.k_order_layout(p, k)
        for n in itertools.product([1, 2, 3], repeat=p):
            for pi in itertools.permutations(range(1, p + 1)):
                assert _lib.strides(list(n), list(pi)) == reference.strides(list(n), list(pi)), (n, pi)


CXX_PROBE = r"""
#include <tlib/ttm.h>
#include <cassert>
#include <vector>
using namespace tlib::ttm;
int main() {
    // shape / layout / strides predicates, gtest_tlib_shape.cpp:65-139
    std::vector<std::vector<unsigned>> s = {{}, {0}, {1}, {2}, {0,1}, {1,0}, {1,1}, {2,1}, {3,1}, {1,2}, {1,3},
        {2,2}, {3,3}, {0,1,1}, {1,1,0}, {1,1,1}, {1,1,2}, {1,2,1}, {1,2,2}, {2,1,1}, {2,1,2}, {2,2,1}, {2,2,2}};
    std::vector<int> scal = {2,6,15}, vec = {3,7,8,9,10,17,19}, mat = {11,12,21}, ten = {16,18,20,22}, inv = {0,1,4,5,13,14};
    auto in = [](std::vector<int> const& v, int i){ for (int x : v) if (x == i) return true; return false; };
    for (int i = 0; i < (int)s.size(); ++i) {
        auto b = s[i].begin(), e = s[i].end();
        if (detail::is_scalar(b,e) != in(scal,i)) return 10 + i;
        if (detail::is_vector(b,e) != in(vec,i)) return 40 + i;
        if (detail::is_matrix(b,e) != in(mat,i)) return 70 + i;
        if (detail::is_tensor(b,e) != in(ten,i)) return 100 + i;
        if (detail::is_valid_shape(b,e) == in(inv,i)) return 130 + i;
    }
    std::vector<std::vector<unsigned>> bad = {{}, {0}, {0,1}, {1,0}, {0,2}, {2,0}, {2,1,0}, {3,0,2}, {3,1,4}, {1,3,4}, {1,3,5}};
    for (auto const& l : bad) if (detail::is_valid_layout(l.begin(), l.end())) return 160;
    std::size_t pi3[3] = {2,1,3};
    if (!detail::is_case<8>(3u, 1, pi3) || detail::is_case<6>(3u, 1, pi3) || !detail::is_case<6>(3u, 2, pi3)) return 170;
    auto A = tensor<float>({4,3,2});
    if (A.strides() != std::vector<std::size_t>({1,4,12})) return 180;
    try { A(4); return 190; } catch (std::runtime_error const&) {}
    return 0;
}
"""


def test_cpp_headers_compile_and_predicates(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    src = tmp_path / "probe.cpp"
    src.write_text(CXX_PROBE)
    exe = tmp_path / "probe"
    subprocess.run([gxx, "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", os.path.join(ROOT, "ttm_b200"), "-ltlibttm_cuda",
                    "-Wl,-rpath," + os.path.join(ROOT, "ttm_b200")], check=True)
    r = subprocess.run([str(exe)])
    assert r.returncode == 0, r.returncode


@pytest.mark.parametrize("name", ["interfaces", "device_tensor"])
def test_cpp_test_programs_build_and_link(tmp_path, name):
    """The C++ programs that tests/test_gpu_dropin.py runs on the GPU compile warning-free and
    resolve every symbol against libtlibttm_cuda.so (device_tensor needs no CUDA header)."""
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    lib = os.path.join(ROOT, "ttm_b200")
    exe = tmp_path / name
    subprocess.run([gxx, "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
                    os.path.join(cuda_home, "include"), os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-o",
                    str(exe), "-L", lib, "-ltlibttm_cuda", "-L", os.path.join(cuda_home, "lib64"), "-lcudart",
                    f"-Wl,-rpath,{lib}:{os.path.join(cuda_home, 'lib64')}"], check=True)
    r = subprocess.run(["ldd", "-r", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and "undefined symbol" not in r.stdout + r.stderr, r.stdout + r.stderr


@pytest.mark.parametrize("name", ["interface1", "interface2", "interface3", "measure"])
def test_reference_examples_built_unchanged(name):
    """The reference's own example programs, compiled unchanged against include/ and linked with
    libtlibttm_cuda.so by oracle/Makefile (`examples`), load and resolve every symbol (running them
    needs a GPU: tests/test_gpu_dropin.py)."""
    from oracle import EXAMPLES_DIR
    exe = os.path.join(EXAMPLES_DIR, name + "_b200")
    if not os.path.exists(exe):
        pytest.skip("reference example programs not built (oracle/Makefile examples)")
    r = subprocess.run(["ldd", "-r", exe], capture_output=True, text=True)
    assert r.returncode == 0 and "undefined symbol" not in r.stdout + r.stderr, r.stdout + r.stderr
    assert "libtlibttm_cuda.so" in r.stdout and "not found" not in r.stdout, r.stdout


def test_printer_matches_reference_text(tmp_path):
    """operator<< prints the reference's MATLAB-style text byte for byte (orders 1-5, both layouts;
    tests/golden/printer_ref.txt was written by the reference's own printer, oracle/Makefile `printer`)."""
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    exe = tmp_path / "printer"
    subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "golden", "printer_cases.cpp"), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    want = open(os.path.join(ROOT, "tests", "golden", "printer_ref.txt")).read()
    assert got == want


FASTDIV_PROBE = r"""
#include "common.cuh"
#include <cstdio>
int main() {
    using namespace tlibttm;
    uint64_t s = 88172645463325252ull;
    auto rnd = [&]() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; };
    long bad = 0;
    for (uint32_t t = 0; t < 100000; ++t) {
        uint32_t d = t < 50000 ? t + 1 : (uint32_t)(rnd() >> (rnd() % 33 + 31));
        if (!d) d = 1;
        const FastDiv f = make_fastdiv(d);
        const uint32_t ns[6] = {0u, 1u, d - 1, d, 0xffffffffu, (uint32_t)rnd()};
        for (uint32_t n : ns) bad += fast_div(n, f) != n / d;
        for (int k = 0; k < 8; ++k) { const uint32_t n = (uint32_t)rnd(); bad += fast_div(n, f) != n / d; }
    }
    std::printf("%ld\n", bad);
    return bad != 0;
}
"""


def test_fast_division_by_invariant_divisors(tmp_path):
    """The multiplicative divisors the stream kernel uses for its unit -> tile -> slice indices
    (common.cuh, host build of the same code) equal integer division: divisors 1..50000 and
    random ones up to 2^32 - 1, numerators 0, 1, d - 1, d, 2^32 - 1 and random."""
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    src = tmp_path / "fastdiv.cpp"
    src.write_text(FASTDIV_PROBE)
    exe = tmp_path / "fastdiv"
    subprocess.run([gxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "ttm_b200", "csrc"), "-I",
                    os.path.join(cuda_home, "include"), str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "0", r.stdout
