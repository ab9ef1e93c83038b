"""The drop-in boundary run for real: the reference's own example programs and a C++ program of
all three tlib::ttm interfaces, linked against libtlibttm_cuda.so and executed on the GPU.

oracle/Makefile (`examples`) compiles each of the reference's example/*.cpp unchanged twice:
`<name>_b200` against include/ and this library, `<name>_ref` against the reference headers and
OpenBLAS. Both run here and must print the same text.
"""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _examples_dir():
    from oracle import EXAMPLES_DIR
    if not os.path.exists(os.path.join(EXAMPLES_DIR, "interface1_b200")):
        pytest.skip("reference example programs not built (oracle/Makefile examples)")
    return EXAMPLES_DIR


def _run(exe, *args):
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (exe, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


@pytest.mark.parametrize("name", ["interface1", "interface2", "interface3"])
def test_reference_example_prints_what_the_reference_prints(cuda, name):
    d = _examples_dir()
    ours = _run(os.path.join(d, name + "_b200"))
    ref = _run(os.path.join(d, name + "_ref"))
    assert ours == ref


def test_reference_measure_program(cuda):
    """example/measure.cpp with all six policies (method 7) in double: same problem text, sizes and
    work figures as the reference's run (timings differ)."""
    d = _examples_dir()
    args = ("7", "3", "2", "64", "48", "40")
    ours = _run(os.path.join(d, "measure_b200"), *args)
    ref = _run(os.path.join(d, "measure_ref"), *args)
    keep = lambda t: [ln for ln in t.splitlines() if not ln.startswith(("Time", "Performance"))]  # noqa: E731
    assert keep(ours) == keep(ref)
    assert ours.count("Performance :") == 12


def _cpp_program(name, tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = tmp_path / name
    lib = os.path.join(ROOT, "ttm_b200")
    subprocess.run([gxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I",
                    os.path.join(cuda_home, "include"), os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
                    "-o", str(exe), "-L", lib, "-ltlibttm_cuda", "-L", os.path.join(cuda_home, "lib64"), "-lcudart",
                    f"-Wl,-rpath,{lib}:{os.path.join(cuda_home, 'lib64')}"], check=True)
    return _run(str(exe))


def test_cpp_program_of_all_three_interfaces(cuda, tmp_path):
    out = _cpp_program("interfaces", tmp_path)
    assert "interfaces ok" in out, out


def test_cpp_device_resident_tensor(cuda, tmp_path):
    """tlib::ttm::device_tensor: A(q) * B and ttm(q, A, B, ...) on device-resident tensors give the
    host interfaces' exact bits, keep C on the device, and keep the host tensor's error texts."""
    out = _cpp_program("device_tensor", tmp_path)
    assert "device_tensor ok" in out, out


def test_top_level_ttmpy_module_runs_the_reference_calls(cuda):
    """`import ttmpy as tp` as the reference's Python test does (ttmpy/tests/test.py:3), on its
    exact-integer einsum cases (restated: the same arange inputs and einsum strings)."""
    import numpy as np
    import ttmpy as tp
    A = np.arange(3 * 2 * 4, dtype=np.float64).reshape(3, 2, 4)
    for q, sub, k in ((1, "ijk,xi->xjk", 3), (2, "ijk,xj->ixk", 2), (3, "ijk,xk->ijx", 4)):
        B = np.arange(5 * k, dtype=np.float64).reshape(5, k)
        assert np.all(tp.ttm(q, A, B) == np.einsum(sub, A, B))
    A = np.arange(3 * 2 * 4 * 5, dtype=np.float64).reshape(3, 2, 4, 5)
    B = [np.arange(2 * 6, dtype=np.float64).reshape(6, 2), np.arange(4 * 7, dtype=np.float64).reshape(7, 4),
         np.arange(5 * 9, dtype=np.float64).reshape(9, 5)]
    D = np.einsum("ijkl,yj->iykl", A, B[0])
    D = np.einsum("ijkl,yk->ijyl", D, B[1])
    D = np.einsum("ijkl,yl->ijky", D, B[2])
    for order in ("forward", "backward", "optimal"):
        assert np.all(tp.ttms(1, A, B, order) == D)
