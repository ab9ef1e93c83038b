"""B200-native mode-q tensor-times-matrix product with the tlib::ttm API.

* ``ttm_b200.ttmpy`` — drop-in for the reference's Python binding (``ttm``, ``ttms``).
* ``ttm_b200._lib``  — ctypes binding of the C ABI (include/tlibttm.h).
* ``ttm_b200.build`` — builds ``libtlibttm_cuda.so`` with nvcc for sm_100a.

The C++ drop-in (``#include <tlib/ttm.h>``) lives in ``include/``.
"""
from . import _lib  # noqa: F401
from . import ttmpy  # noqa: F401

__all__ = ["ttmpy"]
