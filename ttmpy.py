"""The reference binding's module name: ``import ttmpy as tp`` (reference ttmpy/tests/test.py:3).

Callers of the reference's pybind11 module ``ttmpy`` (ttmpy/src/wrapped_ttm.cpp:226-231) import
this module unchanged; ``tp.ttm(q, A, B)`` and ``tp.ttms(q, A, Bs, order)`` run on the GPU through
the C ABI. The implementation and its contract are in ``ttm_b200.ttmpy``.
"""
from ttm_b200.ttmpy import ttm, ttms  # noqa: F401

__all__ = ["ttm", "ttms"]
