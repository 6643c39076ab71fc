"""pigfem_b200: B200-native finite-element assembly path of PIGFEM (IGFEM fiber-composite RVEs).

The product is the CUDA library ``_lib/libpigfem_b200.so`` behind the C ABI in
``include/pigfem_b200.h``; :mod:`pigfem_b200.assembler` mirrors the reference's
``Assembler`` / ``Problem`` host interface on top of it.
"""
from .capi import Problem, ProblemDesc, load_library, LIB_PATH  # noqa: F401
from . import capi  # noqa: F401

__all__ = ["Problem", "ProblemDesc", "load_library", "LIB_PATH", "capi"]
