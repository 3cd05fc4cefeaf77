"""desalm -- host-side Python binding of the B200 DES-ALM pseudo-time iteration.

The product is the C ABI in include/desalm.h, implemented by the CUDA library
libdesalm.so built from des-alm_b200/csrc.  This package loads that library
(ctypes) and generates the seeded synthetic workloads.
"""
from .abi import Case, StepReport, level_dims  # noqa: F401
from . import cases  # noqa: F401
