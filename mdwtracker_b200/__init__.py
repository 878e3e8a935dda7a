"""mdwtracker_b200 -- B200-native multi-density Woodcock tracker.

The product is ``libmdwt.so`` (C ABI in ``include/mdwt.h``; C++ host + sm_100a CUDA
kernels in ``csrc/``).  This package holds its Python mirror of the reference
renderer API (:class:`Renderer`) and the seeded synthetic scene generators used by the
benchmark and the tests.
"""
from .renderer import (FORMATS, LIB_PATH, MDWT_HOST_ONLY, MdwtError, Renderer,  # noqa: F401
                       load_library)

__all__ = ["Renderer", "MdwtError", "load_library", "LIB_PATH", "MDWT_HOST_ONLY", "FORMATS"]
