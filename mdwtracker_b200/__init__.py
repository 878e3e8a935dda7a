"""mdwtracker_b200 -- B200-native multi-density Woodcock tracker.

The product is ``libmdwt.so`` (C ABI in ``include/mdwt.h``; C++ host + sm_100a CUDA
kernels in ``csrc/``).  This package holds its Python mirror of the reference
renderer API (:class:`Renderer`), the learned denoiser's binding (:class:`Denoiser`,
``include/mdwt_denoiser.h``) and the seeded synthetic scene generators used by the
benchmark and the tests.
"""
from .renderer import (FORMATS, LIB_PATH, MDWT_HOST_ONLY, MdwtError, Renderer,  # noqa: F401
                       load_library)
from .denoiser import Denoiser  # noqa: F401
from .batch import Batch  # noqa: F401

__all__ = ["Renderer", "Denoiser", "Batch", "MdwtError", "load_library", "LIB_PATH", "MDWT_HOST_ONLY", "FORMATS"]
