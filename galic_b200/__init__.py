"""galic_b200: B200 (sm_100a) implementation of GALIC's orbit-response hot path.

The product is libgalic_cuda.so (C ABI in include/galic_gpu.h); this package
builds it (`build.build()`), loads it (`_ffi.load_library()`), wraps a context
(`Context`) and generates seeded synthetic models of the benchmark shapes
(`synth`).
"""
from ._ffi import GALIC_FORM_FP32, GALIC_FORM_FP64, GalicParams, load_library  # noqa: F401
from .context import Context, GalicError  # noqa: F401
