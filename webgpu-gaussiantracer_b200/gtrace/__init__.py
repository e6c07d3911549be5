"""gtrace — host side of the B200-native Gaussian ray tracer.

The tracing itself runs in the CUDA library ``libgtrace.so`` (C ABI declared
in include/gtrace.h).  This package mirrors the reference's host code
(PLY loader, uniform block, camera) and binds the library through ctypes.
"""
from .ply import PackedGaussians, load_gaussian_splatting, write_ply  # noqa: F401
from .uniforms import look_at, pack_uniforms, unpack_uniforms, with_fields  # noqa: F401
