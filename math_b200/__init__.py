"""math_b200: B200-native n-space path tracer (drop-in for the painter of templeblock/math).

The hot path is CUDA for sm_100a behind the C ABI in include/ntrace.h (library
math_b200/libntrace.so); :mod:`math_b200.ntrace` mirrors the painter's scene interface over it and
:mod:`math_b200.scenes` prepares the measured scenes.
"""

from .ntrace import NtraceError, Scene, cosine_sphere_coefficient, effective_spp, library  # noqa: F401
