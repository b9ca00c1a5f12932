"""kcfd: B200-native (sm_100a) SIMPLE inner loop for unstructured finite-volume meshes.

Host package over the native library libkcfd.so (CUDA kernels + C ABI, see
include/kcfd.h). Mirrors the K-CFD reference's core/ interface for the hot path.
"""
__version__ = "0.1.0"
