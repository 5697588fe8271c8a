"""dugma_b200: B200-native (sm_100a) DUGMA hot path behind a C ABI.

The compute lives in libdugma_b200.so (hand-written CUDA kernels + C++ host
code); this package is the Python mirror of the reference's plugin interface
(init / update_sig / compi / fr_m and the DUGMA driver) over ctypes.
"""
