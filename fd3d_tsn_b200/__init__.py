"""B200 (sm_100a) implementation of the FD3D_TSN time-stepping hot path.

The product is ``libfd3d_gpu.so`` (CUDA kernels behind the C ABI of
``include/fd3d_gpu.h``); this package holds its Python mirror (``solver``), the
ctypes view of the ABI (``abi``), host-side model set-up (``configs``) and the
build script (``build``).
"""
__all__ = ["abi", "configs", "solver", "build"]
