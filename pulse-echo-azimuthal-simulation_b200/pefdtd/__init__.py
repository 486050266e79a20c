"""pefdtd — B200-native label-indexed anisotropic elastic FDTD.

``pefdtd.fdtd`` is the drop-in for the reference module sim/core/fdtd.py of
Jerome-Graves/pulse-echo-azimuthal-simulation; the CUDA kernels behind it are
in ``csrc/`` and reached through the C ABI of include/pefdtd.h.
"""
__version__ = "0.1.0"
