"""B200-native method-of-moments RCS solve path (2-D pulse EFIE/MFIE and body-of-revolution).

Host code is Python over PyTorch (device memory, streams); every arithmetic kernel
is hand-written sm_100a CUDA in ``libgrimgpu.so`` behind the C ABI of
``include/grimgpu.h``.  There is no CPU fallback.
"""
__version__ = '0.1.0'
