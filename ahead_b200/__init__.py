"""ahead_b200: B200-native AN-hardened BAT operators and star-join pipelines.

The compute path is hand-written sm_100a CUDA in ``libahead_b200.so`` behind
the C ABI of ``include/ahead_gpu.h``; this package is the host-side mirror of
the reference's operator interface (``ahead::bat::ops``) on top of it.  The
library is loaded on first use; if it is missing or no CUDA device is
present, every operator raises instead of computing anything on the CPU.
"""
from .model import *  # noqa: F401,F403
