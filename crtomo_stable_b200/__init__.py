"""B200-native CRTomo forward / sensitivity / Gauss-Newton inner-solve path.

The compute path is libcrt_b200.so (hand-written sm_100a CUDA behind the C
ABI of include/crt_b200.h); this package holds its ctypes binding, the
tomodir readers / writers and the host drivers that replay the CRMod and
CRTomo call sequences.
"""
from . import io  # noqa: F401

__all__ = ["io", "lib", "regularization", "inversion", "crmod", "synth"]
