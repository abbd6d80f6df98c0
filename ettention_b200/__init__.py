"""B200-native (sm_100a) block-iterative tomographic reconstruction path of Ettention.

The compute path is libettention_b200.so (CUDA, C ABI in include/ettention_b200.h);
``ettention_b200.operators`` mirrors libReconstruction's operator surface over it.
"""
from ._abi import EttentionError  # noqa: F401

__all__ = ["EttentionError"]
